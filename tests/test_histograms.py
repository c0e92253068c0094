"""Device-side analysis of a run: the volume histogram (the per-cell volume
of src/volume.cu:5-163 at the current positions, binned on the GPU) and the
population curve N(t) (the curve scripts/pop.py draws from a trajectory, here
from the division events).  Exact against the oracle on identical positions;
against the reference's own kernels over a long growth run the curves and
distributions agree statistically (the FP32 and FP64 trajectories separate
slowly)."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import workloads as W

from parity import make_pair, topo_for

pytestmark = pytest.mark.gpu


def _bins(v, lo, hi, nb):
    out = np.zeros(nb + 2, np.int64)
    for x in np.asarray(v, np.float32):
        if not x >= lo:
            out[0] += 1
        elif not x < hi:
            out[nb + 1] += 1
        else:
            out[min(nb, 1 + int((float(x) - lo) / (hi - lo) * nb))] += 1
    return out


def test_volume_histogram_matches_oracle(mesh):
    """After 600 steps of the 8-cell dividing configuration: every cell's
    volume against the oracle's on the same positions, and the bin counts."""
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, 256, record_pairs=False)
    sim.step(600)
    s = sim.state()
    n = s["n"]
    counts, vols = sim.volume_histogram(lo=0.0, hi=12.0, nbins=48, volumes=True)
    O = oracle.System(256, p, orc._t)
    O.load(s["X"], s["Y"], s["Z"], n=n)
    ref_v = O.compute_volumes()
    rel = np.max(np.abs(vols.astype(np.float64) - ref_v) / np.abs(ref_v))
    print("volume histogram: %d cells, max relative volume difference %.2e, counts %s" % (n, rel, counts.tolist()))
    assert rel < 1e-6
    assert counts.sum() == n
    assert counts[0] == counts[-1] == 0
    assert np.array_equal(counts, _bins(vols, 0.0, 12.0, 48))
    # the same counts from the oracle's volumes unless one sits on a bin edge
    assert np.abs(counts - _bins(ref_v, 0.0, 12.0, 48)).sum() <= 2
    # population curve from the events
    pop = sim.population(0)
    assert pop[0] == 8 and pop[-1] == n and len(pop) == 601 and np.all(np.diff(pop) >= 0)
    O.close()
    orc.close()
    sim.close()


def test_volume_histogram_edges_and_empty_bins(mesh):
    """Values below lo and at or above hi land in the two outer counts."""
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    counts, vols = sim.volume_histogram(lo=10.0, hi=20.0, nbins=5, volumes=True)
    assert counts[0] == 8 and counts[1:].sum() == 0          # every cell is below lo
    counts = sim.volume_histogram(lo=0.1, hi=float(vols.min()), nbins=3)
    assert counts[-1] == 8                                    # every cell at or above hi
    with pytest.raises(cs.CS3DError):
        sim.volume_histogram(lo=2.0, hi=1.0, nbins=4)
    sim.close()


def test_population_and_volumes_against_reference_kernels(mesh):
    """A colony grown from one cell for 9000 steps (about 100 cells; from about
    12000 steps on the reference's 32-slot grid bins overflow) by the
    reference's own kernels and by the CUDA path: the population curves and
    the final volume distributions (both binned by the same device
    function)."""
    from oracle import ref
    from scipy import stats
    if not ref.available():
        pytest.skip("oracle/_ref/cs3d_ref not built")
    p, st, _ = W.config2()
    steps = 9000
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 2048, steps)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 2048)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(steps)
    pop = sim.population(0)
    born = np.bincount(r["events"][:, 0], minlength=steps + 1)[: steps + 1]
    pop_ref = st["n"] + np.cumsum(born)
    # the reference's final state through the same device volume function
    other = cs.Simulation(p, topo, 2048)
    other.load_state(r["X"], r["Y"], r["Z"], n_cells=r["n"])
    c1, v1 = sim.volume_histogram(lo=0.0, hi=12.0, nbins=24, volumes=True)
    c2, v2 = other.volume_histogram(lo=0.0, hi=12.0, nbins=24, volumes=True)
    ks = stats.ks_2samp(v1, v2)
    gap = np.abs(pop - pop_ref).max()
    print("colony %d steps: cells %d (reference %d), largest population gap %d, volume KS p %.3f, "
          "first differing step %s, histograms %s / %s" % (steps, pop[-1], pop_ref[-1], gap, ks.pvalue,
                                                           int(np.argmax(pop != pop_ref)) if gap else None,
                                                           c1.tolist(), c2.tolist()))
    assert abs(pop[-1] - pop_ref[-1]) <= max(2, 0.15 * pop_ref[-1])
    assert ks.pvalue > 1e-3
    sim.close()
    other.close()


@pytest.mark.parametrize("config,steps", [("config1", 5000), ("config2", 8000)])
def test_statistics_across_seeds_against_reference_kernels(mesh, config, steps):
    """Beyond the first 2000 steps the FP32 reference and this library (FP64
    force terms) separate chaotically, so the comparison is statistical, as
    scripts/pop.py analyses a run: eight seeds (RANMAR (s, 100 s), s = 1..8)
    of the same configuration run by the reference's own kernels and by the
    CUDA path.  Two-sample KS tests on the pooled final cell volumes (every
    cell of every seed, computed by the same device function), on the final
    populations of the eight seeds, and on the populations at every 500th
    step of all seeds pooled; the mean final populations agree within 15 %."""
    from oracle import ref
    from scipy import stats
    if not ref.available():
        pytest.skip("oracle/_ref/cs3d_ref not built")
    p0, st, _ = getattr(W, config)()
    topo, _ = topo_for(st, mesh)
    cap = 2048
    checkpoints = np.arange(500, steps + 1, 500)
    pops, pops_ref, vols, vols_ref, curve, curve_ref = [], [], [], [], [], []
    for s in range(1, 9):
        p = dict(p0, rng_ij=s, rng_kl=100 * s)
        r = ref.run(p, mesh, st, cap, steps)
        assert r["status"] == 0, (s, r["status_text"])
        sim = cs.Simulation(p, topo, cap)
        sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
        sim.step(steps)
        pop = sim.population(0)
        born = np.bincount(r["events"][:, 0], minlength=steps + 1)[: steps + 1]
        pop_ref = st["n"] + np.cumsum(born)
        other = cs.Simulation(p, topo, cap)
        other.load_state(r["X"], r["Y"], r["Z"], n_cells=r["n"])
        _, v1 = sim.volume_histogram(lo=0.0, hi=12.0, nbins=24, volumes=True)
        _, v2 = other.volume_histogram(lo=0.0, hi=12.0, nbins=24, volumes=True)
        pops.append(int(pop[-1]))
        pops_ref.append(int(pop_ref[-1]))
        curve.extend(pop[checkpoints].tolist())
        curve_ref.extend(pop_ref[checkpoints].tolist())
        vols.extend(v1.tolist())
        vols_ref.extend(v2.tolist())
        assert sim.last_error() == 0, s
        sim.close()
        other.close()
    ks_v = stats.ks_2samp(vols, vols_ref)
    ks_p = stats.ks_2samp(pops, pops_ref)
    ks_c = stats.ks_2samp(curve, curve_ref)
    print("%s, 8 seeds x %d steps: final populations %s (reference %s); KS p: volumes %.3f (%d / %d cells), "
          "final populations %.3f, populations every 500 steps %.3f"
          % (config, steps, pops, pops_ref, ks_v.pvalue, len(vols), len(vols_ref), ks_p.pvalue, ks_c.pvalue))
    assert ks_v.pvalue > 1e-3
    assert ks_p.pvalue > 1e-3
    assert ks_c.pvalue > 1e-3
    assert abs(np.mean(pops) - np.mean(pops_ref)) <= 0.15 * np.mean(pops_ref)
