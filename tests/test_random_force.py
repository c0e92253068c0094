"""Langevin random force (rand_params.add_rands, src/propagate.cu:668-678).

The reference draws it from curand XORWOW; this library from Philox4x32-10
keyed by rand_seed and counted by (node, step).  Only the distribution can
match the reference: rand_scale_factor times independent standard normals.
Checked here: the oracle's generator against an independent numpy
restatement of Philox4x32-10 + Box-Muller, the distribution (mean, variance,
Kolmogorov-Smirnov against the normal), independence across steps and
nodes; on the GPU, single steps with the random force against the oracle,
and the device's draws against the same distribution tests."""
import numpy as np
import pytest
from scipy import stats

import oracle
from cellsim3d_b200 import workloads as W

M32 = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC'11) on numpy uint64
    arrays holding 32-bit words: ctr (4, n), key (2,)."""
    c = [np.asarray(w, dtype=np.uint64) & M32 for w in ctr]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(M32)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(M32)
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(0x9E3779B9)) & np.uint64(M32)
        k1 = (k1 + np.uint64(0xBB67AE85)) & np.uint64(M32)
    return c


def normals(seed, scale, nodes, step):
    nodes = np.asarray(nodes, dtype=np.uint64)
    z = np.zeros_like(nodes)
    r = philox4x32_10([nodes, z + np.uint64(step), z, z], (seed, 0x2545F491))
    u = [((w >> np.uint64(8)).astype(np.float32) + np.float32(0.5)) * np.float32(1.0 / 16777216.0) for w in r]
    ra = np.sqrt(np.float32(-2.0) * np.log(u[0]))
    rb = np.sqrt(np.float32(-2.0) * np.log(u[2]))
    ta, tb = np.float32(6.28318531) * u[1], np.float32(6.28318531) * u[3]
    s = np.float32(scale)
    return np.stack([s * (ra * np.cos(ta)), s * (ra * np.sin(ta)), s * (rb * np.cos(tb))], -1)


def _params():
    return W.base_params(add_rands=1, rand_scale_factor=0.1, rand_seed=1234)


def test_oracle_generator_matches_independent_restatement():
    p = _params()
    nodes = np.arange(0, 192 * 40)
    got = np.array([oracle.random_force(p, int(n), 17) for n in nodes])
    ref = normals(1234, 0.1, nodes, 17)
    # the same integers and float steps; libm and numpy may differ by an ulp
    np.testing.assert_allclose(got, ref, rtol=2e-6, atol=1e-8)


def _check_distribution(v, scale):
    z = v.reshape(-1) / scale
    n = z.size
    assert abs(z.mean()) < 5.0 / np.sqrt(n), z.mean()
    assert abs(z.std() - 1.0) < 5.0 * np.sqrt(0.5 / n) + 1e-3, z.std()
    assert stats.kstest(z, "norm").pvalue > 1e-4


def test_distribution_and_independence():
    nodes = np.arange(0, 192 * 200)
    a = normals(99, 0.1, nodes, 5)
    b = normals(99, 0.1, nodes, 6)
    c = normals(100, 0.1, nodes, 5)
    for v in (a, b, c):
        _check_distribution(v, 0.1)
    for x, y in ((a, b), (a, c)):
        r = np.corrcoef(x.reshape(-1), y.reshape(-1))[0, 1]
        assert abs(r) < 5.0 / np.sqrt(x.size), r
    # components of one node are independent too
    r = np.corrcoef(a[:, 0], a[:, 2])[0, 1]
    assert abs(r) < 5.0 / np.sqrt(len(a)), r


@pytest.mark.gpu
def test_random_force_single_steps_against_oracle(mesh):
    from parity import make_pair, single_step_check
    c, vel, L = W.packed_fcc(64, phi=0.5, seed=11)
    p = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                      div_time_steps=5000, add_rands=1, rand_scale_factor=0.1, rand_seed=4321)
    st = W.state(c, velocities=vel)
    sim, orc = make_pair(p, st, mesh, capacity=64)
    for target in (1, 2, 3, 10):
        cur = sim.stats()["steps"]
        if target - 1 > cur:
            sim.step(target - 1 - cur)
        single_step_check(sim, "random force step %d" % target)
    fr = sim.random_force()
    n = sim.n_cells()
    v = np.stack([fr["FRX"], fr["FRY"], fr["FRZ"]], -1).reshape(n, 192, 3)[:, :180]
    _check_distribution(v, 0.1)
    # the device draws are the generator's
    step = sim.stats()["steps"]
    nodes = (np.arange(n)[:, None] * 192 + np.arange(180)[None, :]).reshape(-1)
    np.testing.assert_allclose(v.reshape(-1, 3), normals(4321, 0.1, nodes, step), rtol=2e-6, atol=1e-8)
    sim.close()
    orc.close()
