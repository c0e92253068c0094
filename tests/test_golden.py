"""Oracle and host utilities against the reference's golden data: the RANMAR
known-answer test (src/marsaglia.h:66-72), the mesh fixture, the trajectory
format as read by the reference's scripts/celldiv.py."""
import json
import os

import numpy as np

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import traj
from cellsim3d_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_ranmar_kat_oracle():
    k = json.load(open(os.path.join(GOLD, "ranmar_kat.json")))
    r = oracle.Ranmar(k["ij"], k["kl"])
    r.draw(k["skip"])
    got = r.draw(6).astype(np.float64) * 4096 * 4096
    assert got.tolist() == k["expect_x4096sq"]


def test_ranmar_kat_native():
    k = json.load(open(os.path.join(GOLD, "ranmar_kat.json")))
    r = cs.Ranmar(k["ij"], k["kl"])
    r.draw(k["skip"])
    got = r.draw(6).astype(np.float64) * 4096 * 4096
    assert got.tolist() == k["expect_x4096sq"]


def test_ranmar_native_matches_oracle_bitwise():
    for ij, kl in [(42, 4200), (7, 700), (1802, 9373), (0, 0), (31328, 30081)]:
        a, b = cs.Ranmar(ij, kl), oracle.Ranmar(ij, kl)
        assert np.array_equal(a.draw(1000).view(np.uint32), b.draw(1000).view(np.uint32))
        for _ in range(200):
            assert np.array_equal(a.random_vector().view(np.uint32), b.random_vector().view(np.uint32))


def test_random_vector_is_unit():
    r = cs.Ranmar(42, 4200)
    for _ in range(1000):
        n = r.random_vector().astype(np.float64)
        assert abs(np.linalg.norm(n) - 1) < 1e-3   # src/postscriptinit.cu:215


def test_seed_map():
    assert cs.seed_map(42) == (42, 4200)
    assert cs.seed_map(300) == (300, 30000)
    for s in (1000, 1063, 123456):
        ij, kl = cs.seed_map(s)
        assert (ij, kl) == oracle.seed_map(s) == W.seed_pair(s)
        assert 0 <= ij <= 31328 and 0 <= kl <= 30081


def test_rmarin_rejects_out_of_range():
    import pytest
    with pytest.raises(cs.CS3DError):
        cs.Ranmar(40000, 1)


def test_mesh_invariants(mesh):
    nn, sign, bonds, faces = mesh["nn"], mesh["sign"], mesh["bonds"], mesh["faces"]
    assert mesh["xyz"].shape == (180, 3)
    assert set(np.unique(sign)) <= {-1, 1}
    assert bonds.shape == (270, 2)
    assert faces.shape == (92, 7)
    assert np.all(nn[:, :180] >= 0) and np.all(nn[:, :180] < 180)
    # each node has 3 distinct neighbours, the relation is symmetric
    for i in range(180):
        assert len(set(nn[:, i])) == 3
        for k in range(3):
            assert i in nn[:, nn[k, i]]
    # bonds are exactly the neighbour pairs
    pairs = {tuple(sorted((i, int(nn[k, i])))) for i in range(180) for k in range(3)}
    assert pairs == {tuple(sorted(map(int, b))) for b in bonds}
    # 12 pentagons, 80 hexagons; every node on 3 faces
    count = np.zeros(180, int)
    for f in range(92):
        m = 5 if f < 12 else 6
        for q in range(m):
            count[faces[f, q]] += 1
        assert faces[f, m] == faces[f, 0]
    assert np.all(count == 3)


def test_native_mesh_reader_matches_fixture(tmp_path, mesh):
    d = tmp_path
    with open(d / "C180", "w") as f:
        for p in mesh["xyz"]:
            f.write("%.9g  %.9g  %.9g\n" % tuple(float(v) for v in p))
    with open(d / "C180NN", "w") as f:
        for i in range(180):
            f.write(" %d,  %d,  %d,  %d\n" % (mesh["nn"][0, i] + 1, mesh["nn"][1, i] + 1, mesh["nn"][2, i] + 1, mesh["sign"][i]))
    with open(d / "C180C", "w") as f:
        for a, b in mesh["bonds"]:
            f.write(" %d,  %d\n" % (a + 1, b + 1))
    with open(d / "C180_pentahexa", "w") as f:
        for k in range(92):
            m = 5 if k < 12 else 6
            f.write("  ".join(str(v) for v in mesh["faces"][k, :m]) + "\n")
    m = cs.read_fullerene_nn(str(d))
    assert np.array_equal(np.frombuffer(m.xyz, np.float32).reshape(180, 3), mesh["xyz"])
    assert np.array_equal(np.frombuffer(m.nn, np.int32).reshape(3, 192)[:, :180], mesh["nn"][:, :180])
    assert np.array_equal(np.frombuffer(m.faces, np.int32).reshape(92, 7), mesh["faces"])
    assert np.array_equal(np.frombuffer(m.bonds, np.int32).reshape(270, 2), mesh["bonds"])


def test_traj_writer_matches_golden(tmp_path):
    gold = json.load(open(os.path.join(GOLD, "traj_small.json")))
    rng = np.random.default_rng(5)
    path = tmp_path / "t.bin"
    with traj.TrajWriter(path, max_cells=16, variable_stiffness=False, max_frames=2) as w:
        for k, (step, n) in enumerate([(0, 2), (10, 3)]):
            X = rng.standard_normal((n, 192)).astype(np.float32)
            Y = rng.standard_normal((n, 192)).astype(np.float32)
            Z = rng.standard_normal((n, 192)).astype(np.float32)
            w.write_frame(step, k + 1, X, Y, Z)
        w.set_final_cells(3)
    assert open(path, "rb").read() == open(os.path.join(GOLD, "traj_small.bin"), "rb").read()
    hdr, frames = traj.read_traj(path)
    assert hdr["max_cells"] == gold["maxNCells"]
    assert hdr["max_frames"] == gold["maxFrames"]
    for f, g in zip(frames, gold["frames"]):
        assert f["step"] == g["step"] and f["frame"] == g["frame"] and len(f["X"]) == g["n"]
        s = float(np.stack([f["X"], f["Y"], f["Z"]], -1).astype(np.float64).sum())
        assert abs(s - g["sum"]) < 1e-9 * max(1, abs(g["sum"]))
        assert [float(f["X"][0, 0]), float(f["Y"][0, 0]), float(f["Z"][0, 0])] == g["first"]


def _fma_case():
    c = np.load(os.path.join(GOLD, "fma_boundary_case.npz"))
    st = {k: c[k] for k in ("X", "Y", "Z", "VX", "VY", "VZ")}
    st["n"] = 2
    return c, st


def test_fma_boundary_case_fixture():
    """The fixture's pair lies at the cut-off in the uncontracted float
    expression and above it in the contracted one that the reference's build
    evaluates (fma(dz, dz, fma(dx, dx, dy*dy)))."""
    from fractions import Fraction
    c, st = _fma_case()
    i, j = int(c["i"]), int(c["j"])
    f32 = np.float32
    d = [f32(st[k].reshape(2, 192)[0, i] - st[k].reshape(2, 192)[1, j]) for k in ("X", "Y", "Z")]
    fma = lambda a, b, z: f32(float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(z))))
    plain = f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))
    contracted = fma(d[2], d[2], fma(d[0], d[0], f32(d[1] * d[1])))
    ra2 = f32(f32(0.3) * f32(0.3))
    assert plain == c["r2_plain"] and contracted == c["r2_fma"]
    assert plain <= ra2 < contracted


def test_oracle_decides_the_boundary_pair_as_the_reference_build():
    """With the contracted squared distance the oracle leaves the pair out of
    the dissipative set, so node i feels no friction (its neighbours and
    itself rest); tests/test_ref_cuda.py shows the reference's own kernels
    leave it out too."""
    c, st = _fma_case()
    i, j = int(c["i"]), int(c["j"])
    mesh = W.load_mesh()
    p = W.base_params(box_len=(30.0, 30.0, 30.0))
    r0, th = oracle.r0_theta0(st["X"][:192], st["Y"][:192], st["Z"][:192], mesh["nn"])
    O = oracle.System(2, p, oracle.make_topo(mesh["nn"], mesh["sign"], r0, th, mesh["faces"]))
    O.load(st["X"], st["Y"], st["Z"], st["VX"], st["VY"], st["VZ"], n=2)
    O.seed(1, 100)
    O.set_record(True)
    O.init()
    pairs = {tuple(x) for x in O.recorded_pairs(1).tolist()}
    assert (0, i, 1, j) not in pairs and (1, j, 0, i) not in pairs
    assert all(float(O.FD[q][i]) == 0.0 for q in range(3))
    O.close()
