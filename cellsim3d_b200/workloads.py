"""Seeded synthetic initial states for the benchmark configurations.

The reference can only place cells on a 2-D lattice or by random insertion
(src/GPUbounce.cu:1655-1771); the benchmark configurations need 3-D lattices,
packed systems and Gaussian velocities, so their initial states are generated
here and loaded through cs3d_load_state (the reference harness loads the same
arrays).  Every generator is deterministic in its seed.

Mesh: the reference's C180 scaled to mean radius 1.0 (factor 1.718846), then
centred with the reference's float arithmetic (src/GPUbounce.cu:1631-1653).
"""
import math
import os

import numpy as np

MESH_SCALE = 1.718846
_GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")


def load_mesh(path=None):
    """C180 mesh arrays (xyz float32 (180,3), nn (3,192), sign, bonds, faces (92,7))."""
    path = path or os.path.join(_GOLDEN, "c180_mesh.npz")
    d = np.load(path)
    return {k: d[k] for k in d.files}


def scaled_xyz(mesh, scale=MESH_SCALE):
    return (mesh["xyz"].astype(np.float64) * scale).astype(np.float32)


def centred(xyz):
    """Centre as initialize_C180s does: sequential float sums, /180.0 in
    double then float, float subtraction (src/GPUbounce.cu:1631-1653)."""
    xyz = np.asarray(xyz, dtype=np.float32)
    s = [np.float32(0)] * 3
    for i in range(180):
        for d in range(3):
            s[d] = np.float32(s[d] + xyz[i, d])
    s = [np.float32(float(v) / 180.0) for v in s]
    out = xyz.copy()
    for d in range(3):
        out[:, d] = (xyz[:, d] - s[d]).astype(np.float32)
    return out


def place(mesh_xyz, centres):
    """Positions (X, Y, Z), 192-stride, of cells at float32 centres."""
    centres = np.asarray(centres, dtype=np.float32)
    n = len(centres)
    out = []
    for d in range(3):
        a = np.zeros((n, 192), dtype=np.float32)
        a[:, :180] = (mesh_xyz[None, :, d] + centres[:, d:d + 1]).astype(np.float32)
        out.append(a.reshape(-1))
    return out


def base_params(**over):
    """Hot-path parameters shared by all benchmark configurations."""
    p = dict(particle_mass=0.04, repulsion_range=0.2, attraction_range=0.3,
             repulsion_strength=100.0, attraction_strength=0.1, youngs_mod=1000.0,
             stiffness1=1000.0, internal_damping=100.0, viscotic_damping=1.0, gamma_visc=1.0,
             division_vol=2.9, time_interval=1e-4, max_pressure=300.0, min_pressure=50.0,
             growth_rate=0.002, thresh_dist=0.01, box_len=(10.0, 10.0, 10.0),
             check_sphericity=1, constrain_angles=1, use_rigid_box=1, daught_same_stiffness=1,
             div_time_steps=20000, rng_ij=42, rng_kl=4200)
    p.update(over)
    return p


def seed_pair(seed):
    """rand_seed -> RANMAR (ij, kl): src/GPUbounce.cu:1796-1799 for seeds <= 300,
    folded into the legal range above that."""
    if 0 <= seed <= 300:
        return seed, 100 * seed
    s = abs(seed)
    return s % 31329, (100 * s) % 30082


def state(centres, mesh=None, velocities=None, pressure=None):
    mesh = mesh or load_mesh()
    xyz = centred(scaled_xyz(mesh))
    X, Y, Z = place(xyz, centres)
    st = {"X": X, "Y": Y, "Z": Z, "n": len(centres)}
    if velocities is not None:
        st["VX"], st["VY"], st["VZ"] = velocities
    if pressure is not None:
        st["pressure"] = pressure
    return st


# ---------------------------------------------------------------- config 1
def config1():
    """8 cells on a 2x2x2 lattice, spacing 2.2, centred in a box of side 10;
    pressure 50 -> 300 at 0.002/step, division at V = 2.9, seed 42."""
    c = np.array([[5 + 1.1 * sx, 5 + 1.1 * sy, 5 + 1.1 * sz]
                  for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], dtype=np.float32)
    p = base_params(box_len=(10.0, 10.0, 10.0), div_time_steps=20000, rng_ij=42, rng_kl=4200)
    return p, state(c), 20000


# ---------------------------------------------------------------- config 2
def config2(capacity=8192):
    """1 cell at the centre of a box of side 60, grown by division, seed 7."""
    c = np.array([[30.0, 30.0, 30.0]], dtype=np.float32)
    p = base_params(box_len=(60.0, 60.0, 60.0), div_time_steps=10 ** 9, rng_ij=7, rng_kl=700)
    return p, state(c), capacity


# ---------------------------------------------------------------- config 3
def packed_fcc(n_cells, phi=0.5, seed=123, jitter=0.1, min_dist=1.9, vel_sigma=0.01):
    """Jittered FCC packing at volume fraction phi of unit-radius cells: a
    k x k x k FCC lattice (4 k^3 >= n sites) in a cube of side
    L = (n (4/3) pi / phi)^(1/3), random deletion down to n sites, uniform
    jitter in [-jitter, jitter]^3 rejected if it brings two centres closer than
    min_dist.  Velocities N(0, vel_sigma^2) per node component."""
    rng = np.random.default_rng(seed)
    L = (n_cells * (4.0 / 3.0) * math.pi / phi) ** (1.0 / 3.0)
    k = int(math.ceil((n_cells / 4.0) ** (1.0 / 3.0)))
    a = L / k
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"), -1).reshape(-1, 3)
    sites = ((g[:, None, :] + basis[None, :, :]).reshape(-1, 3) + 0.25) * a
    keep = np.sort(rng.choice(len(sites), size=n_cells, replace=False))
    c = sites[keep].copy()
    # jitter every centre, then undo the jitter of any centre that ends up
    # closer than min_dist to another (repeat until none is left)
    from scipy.spatial import cKDTree
    trial = c + rng.uniform(-jitter, jitter, c.shape)
    for _ in range(50):
        pairs = cKDTree(trial).query_pairs(min_dist, output_type="ndarray")
        if len(pairs) == 0:
            break
        bad = np.unique(pairs.reshape(-1))
        trial[bad] = c[bad]
    c = trial
    vel = [rng.normal(0.0, vel_sigma, (n_cells, 192)).astype(np.float32) for _ in range(3)]
    for v in vel:
        v[:, 180:] = 0
    return c.astype(np.float32), [v.reshape(-1) for v in vel], L


def config3(n_cells=100_000, seed=123):
    """100k non-dividing cells, FCC packing at phi = 0.5, pressure fixed at
    200, Gaussian node velocities sigma 0.01, 5000 steps."""
    c, vel, L = packed_fcc(n_cells, phi=0.5, seed=seed)
    p = base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                    div_time_steps=5000, rng_ij=seed, rng_kl=100 * seed)
    return p, state(c, velocities=vel), 5000


# ---------------------------------------------------------------- configs 4/5
def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x, z ^ (z >> 31)


class SplitMix:
    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def uniform(self):
        self.s, z = splitmix64(self.s)
        return (z >> 11) * (1.0 / 9007199254740992.0)


def random_centres(n, box, rng, min_dist=1.9, margin=1.05):
    """Random sequential insertion in [margin, box - margin]^3."""
    out = []
    cellsz = min_dist
    nb = max(1, int(box / cellsz))
    grid = {}
    tries = 0
    while len(out) < n:
        tries += 1
        if tries > 2_000_000:
            raise RuntimeError("random insertion did not converge")
        p = np.array([margin + rng.uniform() * (box - 2 * margin) for _ in range(3)])
        k = tuple(np.clip((p / (box / nb)).astype(int), 0, nb - 1))
        bad = False
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                        if np.sum((out[q] - p) ** 2) < min_dist * min_dist:
                            bad = True
        if not bad:
            grid.setdefault(k, []).append(len(out))
            out.append(p)
    return np.array(out, dtype=np.float32)


def soft_params(p, soft_factor=0.8, **over):
    """`p` with variable stiffness on: stiffness2 = fl(softStiffFactor x
    Youngs_mod), as the reference computes it (src/GPUbounce.cu:2048)."""
    q = dict(p, use_different_stiffnesses=1, soft_stiff_factor=soft_factor,
             stiffness2=float(np.float32(soft_factor) * np.float32(p["youngs_mod"])))
    q.update(over)
    return q


def config4(n_inst=256, master_seed=2024):
    """256 instances: N0 = round(exp(U[0, ln 512])) >= 1 cells, growth rate
    U[0.001, 0.004], division volume U[2.6, 3.2], box 30, seed i."""
    sm = SplitMix(master_seed)
    inst = []
    for i in range(n_inst):
        n0 = max(1, int(round(math.exp(sm.uniform() * math.log(512)))))
        gr = 0.001 + 0.003 * sm.uniform()
        dv = 2.6 + 0.6 * sm.uniform()
        c = random_centres(n0, 30.0, sm)
        ij, kl = seed_pair(i)
        p = base_params(box_len=(30.0, 30.0, 30.0), growth_rate=gr, division_vol=dv,
                        div_time_steps=10 ** 9, rng_ij=ij, rng_kl=kl)
        inst.append((p, state(c)))
    return inst


def rsa_centres(n, box, rng, min_dist=1.9, margin=1.05):
    """Random sequential insertion in [margin, box - margin]^3, vectorised:
    candidates come in batches from the numpy generator `rng`; a candidate is
    kept if no earlier kept centre (earlier batches, then earlier candidates
    of its own batch, in order) lies within min_dist, which is sequential
    insertion of the same candidate stream."""
    from scipy.spatial import cKDTree
    pts = np.empty((0, 3))
    tries = 0
    while len(pts) < n:
        m = max(4096, 8 * (n - len(pts)))
        cand = margin + rng.random((m, 3)) * (box - 2 * margin)
        tries += m
        if tries > 50_000_000:
            raise RuntimeError("random insertion did not converge")
        if len(pts):
            d, _ = cKDTree(pts).query(cand, k=1, distance_upper_bound=min_dist)
            cand = cand[~(d < min_dist)]
        if len(cand) == 0:
            continue
        earlier = [[] for _ in range(len(cand))]
        for i, j in cKDTree(cand).query_pairs(min_dist, output_type="ndarray"):
            earlier[max(i, j)].append(min(i, j))
        keep = np.zeros(len(cand), bool)
        need, taken = n - len(pts), 0
        for i in range(len(cand)):
            if not any(keep[j] for j in earlier[i]):
                keep[i] = True
                taken += 1
                if taken == need:
                    break
        pts = np.concatenate([pts, cand[keep]])
    return pts.astype(np.float32)


def config5_sizes(n_inst=64, master_seed=2025):
    """The initial cell counts of config5's instances (no placement)."""
    sm = SplitMix(master_seed)
    out = []
    for _ in range(n_inst):
        out.append(256 + int(sm.uniform() * (8192 - 256 + 1)))
        sm.uniform()
    return out


def config5(n_inst=64, master_seed=2025, only=None):
    """64 instances: N0 ~ U{256..8192}, random centres at packing 0.4 of the
    region the centres occupy (box side (N0 (4/3) pi / 0.4)^(1/3) + 2 x 1.05,
    centres at least 1.05 from each wall and 1.9 apart), bond stiffness
    U[500, 2000] (stiffFactor1 = k/1000), dividing, seeds 1000..1063.
    only: the instance indices to generate (default all), in index order;
    each is identical to its instance in the full ensemble."""
    sm = SplitMix(master_seed)
    inst = []
    for i in range(n_inst):
        n0 = 256 + int(sm.uniform() * (8192 - 256 + 1))
        k = 500 + 1500 * sm.uniform()
        if only is not None and i not in only:
            continue
        box = (n0 * (4.0 / 3.0) * math.pi / 0.4) ** (1.0 / 3.0) + 2 * 1.05
        c = rsa_centres(n0, box, np.random.default_rng([master_seed, i]))
        ij, kl = seed_pair(1000 + i)
        p = base_params(box_len=(box, box, box), stiffness1=float(np.float32(k)),
                        div_time_steps=10 ** 9, rng_ij=ij, rng_kl=kl)
        inst.append((p, state(c)))
    return inst


def inp_json(p, max_cells, steps, traj_write_int, traj_file="traj.bin", seed=42, binary=True, non_div_steps=0):
    """The reference's inp.json (src/GPUbounce.cu:1938-2096 keys) for the
    hot-path parameters `p` (base_params layout); features off the path are
    switched off.  youngs_mod is the contact modulus, stiffness1 the bond
    stiffness (stiffFactor1 = stiffness1 / youngs_mod)."""
    return {
        "core": {"MaxNoofC180s": int(max_cells), "particle_mass": p["particle_mass"],
                 "repulsion_range": p["repulsion_range"], "attraction_range": p["attraction_range"],
                 "repulsion_strength": p["repulsion_strength"], "attraction_strength": p["attraction_strength"],
                 "Youngs_mod": p["youngs_mod"], "stiffFactor1": p["stiffness1"] / p["youngs_mod"],
                 "viscotic_damping": p["viscotic_damping"], "internal_damping": p["internal_damping"],
                 "gamma_visc": p["gamma_visc"], "division_Vol": p["division_vol"], "random_z_offset?": 0,
                 "z_offset": 0.0, "div_time_steps": int(steps), "time_interval": p["time_interval"],
                 "Restart": 0, "trajWriteInt": int(traj_write_int), "non_div_time_steps": int(non_div_steps),
                 "trajFileName": traj_file, "binaryOutput": 1 if binary else 0,
                 "maxPressure": p["max_pressure"], "minPressure": p["min_pressure"],
                 "growth_rate": p["growth_rate"], "checkSphericity": bool(p["check_sphericity"]),
                 "constrainAngles": bool(p["constrain_angles"]), "doAdaptive_dt": False, "dt_max": 1e-4,
                 "dt_tol": 1e-8, "phase_count": int(p.get("phase_count", 2000000000)),
                 "write_cont_force": bool(p.get("write_cont_force", False)),
                 "forces_file": "forces.csv", "correct_com": False},
        "counting": {"mit-index_file_name": "mit-index.dat",
                     "count_only_internal_cells?": bool(p.get("count_internal_radius", 0.0) > 0),
                     "radius_cutoff": float(p.get("count_internal_radius", 0.0)) or 0.6,
                     "overwrite_mit_ind_file?": True,
                     "cell_count_int": max(1, min(1000, int(steps)))},
        "population": {"doPopModel": 0, "totalFood": 5000.0, "regular_consumption": 2.0,
                       "division_consumption": 10.0, "death_release_food": 10.0, "cellLifeTime": 20000,
                       "max_pop": 1024},
        "walls": {"useWalls": 0, "perpAxis": "Z", "dAxis": 1.0, "wallLen": 10.0, "wallWidth": 10.0,
                  "threshDist": p["thresh_dist"]},
        "divParams": {"useDivPlaneBasis": 0, "divPlaneBasisX": 0.0, "divPlaneBasisY": 1.0, "divPlaneBasisZ": 0.0},
        "stiffnessParams": {"useDifferentStiffnesses": bool(p.get("use_different_stiffnesses", 0)),
                            "softStiffFactor": float(p.get("soft_stiff_factor", 1.0)),
                            "numberOfSofterCells": int(p.get("number_of_softer_cells", 0)),
                            "duringGrowth": not p.get("soften_after_growth", 0),
                            "closenessToCenter": float(p.get("closeness_to_center", 0.0)), "startAtPop": 0,
                            "fractionOfSofterCells": float(p.get("fraction_of_softer_cells", 0.0)),
                            "chooseRandomCellIndices": bool(p.get("choose_random_cell_indices", 0)),
                            "daughtSameStiffness": bool(p["daught_same_stiffness"]), "recalc_r0": False},
        "boxParams": {"useRigidSimulationBox": bool(p["use_rigid_box"]), "usePBCs": False,
                      "boxLength": float(p["box_len"][0]), "box_len_x": float(p["box_len"][0]),
                      "box_len_y": float(p["box_len"][1]), "box_len_z": float(p["box_len"][2]),
                      "flatbox": False, "rand_pos": False},
        "rand_params": {"add_rands": False, "rand_seed": int(seed), "rand_dist": 0, "rand_scale_factor": 0.1},
    }


def write_init_file(path, st):
    """The CS3D_INIT_FILE format of the cs3d driver: "CS3DINIT", int32 n,
    float32 X, Y, Z, VX, VY, VZ [n*192], pressure [n], youngs [n]."""
    n = int(st["n"])
    k = n * 192
    zeros = np.zeros(k, np.float32)
    with open(path, "wb") as f:
        f.write(b"CS3DINIT")
        f.write(np.int32(n).tobytes())
        for key in ("X", "Y", "Z", "VX", "VY", "VZ"):
            a = st.get(key)
            f.write((np.asarray(a, np.float32)[:k] if a is not None else zeros).tobytes())
        f.write(np.asarray(st.get("pressure", np.full(n, 0.0)), np.float32)[:n].tobytes())
        f.write(np.asarray(st.get("youngs", np.full(n, 0.0)), np.float32)[:n].tobytes())
