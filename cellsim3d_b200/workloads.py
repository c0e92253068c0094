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


def config5(n_inst=64, master_seed=2025):
    """64 instances: N0 ~ U{256..8192}, random centres at packing 0.4, bond
    stiffness U[500, 2000] (stiffFactor1 = k/1000), seeds 1000..1063."""
    sm = SplitMix(master_seed)
    inst = []
    for i in range(n_inst):
        n0 = 256 + int(sm.uniform() * (8192 - 256 + 1))
        k = 500 + 1500 * sm.uniform()
        box = (n0 * (4.0 / 3.0) * math.pi / 0.4) ** (1.0 / 3.0)
        c = random_centres(n0, box, sm)
        ij, kl = seed_pair(1000 + i)
        p = base_params(box_len=(box, box, box), stiffness1=float(np.float32(k)),
                        div_time_steps=10 ** 9, rng_ij=ij, rng_kl=kl)
        inst.append((p, state(c)))
    return inst
