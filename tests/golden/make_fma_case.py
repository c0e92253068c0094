"""Generate tests/golden/fma_boundary_case.npz: two cells with exactly one
node pair whose dissipative cut-off decision depends on how the squared
distance is rounded.  For that pair the uncontracted float expression
(dx*dx + dy*dy) + dz*dz lies at or below the cut-off ra^2 and the contracted
fma(dz, dz, fma(dx, dx, dy*dy)) above it; every other pair is at least 1e-5
away from the cut-off.  The partner node moves, every other node rests, so
the dissipative force of the first node is the friction of that one pair if
the pair is kept and zero if it is not.

    python tests/golden/make_fma_case.py

Deterministic (seeded); writes the positions and velocities of both cells
(192-stride), the pair and both squared distances.  Needs only numpy and the
mesh fixture c180_mesh.npz."""
import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from cellsim3d_b200 import workloads as W  # noqa: E402

f32 = np.float32
RA = f32(0.3)
RA2 = f32(RA * RA)


def fma32(a, b, c):
    """fmaf: a*b + c exactly, rounded once to float."""
    return f32(float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))))


def r2_plain(dx, dy, dz):
    return f32(f32(f32(dx * dx) + f32(dy * dy)) + f32(dz * dz))


def r2_fma(dx, dy, dz):
    return fma32(dz, dz, fma32(dx, dx, f32(dy * dy)))


def main():
    mesh = W.load_mesh()
    xyz = W.centred(W.scaled_xyz(mesh))

    def place(c):
        return (xyz + np.asarray(c, f32)[None, :]).astype(f32)

    rng = np.random.default_rng(5)
    cA = np.array([12.0, 12.0, 12.0], f32)
    A = place(cA)
    for _ in range(400):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        lo, hi = 1.5, 3.0
        for _ in range(60):
            t = 0.5 * (lo + hi)
            d = np.sqrt(((A[:, None, :].astype(np.float64) - place(cA + t * u)[None, :, :]) ** 2).sum(-1))
            if d.min() < 0.3:
                lo = t
            else:
                hi = t
        cB0 = (cA + 0.5 * (lo + hi) * u).astype(f32)
        d = np.sqrt(((A[:, None, :].astype(np.float64) - place(cB0)[None, :, :]) ** 2).sum(-1))
        srt = np.sort(d.ravel())
        if srt[1] - srt[0] < 2e-3:
            continue
        i, j = np.unravel_index(np.argmin(d), d.shape)
        hit = None
        for k in range(-4000, 4001):
            c = cB0.copy()
            c[0] = f32(cB0[0] + f32(k) * f32(2 ** -20))
            B = place(c)
            dx, dy, dz = (f32(A[i, q] - B[j, q]) for q in range(3))
            p, m = r2_plain(dx, dy, dz), r2_fma(dx, dy, dz)
            if (p > RA2) != (m > RA2):
                hit = (B, p, m)
                break
        if hit is None:
            continue
        B, p, m = hit
        dd = A[:, None, :] - B[None, :, :]
        r2 = ((dd.astype(np.float64)) ** 2).sum(-1)
        r2[i, j] = np.inf
        if np.min(np.abs(r2 - float(RA2))) < 1e-5:
            continue
        X, Y, Z = (np.zeros((2, 192), f32) for _ in range(3))
        V = [np.zeros((2, 192), f32) for _ in range(3)]
        for q, arr in enumerate((X, Y, Z)):
            arr[0, :180] = A[:, q]
            arr[1, :180] = B[:, q]
        ax = np.array([A[i, q] - B[j, q] for q in range(3)], np.float64)
        ax /= np.linalg.norm(ax)
        v = np.cross(ax, [1.0, 0.0, 0.0])
        v /= np.linalg.norm(v)
        for q in range(3):
            V[q][1, j] = f32(v[q])
        np.savez(os.path.join(HERE, "fma_boundary_case.npz"), X=X.ravel(), Y=Y.ravel(), Z=Z.ravel(),
                 VX=V[0].ravel(), VY=V[1].ravel(), VZ=V[2].ravel(), i=int(i), j=int(j), r2_plain=p, r2_fma=m,
                 ra2=RA2)
        print("pair (0, %d, 1, %d): uncontracted r2 %.9g, contracted %.9g, ra^2 %.9g" % (i, j, p, m, RA2))
        return
    raise SystemExit("no case found")


if __name__ == "__main__":
    main()
