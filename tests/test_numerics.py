"""The arithmetic identities the kernels rely on, checked on the CPU in exact
rational arithmetic (fractions.Fraction; a conversion to float rounds to
nearest, so RN(x) = float(Fraction) and a fused multiply-add is one rounding
of the exact value).

* The integrator's divisions by the mass (src/propagate.cu:681-736, double
  `0.5 * dt * F / m`): the kernels multiply by the correctly rounded
  reciprocal and correct once with the exact remainder,
  q' = fma(fma(-q, m, a), 1/m, q) with q = RN(a * (1/m)) (cs3d_kernels.cuh,
  div_m).  By Markstein's theorem q' is the correctly rounded quotient; the
  test compares it with RN(a / m) on samples of the integrator's shapes.
* The FP64 reciprocal and reciprocal square root: a seed from the hardware's
  approximate instructions (relative error below 1e-6, measured on a B200)
  refined by one Newton step, y (1.5 - 0.5 x y^2) and r (2 - x r)
  (rsqrt_nr, rcp_nr).  The test refines seeds carrying errors of up to 1e-6
  with the same operations, each rounded (the compiler may fuse a multiply
  and an add, which only drops a rounding), and bounds the result's relative
  error by 2e-12, six orders of magnitude inside the 1e-5 force bar.
"""
import random
from fractions import Fraction as Fr

import numpy as np

F = np.float64


def rn(x):
    """Round an exact rational to the nearest double."""
    return float(x)


def fma(a, b, c):
    return rn(Fr(a) * Fr(b) + Fr(c))


def test_markstein_division_is_the_correctly_rounded_quotient():
    rng = random.Random(20261204)
    n = 0
    for _ in range(4000):
        # a = 0.5 * dt * F with float dt and F as the kernels form it,
        # m a float mass, 1/m correctly rounded on the host
        dt = float(np.float32(rng.choice([1e-4, 2e-4, 5e-5, rng.uniform(1e-5, 1e-3)])))
        f = float(np.float32(rng.uniform(-1e4, 1e4) * 10.0 ** rng.randint(-6, 0)))
        m = float(np.float32(rng.choice([0.04, 1.0, rng.uniform(1e-3, 10.0)])))
        a = float(F(0.5) * (F(dt) * F(f)))
        inv_m = 1.0 / m                      # IEEE division: correctly rounded
        q = float(F(a) * F(inv_m))
        q2 = fma(fma(-q, m, a), inv_m, q)
        assert q2 == rn(Fr(a) / Fr(m)), (a, m, q, q2)
        n += q != q2
    # the correction is not idle: the plain product is off in some cases
    assert n > 0


def _decimal_rsqrt(x):
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    return Fr(1) / Fr(Decimal(x).sqrt())


def test_one_newton_step_on_1e6_seeds():
    rng = random.Random(7)
    worst_r, worst_c = 0.0, 0.0
    for _ in range(3000):
        x = 10.0 ** rng.uniform(-8, 8)
        eps = rng.choice([1e-6, -1e-6, rng.uniform(-1e-6, 1e-6)])
        # reciprocal square root: y (1.5 - 0.5 x y^2), the kernel's operation order
        t = _decimal_rsqrt(x)
        y = float(t * (1 + Fr(eps)))
        y1 = F(y) * (F(1.5) - F(0.5) * F(x) * F(y) * F(y))
        worst_r = max(worst_r, abs(float((Fr(float(y1)) - t) / t)))
        # reciprocal: r (2 - x r)
        c = Fr(1) / Fr(x)
        r = float(c * (1 + Fr(eps)))
        r1 = F(r) * (F(2.0) - F(x) * F(r))
        worst_c = max(worst_c, abs(float((Fr(float(r1)) - c) / c)))
    assert worst_r < 2e-12, worst_r
    assert worst_c < 2e-12, worst_c
