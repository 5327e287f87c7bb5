"""The Jacobi stop rule's decision: the reference against the GPU's exact residual.

The reference continues while tolerance < SUM(ABS(sol - solp)) / n
(jacobi_iteration.f90:69,72,77), a sequentially rounded FP64 sum divided by n.  The
GPU solvers sum every |dx| exactly (each truncated to a multiple of 2^-100 and
carried in integer limbs, so the sum does not depend on tiling or atomic order) and
stop when that sum <= the limbs of fl(tol * n).  The two decisions agree except when
the exact sum lies within the rounding error of the reference's sum (and of the
division and the product) of the threshold; there the stop index can differ by one
sweep.  This test states that margin and checks the decisions agree outside it.
"""
import math

import numpy as np

TOL = 1e-16


def reference_continues(vals):
    """jacobi_iteration.f90: residual = SUM(ABS(...))/n, continue while tol < residual
    (the sum rounded term by term, left to right)."""
    s = 0.0
    for v in vals:
        s += v
    return TOL < s / len(vals)


def gpu_continues(vals):
    """The exact rule: sum of floor(|dx| * 2^100) against floor(fl(tol * n) * 2^100)."""
    total = sum(int(math.ldexp(v, 100)) for v in vals)
    thresh = int(math.ldexp(TOL * len(vals), 100))
    return not total <= thresh


def margin(vals):
    """Bound on |rounded sum / n - exact sum / n| relative to tol: (n - 1) u for the
    sequential sum plus u for the division and u for fl(tol * n), u = 2^-53, plus the
    2^-100 truncation of every term."""
    n = len(vals)
    u = 2.0 ** -53
    s = math.fsum(vals)
    return (n + 1) * u * s + u * TOL * n + n * 2.0 ** -100


def test_decisions_agree_outside_the_rounding_margin():
    rng = np.random.default_rng(3)
    disagreements, checked = 0, 0
    for trial in range(400):
        n = int(rng.integers(2, 3000))
        # |dx| spread over three decades around the threshold, then scaled so that the
        # exact mean lands within a few margins of tol (both sides)
        v = 10.0 ** rng.uniform(-18, -15, n)
        target = TOL * n * (1.0 + rng.uniform(-1, 1) * 4 * n * 2.0 ** -53)
        v = v * (target / math.fsum(v))
        vals = [float(x) for x in v]
        ref, gpu = reference_continues(vals), gpu_continues(vals)
        exact = math.fsum(vals)
        if ref != gpu:
            disagreements += 1
            assert abs(exact - TOL * n) <= margin(vals), (n, exact, TOL * n)
        elif abs(exact - TOL * n) > margin(vals):
            checked += 1
    assert checked > 100  # plenty of cases outside the margin, all agreeing
    # inside the margin the two rules do split: the stop index may differ by one sweep
    assert disagreements >= 1
