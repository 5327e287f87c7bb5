"""The split form's rewritten arithmetic, checked on the CPU against the oracle.

The split-precision RHS (FP32 WENO on deviations) evaluates WENO5 point values in
the candidate-quadratic form: on the cell xi in [-1/2, 1/2] the quadratic of
candidate stencil k is q0 +- hx r_k + tau s_k (+ for k = 1) with hx = xi/2 and
tau = (xi^2 - 1/12)/2, where r_k and s_k are the same slope and second-difference
terms the Jiang-Shu smoothness indicators square.  The kernel reads hx and tau of each Gauss
node off the reference's tabulated candidate-2 coefficients (reconstruction.f90:
999-1136).  These tests pin that rewrite in FP64 against the oracle's literal
restatement of the reference, and the exactness argument of the positivity
limiter's shortcut (theta = 1 without dividing when |a| >= |m|).
"""
import numpy as np
import pytest

import oracle as O

# candidate-2 coefficients (of qm1 and qp1) of the four second-sweep Gauss nodes,
# reconstruction.f90:999-1136 (the kernel's gp_hx / gp_tau arguments)
C2 = [(0.2663118796250726, -0.1642562761719537), (0.0577769829791784, -0.1122135388132497),
      (-0.1122135388132497, 0.0577769829791784), (-0.1642562761719537, 0.2663118796250726)]
# linear weights of the four nodes (same source)
G2 = [(0.2658420974778319, 0.6112504900322486, 0.1229074124899195),
      (0.1281641584355059, 0.5219691498503563, 0.3498666917141379),
      (0.3498666917141379, 0.5219691498503563, 0.1281641584355059),
      (0.1229074124899195, 0.6112504900322486, 0.2658420974778319)]
EPS = 1e-24  # the reference's WENO epsilon (FP64)


def candidate_parts(q):
    qm2, qm1, q0, qp1, qp2 = q
    s = np.array([qm2 - 2 * qm1 + q0, qm1 - 2 * q0 + qp1, q0 - 2 * qp1 + qp2])
    r = np.array([qm2 - 4 * qm1 + 3 * q0, qm1 - qp1, 3 * q0 - 4 * qp1 + qp2])
    return s, r


def weno_point_quadratic(q, g, hx, tau):
    """sum_k omega_k p_k(xi) = q0 + sum_k g_k i_k (+-hx r_k + tau s_k) / sum_k g_k i_k."""
    s, r = candidate_parts(q)
    i = 1.0 / (EPS + 13.0 / 12.0 * s * s + 0.25 * r * r) ** 2
    sgn = np.array([1.0, -1.0, -1.0])
    a = np.asarray(g) * i
    return q[2] + (a * (sgn * hx * r + tau * s)).sum() / a.sum()


def test_node_parameters_from_the_table():
    # hx = (c_qp1 - c_qm1)/2 and tau = (c_qm1 + c_qp1)/2 are xi/2 and (xi^2 - 1/12)/2
    qn, _ = O.quadrature()
    for g, (cm1, cp1) in enumerate(C2):
        hx, tau = 0.5 * (cp1 - cm1), 0.5 * (cm1 + cp1)
        assert abs(hx - qn[g] / 2) < 1e-15
        assert abs(tau - (qn[g] ** 2 - 1.0 / 12.0) / 2) < 1e-15


def test_candidate_rows_reproduce_the_table():
    # every tabulated candidate row of the four nodes (coefficients of qm2..qp2)
    qn, _ = O.quadrature()
    for g in range(4):
        hx, tau = qn[g] / 2, (qn[g] ** 2 - 1.0 / 12.0) / 2
        # p_1 = q0 + hx (qm2 - 4qm1 + 3q0) + tau (qm2 - 2qm1 + q0)
        row1 = [hx + tau, -4 * hx - 2 * tau, 1 + 3 * hx + tau]
        # p_2 = q0 - hx (qm1 - qp1) + tau (qm1 - 2q0 + qp1)
        row2 = [-hx + tau, 1 - 2 * tau, hx + tau]
        assert abs(row2[0] - C2[g][0]) < 1e-15 and abs(row2[2] - C2[g][1]) < 1e-15
        # p_1 and p_3 of node g are mirror images of node 3-g
        row3 = [1 - 3 * hx + tau, 4 * hx - 2 * tau, -hx + tau]
        m = 3 - g
        hxm, taum = qn[m] / 2, (qn[m] ** 2 - 1.0 / 12.0) / 2
        assert np.allclose(row1[::-1], [1 - 3 * hxm + taum, 4 * hxm - 2 * taum, -hxm + taum],
                           rtol=0, atol=1e-15)
        assert np.allclose(row3[::-1], [hxm + taum, -4 * hxm - 2 * taum, 1 + 3 * hxm + taum],
                           rtol=0, atol=1e-15)


# Deviations of O(scale) around zero, as the split form reconstructs them: the
# reference's expanded smoothness indicators then lose nothing to cancellation, so
# both forms agree to rounding.  (Around an O(1) value the expanded form's
# cancellation alone moves the weights; the sum-of-squares form is the accurate one.)
@pytest.mark.parametrize("scale", [1.0, 1e-3, 1e-7])
def test_second_sweep_quadratic_form_matches_oracle(scale):
    rng = np.random.default_rng(11)
    for _ in range(300):
        q = scale * rng.standard_normal(5)
        ref = O.weno5_second(q)
        got = [weno_point_quadratic(q, G2[g], 0.5 * (C2[g][1] - C2[g][0]),
                                    0.5 * (C2[g][0] + C2[g][1])) for g in range(4)]
        assert np.allclose(got, ref, rtol=0, atol=1e-13 * scale)


def test_first_sweep_quadratic_form_matches_oracle():
    # faces xi = -1/2 (hx = -1/4, tau = 1/12, gamma = 3/10, 3/5, 1/10) and xi = +1/2
    rng = np.random.default_rng(12)
    for _ in range(300):
        q = rng.standard_normal(5)  # O(1) deviations around zero
        wm, wp = O.weno5_first(q)
        gm = weno_point_quadratic(q, (0.3, 0.6, 0.1), -0.25, 1.0 / 12.0)
        gp = weno_point_quadratic(q, (0.1, 0.6, 0.3), 0.25, 1.0 / 12.0)
        assert abs(gm - wm) <= 1e-13 * max(1.0, abs(wm))
        assert abs(gp - wp) <= 1e-13 * max(1.0, abs(wp))


def test_limiter_shortcut_is_exact():
    # theta = min(1, |a/m|) (finitevolume.f90:671-691) equals 1 whenever |a| >= |m|:
    # the quotient is >= 1 and rounding keeps it there, so the division is skipped
    rng = np.random.default_rng(13)
    a = np.abs(rng.standard_normal(200000)) * 10.0 ** rng.integers(-12, 3, 200000)
    m = rng.standard_normal(200000) * 10.0 ** rng.integers(-12, 3, 200000)
    a = np.concatenate([a, [1.0, 2.5e-7, 0.0, 3.0]])
    m = np.concatenate([m, [-1.0, -2.5e-7, -1e-300, 3.0]])
    with np.errstate(divide="ignore", invalid="ignore"):
        full = np.minimum(1.0, np.abs(a / m))
    short = np.where(np.abs(a) >= np.abs(m), 1.0, full)
    assert np.array_equal(full, short)
