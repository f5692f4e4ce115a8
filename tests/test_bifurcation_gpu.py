"""GPU tests of the bifurcation drivers: LinearEvolve about a frozen state
(StateVector.cpp:107-156), InverseIteration (InverseIteration.cpp),
FindCriticalPoint (FindCriticalPoint.cpp) and FindHopf (FindHopf.cpp).

Checks:
  * linear_evolve equals the solver's own TimeStepLinear about the same
    frozen base (SetBase + TimeStepLinear) to 1e-6: the two paths differ only
    in how the base reaches the device;
  * the drivers' residual functions equal their definitions assembled from
    evolve / linear_evolve and FP64 inner products on the host, to 1e-5
    relative (FP32 state, one subtraction);
  * the constraints leave what the reference's leave: v orthogonal to ddx x,
    the means of v's u1 and b zero, Energy(v) = weight; v1.A = 1, v2.A = 0
    with (v1, v2) still in the plane of the input pair (to 1e-5);
  * inverse iteration about the laminar shear layer, shifted next to the
    Kelvin-Helmholtz growth factor that the Arnoldi driver finds, converges
    to that mode: its eigenvalue estimate matches to 1e-3 and the residual
    |L b - mu b| (|b| = 1) falls below 1e-2 mu (each solve stops at a 5%
    GMRES residual, as the reference's);
  * a Newton-Krylov step of FindCriticalPoint from the laminar state and
    the Kelvin-Helmholtz mode lowers the residual.
"""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, rel_l2
from tests.test_gpu_parity import gpu_solver
from tests.test_vecs_drivers_gpu import _enforce_bcs, _flow

pytestmark = pytest.mark.gpu

CFG = CONFIGS["kh2d"]


def _kept(cfg, seed, amp):
    s = gpu_solver(cfg)
    s.set_state(0, make_ic(cfg, seed=seed, amp=amp))
    s.Prepare()
    s.synchronize()
    return _enforce_bcs(s.get_state_kept()[0])


def _dot(flow, a, b, Ri):
    from stratiflow_b200 import drivers as D
    return D.ext_dot(flow, (a, 0.0), (b, 0.0), Ri)


def _ddx(flow, a):
    K1 = flow.N1 // 3
    K2 = 2 * (flow.N2 // 3) - 1 if flow.N2 > 1 else 1
    m = np.arange(flow.plane)
    kx = np.where(m < K1 * K2, 2 * np.pi * (m % K1) / flow.L1, 0.0)
    out = a.astype(np.complex128) * (1j * kx)[None, None, :]
    out[4] = 0
    return out


def test_linear_evolve_matches_solver_linear_step():
    from stratiflow_b200 import drivers as D
    flow = _flow(CFG)
    base = make_ic(CFG, seed=11, amp=5e-2)
    pert = make_ic(CFG, seed=12, amp=1e-3)
    s = gpu_solver(CFG)
    s.set_state(0, base)
    about = s.get_state_kept()[0]
    s.set_state(0, pert)
    s.Prepare()
    d = s.get_state_kept()[0].copy()
    d[4] = 0
    T, n = 0.3, 30
    got = D.linear_evolve(flow, about, d, T)
    s.SetBase(0, base["u1"], base["u2"], base["u3"], base["b"])
    s.set_state_kept(d[None])
    s.Prepare()
    s.TimeStepLinear(n)
    s.synchronize()
    want = _enforce_bcs(s.get_state_kept()[0])
    assert rel_l2(got[:4], want[:4]) < 1e-6


def test_critical_point_function_matches_its_definition():
    from stratiflow_b200 import drivers as D
    flow = _flow(CFG)
    x = _kept(CFG, 21, 5e-2)
    v = _kept(CFG, 22, 1e-2)
    Ri, T, w = 0.11, 0.5, 0.7
    Fx, Fv, Fp = D.critical_point_function(flow, x, v, Ri, T=T, weight=w)
    ex = D.evolve(flow, x, T, Ri)[0].astype(np.complex128) - x
    ev = D.linear_evolve(flow, x, v, T, Ri).astype(np.complex128) - v
    assert rel_l2(Fx[:4], ex[:4]) < 1e-5
    assert rel_l2(Fv[:4], ev[:4]) < 1e-5
    want_p = 0.5 * _dot(flow, v, v, Ri) - w
    assert abs(Fp - want_p) <= 1e-6 * (abs(want_p) + w)


def test_critical_point_constraints():
    from stratiflow_b200 import drivers as D
    from stratiflow_b200.grid import vertical_points
    flow = _flow(CFG)
    x = _kept(CFG, 31, 5e-2)
    v = _kept(CFG, 32, 1e-2)
    Ri, w = 0.12, 0.4
    x2, v2, ri2 = D.critical_point_constraints(flow, x, v, Ri, weight=w)
    assert ri2 == Ri
    assert np.array_equal(x2[:4], x[:4])
    ps = _ddx(flow, x2)
    assert abs(_dot(flow, v2, ps, Ri)) <= 1e-5 * np.sqrt(_dot(flow, v2, v2, Ri) * _dot(flow, ps, ps, Ri))
    # the (0,0) columns of u1 and b: RemoveAverage (Integration.h:72-75) of the
    # input's (ddx x has no (0,0) part and the projection leaves these columns
    # alone), times the one factor of Rescale
    z = vertical_points(flow.L3, flow.N3)
    scale = []
    for f in (0, 3):
        col = v[f, :, 0].real.astype(np.float64)
        integ = np.sum((z[2:flow.N3] - z[1:flow.N3 - 1]) * col[1:flow.N3 - 1])
        after = col - integ / flow.L3 / 2
        got = v2[f, :, 0].real.astype(np.float64)
        if not after.any():   # a field the input leaves at zero stays zero
            assert not got.any(), f
            continue
        s = got @ after / (after @ after)
        assert np.linalg.norm(got - s * after) <= 1e-5 * np.linalg.norm(got), f
        scale.append(s)
    assert scale and max(scale) - min(scale) <= 1e-5 * abs(scale[0])
    assert abs(0.5 * _dot(flow, v2, v2, Ri) - w) <= 1e-5 * w


def test_hopf_constraints_and_function():
    from stratiflow_b200 import drivers as D
    flow = _flow(CFG)
    x = _kept(CFG, 41, 5e-2)
    v1 = _kept(CFG, 42, 1e-2)
    v2 = _kept(CFG, 43, 1e-2)
    Ri, theta, T = 0.1, 0.3, 0.5
    n1 = np.sqrt(_dot(flow, v1, v1, Ri))
    A = v1 / n1
    _, c1, c2, ri, th = D.hopf_constraints(flow, x, v1, v2, Ri, theta)
    assert ri == Ri and th == theta
    assert abs(_dot(flow, c1, A, Ri) - 1.0) < 1e-5
    assert abs(_dot(flow, c2, A, Ri)) < 1e-5 * np.sqrt(_dot(flow, c2, c2, Ri) * _dot(flow, A, A, Ri))
    # (c1, c2) in the plane of (v1, v2)
    B = np.stack([v1[:4].ravel(), v2[:4].ravel()], axis=1).astype(np.complex128)
    for c in (c1, c2):
        coef, *_ = np.linalg.lstsq(B, c[:4].ravel().astype(np.complex128), rcond=None)
        assert rel_l2(B @ coef, c[:4].ravel()) < 1e-5
    # the residual function, on the input rescaled by |v1| as FindHopf's main does
    Fx, F1, F2, Fp, Ft = D.hopf_function(flow, x, v1, v2, Ri, theta, T=T)
    w1, w2 = v1 / n1, v2 / n1
    L1 = D.linear_evolve(flow, x, w1, T, Ri).astype(np.complex128)
    L2 = D.linear_evolve(flow, x, w2, T, Ri).astype(np.complex128)
    e1 = L1 - np.cos(theta) * w1 + np.sin(theta) * w2
    e2 = L2 - np.sin(theta) * w1 - np.cos(theta) * w2
    ex = D.evolve(flow, x, T, Ri)[0].astype(np.complex128) - x
    assert rel_l2(Fx[:4], ex[:4]) < 1e-5
    assert rel_l2(F1[:4], e1[:4]) < 1e-5
    assert rel_l2(F2[:4], e2[:4]) < 1e-5
    assert abs(Ft) < 1e-5   # v1.A - 1 with A = v1
    assert abs(Fp - _dot(flow, w2, w1, Ri)) < 1e-5


T_KH = 4.0


def _kh_mode(flow):
    from stratiflow_b200 import drivers as D
    zero = np.zeros(flow.state_shape, dtype=np.complex64)
    ev, vr, vi, _ = D.arnoldi(flow, zero, T=T_KH, block=8, krylov=96, tol=1e-8, nev=2, vectors=True)
    return zero, ev, vr


def test_inverse_iteration_finds_the_kh_mode():
    from stratiflow_b200 import drivers as D
    flow = _flow(CFG)
    zero, ev, _ = _kh_mode(flow)
    lam = ev[0]
    # the growing, stationary KH mode (a double real eigenvalue in the real
    # space, split by rounding into a pair 1e-5 apart)
    assert abs(lam.imag) < 1e-3 * abs(lam) and lam.real > 1.0
    b0 = _kept(CFG, 51, 1e-3)
    b, hist = D.inverse_iteration(flow, zero, b0, T=T_KH, mu=1.01 * lam.real, eps=0.05, iters=3, krylov=256)
    assert abs(hist["eigenvalue"][-1] - lam.real) < 1e-3 * lam.real, hist
    assert hist["residual"][-1] < 1e-2 * lam.real, hist
    assert hist["residual"][-1] < hist["residual"][0]


def test_critical_point_newton_lowers_the_residual():
    from stratiflow_b200 import drivers as D
    flow = _flow(CFG)
    zero, ev, vr = _kh_mode(flow)
    opts = D.NKOptions(max_newton=2, krylov=30, gmres_tol=1e-2, jacobian="fd", block=0)
    x, v, Ri, st = D.find_critical_point(flow, zero, vr, CFG["Ri"], T=T_KH, weight=1e-4, opts=opts)
    assert st["newton_iterations"] >= 1
    assert st["residuals"][-1] < st["residuals"][0], st
    assert np.isfinite(Ri)
