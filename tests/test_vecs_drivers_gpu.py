"""GPU tests of the device state vectors (sf_vecs_*, the StateVector algebra
of StateVector.h:40-149) and of the host drivers' Jacobian actions.

Bounds: copies are exact; axpy / lincomb / scale agree with numpy on the same
FP32 inputs to 1e-6 relative (one FP32 rounding per element); the FP64 dot
products agree with the FP64 oracle energies and with a numpy FP64
restatement of StateVector::Dot to 1e-7 of |x|^2: the device sums FP64
products but holds the vertical quadrature weights in FP32, as the
reference's FP32 build does.
"""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu


def _solver_with_states(name, n, amp=5e-2):
    cfg = CONFIGS[name]
    s = gpu_solver(cfg, nrun=n)
    for r in range(n):
        s.set_state(r, make_ic(cfg, seed=60 + r, amp=amp))
    s.Prepare()
    s.TimeStep(3)
    s.synchronize()
    return cfg, s


def _flow(cfg):
    from stratiflow_b200 import drivers as D
    return D.Flow(cfg["N1"], cfg["N2"], cfg["N3"], cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Pr"],
                  cfg["Ri"], cfg["dt"], cfg["bg"])


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_vecs_copy_and_algebra(name):
    import stratiflow_b200 as sf
    cfg, s = _solver_with_states(name, 2)
    runs = s.get_state_kept()
    V = sf.Vecs(s, 3)
    V.from_run(0, 0, 2)
    a, b = V.get(0), V.get(1)
    assert np.array_equal(a, runs[0]) and np.array_equal(b, runs[1])
    V.copy(2, V, 0)
    V.axpy(2, 0.5, V, 1)   # MulAdd: u1..b only, p untouched
    c = V.get(2)
    assert rel_l2(c[:4], a[:4] + np.float32(0.5) * b[:4]) < 1e-6
    assert np.array_equal(c[4], a[4])
    V.lincomb(2, 2.0, -1.0, V, 1)
    d = V.get(2)
    assert rel_l2(d, 2 * c - b) < 1e-6
    V.scale(2, 3.0)
    assert rel_l2(V.get(2), 3 * d) < 1e-6
    # to_run writes back exactly
    V.to_run(2, 1)
    assert np.array_equal(s.get_state_kept()[1], V.get(2))


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_vecs_dots_match_fp64(name):
    import stratiflow_b200 as sf
    from stratiflow_b200 import drivers as D
    cfg, s = _solver_with_states(name, 2)
    V = sf.Vecs(s, 2)
    V.from_run(0, 0, 2)
    Ri = cfg["Ri"]
    dd = V.dots(0, 2, V, 0, Ri)
    o = make_oracle(cfg, 64)
    o.set_state(s.get_state(0))
    ke, pe = o.energy()
    # StateVector::Dot = 2 (KE + PE); the oracle sums its quadrature in another order
    assert abs(dd[0] - 2 * (ke + pe)) <= 1e-7 * abs(dd[0])
    flow = _flow(cfg)
    a, b = V.get(0), V.get(1)
    ref01 = D.ext_dot(flow, (a, 0.0), (b, 0.0), Ri)
    assert abs(dd[1] - ref01) <= 1e-7 * abs(dd[0])
    tot = V.dot_sum(0, V, 0, 2, Ri)
    ref = D.ext_dot(flow, (a, 0.0), (a, 0.0), Ri) + D.ext_dot(flow, (b, 0.0), (b, 0.0), Ri)
    assert abs(tot - ref) <= 1e-7 * abs(ref)


def test_phase_shift_and_average_match_reference_formulas():
    """RemovePhaseShift (StateVector.h:103-120): shift = -arg u1(1,0,N3/2) +
    pi/2, every kept mode times exp(i j1 shift); RemoveAverage
    (Integration.h:72-75): the (0,0) stack minus its vertical integral / 2 L3."""
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import vertical_points
    cfg, s = _solver_with_states("shear3d_small", 1)
    V = sf.Vecs(s, 1)
    V.from_run(0, 0)
    a = V.get(0).astype(np.complex128)
    N3, K1 = s.N3, s.K1
    P = s.K1 * s.K2
    shift = V.phase_shift(0)
    want = -np.angle(a[0, N3 // 2, 1]) + np.pi / 2
    assert abs(shift - want) < 1e-6
    j1 = np.arange(s.plane) % K1
    ph = np.where(np.arange(s.plane) < P, np.exp(1j * j1 * want), 1.0)
    exp = a.copy()
    exp[:4] *= ph[None, None, :]
    got = V.get(0)
    assert rel_l2(got, exp) < 1e-6
    assert abs(np.angle(got[0, N3 // 2, 1]) - np.pi / 2) < 1e-5
    cfg_L3 = cfg["L3"]
    z = vertical_points(cfg_L3, N3)
    for f in (0, 3):
        col = V.get(0)[f, :, 0].real.astype(np.float64)
        integ = np.sum((z[2:N3] - z[1:N3 - 1]) * col[1:N3 - 1])
        V.remove_average(0, f, cfg_L3)
        after = V.get(0)[f, :, 0].real.astype(np.float64)
        assert np.allclose(after, col - integ / cfg_L3 / 2, rtol=0, atol=1e-6 * max(1e-30, np.abs(col).max()))


def _enforce_bcs(a):
    """StateVector::EnforceBCs (StateVector.h:415-421) in numpy."""
    a = a.copy()
    N3 = a.shape[1]
    a[2, [0, 1, 2, N3 - 2, N3 - 1]] = 0
    for f in (0, 1, 3):
        a[f, 0] = a[f, 1]
        a[f, N3 - 1] = a[f, N3 - 2]
    return a


def test_enforce_bcs_matches_reference_formula():
    """StateVector::EnforceBCs (StateVector.h:415-421): u3 ZeroEnds (levels
    0, 1, 2, N3-2, N3-1 of a Dirichlet field, Field.h:475-486), u1, u2, b
    NeumannEnds (level 0 = level 1, N3-1 = N3-2, Field.h:488-500)."""
    import stratiflow_b200 as sf
    cfg, s = _solver_with_states("shear3d_small", 1)
    V = sf.Vecs(s, 1)
    V.from_run(0, 0)
    a = V.get(0)
    V.enforce_bcs(0)
    want = _enforce_bcs(a)
    want[:, :, s.K1 * s.K2:] = a[:, :, s.K1 * s.K2:]
    assert np.array_equal(V.get(0), want)


def test_driver_tangent_matches_central_difference():
    """Phi'(x) d of the multiple-shooting driver (2 segments, 50 steps each)
    against the central difference of its own Evolve with e d = 1e-2 |x|:
    the O(e^2) truncation and the FP32 rounding of the difference both stay
    below 1e-3 relative."""
    from stratiflow_b200 import drivers as D
    cfg = CONFIGS["kh2d"]
    flow = _flow(cfg)
    tmp = gpu_solver(cfg, nrun=2)
    for i in range(2):
        tmp.set_state(i, make_ic(cfg, seed=70 + i, amp=5e-2))
    X = tmp.get_state_kept()
    for i in range(2):
        tmp.set_state(i, make_ic(cfg, seed=80 + i, amp=1e-3))
    Dd = tmp.get_state_kept()
    tau = 0.5
    j = D.evolve_tangent(flow, X, Dd, tau, M=2)
    eps = 0.5
    fp = D.evolve(flow, X + eps * Dd, tau, M=2)
    fm = D.evolve(flow, X - eps * Dd, tau, M=2)
    fd = (fp.astype(np.complex128) - fm) / (2 * eps)
    assert rel_l2(j[:, :4], fd[:, :4]) < 1e-3


def test_block_gram_update_and_band():
    """sf_vecs_gram / sf_vecs_update / sf_vecs_band against numpy and the
    one-pair dot product."""
    import stratiflow_b200 as sf
    cfg, s = _solver_with_states("kh2d", 3)
    V = sf.Vecs(s, 6)
    V.from_run(0, 0, 3)
    V.from_run(3, 0, 3)
    V.scale(3, -0.5, 3)
    Ri = cfg["Ri"]
    G = V.gram(0, 3, V, 3, 3, Ri)
    for i in range(3):
        for k in range(3):
            d = V.dots(i, 1, V, 3 + k, Ri)[0]
            assert abs(G[i, k] - d) <= 1e-12 * abs(V.dots(i, 1, V, i, Ri)[0])
    a = [V.get(i) for i in range(6)]
    C = np.array([[1.0, 0.5, -2.0], [0.25, -1.0, 3.0], [0.0, 2.0, 1.0]])
    V.update(3, 3, 0.75, V, 0, 3, C)
    for k in range(3):
        want = a[3 + k].astype(np.complex128)
        want[:4] += 0.75 * sum(C[i, k] * a[i][:4] for i in range(3))
        assert rel_l2(V.get(3 + k), want) < 1e-6
    V.band(0, 0b1001, 1, 4)   # u1 and b, 1 <= j1 < 4
    got = V.get(0)
    j1 = np.arange(s.plane) % s.K1
    keep = (j1 >= 1) & (j1 < 4) & (np.arange(s.plane) < s.K1 * s.K2)
    want = np.zeros_like(a[0])
    for f in (0, 3):
        want[f][:, keep] = a[0][f][:, keep]
    assert np.array_equal(got, want)


def test_block_newton_step_solves_the_linear_model():
    """One block Newton-Krylov step of Phi_T(x) = x (T = 0.3, 16 directions
    per batched Jacobian action, trust region wide open): the step dx it
    takes leaves |J dx + F| / |F| equal to the block GMRES residual it
    reports, with J dx = Phi'(x) dx - dx from the tangent-linear driver."""
    from stratiflow_b200 import drivers as D
    cfg = CONFIGS["kh2d"]
    flow = _flow(cfg)
    s = gpu_solver(cfg)
    s.set_state(0, make_ic(cfg, seed=91, amp=5e-2))
    s.Prepare()
    x = _enforce_bcs(s.get_state_kept()[0])
    x[4] = 0
    T = 0.3
    out, st = D.newton_fixed(flow, x, T, M=1, constrain=False,
                             opts=D.NKOptions(max_newton=1, krylov=96, gmres_tol=1e-3, Delta=1e6, block=16))
    assert st["newton_iterations"] == 1 and st["residuals"][1] < st["residuals"][0]
    dx = out[0].astype(np.complex128) - x
    dx[4] = 0
    F = D.evolve(flow, x, T)[0].astype(np.complex128) - x
    F[4] = 0
    Jdx = D.evolve_tangent(flow, x, dx.astype(np.complex64), T)[0].astype(np.complex128) - dx
    r = Jdx + F
    rel = np.sqrt(D.ext_dot(flow, (r, 0.0), (r, 0.0), cfg["Ri"]) / D.ext_dot(flow, (F, 0.0), (F, 0.0), cfg["Ri"]))
    assert abs(rel - st["gmres_residuals"][0]) < 0.02, (rel, st["gmres_residuals"][0])
