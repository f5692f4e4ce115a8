"""Newton-Krylov, periodic-orbit and pseudo-arclength drivers (the C++
library libstratiflow_host.so, built from host/) and the continuation loop.

States are numpy complex64 arrays in the kept layout [5][N3][plane] (one
state) or [M][5][N3][plane] (M shooting segments).
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import SFError, load_library

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB = os.path.join(HERE, "libstratiflow_host.so")
_host = None


def load_host():
    global _host
    if _host is None:
        load_library()   # the CUDA library first (and its error if missing)
        if not os.path.exists(HOST_LIB):
            raise SFError(f"{HOST_LIB} is missing: build it with `python -m stratiflow_b200.build`")
        L = C.CDLL(HOST_LIB)
        dp, fp, i, d = C.POINTER(C.c_double), C.c_void_p, C.c_int, C.c_double
        L.sfh_last_error.restype = C.c_char_p
        L.sfh_newton_fixed.argtypes = [dp, i, d, i, fp, dp, fp, dp, i]
        L.sfh_periodic_orbit.argtypes = [dp, i, d, fp, dp, fp, dp, dp, i]
        L.sfh_arclength.argtypes = [dp, i, d, fp, d, fp, d, d, fp, d, dp, fp, dp, dp, i]
        L.sfh_evolve.argtypes = [dp, i, d, d, fp, fp]
        L.sfh_evolve_tangent.argtypes = [dp, i, d, d, fp, fp, fp]
        L.sfh_arnoldi.argtypes = [dp, fp, d, i, i, d, i, C.c_ulonglong, dp, dp, i, C.POINTER(i), fp, fp, dp]
        L.sfh_arnoldi.restype = C.c_int
        L.sfh_full_evolve.argtypes = [C.c_void_p, d, d, i, dp]
        L.sfh_full_evolve.restype = C.c_int
        L.sfh_linear_evolve.argtypes = [dp, fp, fp, d, fp]
        L.sfh_inverse_iteration.argtypes = [dp, fp, fp, d, d, d, i, i, dp, i]
        L.sfh_critical_point.argtypes = [dp, i, d, d, fp, dp, dp, dp, i]
        L.sfh_find_hopf.argtypes = [dp, i, d, fp, dp, dp, dp, dp, i]
        for f in ("sfh_linear_evolve", "sfh_inverse_iteration", "sfh_critical_point", "sfh_find_hopf"):
            getattr(L, f).restype = C.c_int
        for f in ("sfh_newton_fixed", "sfh_periodic_orbit", "sfh_arclength", "sfh_evolve", "sfh_evolve_tangent"):
            getattr(L, f).restype = C.c_int
        _host = L
    return _host


BACKGROUNDS = {"tanh": 0, "holmboe": 1, "linear": 2}


class Flow:
    """Grid + flow parameters of a driver call (Parameters.h:6-43)."""

    def __init__(self, N1, N2, N3, L1, L2, L3, Re, Pr, Ri, dt, background="tanh"):
        self.N1, self.N2, self.N3 = int(N1), int(N2), int(N3)
        self.L1, self.L2, self.L3 = float(L1), float(L2), float(L3)
        self.Re, self.Pr, self.Ri, self.dt = float(Re), float(Pr), float(Ri), float(dt)
        self.background = background
        K1 = self.N1 // 3
        K2 = 2 * (self.N2 // 3) - 1 if self.N2 > 1 else 1
        self.plane = (K1 * K2 + 15) // 16 * 16
        self.state_shape = (5, self.N3, self.plane)

    def array(self):
        return np.array([self.N1, self.N2, self.N3, self.L1, self.L2, self.L3, self.Re, self.Pr, self.Ri,
                         self.dt, BACKGROUNDS[self.background]], dtype=np.float64)


class NKOptions:
    """jacobian: "tangent" (exact actions by the tangent-linear batch) or
    "fd" (finite differences with step fd_eps |x|, NewtonKrylov.h:218-235).
    block: directions per batched Jacobian action of the block Krylov solver
    (single shooting, M = 1); 0 selects the one-direction solver, which also
    runs multiple shooting. krylov: basis vectors before the solve stops.
    precondition: the block solvers' mean-flow preconditioner (the (0,0)
    profiles of u1 and b relax by diffusion alone and are otherwise the
    slowest directions for GMRES). relative: newton_fixed's block solver
    takes the x shift as an unknown with a phase condition (relative
    equilibria) instead of removing the phase after each update."""

    def __init__(self, max_newton=20, krylov=80, target=1e-6, gmres_tol=0.01, Delta=100.0, fd_eps=3e-4,
                 jacobian="tangent", block=16, precondition=True, relative=False):
        assert jacobian in ("tangent", "fd")
        self.v = np.array([max_newton, krylov, target, gmres_tol, Delta, fd_eps,
                           0.0 if jacobian == "tangent" else 1.0, block, float(bool(precondition)),
                           float(bool(relative))], dtype=np.float64)


def _opts(opts, M):
    """The options as passed: multiple shooting (M > 1) runs the
    one-direction solver."""
    v = (opts or NKOptions()).v.copy()
    if M > 1:
        v[7] = 0
    return v


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.c_void_p)


def _segments(flow, x, M):
    x = np.ascontiguousarray(x, dtype=np.complex64)
    if x.shape == flow.state_shape:
        x = np.broadcast_to(x, (M,) + flow.state_shape).copy()
    assert x.shape == (M,) + flow.state_shape, x.shape
    return x


def _stats(st):
    n = int(st[7])
    ng = max(0, min(n - 1, (len(st) - 8 - n) // 2))
    g = st[8 + n:8 + n + 2 * ng]
    return {"newton_iterations": int(st[0]), "jacobian_actions": int(st[1]), "integrations": int(st[2]),
            "seconds": float(st[3]), "integration_seconds": float(st[4]), "residual": float(st[5]),
            "converged": bool(st[6] > 0.5), "residuals": [float(v) for v in st[8:8 + n]],
            "gmres_residuals": [float(v) for v in g[0::2]], "gmres_vectors": [int(v) for v in g[1::2]]}


def _call(rc):
    if rc != 0:
        raise SFError(load_host().sfh_last_error().decode(errors="replace"))


def newton_fixed(flow: Flow, x, T, M=1, opts: NKOptions | None = None, constrain=True):
    """Phi_T(x) = x by Newton-Krylov with M shooting segments
    (BasicNewtonKrylov, BasicNewtonKrylov.h:5-14; constraints of
    PseudoArclength.h:15-20)."""
    L = load_host()
    xs = _segments(flow, x, M)
    out = np.zeros_like(xs)
    st = np.zeros(8 + 3 * 64)
    ov = _opts(opts, M)
    _call(L.sfh_newton_fixed(_dp(flow.array()), M, float(T), int(constrain), _fp(xs), _dp(ov), _fp(out),
                             _dp(st), len(st)))
    return out, _stats(st)


def periodic_orbit(flow: Flow, x, T0, M=16, opts: NKOptions | None = None):
    """FindPeriodic (FindPeriodic.cpp:4-28) by multiple shooting: returns the
    M segments, the period and the statistics."""
    L = load_host()
    xs = _segments(flow, x, M)
    out = np.zeros_like(xs)
    T = C.c_double()
    st = np.zeros(8 + 3 * 64)
    ov = _opts(opts, M)
    _call(L.sfh_periodic_orbit(_dp(flow.array()), M, float(T0), _fp(xs), _dp(ov), _fp(out), C.byref(T),
                               _dp(st), len(st)))
    return out, T.value, _stats(st)


def arclength_correct(flow: Flow, x0, Ri0, v, vRi, ds, guess, Ri_guess, T, M=1, opts: NKOptions | None = None):
    """One corrector of the pseudo-arclength continuation
    (PseudoArclength.h:6-42)."""
    L = load_host()
    X0, V, G = (_segments(flow, a, M) for a in (x0, v, guess))
    out = np.zeros_like(G)
    ri = C.c_double()
    st = np.zeros(8 + 3 * 64)
    ov = _opts(opts, M)
    _call(L.sfh_arclength(_dp(flow.array()), M, float(T), _fp(X0), float(Ri0), _fp(V), float(vRi), float(ds),
                          _fp(G), float(Ri_guess), _dp(ov), _fp(out), C.byref(ri), _dp(st), len(st)))
    return out, ri.value, _stats(st)


def evolve(flow: Flow, x, tau, Ri=None, M=1):
    L = load_host()
    xs = _segments(flow, x, M)
    out = np.zeros_like(xs)
    _call(L.sfh_evolve(_dp(flow.array()), M, float(tau), float(flow.Ri if Ri is None else Ri), _fp(xs),
                       _fp(out)))
    return out


def evolve_tangent(flow: Flow, x, dx, tau, Ri=None, M=1):
    """Phi'(x) dx over tau for each of the M segments (exact tangent-linear
    integration about the moving base)."""
    L = load_host()
    xs, ds = _segments(flow, x, M), _segments(flow, dx, M)
    out = np.zeros_like(xs)
    _call(L.sfh_evolve_tangent(_dp(flow.array()), M, float(tau), float(flow.Ri if Ri is None else Ri), _fp(xs),
                               _fp(ds), _fp(out)))
    return out


def arnoldi(flow: Flow, about, T=11.0, block=16, krylov=320, tol=1e-6, nev=6, seed=1, vectors=False):
    """Eigenvalues (by decreasing modulus) of the linearised evolution over T
    about the state `about` (BasicArnoldi, Arnoldi.h:15-226; LinearEvolve,
    StateVector.cpp:107-155), with `block` directions per batched
    integration. With vectors=True also the real and imaginary parts of the
    leading eigenvector. Returns (eigenvalues, [vec_re, vec_im,] stats)."""
    L = load_host()
    x = np.ascontiguousarray(np.asarray(about, dtype=np.complex64).reshape(flow.state_shape))
    cap = 4096
    re, im = np.zeros(cap), np.zeros(cap)
    n = C.c_int()
    st = np.zeros(3)
    vr = np.zeros(flow.state_shape, dtype=np.complex64) if vectors else None
    vi = np.zeros(flow.state_shape, dtype=np.complex64) if vectors else None
    _call(L.sfh_arnoldi(_dp(flow.array()), _fp(x), float(T), int(block), int(krylov), float(tol), int(nev), int(seed),
                        _dp(re), _dp(im), cap, C.byref(n), _fp(vr) if vectors else None,
                        _fp(vi) if vectors else None, _dp(st)))
    ev = re[:n.value] + 1j * im[:n.value]
    stats = {"directions": int(st[0]), "integrations": int(st[1]), "seconds": float(st[2])}
    return (ev, vr, vi, stats) if vectors else (ev, stats)


# ---------------------------------------------------------- bifurcations
def linear_evolve(flow: Flow, about, d, T, Ri=None):
    """LinearEvolve (StateVector.cpp:107-156): d advanced over T by
    TimeStepLinear about the frozen state `about` (SetBackground,
    IMEXRK.h:334-352), in equal steps of at most flow.dt."""
    L = load_host()
    f = _flow_at(flow, Ri)
    a = np.ascontiguousarray(np.asarray(about, dtype=np.complex64).reshape(flow.state_shape))
    x = np.ascontiguousarray(np.asarray(d, dtype=np.complex64).reshape(flow.state_shape))
    out = np.zeros_like(x)
    _call(L.sfh_linear_evolve(_dp(f.array()), _fp(a), _fp(x), float(T), _fp(out)))
    return out


def _flow_at(flow: Flow, Ri):
    if Ri is None:
        return flow
    f = Flow(flow.N1, flow.N2, flow.N3, flow.L1, flow.L2, flow.L3, flow.Re, flow.Pr, Ri, flow.dt, flow.background)
    return f


def inverse_iteration(flow: Flow, about, b0, T=5.0, mu=1.0, eps=0.05, iters=5, krylov=512, Ri=None):
    """InverseIteration (InverseIteration.cpp:1-124): the eigenvector of the
    linearised evolution over T about `about` whose eigenvalue is nearest mu,
    from the start b0. Each iteration solves (L - mu) y = b by GMRES to
    relative residual eps and normalises. Returns (b, history) with history
    {"eigenvalue": |L b| / |b| before each solve, "residual": |L b -
    eigenvalue b|, "krylov": GMRES vectors of each solve}."""
    L = load_host()
    f = _flow_at(flow, Ri)
    a = np.ascontiguousarray(np.asarray(about, dtype=np.complex64).reshape(flow.state_shape))
    b = np.ascontiguousarray(np.asarray(b0, dtype=np.complex64).reshape(flow.state_shape)).copy()
    hist = np.zeros(1 + 3 * iters)
    _call(L.sfh_inverse_iteration(_dp(f.array()), _fp(a), _fp(b), float(T), float(mu), float(eps), int(iters),
                                  int(krylov), _dp(hist), len(hist)))
    n = int(hist[0])
    return b, {"eigenvalue": list(hist[1:1 + n]), "residual": list(hist[1 + n:1 + 2 * n]),
               "krylov": [int(v) for v in hist[1 + 2 * n:1 + 3 * n]]}


def _critical(flow, mode, x, v, Ri, T, weight, opts):
    L = load_host()
    xv = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.complex64).reshape(flow.state_shape),
                                        np.asarray(v, dtype=np.complex64).reshape(flow.state_shape)]))
    ri = np.array([Ri], dtype=np.float64)
    st = np.zeros(8 + 3 * 64)
    ov = (opts or NKOptions(jacobian="fd", block=0)).v.copy()
    ov[7] = 0
    _call(L.sfh_critical_point(_dp(flow.array()), int(mode), float(T), float(weight), _fp(xv), _dp(ri), _dp(ov),
                               _dp(st), len(st)))
    return xv[0], xv[1], float(ri[0]), st


def find_critical_point(flow: Flow, x, v, Ri, T=11.0, weight=1.0, opts: NKOptions | None = None):
    """FindCriticalPoint (FindCriticalPoint.cpp:110-213): a state x, an
    eigenvector v with eigenvalue 1 of the evolution over T linearised about
    x, and the Ri at which they exist, by Newton-Krylov (finite-difference
    Jacobian actions, as the reference's NewtonKrylov) on F = (Phi_T(x) - x,
    L_T(x) v - v, Energy(v) - weight) after the constraints (v orthogonal to
    ddx x, mean of u1 and b removed, Energy(v) = weight).
    Returns (x, v, Ri, stats)."""
    x, v, ri, st = _critical(flow, 0, x, v, Ri, T, weight, opts)
    return x, v, ri, _stats(st)


def critical_point_constraints(flow: Flow, x, v, Ri, weight=1.0):
    """FindCriticalPoint::EnforceConstraints (FindCriticalPoint.cpp:114-134) alone."""
    x, v, ri, _ = _critical(flow, 1, x, v, Ri, 1.0, weight, None)
    return x, v, ri


def critical_point_function(flow: Flow, x, v, Ri, T=11.0, weight=1.0):
    """FindCriticalPoint::EvalFunction (FindCriticalPoint.cpp:136-150): (F_x, F_v, F_p)."""
    return _critical(flow, 2, x, v, Ri, T, weight, None)[:3]


def _hopf(flow, mode, x, v1, v2, Ri, theta, T, opts):
    L = load_host()
    xv = np.ascontiguousarray(np.stack([np.asarray(a, dtype=np.complex64).reshape(flow.state_shape)
                                        for a in (x, v1, v2)]))
    ri = np.array([Ri], dtype=np.float64)
    th = np.array([theta], dtype=np.float64)
    st = np.zeros(8 + 3 * 64)
    ov = (opts or NKOptions(jacobian="fd", block=0)).v.copy()
    ov[7] = 0
    _call(L.sfh_find_hopf(_dp(flow.array()), int(mode), float(T), _fp(xv), _dp(ri), _dp(th), _dp(ov), _dp(st),
                          len(st)))
    return xv[0], xv[1], xv[2], float(ri[0]), float(th[0]), st


def find_hopf(flow: Flow, x, v1, v2, Ri, theta, T=11.0, opts: NKOptions | None = None):
    """FindHopf (FindHopf.cpp:4-101): a state x and a complex eigenvector
    v1 + i v2 with eigenvalue exp(i theta) (modulus 1) of the evolution over
    T linearised about x, and the Ri at which they exist, by Newton-Krylov
    with finite-difference Jacobian actions. v1, v2 are first divided by |v1|
    and A = v1 fixes the eigenvector's phase and size (v1.A = 1, v2.A = 0).
    Returns (x, v1, v2, Ri, theta, stats)."""
    x, v1, v2, ri, th, st = _hopf(flow, 0, x, v1, v2, Ri, theta, T, opts)
    return x, v1, v2, ri, th, _stats(st)


def hopf_constraints(flow: Flow, x, v1, v2, Ri, theta):
    """FindHopf::EnforceConstraints (FindHopf.cpp:9-20) after the initial
    rescaling by |v1| (FindHopf.cpp:88-93)."""
    return _hopf(flow, 1, x, v1, v2, Ri, theta, 1.0, None)[:5]


def hopf_function(flow: Flow, x, v1, v2, Ri, theta, T=11.0):
    """FindHopf::EvalFunction (FindHopf.cpp:22-50) after the initial
    rescaling by |v1|: (F_x, F_v1, F_v2, F_p = v2.A, F_theta = v1.A - 1)."""
    return _hopf(flow, 2, x, v1, v2, Ri, theta, T, None)[:5]


# ------------------------------------------------------------ continuation
def ext_dot(flow: Flow, a, b, Ri):
    """ExtendedStateVector::Dot (ExtendedStateVector.h:12-15) on host arrays:
    StateVector::Dot (StateVector.h:122-134) of the states plus p p'."""
    from .grid import vertical_points, vertical_points_fractional
    xa, pa = a
    xb, pb = b
    N3 = flow.N3
    z = vertical_points(flow.L3, N3)
    zf = vertical_points_fractional(flow.L3, N3)
    wzn = np.zeros(N3)
    wzn[1:N3 - 1] = z[2:N3] - z[1:N3 - 1]
    wzd = np.zeros(N3)
    wzd[2:N3 - 1] = zf[2:N3 - 1] - zf[1:N3 - 2]
    K1 = flow.N1 // 3
    K2 = 2 * (flow.N2 // 3) - 1 if flow.N2 > 1 else 1
    P = K1 * K2
    wm = np.zeros(flow.plane)
    wm[:P] = 2.0
    wm[0] = 1.0
    xa = xa.reshape((-1,) + flow.state_shape)
    xb = xb.reshape((-1,) + flow.state_shape)
    tot = 0.0
    for f, (wz, wf) in enumerate(((wzn, 1.0), (wzn, 1.0), (wzd, 1.0), (wzn, Ri))):
        if f == 1 and flow.N2 == 1:
            continue
        t = (xa[:, f].real.astype(np.float64) * xb[:, f].real + xa[:, f].imag.astype(np.float64) * xb[:, f].imag)
        tot += wf * float(np.einsum("sjm,j,m->", t, wz, wm))
    return tot + pa * pb


def secant_predictor(flow: Flow, p1, p2, ds):
    """PseudoArclength.cpp:33-61: unit tangent from two converged points in
    the extended norm; guess = x2 + ds v. Returns (guess, tangent)."""
    (x1, r1), (x2, r2) = p1, p2
    dx = x2.astype(np.complex128) - x1
    if r2 == r1:
        n = np.sqrt(ext_dot(flow, (dx, 0.0), (dx, 0.0), r2))
        v = (dx / n, 0.0)
    else:
        vx = dx / (r2 - r1)
        vp = 1.0 / np.sqrt(1.0 + ext_dot(flow, (vx, 0.0), (vx, 0.0), r2))
        vx = vx * vp
        if r2 < r1:
            vx, vp = -vx, -vp
        v = (vx, vp)
    guess = (x2 + ds * v[0], r2 + ds * v[1])
    return (guess[0].astype(np.complex64), guess[1]), (v[0].astype(np.complex64), v[1])


def continuation(flow: Flow, start_points, ds, npoints, T=11.0, M=1, opts=None, predictor=None, log=None,
                 fallback_after=6, stop_on_failure=False):
    """Pseudo-arclength continuation from two converged points
    ((x, Ri), (x, Ri)). `predictor(history, ds)` may replace the secant: it
    gets the converged points so far and returns a guess (x, Ri); the secant
    tangent is always used for the arclength constraint. A learned guess
    gets `fallback_after` Newton iterations; if it has not converged by then
    the point is solved again from the secant guess. A point that does not
    converge is kept at Newton's last iterate (and ends the run with
    `stop_on_failure`). Returns the points and the per-point statistics."""
    pts = list(start_points)
    stats = []
    opts = opts or NKOptions()
    for k in range(npoints):
        t0 = time.perf_counter()
        sec_guess, (vx, vp) = secant_predictor(flow, pts[-2], pts[-1], ds)
        guess = predictor(pts, ds) if predictor is not None else sec_guess
        used = "learned" if predictor is not None else "secant"
        o = opts
        if predictor is not None:
            o = NKOptions()
            o.v = opts.v.copy()
            o.v[0] = min(opts.v[0], fallback_after)
        x, Ri, st = arclength_correct(flow, pts[-1][0], pts[-1][1], vx, vp, ds, guess[0], guess[1], T, M, o)
        if not st["converged"] and predictor is not None:
            # the secant predictor remains the fallback
            x, Ri, st2 = arclength_correct(flow, pts[-1][0], pts[-1][1], vx, vp, ds, sec_guess[0], sec_guess[1],
                                           T, M, opts)
            for key in ("newton_iterations", "jacobian_actions", "integrations", "seconds", "integration_seconds"):
                st2[key] += st[key]
            st2["fallback_from"] = st
            st = st2
            used = "secant (fallback)"
        st["predictor"] = used
        st["wall_seconds"] = time.perf_counter() - t0
        st["Ri"] = Ri
        stats.append(st)
        pts.append((x.reshape(flow.state_shape) if M == 1 else x, Ri))
        if log:
            log(k, st)
        if not st["converged"] and stop_on_failure:
            break
    return pts, stats


# ------------------------------------------------------- learned predictor
class LearnedPredictor:
    """The convolutional predictor of the next branch point (sf_net, BF16
    operands and FP32 accumulation on the tensor cores), used in place of the
    secant guess of PseudoArclength.cpp:60-61 with the secant as fallback.

    Features along z (the convolution axis), per level: the real and
    imaginary parts of the kept modes of u1, u3 and b of the last converged
    state and of its difference from the one before, plus the step ds and Ri
    as constant channels. The network predicts the correction that takes the
    secant guess to the converged point, in units of its training RMS. 2D
    only (one kept wavenumber row)."""

    def __init__(self, flow: Flow, hidden=256, layers=4, seed=0, max_batch=64):
        from . import Net
        assert flow.N2 == 1, "the learned predictor is 2D"
        self.flow = flow
        self.P = flow.N1 // 3
        self.fields = (0, 2, 3)
        self.nc = len(self.fields) * self.P * 2
        self.cin = (2 * self.nc + 2 + 7) // 8 * 8
        self.cout = (self.nc + 7) // 8 * 8
        self.channels = [self.cin] + [hidden] * (layers - 1) + [self.cout]
        self.net = Net(self.channels, flow.N3, max_batch, seed=seed)
        self.scale = None
        self.losses = None

    def _feat(self, x):
        x = np.asarray(x).reshape(self.flow.state_shape)
        sel = x[list(self.fields), :, :self.P]
        f = np.stack([sel.real, sel.imag], axis=-1)            # [field][z][mode][re|im]
        return f.transpose(1, 0, 2, 3).reshape(self.flow.N3, self.nc).astype(np.float64)

    def _unfeat(self, f):
        x = np.zeros(self.flow.state_shape, dtype=np.complex128)
        g = f.reshape(self.flow.N3, len(self.fields), self.P, 2).transpose(1, 0, 2, 3)
        for i, fld in enumerate(self.fields):
            x[fld, :, :self.P] = g[i, ..., 0] + 1j * g[i, ..., 1]
        return x

    def _inputs(self, p1, p2, ds):
        (x1, r1), (x2, r2) = p1, p2
        a, b = self._feat(x2), self._feat(x2) - self._feat(x1)
        sx, sd, sds, sri = self.scale["x"], self.scale["d"], self.scale["ds"], self.scale["Ri"]
        out = np.zeros((self.flow.N3, self.cin), dtype=np.float32)
        out[:, :self.nc] = a / sx
        out[:, self.nc:2 * self.nc] = b / sd
        out[:, 2 * self.nc] = ds / sds
        out[:, 2 * self.nc + 1] = r2 / sri
        return out

    def fit(self, points, ds, steps=600, lr=1e-3, holdout=2, chunk=50):
        """Train on consecutive triples of converged points (x, Ri): inputs
        from the first two, target = third - secant guess. The last
        `holdout` triples are held out: training keeps the parameters with
        the lowest held-out loss, and if no parameters beat the secant guess
        there (a zero correction) the predictor returns the secant guess.
        Returns the training losses."""
        triples = [(points[k - 2], points[k - 1], points[k]) for k in range(2, len(points))]
        assert triples, "need at least three converged points"
        feats = [self._feat(p[0]) for p in points]
        diffs = [feats[k] - feats[k - 1] for k in range(1, len(points))]
        tg = []
        for p1, p2, p3 in triples:
            (gx, _), _ = secant_predictor(self.flow, p1, p2, ds)
            tg.append(self._feat(p3[0]) - self._feat(gx))
        rms = lambda arrs: float(np.sqrt(np.mean([np.mean(a ** 2) for a in arrs]))) or 1.0
        self.scale = {"x": rms(feats), "d": rms(diffs), "t": rms(tg), "ds": abs(ds) or 1.0,
                      "Ri": max(abs(p[1]) for p in points) or 1.0}
        X = np.stack([self._inputs(p1, p2, ds) for p1, p2, _ in triples])
        Y = np.zeros((len(triples), self.flow.N3, self.cout), dtype=np.float32)
        for i, t in enumerate(tg):
            Y[i, :, :self.nc] = t / self.scale["t"]
        nh = holdout if len(triples) > holdout else 0
        Xt, Yt = (X[:-nh], Y[:-nh]) if nh else (X, Y)
        self.val_baseline = float(np.mean(Y[-nh:] ** 2)) if nh else None
        best, best_loss, losses, self.val_losses = None, self.val_baseline, [], []
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            self.net.set_data(Xt, Yt)
            losses.extend(self.net.train(n, lr))
            done += n
            if nh:
                v = float(np.mean((self.net.forward(X[-nh:]) - Y[-nh:]) ** 2))
                self.val_losses.append(v)
                if v < best_loss:
                    best, best_loss = self.net.get_params(), v
        if nh:
            self.use_net = best is not None
            if best is not None:
                self.net.set_params(best)
        else:
            self.use_net = True
        self.losses = np.array(losses)
        return self.losses

    def __call__(self, pts, ds):
        sec_guess, _ = secant_predictor(self.flow, pts[-2], pts[-1], ds)
        if not getattr(self, "use_net", True):
            return sec_guess
        y = self.net.forward(self._inputs(pts[-2], pts[-1], ds)[None])[0]
        corr = self._unfeat(y[:, :self.nc].astype(np.float64) * self.scale["t"])
        return (sec_guess[0] + corr).astype(np.complex64), sec_guess[1]


# ----------------------------------------------- adjoint optimisation step
def solve_quadratic(a, b, c, positive=False):
    """SolveQuadratic (Integration.cpp:3-22): a root of a x^2 + b x + c, 0 if
    the roots are complex."""
    disc = b * b - 4 * a * c
    if disc < 0:
        return 0.0
    return (-b + np.sqrt(disc)) / (2 * a) if positive else (-b - np.sqrt(disc)) / (2 * a)


def optimal_mixing_step(solver, x0, steps, epsilon):
    """One update of the initial perturbation towards more mixing
    (Adjoint.cpp:11-103): the adjoint of the mixing objective from a zero
    final state back to t = 0 through `steps` fixed steps of run 0
    (IMEXRK.AdjointEvolve), b of the adjoint divided by Ri, a step of size
    epsilon along the gradient projected onto the sphere of the initial
    energy (lambda from SolveQuadratic, epsilon halved while it has no real
    root), then Rescale (StateVector.cpp:189-226) to that energy.
    x0: kept-layout state [5][N3][plane]. Returns (new state, info)."""
    from . import Vecs
    assert solver.nrun == 1, "one run"
    x0 = np.asarray(x0, dtype=np.complex64).reshape(solver.kept_shape[1:])
    zero = np.zeros(solver.kept_shape, dtype=np.complex64)
    adj = solver.AdjointEvolve(x0[None], zero, steps)[0].copy()
    Ri = float(solver.Ri[0])
    adj[3] /= Ri
    V = Vecs(solver, 3)
    V.set(0, x0)
    V.set(1, adj)
    udotu, udotv = V.dots(0, 2, V, 0, Ri)
    vdotv = V.dots(1, 1, V, 1, Ri)[0]
    lam = 0.0
    while lam == 0.0:
        lam = solve_quadratic(epsilon * udotu, 2 * epsilon * udotv - 2 * udotu, epsilon * vdotv - 2 * udotv)
        if lam == 0.0:
            epsilon /= 2
    # deriv = adjoint + lambda x0; result = x0 - epsilon deriv (on u1..b)
    V.copy(2, V, 1)
    V.axpy(2, lam, V, 0)
    residual = V.dots(2, 1, V, 2, Ri)[0]
    V.lincomb(2, -epsilon, 1.0, V, 0)
    # Rescale to the energy of x0: project, scale, project
    energy = 0.5 * udotu
    V.zero_pressure(2)
    V.to_run(2, 0)
    solver.Prepare()
    V.from_run(2, 0)
    e_before = 0.5 * V.dots(2, 1, V, 2, Ri)[0]
    V.scale(2, np.sqrt(energy / e_before) if e_before != 0 else 0.0)
    V.to_run(2, 0)
    solver.Prepare()
    out = solver.get_state_kept()[0]
    return out, {"epsilon": epsilon, "lambda": lam, "residual": residual, "udotu": udotu, "udotv": udotv,
                 "vdotv": vdotv, "bound_epsilon": -2 * udotu / udotv if udotv != 0 else None}
