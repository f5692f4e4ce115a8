"""GPU test of BasicArnoldi (Arnoldi.h:15-226): the eigenvalues of the
linearised evolution over T about the laminar shear layer (the
Kelvin-Helmholtz modes), from the block Arnoldi driver (8 directions per
batched TimeStepLinear integration, FP64 Hessenberg numerics), against a
plain Arnoldi iteration in numpy whose matrix-vector product is the FP64
oracle's TimeStepLinear (IMEXRK.cpp:26-41) over the same T.

The driver works in the real vector space of the kept coefficients, where
each eigenvalue of the complex-linear operator about an x-homogeneous base
appears with its conjugate (a real one twice); the numpy reference works in
the complex space. Bound: the growth factor of the Kelvin-Helmholtz mode
(the largest modulus) agrees to 1e-4 relative (the FP32 linear integration
over 400 steps against the FP64 one), and both find it real."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_oracle

pytestmark = pytest.mark.gpu

T = 4.0


def oracle_eigenvalues(cfg, k=40, seed=5):
    o = make_oracle(cfg, prec=64)
    shape = o.modal_shape
    zero = np.zeros(shape, dtype=np.complex128)
    o.set_base(zero, zero, zero, zero)
    rng = np.random.default_rng(seed)
    names = ("u1", "u3", "b")

    def pack(st):
        return np.concatenate([st[n].ravel() for n in names])

    def unpack(v):
        n = int(np.prod(shape))
        return {nm: v[i * n:(i + 1) * n].reshape(shape) for i, nm in enumerate(names)}

    def matvec(v):
        st = unpack(v)
        st["u2"] = zero
        st["p"] = zero
        o.set_state(st)
        o.prepare()
        o.step_linear(int(round(T / cfg["dt"])))
        return pack(o.get_state())

    # a random start projected by the oracle itself (only kept, divergence-free modes)
    o.make_ic(seed, amp=1e-3, nx_lo=8, ny_lo=8, fields=("u1", "u3"))
    o.prepare()
    q = [pack(o.get_state())]
    q[0] /= np.linalg.norm(q[0])
    H = np.zeros((k + 1, k), dtype=np.complex128)
    for j in range(k):
        w = matvec(q[j])
        for _ in range(2):
            for i in range(j + 1):
                h = np.vdot(q[i], w)
                H[i, j] += h
                w = w - h * q[i]
        H[j + 1, j] = np.linalg.norm(w)
        q.append(w / H[j + 1, j])
    ev = np.linalg.eigvals(H[:k, :k])
    return ev[np.argsort(-np.abs(ev))]


def test_arnoldi_matches_oracle_kh_modes():
    from stratiflow_b200 import drivers as D
    cfg = CONFIGS["lin2d"]
    flow = D.Flow(cfg["N1"], 1, cfg["N3"], cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Pr"], cfg["Ri"],
                  cfg["dt"], cfg["bg"])
    zero = np.zeros(flow.state_shape, dtype=np.complex64)
    ev, vr, vi, st = D.arnoldi(flow, zero, T=T, block=8, krylov=160, tol=1e-9, nev=4, vectors=True)
    ref = oracle_eigenvalues(cfg)
    assert abs(ev[0]) > 1.0   # Kelvin-Helmholtz growth at Ri = 0.1
    assert abs(abs(ev[0]) - abs(ref[0])) <= 1e-4 * abs(ref[0]), (ev[:4], ref[:4])
    assert abs(ev[0].imag) <= 1e-6 * abs(ev[0]) and abs(ref[0].imag) <= 1e-6 * abs(ref[0])
    assert abs(abs(ev[1]) - abs(ev[0])) <= 1e-5 * abs(ev[0])   # its copy in the real space (FP32 apart)
    # the leading eigenvector is not zero and lies in the perturbation fields
    assert np.linalg.norm(vr[:4]) + np.linalg.norm(vi[:4]) > 0
