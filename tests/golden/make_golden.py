"""Generates the golden fixtures of tests/golden/ with the literal dense-matrix
transcription of the reference (oracle/dense_ref.py, FP64, numpy FFT).

    python tests/golden/make_golden.py

The reference has no tests or fixtures of its own and cannot be built here,
so these vectors pin the banded C++ oracle to the reference's own operator
construction (Differentiation.cpp, Tridiagonal.h, IMEXRK.h/.cpp) rather than
to outputs of the reference binary.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import dense_ref as D  # noqa: E402

CASES = {
    # name: (N1, N2, N3, Re, Ri, Pr, dt, background)
    "small2d": (16, 1, 16, 1000.0, 0.1, 1.0, 0.01, "linear"),
    "small2d_tanh": (32, 1, 24, 500.0, 0.2, 2.0, 0.02, "tanh"),
    "small3d": (16, 16, 16, 1000.0, 0.16, 1.0, 0.01, "holmboe"),
}


def seeded_state(imex: D.IMEXRK, seed: int, amp: float):
    rng = np.random.default_rng(seed)
    st = {}
    for name in ("u1", "u2", "u3", "b"):
        a = np.zeros((imex.N2, imex.M1, imex.N3), complex)
        if name == "u2" and not imex.dim3:
            st[name] = a
            continue
        a[imex.kept] = amp * (rng.standard_normal((imex.kept.sum(), imex.N3))
                              + 1j * rng.standard_normal((imex.kept.sum(), imex.N3)))
        # real-valued nodal field: Hermitian j1 = 0 column
        a[0, 0] = a[0, 0].real
        if imex.dim3:
            for j2 in range(1, imex.N2):
                if imex.kept[j2, 0] and j2 < imex.N2 // 2:
                    a[imex.N2 - j2, 0] = np.conj(a[j2, 0])
        # StateVector::EnforceBCs (StateVector.h:415-421)
        if name == "u3":
            a[..., [0, 1, 2, -2, -1]] = 0
        else:
            a[..., 0] = a[..., 1]
            a[..., -1] = a[..., -2]
        st[name] = a
    return st


def profiles(kind, L3, N3):
    zf = D.vertical_points_fractional(L3, N3)
    U = np.tanh(zf)
    U[1] = U[2]; U[0] = U[1]; U[-2] = U[-3]; U[-1] = U[-2]
    dB = {"linear": np.ones(N3), "tanh": 1 / np.cosh(zf) ** 2, "holmboe": 3 / np.cosh(3 * zf) ** 2}[kind]
    return U, dB


def main():
    L1 = 2 * np.pi / 0.44
    for name, (N1, N2, N3, Re, Ri, Pr, dt, bg) in CASES.items():
        imex = D.IMEXRK(N1, N2, N3, L1, L1 / 2, 10.0, Re, Ri, Pr, dt)
        U, dB = profiles(bg, 10.0, N3)
        imex.U_ = U
        imex.dBdz = dB
        st = seeded_state(imex, seed=20240 + N1 + N2 + N3, amp=0.05)
        for k, v in st.items():
            setattr(imex, k, v.copy())
        imex.p[:] = 0
        out = {"params": np.array([N1, N2, N3, L1, L1 / 2, 10.0, Re, Ri, Pr, dt]), "U": U, "dBdz": dB}
        for k in ("u1", "u2", "u3", "b"):
            out["in_" + k] = st[k]
        imex.Prepare()
        for k in ("u1", "u2", "u3", "b", "p"):
            out["prep_" + k] = getattr(imex, k).copy()
        for _ in range(3):
            imex.TimeStep()
        for k in ("u1", "u2", "u3", "b", "p"):
            out["step3_" + k] = getattr(imex, k).copy()
        out["step3_energy"] = np.array([imex.KE(), imex.PE()])
        base = {k: getattr(imex, k).copy() for k in ("u1", "u2", "u3", "b")}
        imex.SetBase(base["u1"], base["u2"], base["u3"], base["b"])
        for _ in range(2):
            imex.TimeStepLinear()
        for k in ("u1", "u2", "u3", "b", "p"):
            out["lin2_" + k] = getattr(imex, k).copy()
        # two adjoint steps between the prepared input (below) and the
        # 3-step state (above), from the linear result as the adjoint state
        below = {k: out["prep_" + k] for k in ("u1", "u2", "u3", "b")}
        above = {k: out["step3_" + k] for k in ("u1", "u2", "u3", "b")}
        imex.p[:] = 0
        imex.Prepare()
        for k in ("u1", "u2", "u3", "b", "p"):
            out["adjin_" + k] = getattr(imex, k).copy()
        for _ in range(2):
            imex.TimeStepAdjoint(below, above)
        for k in ("u1", "u2", "u3", "b", "p"):
            out["adj2_" + k] = getattr(imex, k).copy()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")


if __name__ == "__main__":
    main()
