"""ctypes front end of the CPU oracle (``libsforacle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` as the
checker and the CPU baseline. The product path never imports this module.

The oracle restates jeremypparker/Stratiflow's IMEXRK time step (IMEXRK.cpp:8-258,
IMEXRK.h:37-545) on the CPU in float (the reference's default build) or double
(its -DDOUBLE build). Fields cross this interface in the reference's own
storage layout: complex modal data z-fastest, index (M1*n2 + n1)*N3 + n3 with
M1 = N1/2+1 (Field.h:399, 410).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsforacle.so")
SRC = os.path.join(HERE, "sf_oracle.cpp")

FIELDS = {"u1": 0, "u2": 1, "u3": 2, "b": 3, "p": 4, "r1": 5, "r2": 6, "r3": 7, "rB": 8}


def build(force: bool = False) -> str:
    """Compile the oracle with g++ (OpenMP). Returns the library path."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
               SRC, "-o", LIB]
        subprocess.check_call(cmd)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, i, d, dp = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)
        L.sfo_create.restype = vp
        L.sfo_create.argtypes = [i, i, i, i, d, d, d, d, d, d, d]
        for name, args in [
            ("sfo_destroy", [vp]), ("sfo_set_dt", [vp, d]), ("sfo_set_ri", [vp, d]),
            ("sfo_set_background", [vp, dp, dp]), ("sfo_get_grid", [vp, i, dp]),
            ("sfo_set_field", [vp, i, dp]), ("sfo_get_field", [vp, i, dp]),
            ("sfo_get_nodal", [vp, i, dp]), ("sfo_prepare", [vp]), ("sfo_step", [vp, i]),
            ("sfo_step_linear", [vp, i]), ("sfo_remove_divergence", [vp, d]),
            ("sfo_populate_nodal", [vp]), ("sfo_filter_all", [vp]),
            ("sfo_set_base", [vp, dp, dp, dp, dp]), ("sfo_energy", [vp, dp, dp]),
            ("sfo_dissipation", [vp, dp, dp]),
            ("sfo_to_nodal", [vp, dp, dp]), ("sfo_to_modal", [vp, dp, dp]),
            ("sfo_make_ic", [vp, C.c_uint64, d, i, i, i]), ("sfo_set_threads", [i]),
            ("sfo_step_adjoint", [vp, dp, dp]),
        ]:
            fn = getattr(L, name)
            fn.restype = None
            fn.argtypes = args
        L.sfo_get_threads.restype = i
        L.sfo_get_threads.argtypes = []
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().sfo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().sfo_get_threads())


class Oracle:
    """One CPU solver: a restatement of ``IMEXRK`` (IMEXRK.h:31-670) with a
    runtime grid. ``prec`` is 32 or 64."""

    def __init__(self, N1, N2, N3, L1, L2, L3, Re, Ri, Pr, dt, prec=32):
        self.N1, self.N2, self.N3 = int(N1), int(N2), int(N3)
        self.M1 = self.N1 // 2 + 1
        self.prec = prec
        self.Ri = float(Ri)
        self.h = lib().sfo_create(prec, self.N1, self.N2, self.N3, L1, L2, L3, Re, Ri, Pr, dt)
        if not self.h:
            raise ValueError("oracle grid: N1, N2 must be powers of two (N1 >= 8), N3 % 4 == 0")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().sfo_destroy(h)
            self.h = None

    @property
    def modal_shape(self):
        return (self.N2, self.M1, self.N3)

    @property
    def nodal_shape(self):
        return (self.N2, self.N1, self.N3)

    def set_dt(self, dt):
        lib().sfo_set_dt(self.h, float(dt))

    def set_ri(self, ri):
        self.Ri = float(ri)
        lib().sfo_set_ri(self.h, float(ri))

    def set_background(self, U, dBdz):
        U = np.ascontiguousarray(U, dtype=np.float64)
        dB = np.ascontiguousarray(dBdz, dtype=np.float64)
        lib().sfo_set_background(self.h, _dp(U), _dp(dB))

    def grid(self, which):
        out = np.zeros(self.N3)
        lib().sfo_get_grid(self.h, {"z": 0, "zf": 1, "DY": 2, "DYF": 3}[which], _dp(out))
        return out

    def set_field(self, name, arr):
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.complex128).reshape(self.modal_shape))
        lib().sfo_set_field(self.h, FIELDS[name], _dp(a.view(np.float64)))

    def get_field(self, name):
        out = np.zeros(self.modal_shape, dtype=np.complex128)
        lib().sfo_get_field(self.h, FIELDS[name], _dp(out.view(np.float64)))
        return out

    def get_nodal(self, which):
        out = np.zeros(self.nodal_shape)
        lib().sfo_get_nodal(self.h, {"U1": 0, "U2": 1, "U3": 2, "B": 3}[which], _dp(out))
        return out

    def set_state(self, st: dict):
        for k, v in st.items():
            self.set_field(k, v)

    def get_state(self, names=("u1", "u2", "u3", "b", "p")):
        return {k: self.get_field(k) for k in names}

    def prepare(self):
        lib().sfo_prepare(self.h)

    def step(self, n=1):
        lib().sfo_step(self.h, int(n))

    def step_linear(self, n=1):
        lib().sfo_step_linear(self.h, int(n))

    def remove_divergence(self, pm):
        lib().sfo_remove_divergence(self.h, float(pm))

    def populate_nodal(self):
        lib().sfo_populate_nodal(self.h)

    def filter_all(self):
        lib().sfo_filter_all(self.h)

    def set_base(self, u1, u2, u3, b):
        arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(self.modal_shape))
                for a in (u1, u2, u3, b)]
        lib().sfo_set_base(self.h, *[_dp(a.view(np.float64)) for a in arrs])

    def step_adjoint(self, below: dict, above: dict):
        """IMEXRK::TimeStepAdjoint with the direct state below (earlier) and
        above (later): dicts of modal u1, u2, u3, b."""
        def pack(st):
            return np.ascontiguousarray(np.stack([np.asarray(st[k], dtype=np.complex128).reshape(self.modal_shape)
                                                  for k in ("u1", "u2", "u3", "b")]))
        bl, ab = pack(below), pack(above)
        lib().sfo_step_adjoint(self.h, _dp(bl.view(np.float64)), _dp(ab.view(np.float64)))

    def energy(self):
        ke, pe = C.c_double(), C.c_double()
        lib().sfo_energy(self.h, C.byref(ke), C.byref(pe))
        return ke.value, pe.value

    def dissipation(self):
        """(eps, chi): (1/Re) sum_i InnerProd(grad u_i, grad u_i) and
        Ri/(Re Pr) InnerProd(grad b, grad b), the sinks of KE and PE."""
        e, c = C.c_double(), C.c_double()
        lib().sfo_dissipation(self.h, C.byref(e), C.byref(c))
        return e.value, c.value

    def to_nodal(self, modal):
        a = np.ascontiguousarray(np.asarray(modal, dtype=np.complex128).reshape(self.modal_shape))
        out = np.zeros(self.nodal_shape)
        lib().sfo_to_nodal(self.h, _dp(a.view(np.float64)), _dp(out))
        return out

    def to_modal(self, nodal):
        a = np.ascontiguousarray(np.asarray(nodal, dtype=np.float64).reshape(self.nodal_shape))
        out = np.zeros(self.modal_shape, dtype=np.complex128)
        lib().sfo_to_modal(self.h, _dp(a), _dp(out.view(np.float64)))
        return out

    def make_ic(self, seed, amp=1e-3, nx_lo=8, ny_lo=8, fields=("u1", "u3")):
        mask = 0
        for f in fields:
            mask |= 1 << {"u1": 0, "u2": 1, "u3": 2, "b": 3}[f]
        lib().sfo_make_ic(self.h, int(seed), float(amp), int(nx_lo), int(ny_lo), mask)
