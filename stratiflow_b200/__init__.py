"""stratiflow_b200 — B200-native IMEX-RK time step of a stratified shear flow.

Python front end over the C-ABI in ``include/stratiflow_b200.h``. The
solver object mirrors the reference's ``IMEXRK`` (IMEXRK.h:31-670): the same
operations under the same names, on a batch of runs held on one GPU.

The CUDA library must have been built (``python -m stratiflow_b200.build``);
there is no CPU fallback: importing this package without it raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .grid import (background_profile, kept_modes, neumann_profile, vertical_points,
                   vertical_points_fractional)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstratiflow_b200.so")

U1, U2, U3, B, P = 0, 1, 2, 3, 4
FIELD = {"u1": U1, "u2": U2, "u3": U3, "b": B, "p": P}

# every entry point declared in include/stratiflow_b200.h
EXPORTS = [
    "sf_create", "sf_destroy", "sf_last_error", "sf_set_dt", "sf_set_ri", "sf_set_background",
    "sf_set_field", "sf_get_field", "sf_set_state_kept", "sf_get_state_kept", "sf_step_host_async", "sf_state_device",
    "sf_set_state_device", "sf_prepare", "sf_remove_divergence", "sf_step", "sf_set_base",
    "sf_step_linear", "sf_energy", "sf_dissipation", "sf_dot", "sf_synchronize", "sf_stream", "sf_launch_count",
    "sf_profile_step", "sf_profile_names", "sf_remove_divergence_noalloc",
    "sf_vecs_create", "sf_vecs_destroy", "sf_vecs_count", "sf_vecs_device", "sf_vecs_from_run", "sf_vecs_to_run",
    "sf_vecs_copy", "sf_vecs_set_host", "sf_vecs_get_host", "sf_vecs_axpy", "sf_vecs_lincomb", "sf_vecs_scale",
    "sf_vecs_dots", "sf_vecs_dot_sum", "sf_vecs_enforce_bcs", "sf_vecs_phase_shift", "sf_vecs_remove_average",
    "sf_vecs_zero_pressure", "sf_vecs_synchronize", "sf_set_tangent",
    "sf_net_create", "sf_net_destroy", "sf_net_num_params", "sf_net_get_params", "sf_net_set_params",
    "sf_net_forward", "sf_net_set_data", "sf_net_gradient", "sf_net_train",
    "sf_vecs_gram", "sf_vecs_update", "sf_vecs_band", "sf_vecs_column", "sf_set_xpass_slabs", "sf_set_xy_bands", "sf_set_z_chunks", "sf_set_xpass_groups", "sf_set_xpass_kernel", "sf_set_z_kernel",
    "sf_ensemble_create", "sf_ensemble_destroy", "sf_ensemble_member", "sf_ensemble_step",
    "sf_ensemble_synchronize", "sf_ensemble_launch_count", "sf_ensemble_stream", "sf_ensemble_profile", "sf_set_base_device",
    "sf_get_nodal", "sf_set_nodal", "sf_velocity_maxima", "sf_cfl", "sf_get_dt", "sf_get_runs", "sf_step_adjoint",
]


class SFError(RuntimeError):
    pass


class _Grid(C.Structure):
    _fields_ = [("N1", C.c_int), ("N2", C.c_int), ("N3", C.c_int), ("nrun", C.c_int)]


class _Flow(C.Structure):
    _fields_ = [("L1", C.c_double), ("L2", C.c_double), ("L3", C.c_double), ("Re", C.c_double),
                ("Pr", C.c_double)]


_lib = None


def load_library(path: str | None = None):
    """Load ``libstratiflow_b200.so``; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise SFError(f"{path} is missing: build it with `python -m stratiflow_b200.build`")
    L = C.CDLL(path)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    dp, fp = C.POINTER(C.c_double), C.c_void_p
    sig = {
        "sf_create": [C.POINTER(_Grid), C.POINTER(_Flow), d, i, C.POINTER(vp)],
        "sf_destroy": [vp], "sf_set_dt": [vp, d], "sf_set_ri": [vp, i, d],
        "sf_set_background": [vp, i, dp, dp], "sf_set_field": [vp, i, i, fp],
        "sf_get_field": [vp, i, i, fp], "sf_set_state_kept": [vp, fp], "sf_get_state_kept": [vp, fp],
        "sf_step_host_async": [vp, fp, fp, i],
        "sf_state_device": [vp, C.POINTER(vp), C.POINTER(C.c_size_t)], "sf_set_state_device": [vp, vp],
        "sf_prepare": [vp], "sf_remove_divergence": [vp, d], "sf_step": [vp, i],
        "sf_set_base": [vp, i, fp, fp, fp, fp], "sf_step_linear": [vp, i],
        "sf_energy": [vp, i, dp, dp], "sf_dissipation": [vp, i, dp, dp], "sf_dot": [vp, i, vp, i, dp], "sf_synchronize": [vp],
        "sf_stream": [vp, C.POINTER(vp)], "sf_launch_count": [vp, C.POINTER(C.c_longlong)],
        "sf_profile_step": [vp, i, i, i, dp, C.POINTER(i)], "sf_profile_names": [vp, C.c_char_p, C.c_size_t],
        "sf_remove_divergence_noalloc": [C.POINTER(_Grid), C.POINTER(_Flow), d, vp, vp, vp, vp, vp, vp],
        "sf_vecs_create": [vp, i, C.POINTER(vp)], "sf_vecs_destroy": [vp], "sf_vecs_count": [vp, C.POINTER(i)],
        "sf_vecs_device": [vp, i, C.POINTER(vp)], "sf_vecs_from_run": [vp, i, vp, i, i], "sf_vecs_to_run": [vp, i, vp, i, i],
        "sf_vecs_copy": [vp, i, vp, i], "sf_vecs_set_host": [vp, i, fp], "sf_vecs_get_host": [vp, i, fp],
        "sf_vecs_axpy": [vp, i, d, vp, i, i], "sf_vecs_lincomb": [vp, i, d, d, vp, i, i],
        "sf_vecs_scale": [vp, i, d, i], "sf_vecs_dots": [vp, i, i, vp, i, d, dp],
        "sf_vecs_dot_sum": [vp, i, vp, i, i, d, dp], "sf_vecs_enforce_bcs": [vp, i, i],
        "sf_vecs_phase_shift": [vp, i, i, dp], "sf_vecs_remove_average": [vp, i, i, d], "sf_vecs_synchronize": [vp],
        "sf_vecs_zero_pressure": [vp, i, i], "sf_set_tangent": [vp, i],
        "sf_net_create": [i, C.POINTER(i), i, i, C.c_ulonglong, vp, C.POINTER(vp)], "sf_net_destroy": [vp],
        "sf_net_num_params": [vp, C.POINTER(C.c_longlong)], "sf_net_get_params": [vp, fp],
        "sf_net_set_params": [vp, fp], "sf_net_forward": [vp, fp, i, fp], "sf_net_set_data": [vp, fp, fp, i],
        "sf_net_gradient": [vp, fp, dp], "sf_net_train": [vp, i, d, dp],
        "sf_vecs_gram": [vp, i, i, vp, i, i, d, dp], "sf_vecs_update": [vp, i, i, d, vp, i, i, dp],
        "sf_vecs_band": [vp, i, i, i, i], "sf_vecs_column": [vp, i, i, i, fp, i], "sf_set_xpass_slabs": [vp, i], "sf_set_xy_bands": [vp, i], "sf_set_z_chunks": [vp, i], "sf_set_xpass_groups": [vp, i], "sf_set_xpass_kernel": [vp, i], "sf_set_z_kernel": [vp, i], "sf_set_base_device": [vp, i, vp],
        "sf_get_nodal": [vp, i, i, fp], "sf_set_nodal": [vp, i, i, fp], "sf_velocity_maxima": [vp, i, dp],
        "sf_cfl": [vp, i, dp], "sf_get_dt": [vp, dp], "sf_get_runs": [vp, C.POINTER(i)],
        "sf_step_adjoint": [vp, vp, vp],
        "sf_ensemble_create": [i, C.POINTER(_Grid), C.POINTER(_Flow), dp, i, C.POINTER(vp)],
        "sf_ensemble_destroy": [vp], "sf_ensemble_member": [vp, i, C.POINTER(vp)], "sf_ensemble_step": [vp, i],
        "sf_ensemble_synchronize": [vp], "sf_ensemble_launch_count": [vp, C.POINTER(C.c_longlong)],
        "sf_ensemble_stream": [vp, C.POINTER(vp)], "sf_ensemble_profile": [vp, i, dp, dp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.sf_last_error.argtypes = []
    L.sf_last_error.restype = C.c_char_p
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        msg = load_library().sf_last_error().decode(errors="replace")
        raise SFError(f"stratiflow_b200 error {rc}: {msg}")


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class IMEXRK:
    """A batch of ``nrun`` independent IMEX-RK integrations of one grid on one
    GPU; the device-resident counterpart of the reference's ``IMEXRK``
    (IMEXRK.h:31-670) with runtime grid sizes (Parameters.h:42-43)."""

    def __init__(self, N1, N2, N3, L1, L2, L3, Re, Pr, dt, nrun=1, device=0):
        L = load_library()
        self.N1, self.N2, self.N3, self.nrun = int(N1), int(N2), int(N3), int(nrun)
        self.device = int(device)
        self.M1 = self.N1 // 2 + 1
        self.L1, self.L2, self.L3, self.Re, self.Pr = float(L1), float(L2), float(L3), float(Re), float(Pr)
        self.deltaT = float(dt)
        g = _Grid(self.N1, self.N2, self.N3, self.nrun)
        f = _Flow(self.L1, self.L2, self.L3, self.Re, self.Pr)
        h = C.c_void_p()
        _check(L.sf_create(C.byref(g), C.byref(f), self.deltaT, int(device), C.byref(h)))
        self._h = h
        self.dim3 = self.N2 > 1
        self.K1 = self.N1 // 3
        self.K2 = 2 * (self.N2 // 3) - 1 if self.dim3 else 1
        self.plane = (self.K1 * self.K2 + 15) // 16 * 16
        self.Ri = np.zeros(self.nrun)

    @classmethod
    def _member(cls, handle, N1, N2, N3, L1, L2, L3, Re, Pr, dt, device=0):
        """A view of a solver owned by something else (an Ensemble member):
        every method works, close() does not destroy it."""
        self = cls.__new__(cls)
        self.N1, self.N2, self.N3, self.nrun = int(N1), int(N2), int(N3), 1
        self.device = int(device)
        self.M1 = self.N1 // 2 + 1
        self.L1, self.L2, self.L3, self.Re, self.Pr = float(L1), float(L2), float(L3), float(Re), float(Pr)
        self.deltaT = float(dt)
        self._h = handle
        self._owned = False
        self.dim3 = self.N2 > 1
        self.K1 = self.N1 // 3
        self.K2 = 2 * (self.N2 // 3) - 1 if self.dim3 else 1
        self.plane = (self.K1 * self.K2 + 15) // 16 * 16
        self.Ri = np.zeros(1)
        return self

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                load_library().sf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- parameters ----
    def UpdateForTimestep(self, dt=None):
        """deltaT assignment + UpdateForTimestep (IMEXRK.h:502-545)."""
        if dt is not None:
            self.deltaT = float(dt)
        _check(load_library().sf_set_dt(self._h, self.deltaT))

    def set_ri(self, run, Ri):
        self.Ri[run] = float(Ri)
        _check(load_library().sf_set_ri(self._h, int(run), float(Ri)))

    def SetBackground(self, run, U, dBdz=None):
        """IMEXRK::SetBackground(Neumann1D) (IMEXRK.h:321-332) plus the
        background stratification profile (ones = the reference)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        dB = np.ones(self.N3) if dBdz is None else np.ascontiguousarray(dBdz, dtype=np.float64)
        _check(load_library().sf_set_background(self._h, int(run), U.ctypes.data_as(C.POINTER(C.c_double)),
                                                dB.ctypes.data_as(C.POINTER(C.c_double))))

    # ---- fields (reference layout [N2][M1][N3] complex64) ----
    @property
    def modal_shape(self):
        return (self.N2, self.M1, self.N3)

    def set_field(self, run, name, arr):
        a = np.ascontiguousarray(np.asarray(arr).reshape(self.modal_shape), dtype=np.complex64)
        _check(load_library().sf_set_field(self._h, int(run), FIELD[name], _fptr(a)))

    def get_field(self, run, name):
        out = np.zeros(self.modal_shape, dtype=np.complex64)
        _check(load_library().sf_get_field(self._h, int(run), FIELD[name], _fptr(out)))
        return out

    def set_state(self, run, st: dict):
        for k, v in st.items():
            self.set_field(run, k, v)

    def get_state(self, run, names=("u1", "u2", "u3", "b", "p")):
        return {k: self.get_field(run, k) for k in names}

    # ---- kept layout, all runs at once ----
    @property
    def kept_shape(self):
        return (self.nrun, 5, self.N3, self.plane)

    def set_state_kept(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex64).reshape(self.kept_shape)
        _check(load_library().sf_set_state_kept(self._h, _fptr(a)))

    def get_state_kept(self, out=None):
        if out is None:
            out = np.zeros(self.kept_shape, dtype=np.complex64)
        _check(load_library().sf_get_state_kept(self._h, _fptr(out)))
        return out

    def step_host_async(self, host_in, host_out, n=1):
        """sf_step_host_async: copy host_in (kept layout, all runs) in, n x
        TimeStep, copy the result to host_out, without waiting; consecutive
        calls overlap their copies with each other's steps. The arrays must
        stay alive, host_in unchanged and host_out unread until synchronize()."""
        for a in (host_in, host_out):
            if a.dtype != np.complex64 or a.size != int(np.prod(self.kept_shape)) or not a.flags.c_contiguous:
                raise SFError("step_host_async takes contiguous complex64 arrays of the kept shape")
        _check(load_library().sf_step_host_async(self._h, _fptr(host_in), _fptr(host_out), int(n)))

    def state_device_ptr(self):
        p, n = C.c_void_p(), C.c_size_t()
        _check(load_library().sf_state_device(self._h, C.byref(p), C.byref(n)))
        return p.value, n.value

    def set_state_device(self, ptr):
        _check(load_library().sf_set_state_device(self._h, C.c_void_p(ptr)))

    # ---- the scheme ----
    def Prepare(self):
        """FilterAll + RemoveDivergence(0) (StateVector.cpp:94-97)."""
        _check(load_library().sf_prepare(self._h))

    def RemoveDivergence(self, pressure_multiplier=1.0):
        _check(load_library().sf_remove_divergence(self._h, float(pressure_multiplier)))

    def TimeStep(self, n=1):
        """n x IMEXRK::TimeStep (IMEXRK.cpp:8-24) on every run; asynchronous."""
        _check(load_library().sf_step(self._h, int(n)))

    def SetBase(self, run, u1, u2, u3, b):
        """IMEXRK::SetBackground(u1,u2,u3,b) (IMEXRK.h:334-352)."""
        arrs = [np.ascontiguousarray(np.asarray(x).reshape(self.modal_shape), dtype=np.complex64)
                for x in (u1, u2, u3, b)]
        _check(load_library().sf_set_base(self._h, int(run), *[_fptr(x) for x in arrs]))

    # ---- nodal fields, .fields files, CFL ----
    @property
    def nodal_shape(self):
        """The reference's nodal layout (N1 n2 + n1) N3 + n3 as [N2][N1][N3]."""
        return (self.N2, self.N1, self.N3)

    def get_nodal(self, run, name):
        out = np.zeros(self.nodal_shape, dtype=np.float32)
        _check(load_library().sf_get_nodal(self._h, int(run), FIELD[name], _fptr(out)))
        return out

    def set_nodal(self, run, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float32).reshape(self.nodal_shape)
        _check(load_library().sf_set_nodal(self._h, int(run), FIELD[name], _fptr(a)))

    def SaveFlow(self, run, filename):
        """IMEXRK::SaveFlow (IMEXRK.h:415-423): the nodal U1, U2, U3, B as raw
        float32 in the reference's layout, one after the other."""
        with open(filename, "wb") as f:
            for name in ("u1", "u2", "u3", "b"):
                f.write(self.get_nodal(run, name).tobytes())

    def LoadFlow(self, run, filename, two_dimensional=False):
        """IMEXRK::LoadFlow (IMEXRK.h:425-443): reads the four nodal fields and
        takes them to modal space (ToModal). A two-dimensional file holds one
        y-plane per field, repeated along y; U2 is then zero."""
        per = self.N1 * self.N3 if two_dimensional else self.N1 * self.N2 * self.N3
        raw = np.fromfile(filename, dtype=np.float32)
        if raw.size != 4 * per:
            raise SFError(f"{filename}: {raw.size} floats, expected {4 * per}")
        for i, name in enumerate(("u1", "u2", "u3", "b")):
            a = raw[i * per:(i + 1) * per]
            if two_dimensional:
                a = np.broadcast_to(a.reshape(1, self.N1, self.N3), self.nodal_shape)
            if two_dimensional and name == "u2":
                a = np.zeros(self.nodal_shape, dtype=np.float32)
            self.set_nodal(run, name, a)

    def velocity_maxima(self, run=0):
        out = (C.c_double * 3)()
        _check(load_library().sf_velocity_maxima(self._h, int(run), out))
        return tuple(out)

    def CFL(self, run=0):
        """IMEXRK::CFL's number at the current dt (IMEXRK.h:355-366)."""
        c = C.c_double()
        _check(load_library().sf_cfl(self._h, int(run), C.byref(c)))
        return c.value

    def FullEvolve(self, T, target_cfl=0.8, interval=100):
        """StateVector::FullEvolve's loop (StateVector.cpp:3-84) on the device
        state: RemoveDivergence(0), then steps whose dt is reset every
        `interval` steps to bring the CFL number (largest over the runs) to
        `target_cfl`, the last ones shortened to end exactly at T. Returns
        {"steps", "t", "dt", "cfl_checks", "seconds"}; deltaT holds the last dt."""
        from .drivers import load_host
        st = (C.c_double * 5)()
        rc = load_host().sfh_full_evolve(self._h, float(T), float(target_cfl), int(interval), st)
        if rc != 0:
            raise SFError(load_host().sfh_last_error().decode(errors="replace"))
        self.deltaT = st[2]
        return {"steps": int(st[0]), "t": st[1], "dt": st[2], "cfl_checks": int(st[3]), "seconds": st[4]}

    def TimeStepAdjoint(self, below, above):
        """IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126): one step of every run's
        adjoint state, given the direct states at the step's ends (below the
        earlier, above the later) as Vecs of nrun states or as host arrays in
        the kept layout [nrun][5][N3][plane]; a (Vecs, i) pair names the nrun
        states from vector i on."""
        L = load_library()
        keep = []

        def dev(x):
            if isinstance(x, tuple) and isinstance(x[0], Vecs):
                p = C.c_void_p()
                _check(L.sf_vecs_device(x[0]._h, int(x[1]), C.byref(p)))
                return p
            if isinstance(x, Vecs):
                return dev((x, 0))
            v = Vecs(self, self.nrun)
            a = np.ascontiguousarray(x, dtype=np.complex64).reshape(self.kept_shape)
            for r in range(self.nrun):
                v.set(r, a[r])
            keep.append(v)
            return dev(v)
        _check(L.sf_step_adjoint(self._h, dev(below), dev(above)))
        self.synchronize()
        del keep

    def AdjointEvolve(self, direct0, adjoint_T, steps):
        """StateVector::AdjointEvolve (StateVector.cpp:158-187) with its direct
        snapshots: the direct state direct0 (kept layout, all runs) is evolved
        `steps` fixed steps with every state kept on the device, then the
        adjoint state adjoint_T is projected and taken back through the steps,
        each between the stored states at its two ends. The solver holds the
        adjoint state at the start time afterwards; returns it (kept layout)."""
        n = self.nrun
        snaps = Vecs(self, (steps + 1) * n)
        self.set_state_kept(direct0)
        self.Prepare()
        snaps.from_run(0, 0, n)
        for k in range(steps):
            self.TimeStep(1)
            snaps.from_run((k + 1) * n, 0, n)
        self.set_state_kept(adjoint_T)
        self.Prepare()
        for step in range(steps):
            self.TimeStepAdjoint((snaps, (steps - 1 - step) * n), (snaps, (steps - step) * n))
        return self.get_state_kept()

    def set_xpass_slabs(self, slabs):
        """Slabs per x-pass block (0: automatic); a launch setting only."""
        _check(load_library().sf_set_xpass_slabs(self._h, int(slabs)))

    def set_xy_bands(self, bands):
        """Level bands of the 3D x-y pass (1..8; 1: no side streams); a launch
        setting only."""
        _check(load_library().sf_set_xy_bands(self._h, int(bands)))

    def autotune(self, mode="step", steps=8, use_cache=True):
        """Pick this grid's launch settings by timing candidates on the device
        (stratiflow_b200.autotune; FFTW_PATIENT's role in the reference,
        Field.h:719-730); cached per device and grid. Returns the settings."""
        from . import autotune
        return autotune.tune(self, mode=mode, steps=steps, use_cache=use_cache)[0]

    def set_xpass_groups(self, groups):
        """Lane groups per x-pass block (0: automatic); a launch setting only."""
        _check(load_library().sf_set_xpass_groups(self._h, int(groups)))

    def set_xpass_kernel(self, kind):
        """3D nonlinear x pass: 1 level-marching lane groups (default), 0 slab
        blocks; a launch setting (the results change only by rounding)."""
        _check(load_library().sf_set_xpass_kernel(self._h, int(kind)))

    def set_z_kernel(self, kind):
        """z pass: 2 k_z_step_c (default, one lane per complex mode), 0
        k_z_step, 1 k_z_step_tma (TMA-fed first sweeps); a launch setting
        (the results change only by rounding)."""
        _check(load_library().sf_set_z_kernel(self._h, int(kind)))

    def set_z_chunks(self, chunks):
        """Warps per block of the z solves (0: automatic, 8 or 16), each with
        one z-chunk (k_z_step) or two (k_z_step_c); a launch setting (the
        results change only by rounding)."""
        _check(load_library().sf_set_z_chunks(self._h, int(chunks)))

    def set_tangent(self, nbase):
        """Runs >= nbase advance linearised about the live run (r - nbase) % nbase."""
        _check(load_library().sf_set_tangent(self._h, int(nbase)))

    def TimeStepLinear(self, n=1):
        """n x IMEXRK::TimeStepLinear (IMEXRK.cpp:26-41); asynchronous."""
        _check(load_library().sf_step_linear(self._h, int(n)))

    def energy(self, run=0):
        """(KE, PE) of one run (IMEXRK.h:395-411), FP64 accumulation."""
        ke, pe = C.c_double(), C.c_double()
        _check(load_library().sf_energy(self._h, int(run), C.byref(ke), C.byref(pe)))
        return ke.value, pe.value

    def dissipation(self, run=0):
        """(eps, chi): the viscous and diffusive sinks of KE and PE of one run,
        (1/Re) sum_i InnerProd(grad u_i, grad u_i) and
        Ri/(Re Pr) InnerProd(grad b, grad b), FP64 accumulation."""
        e, c = C.c_double(), C.c_double()
        _check(load_library().sf_dissipation(self._h, int(run), C.byref(e), C.byref(c)))
        return e.value, c.value

    def KE(self, run=0):
        return self.energy(run)[0]

    def PE(self, run=0):
        return self.energy(run)[1]

    def dot(self, run_a, other: "IMEXRK", run_b):
        out = C.c_double()
        _check(load_library().sf_dot(self._h, int(run_a), other._h, int(run_b), C.byref(out)))
        return out.value

    def synchronize(self):
        _check(load_library().sf_synchronize(self._h))

    def stream(self):
        p = C.c_void_p()
        _check(load_library().sf_stream(self._h, C.byref(p)))
        return p.value

    def profile_step(self, nsteps=3, linear=False):
        """{kernel slot name: average ms} of one step, timed eagerly with
        CUDA events between launches; advances the state by nsteps steps."""
        L = load_library()
        cap = 64
        ms = (C.c_double * cap)()
        n = C.c_int()
        _check(L.sf_profile_step(self._h, int(nsteps), int(bool(linear)), cap, ms, C.byref(n)))
        buf = C.create_string_buffer(4096)
        _check(L.sf_profile_names(self._h, buf, 4096))
        names = buf.value.decode().split(",")
        if linear:   # TimeStepLinear's x pass is the slab kernel
            names = ["k_xpass" if nm == "k_xmarch" else nm for nm in names]
        return [(f"s{i // (n.value // 3)}:{names[i]}", ms[i]) for i in range(n.value)]

    def launch_count(self):
        n = C.c_longlong()
        _check(load_library().sf_launch_count(self._h, C.byref(n)))
        return n.value


class Ensemble:
    """Independent 2D runs on grids of different sizes stepped together
    (sf_ensemble_*): one launch per RK stage over every run's x-pass and
    z-solve work items, one CUDA graph per step. grids is a list of
    (N1, N3); flows a list of (L1, L3, Re, Pr) or one tuple for all; dt one
    value or a list. members[r] is an IMEXRK view of run r (set_ri,
    SetBackground, set_state, Prepare, get_field, energy, ...)."""

    def __init__(self, grids, flows, dt, device=0):
        L = load_library()
        R = len(grids)
        flows = list(flows) if isinstance(flows, (list, np.ndarray)) and len(flows) == R and \
            not np.isscalar(flows[0]) else [flows] * R
        dts = np.broadcast_to(np.asarray(dt, dtype=np.float64), (R,)).copy()
        g = (_Grid * R)(*[_Grid(int(n1), 1, int(n3), 1) for n1, n3 in grids])
        f = (_Flow * R)(*[_Flow(float(l1), float(l1) / 2, float(l3), float(re), float(pr))
                          for l1, l3, re, pr in flows])
        h = C.c_void_p()
        _check(L.sf_ensemble_create(R, g, f, dts.ctypes.data_as(C.POINTER(C.c_double)), int(device), C.byref(h)))
        self._h = h
        self.members = []
        for r, ((n1, n3), (l1, l3, re, pr)) in enumerate(zip(grids, flows)):
            m = C.c_void_p()
            _check(L.sf_ensemble_member(self._h, r, C.byref(m)))
            self.members.append(IMEXRK._member(m, n1, 1, n3, l1, l1 / 2, l3, re, pr, dts[r], device))

    def step(self, n=1):
        """n x IMEXRK::TimeStep of every run; asynchronous."""
        _check(load_library().sf_ensemble_step(self._h, int(n)))

    def synchronize(self):
        _check(load_library().sf_ensemble_synchronize(self._h))

    def stream(self):
        p = C.c_void_p()
        _check(load_library().sf_ensemble_stream(self._h, C.byref(p)))
        return p.value

    def launch_count(self):
        n = C.c_longlong()
        _check(load_library().sf_ensemble_launch_count(self._h, C.byref(n)))
        return n.value

    def profile(self, nsteps=3):
        """(ms of one x-pass launch, ms of one z-solve launch), all members,
        timed eagerly with CUDA events; advances every run nsteps steps."""
        a, b = C.c_double(), C.c_double()
        _check(load_library().sf_ensemble_profile(self._h, int(nsteps), C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            for m in self.members:
                m._h = None
            load_library().sf_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Vecs:
    """A device store of n states of `solver`'s grid (sf_vecs_*): the
    StateVector algebra of StateVector.h:40-149, states in the kept layout
    [5][N3][plane]."""

    def __init__(self, solver: IMEXRK, n: int):
        self.solver = solver
        self.n = int(n)
        self.shape = (5, solver.N3, solver.plane)
        self._h = C.c_void_p()
        _check(load_library().sf_vecs_create(solver._h, self.n, C.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            load_library().sf_vecs_destroy(h)
            self._h = C.c_void_p()

    def set(self, i, a):
        a = np.ascontiguousarray(a, dtype=np.complex64).reshape(self.shape)
        _check(load_library().sf_vecs_set_host(self._h, int(i), _fptr(a)))

    def get(self, i):
        out = np.zeros(self.shape, dtype=np.complex64)
        _check(load_library().sf_vecs_get_host(self._h, int(i), _fptr(out)))
        return out

    def from_run(self, i, run, count=1):
        _check(load_library().sf_vecs_from_run(self._h, int(i), self.solver._h, int(run), int(count)))

    def to_run(self, i, run, count=1):
        _check(load_library().sf_vecs_to_run(self._h, int(i), self.solver._h, int(run), int(count)))

    def copy(self, dst, other: "Vecs", src):
        _check(load_library().sf_vecs_copy(self._h, int(dst), other._h, int(src)))

    def axpy(self, y, alpha, other: "Vecs", x, count=1):
        _check(load_library().sf_vecs_axpy(self._h, int(y), float(alpha), other._h, int(x), int(count)))

    def lincomb(self, y, a, b, other: "Vecs", x, count=1):
        _check(load_library().sf_vecs_lincomb(self._h, int(y), float(a), float(b), other._h, int(x), int(count)))

    def scale(self, i, alpha, count=1):
        _check(load_library().sf_vecs_scale(self._h, int(i), float(alpha), int(count)))

    def dots(self, first, count, other: "Vecs", x, Ri):
        out = np.zeros(int(count))
        _check(load_library().sf_vecs_dots(self._h, int(first), int(count), other._h, int(x), float(Ri),
                                           out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def dot_sum(self, a, other: "Vecs", b, count, Ri):
        out = C.c_double()
        _check(load_library().sf_vecs_dot_sum(self._h, int(a), other._h, int(b), int(count), float(Ri),
                                               C.byref(out)))
        return out.value

    def enforce_bcs(self, i, count=1):
        _check(load_library().sf_vecs_enforce_bcs(self._h, int(i), int(count)))

    def phase_shift(self, i, shift=None):
        s = C.c_double(0.0 if shift is None else float(shift))
        _check(load_library().sf_vecs_phase_shift(self._h, int(i), int(shift is not None), C.byref(s)))
        return s.value

    def remove_average(self, i, field, L3):
        _check(load_library().sf_vecs_remove_average(self._h, int(i), int(field), float(L3)))

    def gram(self, a, na, other: "Vecs", b, nb, Ri):
        out = np.zeros((int(na), int(nb)))
        _check(load_library().sf_vecs_gram(self._h, int(a), int(na), other._h, int(b), int(nb), float(Ri),
                                           out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def update(self, b, nb, alpha, other: "Vecs", a, na, coef):
        coef = np.ascontiguousarray(coef, dtype=np.float64).reshape(int(na), int(nb))
        _check(load_library().sf_vecs_update(self._h, int(b), int(nb), float(alpha), other._h, int(a), int(na),
                                             coef.ctypes.data_as(C.POINTER(C.c_double))))

    def band(self, i, field_mask, j1_lo, j1_hi):
        _check(load_library().sf_vecs_band(self._h, int(i), int(field_mask), int(j1_lo), int(j1_hi)))

    def column(self, i, field, mode):
        out = np.zeros(self.solver.N3, dtype=np.complex64)
        _check(load_library().sf_vecs_column(self._h, int(i), int(field), int(mode), _fptr(out), 0))
        return out

    def set_column(self, i, field, mode, col):
        col = np.ascontiguousarray(col, dtype=np.complex64)
        assert col.shape == (self.solver.N3,)
        _check(load_library().sf_vecs_column(self._h, int(i), int(field), int(mode), _fptr(col), 1))

    def zero_pressure(self, i, count=1):
        _check(load_library().sf_vecs_zero_pressure(self._h, int(i), int(count)))

    def synchronize(self):
        _check(load_library().sf_vecs_synchronize(self._h))


class Net:
    """The convolutional continuation predictor (sf_net_*): `channels` has
    nlayers + 1 entries; tensors are float32 [batch][Z][C]."""

    def __init__(self, channels, Z, max_batch, seed=0, stream=None):
        self.channels = [int(c) for c in channels]
        self.Z, self.max_batch = int(Z), int(max_batch)
        ch = (C.c_int * len(self.channels))(*self.channels)
        self._h = C.c_void_p()
        _check(load_library().sf_net_create(len(self.channels) - 1, ch, self.Z, self.max_batch, int(seed),
                                            C.c_void_p(stream), C.byref(self._h)))
        n = C.c_longlong()
        _check(load_library().sf_net_num_params(self._h, C.byref(n)))
        self.num_params = n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            load_library().sf_net_destroy(h)
            self._h = C.c_void_p()

    def get_params(self):
        out = np.zeros(self.num_params, dtype=np.float32)
        _check(load_library().sf_net_get_params(self._h, _fptr(out)))
        return out

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.num_params
        _check(load_library().sf_net_set_params(self._h, _fptr(w)))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        B = x.shape[0]
        assert x.shape == (B, self.Z, self.channels[0])
        y = np.zeros((B, self.Z, self.channels[-1]), dtype=np.float32)
        _check(load_library().sf_net_forward(self._h, _fptr(x), B, _fptr(y)))
        return y

    def set_data(self, x, target):
        x = np.ascontiguousarray(x, dtype=np.float32)
        target = np.ascontiguousarray(target, dtype=np.float32)
        B = x.shape[0]
        assert x.shape == (B, self.Z, self.channels[0]) and target.shape == (B, self.Z, self.channels[-1])
        self._data = (x, target)   # the host arrays outlive the asynchronous upload
        _check(load_library().sf_net_set_data(self._h, _fptr(x), _fptr(target), B))

    def gradient(self):
        g = np.zeros(self.num_params, dtype=np.float32)
        loss = C.c_double()
        _check(load_library().sf_net_gradient(self._h, _fptr(g), C.byref(loss)))
        return g, loss.value

    def train(self, steps, lr):
        losses = np.zeros(int(steps))
        _check(load_library().sf_net_train(self._h, int(steps), float(lr),
                                           losses.ctypes.data_as(C.POINTER(C.c_double))))
        return losses


__all__ = ["IMEXRK", "Vecs", "Net", "SFError", "load_library", "EXPORTS", "vertical_points",
           "vertical_points_fractional", "neumann_profile", "background_profile", "kept_modes"]
