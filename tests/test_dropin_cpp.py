"""The C++ drop-in (stratiflow_b200/host/imexrk.hpp): a class with the
reference's IMEXRK surface over the C-ABI. The CPU test compiles and links a
caller written against that surface (tests/cpp/dropin_fixed_evolve.cpp, the
reference's FixedEvolve loop); the GPU test runs it and compares its state
after 10 steps with the Python binding's and with the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_fixed_evolve.cpp")


def _build(tmp):
    from stratiflow_b200 import build as B
    lib = B.build()
    exe = os.path.join(tmp, "dropin_fixed_evolve")
    libdir = os.path.dirname(lib)
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", SRC,
                           "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lstratiflow_b200",
                           f"-Wl,-rpath,{libdir}", "-o", exe])
    return exe


def test_dropin_caller_compiles_and_links(tmp_path):
    exe = _build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_dropin_fixed_evolve_matches_python_and_oracle(tmp_path):
    from stratiflow_b200.grid import background_profile
    from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2
    from tests.test_gpu_parity import gpu_solver
    cfg = CONFIGS["shear3d_small"]
    exe = _build(str(tmp_path))
    ic = make_ic(cfg, seed=77)
    U, dB = background_profile(cfg["bg"], cfg["L3"], cfg["N3"])
    names = ("u1", "u2", "u3", "b", "p")
    with open(tmp_path / "in.bin", "wb") as fh:
        np.array([cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Ri"], cfg["Pr"], cfg["dt"]]).tofile(fh)
        np.asarray(U, np.float64).tofile(fh)
        np.asarray(dB, np.float64).tofile(fh)
        for k in names:
            np.ascontiguousarray(ic[k], dtype=np.complex64).tofile(fh)
    subprocess.check_call([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "10"])
    raw = open(tmp_path / "out.bin", "rb").read()
    shape = (cfg["N2"], cfg["N1"] // 2 + 1, cfg["N3"])
    n = int(np.prod(shape))
    f = np.frombuffer(raw[:5 * n * 8], dtype=np.complex64).reshape(5, *shape)
    ke, pe = np.frombuffer(raw[5 * n * 8:], dtype=np.float64)
    # the drop-in keeps deltaT in stratifloat (float), as IMEXRK.h does; the
    # Python path gets the same float-rounded step (p, which accumulates q/h,
    # would otherwise differ by the last bit of h amplified ~1000 times)
    s = gpu_solver(dict(cfg, dt=float(np.float32(cfg["dt"]))))
    s.set_state(0, ic)
    s.Prepare()
    s.TimeStep(10)
    s.synchronize()
    o = make_oracle(cfg, 64)
    o.set_state(ic)
    o.prepare()
    o.step(10)
    for i, k in enumerate(names):
        assert rel_l2(f[i], s.get_field(0, k)) < 1e-6, k
        assert rel_l2(f[i], o.get_field(k)) < (5e-4 if k == "p" else 1e-5), k
    ke_o, pe_o = o.energy()
    assert abs(ke - ke_o) <= 1e-5 * ke_o and abs(pe - pe_o) <= 1e-5 * pe_o
