"""GPU tests of the nodal fields of a state (sf_get_nodal / sf_set_nodal,
the .fields files of IMEXRK::SaveFlow / LoadFlow), the CFL number and the
adaptive-step FullEvolve loop.

Bounds: nodal fields against the FP64 oracle's PopulateNodalVariables and
modal fields against its ToModal to 1e-6 relative L2 (one FP32 transform);
a nodal -> modal -> nodal round trip of a kept-mode state to 1e-6; the
velocity maxima of IMEXRK::CFL against the oracle's nodal fields to 1e-6."""
import os

import numpy as np
import pytest

from stratiflow_b200.grid import background_profile
from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu

NAMES = {"u1": "U1", "u2": "U2", "u3": "U3", "b": "B"}


def _state(name, seed=7, amp=5e-2):
    cfg = CONFIGS[name]
    ic = make_ic(cfg, seed=seed, amp=amp)
    ic["b"] = 0.3 * ic["u1"]   # a buoyancy field too
    s = gpu_solver(cfg)
    s.set_state(0, ic)
    return cfg, ic, s


def _fields(cfg):
    return ("u1", "u2", "u3", "b") if cfg["N2"] > 1 else ("u1", "u3", "b")


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_nodal_fields_match_oracle(name):
    cfg, ic, s = _state(name)
    o = make_oracle(cfg, 64)
    o.set_state(ic)
    o.populate_nodal()
    for k in _fields(cfg):
        assert rel_l2(s.get_nodal(0, k), o.get_nodal(NAMES[k])) < 1e-6, k


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_to_modal_matches_oracle_and_round_trips(name):
    cfg, ic, s = _state(name)
    o = make_oracle(cfg, 64)
    rng = np.random.default_rng(3)
    for k in _fields(cfg):
        nod = rng.normal(size=o.nodal_shape).astype(np.float32)
        s.set_nodal(0, k, nod)
        assert rel_l2(s.get_field(0, k), o.to_modal(nod.astype(np.float64))) < 1e-6, k
    # kept-mode state -> nodal -> modal
    s.set_state(0, ic)
    for k in _fields(cfg):
        before = s.get_field(0, k)
        s.set_nodal(0, k, s.get_nodal(0, k))
        assert rel_l2(s.get_field(0, k), before) < 1e-6, k


def test_fields_file_round_trip(tmp_path):
    cfg, ic, s = _state("shear3d_small")
    path = os.path.join(tmp_path, "state.fields")
    s.SaveFlow(0, path)
    assert os.path.getsize(path) == 4 * 4 * cfg["N1"] * cfg["N2"] * cfg["N3"]
    t = gpu_solver(cfg)
    t.LoadFlow(0, path)
    for k in _fields(cfg):
        assert rel_l2(t.get_field(0, k), s.get_field(0, k)) < 1e-6, k


def test_velocity_maxima_and_cfl_match_oracle_nodal_fields():
    cfg, ic, s = _state("kh2d")
    o = make_oracle(cfg, 64)
    o.set_state(ic)
    o.populate_nodal()
    U, _ = background_profile(cfg["bg"], cfg["L3"], cfg["N3"])
    m1 = np.max(np.abs(o.get_nodal("U1") + U[None, None, :]))
    m3 = np.max(np.abs(o.get_nodal("U3")))
    got = s.velocity_maxima(0)
    assert abs(got[0] - m1) <= 1e-6 * m1 and abs(got[2] - m3) <= 1e-6 * m3 and got[1] == 0
    z = o.grid("z")
    cfl = (m1 / (cfg["L1"] / cfg["N1"]) + m3 / (z[cfg["N3"] // 2 + 1] - z[cfg["N3"] // 2])) * cfg["dt"]
    assert abs(s.CFL(0) - cfl) <= 1e-6 * cfl


def test_full_evolve_ends_at_T_with_the_target_cfl():
    cfg, ic, s = _state("kh2d")
    st = s.FullEvolve(3.0, target_cfl=0.8, interval=100)
    assert abs(st["t"] - 3.0) < 1e-9 and st["cfl_checks"] >= 1 and st["steps"] >= 1
    # the same evolution again gives the same state
    cfg2, ic2, s2 = _state("kh2d")
    s2.FullEvolve(3.0, target_cfl=0.8, interval=100)
    assert np.array_equal(s.get_state_kept(), s2.get_state_kept())
    # the first check sets dt = dt0 * 0.8 / CFL, then the last steps are
    # shortened to end at T (StateVector.cpp:29-46)
    _, _, s3 = _state("kh2d")
    dt0, c0 = s3.deltaT, s3.CFL(0)
    dt1 = dt0 * 0.8 / c0
    T = 7.5 * dt1
    st3 = s3.FullEvolve(T, target_cfl=0.8, interval=100)
    n = int(T / dt1) + 1
    assert st3["steps"] == n and abs(st3["dt"] - T / n) <= 1e-6 * T / n


def test_load_and_interpolate(tmp_path):
    """StateVector::LoadAndInterpolate (StateVector.h:275-413): onto the same
    grid it returns the state (coincident points get weight 1); onto a finer
    grid each kept mode's z column is the linear interpolation (numpy's
    np.interp, clamped) of the coarse one at interior levels."""
    from stratiflow_b200.grid import vertical_points, vertical_points_fractional
    from stratiflow_b200.regrid import load_and_interpolate
    cfg, ic, s = _state("kh2d")
    path = os.path.join(tmp_path, "coarse.fields")
    s.SaveFlow(0, path)
    same = gpu_solver(cfg)
    load_and_interpolate(same, 0, path, cfg["N1"], cfg["N3"])
    for k in ("u1", "u3", "b"):
        a, b = same.get_field(0, k), s.get_field(0, k)
        assert rel_l2(a[..., 2:-2], b[..., 2:-2]) < 1e-6, k
    fine_cfg = dict(CONFIGS["nk2d"])
    fine = gpu_solver(fine_cfg)
    load_and_interpolate(fine, 0, path, cfg["N1"], cfg["N3"])
    zo, zn = vertical_points_fractional(10.0, cfg["N3"]), vertical_points_fractional(10.0, fine_cfg["N3"])
    src, dst = s.get_field(0, "u1")[0], fine.get_field(0, "u1")[0]
    K1 = cfg["N1"] // 3
    for j1 in range(K1):
        want = np.interp(zn, zo, src[j1].real) + 1j * np.interp(zn, zo, src[j1].imag)
        got = dst[j1]
        sl = slice(2, fine_cfg["N3"] - 2)
        assert np.allclose(got[sl], want[sl], rtol=1e-5, atol=1e-6 * np.abs(src).max()), j1
    assert not np.any(dst[K1:])   # modes the coarse grid did not keep stay zero
    del vertical_points
