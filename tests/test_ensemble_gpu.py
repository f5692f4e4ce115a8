"""Ensembles of 2D runs on different grids (sf_ensemble_*): every run's x pass
and z solves in one launch per RK stage. Three runs
of different N1, N3 and Ri, stepped together, equal three separate FP64
oracle integrations after 10 steps (1e-5 relative L2 per field, 5e-4 for p,
the parity tests' bounds), and the step is three launches."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2

pytestmark = pytest.mark.gpu

RUNS = [(64, 128, 0.05), (128, 256, 0.12), (256, 384, 0.25)]


def _cfg(n1, n3, ri):
    return dict(CONFIGS["kh2d"], N1=n1, N3=n3, Ri=ri)


def test_mixed_grid_ensemble_matches_separate_oracle_runs():
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import background_profile
    cfgs = [_cfg(*r) for r in RUNS]
    e = sf.Ensemble([(c["N1"], c["N3"]) for c in cfgs], [(c["L1"], c["L3"], c["Re"], c["Pr"]) for c in cfgs],
                    [c["dt"] for c in cfgs])
    ics = []
    for r, (c, m) in enumerate(zip(cfgs, e.members)):
        U, dB = background_profile(c["bg"], c["L3"], c["N3"])
        m.set_ri(0, c["Ri"])
        m.SetBackground(0, U, dB)
        ics.append(make_ic(c, seed=40 + r))
        m.set_state(0, ics[r])
        m.Prepare()
    n0 = e.launch_count()
    e.step(10)
    e.synchronize()
    assert e.launch_count() - n0 == 30
    for r, (c, m) in enumerate(zip(cfgs, e.members)):
        o = make_oracle(c, 64)
        o.set_state(ics[r])
        o.prepare()
        o.step(10)
        for k in ("u1", "u3", "b", "p"):
            err = rel_l2(m.get_field(0, k), o.get_field(k))
            assert err < (5e-4 if k == "p" else 1e-5), (RUNS[r], k, err)
    e.close()


def test_ensemble_rejects_3d_members():
    import stratiflow_b200 as sf
    import ctypes as C
    L = sf.load_library()
    g = (sf._Grid * 1)(sf._Grid(64, 32, 64, 1))
    f = (sf._Flow * 1)(sf._Flow(1.0, 1.0, 10.0, 1000.0, 1.0))
    dt = (C.c_double * 1)(0.01)
    h = C.c_void_p()
    assert L.sf_ensemble_create(1, g, f, dt, 0, C.byref(h)) == -1
    assert "2D" in L.sf_last_error().decode()
