"""GPU tests of the tangent-linear batch (sf_set_tangent): runs >= nbase
advance by TimeStepLinear about the live state of their base run, which is
the exact derivative of the discrete step map.

Checks:
  * against the FP64 oracle's central difference
    (Phi(x + e d) - Phi(x - e d)) / 2e, e = 1e-2 on |d| = 1e-3 |x|-scale
    perturbations: truncation O(e^2) is far below FP32 rounding, so the
    bound is the FP32 step's own, 2e-5 relative L2 for u1, u2, u3, b after
    the stated steps and 5e-4 for p (p accumulates q/h);
  * the base runs of a tangent batch equal the same runs of a plain batch
    bit for bit (the base runs take the nonlinear kernels unchanged);
  * linearity: J(d1 + d2) = J d1 + J d2 to 1e-6.
"""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2
from tests.test_gpu_parity import fields, gpu_solver

pytestmark = pytest.mark.gpu

TOL = 2e-5
TOL_P = 5e-4


def _scaled(st, a):
    return {k: v * a for k, v in st.items()}


def _sum(a, b, sa=1.0, sb=1.0):
    return {k: sa * a[k] + sb * b[k] for k in a}


@pytest.mark.parametrize("name,nsteps", [("kh2d", 10), ("shear3d_small", 5)])
def test_tangent_matches_fp64_central_difference(name, nsteps):
    cfg = CONFIGS[name]
    base = make_ic(cfg, seed=21, amp=5e-2)
    d = make_ic(cfg, seed=22, amp=1e-3)
    s = gpu_solver(cfg, nrun=2)
    s.set_tangent(1)
    s.set_state(0, base)
    s.set_state(1, d)
    s.Prepare()
    s.TimeStep(nsteps)
    s.synchronize()
    eps = 1e-2
    out = {}
    for sign in (1, -1):
        o = make_oracle(cfg, 64)
        o.set_state(_sum(base, d, 1.0, sign * eps))
        o.prepare()
        o.step(nsteps)
        out[sign] = o.get_state()
    fd = _sum(out[1], out[-1], 0.5 / eps, -0.5 / eps)
    errs = {k: rel_l2(s.get_field(1, k), fd[k]) for k in fields(cfg) + ("p",)}
    bad = {k: e for k, e in errs.items() if e > (TOL_P if k == "p" else TOL)}
    assert not bad, errs


def test_tangent_bases_equal_plain_runs():
    cfg = CONFIGS["kh2d"]
    xs = [make_ic(cfg, seed=31 + r, amp=5e-2) for r in range(2)]
    ds = [make_ic(cfg, seed=41 + r, amp=1e-3) for r in range(2)]
    t = gpu_solver(cfg, nrun=4)
    t.set_tangent(2)
    p = gpu_solver(cfg, nrun=2)
    for r in range(2):
        t.set_state(r, xs[r])
        t.set_state(2 + r, ds[r])
        p.set_state(r, xs[r])
    for s in (t, p):
        s.Prepare()
        s.TimeStep(7)
        s.synchronize()
    for r in range(2):
        for k in fields(cfg) + ("p",):
            assert np.array_equal(t.get_field(r, k), p.get_field(r, k)), (r, k)


def test_tangent_is_linear():
    cfg = CONFIGS["shear3d_small"]
    x = make_ic(cfg, seed=51, amp=5e-2)
    d1 = make_ic(cfg, seed=52, amp=1e-3)
    d2 = make_ic(cfg, seed=53, amp=1e-3)
    s = gpu_solver(cfg, nrun=4)
    s.set_tangent(1)   # runs 1, 2, 3 all linearised about run 0
    s.set_state(0, x)
    s.set_state(1, d1)
    s.set_state(2, d2)
    s.set_state(3, _sum(d1, d2))
    s.Prepare()
    s.TimeStep(5)
    s.synchronize()
    for k in fields(cfg):
        j12 = s.get_field(3, k)
        assert rel_l2(s.get_field(1, k) + s.get_field(2, k), j12) < 1e-6, k


def test_set_tangent_rejects_bad_counts():
    import stratiflow_b200 as sf
    cfg = CONFIGS["kh2d"]
    s = gpu_solver(cfg, nrun=3)
    for bad in (-1, 2, 3, 4):
        with pytest.raises(sf.SFError):
            s.set_tangent(bad)
    s.set_tangent(1)
    s.set_tangent(0)
