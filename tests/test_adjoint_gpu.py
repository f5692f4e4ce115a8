"""GPU test of IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126; BuildRHSAdjoint,
IMEXRK.cpp:260-379; the mixing objective's forcing of
UpdateAdjointVariables, IMEXRK.h:461-500) against the FP64 oracle's
restatement: three adjoint steps between two direct snapshots, from the same
projected adjoint state, on a batch of two runs with different Ri.

Bound: 1e-5 relative L2 for u1, u3, b and 5e-4 for p, the parity tests'
bounds for the forward step."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu


def _kept(cfg, states):
    s = gpu_solver(cfg, nrun=len(states))
    for r, st in enumerate(states):
        s.set_state(r, st)
    return s.get_state_kept()


def test_adjoint_step_matches_oracle():
    cfg = CONFIGS["kh2d"]
    Ris = [cfg["Ri"], 0.2]
    below = [make_ic(cfg, seed=501 + r, amp=5e-2) for r in range(2)]
    above = [make_ic(cfg, seed=511 + r, amp=5e-2) for r in range(2)]
    adj = [make_ic(cfg, seed=521 + r, amp=1e-3) for r in range(2)]
    s = gpu_solver(cfg, nrun=2, Ri=Ris)
    for r in range(2):
        s.set_state(r, adj[r])
    s.Prepare()
    kb, ka = _kept(cfg, below), _kept(cfg, above)
    for _ in range(3):
        s.TimeStepAdjoint(kb, ka)
    for r in range(2):
        o = make_oracle(cfg, 64, Ri=Ris[r])
        o.set_state(adj[r])
        o.prepare()
        for _ in range(3):
            o.step_adjoint(below[r], above[r])
        for k in ("u1", "u3", "b"):
            assert rel_l2(s.get_field(r, k), o.get_field(k)) < 1e-5, (r, k)
        assert rel_l2(s.get_field(r, "p"), o.get_field("p")) < 5e-4, r


def test_adjoint_evolve_matches_oracle():
    """StateVector::AdjointEvolve (StateVector.cpp:158-187): 4 forward steps
    stored, then 4 adjoint steps back through them, against the same with the
    FP64 oracle (its own forward snapshots). Bound 1e-4: the FP32 forward
    snapshots differ from the FP64 ones by about 1e-6 and feed every adjoint
    step."""
    cfg = CONFIGS["kh2d"]
    x0 = make_ic(cfg, seed=531, amp=5e-2)
    aT = make_ic(cfg, seed=532, amp=1e-3)
    s = gpu_solver(cfg)
    out = s.AdjointEvolve(_kept(cfg, [x0]), _kept(cfg, [aT]), 4)
    o = make_oracle(cfg, 64)
    o.set_state(x0)
    o.prepare()
    snaps = [o.get_state()]
    for _ in range(4):
        o.step(1)
        snaps.append(o.get_state())
    o.set_state(aT)
    o.prepare()
    for step in range(4):
        o.step_adjoint(snaps[3 - step], snaps[4 - step])
    for k in ("u1", "u3", "b"):
        assert rel_l2(s.get_field(0, k), o.get_field(k)) < 1e-4, k
    assert out.shape == s.kept_shape


def test_adjoint_step_3d_matches_oracle():
    """The 3D adjoint step (y transforms of the 12 fields, the 16 products,
    the forward pass's 8 combinations) against the FP64 oracle on the
    64 x 32 x 64 grid, two steps."""
    cfg = CONFIGS["shear3d_small"]
    below = make_ic(cfg, seed=541, amp=5e-2)
    above = make_ic(cfg, seed=542, amp=5e-2)
    adj = make_ic(cfg, seed=543, amp=1e-3)
    s = gpu_solver(cfg)
    s.set_state(0, adj)
    s.Prepare()
    kb, ka = _kept(cfg, [below]), _kept(cfg, [above])
    for _ in range(2):
        s.TimeStepAdjoint(kb, ka)
    o = make_oracle(cfg, 64)
    o.set_state(adj)
    o.prepare()
    for _ in range(2):
        o.step_adjoint(below, above)
    for k in ("u1", "u2", "u3", "b"):
        assert rel_l2(s.get_field(0, k), o.get_field(k)) < 1e-5, k
    assert rel_l2(s.get_field(0, "p"), o.get_field("p")) < 5e-4


def test_optimal_mixing_step_matches_oracle():
    """One update of Adjoint.cpp (adjoint from a zero final state, gradient
    step on the energy sphere, Rescale) against the same arithmetic on the
    FP64 oracle's forward and adjoint integrations (numpy for the update)."""
    from stratiflow_b200 import drivers as D
    from tests.test_vecs_drivers_gpu import _flow
    cfg = CONFIGS["kh2d"]
    x0d = make_ic(cfg, seed=551, amp=5e-2)
    s = gpu_solver(cfg)
    x0 = _kept(cfg, [x0d])[0]
    new, info = D.optimal_mixing_step(s, x0, 3, 0.05)
    # the oracle
    o = make_oracle(cfg, 64)
    o.set_state(x0d)
    o.prepare()
    snaps = [o.get_state()]
    for _ in range(3):
        o.step(1)
        snaps.append(o.get_state())
    zero = {k: np.zeros_like(v) for k, v in x0d.items()}
    o.set_state(zero)
    o.prepare()
    for step in range(3):
        o.step_adjoint(snaps[2 - step], snaps[3 - step])
    adj = o.get_state()
    adj["b"] = adj["b"] / cfg["Ri"]
    flow = _flow(cfg)
    tmp = gpu_solver(cfg)
    def kept(st):
        tmp.set_state(0, st)
        return tmp.get_state_kept()[0].astype(np.complex128)
    xk, vk = kept(x0d), kept(adj)
    xk[4] = 0
    vk[4] = 0
    dot = lambda a, b: D.ext_dot(flow, (a, 0.0), (b, 0.0), cfg["Ri"])
    uu, uv, vv = dot(xk, xk), dot(xk, vk), dot(vk, vk)
    assert abs(info["udotv"] - uv) <= 1e-4 * np.sqrt(uu * vv)
    eps = 0.05
    lam = 0.0
    while lam == 0.0:
        lam = D.solve_quadratic(eps * uu, 2 * eps * uv - 2 * uu, eps * vv - 2 * uv)
        if lam == 0.0:
            eps /= 2
    assert abs(info["lambda"] - lam) <= 1e-3 * abs(lam)
    res = xk - eps * (vk + lam * xk)
    # Rescale on the oracle: project, scale to the energy of x0, project
    tmp.set_state_kept(res[None].astype(np.complex64))
    tmp.Prepare()
    r1 = tmp.get_state_kept()[0].astype(np.complex128)
    r1[4] = 0
    r1 *= np.sqrt(0.5 * uu / (0.5 * dot(r1, r1)))
    tmp.set_state_kept(r1[None].astype(np.complex64))
    tmp.Prepare()
    want = tmp.get_state_kept()[0]
    for f in (0, 2, 3):
        assert rel_l2(new[f], want[f]) < 1e-4, f
