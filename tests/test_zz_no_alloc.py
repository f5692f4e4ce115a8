"""GPU test of sf_remove_divergence_noalloc, the pressure projection for
callers that cannot allocate device memory (a host that only lends this
library pre-sized buffers from its own pool, or a loop that must never enter
the allocator). Its working memory is a fixed device array inside the
library; this test allocates the caller's buffers itself, calls the entry
point through the C-ABI twice in a row, and checks each result against
sf_remove_divergence on a solver holding the same state and against the
FP64 oracle's RemoveDivergence (IMEXRK.cpp:43-73).

The input really has divergence: u1 alone of a divergence-free field is
scaled, so the projection changes u3 by 15-25% and p by ~100%; a wrong solve
cannot pass.

This file is collected last so that a run which stops at the first failure
has already run every other test; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2

pytestmark = pytest.mark.gpu

# velocities: 1e-5 relative L2, the parity tests' bound. p against the other
# GPU entry point: 5e-4 (the two FP32 solves of the ill-conditioned Laplacian
# round differently); p against the FP64 oracle: 1e-4, about 8x the FP32
# oracle's own deviation from FP64 on these inputs (1.2e-5)
TOL = 1e-5
TOL_P = 5e-4
TOL_P64 = 1e-4


def _solver(cfg):
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import background_profile
    s = sf.IMEXRK(cfg["N1"], cfg["N2"], cfg["N3"], cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Pr"],
                  cfg["dt"])
    U, dB = background_profile(cfg["bg"], cfg["L3"], cfg["N3"])
    s.set_ri(0, cfg["Ri"])
    s.SetBackground(0, U, dB)
    return s


def _unprojected_state(cfg, seed):
    """A seeded state with divergence (u1 of a projected field scaled by 1.5)
    and a non-zero p."""
    ic = make_ic(cfg, seed=seed)
    st = dict(ic)
    st["u1"] = 1.5 * ic["u1"]
    st["p"] = 1e-3 * ic["u1"]
    return st


@pytest.mark.parametrize("name", ["nk2d", "shear3d_small"])
def test_noalloc_matches_remove_divergence_twice(name):
    import torch
    import stratiflow_b200 as sf
    L = sf.load_library()
    cfg = CONFIGS[name]
    s = _solver(cfg)
    dev = torch.device("cuda", 0)
    grid = sf._Grid(cfg["N1"], cfg["N2"], cfg["N3"], 1)
    flow = sf._Flow(cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Pr"])
    ptr = lambda t: C.c_void_p(t.data_ptr())
    names = ["u1", "u2", "u3"] if cfg["N2"] > 1 else ["u1", "u3"]
    idx = {"u1": 0, "u2": 1, "u3": 2, "p": 4}
    for call, (seed, pm) in enumerate(((21, 0.5), (22, 2.0))):
        st = _unprojected_state(cfg, seed)
        s.set_state(0, st)
        kept = s.get_state_kept()[0]                  # [5][N3][plane] complex64
        # the caller's own device buffers (allocated here, by the caller)
        buf = [torch.from_numpy(np.ascontiguousarray(kept[f]).view(np.float32).copy()).to(dev)
               for f in range(5)]
        pout = torch.empty_like(buf[4])
        s.RemoveDivergence(pm)
        s.synchronize()
        ref = s.get_state_kept()[0]
        ref_full = {f: s.get_field(0, f) for f in names + ["p"]}
        torch.cuda.synchronize()
        u2 = ptr(buf[1]) if cfg["N2"] > 1 else None
        rc = L.sf_remove_divergence_noalloc(C.byref(grid), C.byref(flow), pm, ptr(buf[0]), u2, ptr(buf[2]),
                                            ptr(buf[4]), ptr(pout), None)
        assert rc == 0, L.sf_last_error().decode()
        torch.cuda.synchronize()
        got = {f: buf[idx[f]] for f in names}
        got["p"] = pout
        # the projection did real work on this input
        assert rel_l2(ref_full["u3"], st["u3"]) > 0.1, (call, rel_l2(ref_full["u3"], st["u3"]))
        assert rel_l2(ref_full["p"], st["p"]) > 0.5
        for f, t in got.items():
            g = t.cpu().numpy().view(np.complex64).reshape(ref[idx[f]].shape)
            tol = TOL_P if f == "p" else TOL
            assert rel_l2(g, ref[idx[f]]) < tol, (call, f, rel_l2(g, ref[idx[f]]))
        # and both equal the FP64 oracle's projection, in the reference layout
        o = make_oracle(cfg, 64)
        o.set_state(st)
        o.remove_divergence(pm)
        mine = ref.copy()
        for f, t in got.items():
            mine[idx[f]] = t.cpu().numpy().view(np.complex64).reshape(ref[idx[f]].shape)
        s.set_state_kept(mine[None])
        for f in names + ["p"]:
            e = rel_l2(s.get_field(0, f), o.get_field(f))
            assert e < (TOL_P64 if f == "p" else TOL), (call, f, "vs FP64 oracle", e)


def test_noalloc_rejects_grids_beyond_its_fixed_memory():
    import stratiflow_b200 as sf
    L = sf.load_library()
    cfg = CONFIGS["shear3d"]   # 256 x 128 x 384: N3 * plane far above the limit
    grid = sf._Grid(cfg["N1"], cfg["N2"], cfg["N3"], 1)
    flow = sf._Flow(cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Pr"])
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = L.sf_remove_divergence_noalloc(C.byref(grid), C.byref(flow), 1.0, dummy, dummy, dummy, dummy, dummy,
                                        None)
    assert rc == -1
    assert "too large" in L.sf_last_error().decode()
