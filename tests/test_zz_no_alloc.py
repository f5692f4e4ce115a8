"""GPU test of sf_remove_divergence_noalloc, the pressure projection for
callers that cannot allocate device memory (a host that only lends this
library pre-sized buffers from its own pool, or a loop that must never enter
the allocator). Its working memory is a fixed device array inside the
library; this test allocates the caller's buffers itself, calls the entry
point through the C-ABI twice in a row, and checks each result against
sf_remove_divergence on a solver holding the same state.

This file is collected last so that a run which stops at the first failure
has already run every other test; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, rel_l2

pytestmark = pytest.mark.gpu

# the tolerances of the parity tests: 1e-5 for the velocity fields and 5e-4
# for p, whose increment q comes from an FP32 solve of the ill-conditioned
# Laplacian and so carries rounding that differs between any two codes
TOL = 1e-5
TOL_P = 5e-4


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
    """A seeded state that is not divergence-free, with a non-zero p."""
    ic = make_ic(cfg, seed=seed)
    st = {k: v * (1.0 + 0.1j) for k, v in ic.items()}
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
    for call, (seed, pm) in enumerate(((21, 0.5), (22, 2.0))):
        s.set_state(0, _unprojected_state(cfg, seed))
        kept = s.get_state_kept()[0]                  # [5][N3][plane] complex64
        # the caller's own device buffers (allocated here, by the caller)
        buf = [torch.from_numpy(np.ascontiguousarray(kept[f]).view(np.float32).copy()).to(dev)
               for f in range(5)]
        pout = torch.empty_like(buf[4])
        s.RemoveDivergence(pm)
        s.synchronize()
        ref = s.get_state_kept()[0]
        torch.cuda.synchronize()
        u2 = ptr(buf[1]) if cfg["N2"] > 1 else None
        rc = L.sf_remove_divergence_noalloc(C.byref(grid), C.byref(flow), pm, ptr(buf[0]), u2, ptr(buf[2]),
                                            ptr(buf[4]), ptr(pout), None)
        assert rc == 0, L.sf_last_error().decode()
        torch.cuda.synchronize()
        got = {f: buf[{"u1": 0, "u2": 1, "u3": 2}[f]] for f in names}
        got["p"] = pout
        for f, t in got.items():
            i = {"u1": 0, "u2": 1, "u3": 2, "p": 4}[f]
            g = t.cpu().numpy().view(np.complex64).reshape(ref[i].shape)
            tol = TOL_P if f == "p" else TOL
            assert rel_l2(g, ref[i]) < tol, (call, f, rel_l2(g, ref[i]))


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
