"""The x pass gives the same step however many z-slabs one block walks
through (sf_set_xpass_slabs): a block that carries the shared levels from one
slab to the next keeps rows another block would form again. Not bit for bit:
the forward transforms take two real product rows per complex FFT, and a
carried row changes which rows are paired, which moves the last FP32 bit of
the transformed rows; after 4 steps the runs agree to the parity tests'
tolerance (1e-5 relative L2 per field, 5e-4 for p). Checked on nonlinear,
frozen-base linear and tangent-linear batches, with slab counts that leave
the last block of a column partly past the top."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, rel_l2
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu


def _run(name, slabs, nrun=1, mode="nonlinear", steps=4):
    cfg = CONFIGS[name]
    s = gpu_solver(cfg, nrun=nrun)
    s.set_xpass_slabs(slabs)
    for r in range(nrun):
        s.set_state(r, make_ic(cfg, seed=300 + r, amp=5e-2 if r == 0 else 1e-3))
    if mode == "linear":
        b = make_ic(cfg, seed=399, amp=5e-2)
        for r in range(nrun):
            s.SetBase(r, b["u1"], b["u2"], b["u3"], b["b"])
    if mode == "tangent":
        s.set_tangent(1)
    s.Prepare()
    if mode == "linear":
        s.TimeStepLinear(steps)
    else:
        s.TimeStep(steps)
    s.synchronize()
    return s.get_state_kept()


@pytest.mark.parametrize("name,nrun,mode,slabs", [
    ("kh2d", 2, "nonlinear", 5),
    ("shear3d_small", 1, "nonlinear", 3),
    ("shear3d_small", 1, "linear", 3),
    ("kh2d", 2, "tangent", 7),
    ("shear3d_small", 2, "tangent", 2),
])
def test_slabs_per_block_do_not_change_the_step(name, nrun, mode, slabs):
    one = _run(name, 1, nrun, mode)
    many = _run(name, slabs, nrun, mode)
    for r in range(nrun):
        for f in range(5):
            tol = 5e-4 if f == 4 else 1e-5
            assert rel_l2(many[r, f], one[r, f]) < tol, (r, f, rel_l2(many[r, f], one[r, f]))


@pytest.mark.parametrize("name,nrun,mode,bands", [
    ("shear3d_small", 1, "nonlinear", 3),
    ("shear3d_small", 2, "nonlinear", 8),
    ("shear3d_small", 1, "linear", 2),
    ("shear3d", 1, "nonlinear", 4),
])
def test_xy_bands_give_the_same_step_bit_for_bit(name, nrun, mode, bands):
    """The banded 3D x-y pass (y transforms of other bands on side streams)
    runs every block and column exactly as the one-band pass does, so the
    step is bit-identical; the band count is a launch setting only."""
    def run(b):
        cfg = CONFIGS[name]
        s = gpu_solver(cfg, nrun=nrun)
        s.set_xy_bands(b)
        for r in range(nrun):
            s.set_state(r, make_ic(cfg, seed=500 + r))
        if mode == "linear":
            base = make_ic(cfg, seed=599, amp=5e-2)
            for r in range(nrun):
                s.SetBase(r, base["u1"], base["u2"], base["u3"], base["b"])
        s.Prepare()
        (s.TimeStepLinear if mode == "linear" else s.TimeStep)(3)
        s.synchronize()
        out = s.get_state_kept()
        s.close()
        return out
    one, many = run(1), run(bands)
    assert np.array_equal(one, many)


@pytest.mark.parametrize("name,nrun,bands", [
    ("shear3d_small", 1, 1),
    ("shear3d_small", 2, 3),
    ("shear3d", 1, 1),
])
def test_marching_x_pass_agrees_with_the_slab_x_pass(name, nrun, bands):
    """The 3D nonlinear x pass as level-marching lane groups (the default,
    sf_set_xpass_kernel 1) and as slab blocks (0) form the same products and
    transforms; they differ in the order the z stencils' terms are summed and
    in the packed two-transform FFT's rounding, so after 4 steps the states
    agree to the parity tests' tolerance (1e-5 relative L2 per field, 5e-4
    for p), with several runs and with the level bands of the x-y pass."""
    def run(kind):
        cfg = CONFIGS[name]
        s = gpu_solver(cfg, nrun=nrun)
        s.set_xpass_kernel(kind)
        s.set_xy_bands(bands)
        for r in range(nrun):
            s.set_state(r, make_ic(cfg, seed=700 + r, amp=5e-2 if r == 0 else 1e-3))
        s.Prepare()
        s.TimeStep(4)
        s.synchronize()
        out = s.get_state_kept()
        s.close()
        return out
    slab, march = run(0), run(1)
    for r in range(nrun):
        for f in range(5):
            tol = 5e-4 if f == 4 else 1e-5
            assert rel_l2(march[r, f], slab[r, f]) < tol, (r, f, rel_l2(march[r, f], slab[r, f]))
