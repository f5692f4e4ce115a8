"""The other z-pass kernels against k_z_step (sf_set_z_kernel 0):
k_z_step_tma (kind 1: each warp brings its first Thomas sweeps' inputs into
a shared-memory ring with tensor-map copies, the sweeps' intermediates live
in tensor memory), the same chunked solve with the same terms in the same
order; and k_z_step_c (kind 2: one lane per complex mode in packed FP32, two
z-chunks per warp: 16 chunks in blocks of 8 warps, 32 in blocks of 16
warps on the grids here that leave SMs idle), the same terms, with the
recurrences split into more chunks. The states agree to the bits
the compilations round differently: for kind 1, 1e-6 relative L2 per field
after 4 steps (5e-5 for p); for kind 2, whose chunking reassociates every
recurrence, to the parity tests' bound against the FP64 oracle (1e-5 per
field, 5e-4 for p; measured about 1e-6). Checked in 2D and 3D, on nonlinear,
frozen-base linear and tangent-linear batches, with the adjoint step, and
with grids whose last chunk is shorter than the others."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic, rel_l2
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu


def _run(name, kind, nrun, mode, steps=4):
    cfg = CONFIGS[name]
    s = gpu_solver(cfg, nrun=nrun)
    if kind in (0, 1):
        s.set_z_chunks(8)   # the tensor-map kernel takes 8 chunks; the baseline the same
    s.set_z_kernel(kind)
    for r in range(nrun):
        s.set_state(r, make_ic(cfg, seed=800 + r, amp=5e-2 if r == 0 else 1e-3))
    if mode == "linear":
        b = make_ic(cfg, seed=899, amp=5e-2)
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
    out = s.get_state_kept()
    s.close()
    return out


def _agree(a, b, kind=1):
    tol, ptol = (1e-6, 5e-5) if kind == 1 else (1e-5, 5e-4)
    for f in range(a.shape[1]):
        err = rel_l2(b[:, f], a[:, f])
        assert err <= (ptol if f == 4 else tol), (f, err)


CASES = [
    ("lin2d", 1, "nonlinear"),
    ("kh2d", 2, "nonlinear"),
    ("kh2d", 2, "tangent"),
    ("shear3d_small", 1, "nonlinear"),
    ("shear3d_small", 2, "linear"),
    ("shear3d", 1, "nonlinear"),
]


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("name,nrun,mode", CASES)
def test_z_pass_kernels_agree_with_the_z_step(name, nrun, mode, kind):
    _agree(_run(name, 0, nrun, mode), _run(name, kind, nrun, mode), kind)


@pytest.mark.parametrize("n3", [100, 36])
def test_complex_lane_z_pass_with_uneven_chunks(n3):
    """k_z_step_c's chunk bounds and end tests against k_z_step: N3 = 100
    gives 16 chunks of 7 levels, the last of 5; N3 = 36 gives 12 chunks of 3
    levels and 4 empty ones (two warps with no levels, which still take part
    in the chunk scans)."""
    name = f"_kh2d_{n3}"
    CONFIGS[name] = dict(CONFIGS["kh2d"], N3=n3)
    try:
        _agree(_run(name, 0, 1, "nonlinear"), _run(name, 2, 1, "nonlinear"), 2)
    finally:
        del CONFIGS[name]


@pytest.mark.parametrize("kind", [1, 2])
def test_z_pass_kernels_agree_in_the_adjoint_step(kind):
    cfg = CONFIGS["kh2d"]

    def run(kind):
        def kept(states):
            k = gpu_solver(cfg, nrun=len(states))
            for r, st in enumerate(states):
                k.set_state(r, st)
            out = k.get_state_kept()
            k.close()
            return out
        below = kept([make_ic(cfg, seed=851 + r, amp=5e-2) for r in range(2)])
        above = kept([make_ic(cfg, seed=861 + r, amp=5e-2) for r in range(2)])
        s = gpu_solver(cfg, nrun=2)
        if kind in (0, 1):
            s.set_z_chunks(8)
        s.set_z_kernel(kind)
        for r in range(2):
            s.set_state(r, make_ic(cfg, seed=871 + r, amp=1e-3))
        s.Prepare()
        for _ in range(3):
            s.TimeStepAdjoint(below, above)
        s.synchronize()
        out = s.get_state_kept()
        s.close()
        return out
    _agree(run(0), run(kind), kind)


@pytest.mark.parametrize("warps", [8, 16])
def test_complex_lane_z_pass_block_sizes(warps):
    """k_z_step_c with 8 warps (16 chunks) and 16 warps (32 chunks) per block,
    forced through sf_set_z_chunks, on the 3D grid 64 x 32 x 64 with two
    runs, against k_z_step."""
    cfg = CONFIGS["shear3d_small"]

    def run(kind, z):
        s = gpu_solver(cfg, nrun=2)
        s.set_z_kernel(kind)
        s.set_z_chunks(z)
        for r in range(2):
            s.set_state(r, make_ic(cfg, seed=880 + r, amp=5e-2))
        s.Prepare()
        s.TimeStep(4)
        s.synchronize()
        out = s.get_state_kept()
        s.close()
        return out
    _agree(run(0, 8), run(2, warps), 2)

