"""GPU test of sf_step_host_async: a stream of independent states stepped
from host memory with the copies of neighbouring calls overlapping each
step. Every output must equal, bit for bit, the same input stepped through
the one-call-at-a-time path (sf_set_state_kept, sf_step, sf_get_state_kept):
the kernels and their inputs are the same, only the copies are reordered."""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_ic
from tests.test_gpu_parity import gpu_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_step_host_async_equals_one_call_at_a_time(name):
    cfg = CONFIGS[name]
    s = gpu_solver(cfg, nrun=2)
    ins = []
    for k in range(5):
        for r in range(2):
            s.set_state(r, make_ic(cfg, seed=100 + 2 * k + r, amp=5e-2))
        s.Prepare()
        ins.append(s.get_state_kept().copy())
    outs = [np.zeros_like(x) for x in ins]
    a = gpu_solver(cfg, nrun=2)
    for x, y in zip(ins, outs):
        a.step_host_async(x, y, 3)
    a.synchronize()
    for x, y in zip(ins, outs):
        s.set_state_kept(x)
        s.TimeStep(3)
        s.synchronize()
        assert np.array_equal(s.get_state_kept(), y)


def test_step_host_async_rejects_wrong_arrays():
    import stratiflow_b200 as sf
    cfg = CONFIGS["kh2d"]
    s = gpu_solver(cfg)
    good = np.zeros(s.kept_shape, dtype=np.complex64)
    with pytest.raises(sf.SFError):
        s.step_host_async(good.astype(np.complex128), good, 1)
    with pytest.raises(sf.SFError):
        s.step_host_async(good, good[..., :8].copy(), 1)
