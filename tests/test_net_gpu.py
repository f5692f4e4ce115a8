"""GPU tests of the learned predictor's kernels (sf_net_*): forward pass and
gradients against the CPU restatement oracle/net_ref.py with the same BF16
rounding points and FP64 accumulation.

Bounds: the GPU accumulates in FP32, so an intermediate activation whose FP32
sum lands on the other side of a BF16 rounding boundary than the FP64 sum
differs by one BF16 ulp (2^-8 relative); such flips are rare and bound the
agreement: forward output <= 2e-3 and each layer's weight gradient <= 1e-2
relative L2 (the output layer's, before any flip can reach it, <= 1e-4).
"""
import numpy as np
import pytest

from oracle import net_ref as R
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _net(ch, Z, B, seed=11):
    import stratiflow_b200 as sf
    n = sf.Net(ch, Z, B, seed=seed)
    p = R.init_params(ch, seed)
    n.set_params(p)
    return n, p


def test_forward_matches_cpu():
    ch = [32, 64, 64, 48]
    Z, B = 40, 3
    n, p = _net(ch, Z, B)
    x = np.random.default_rng(1).normal(0, 1, (B, Z, ch[0])).astype(np.float32)
    y = n.forward(x)
    ref, _ = R.forward(p, ch, x)
    assert rel_l2(y, ref) < 2e-3


def test_gradient_matches_cpu():
    ch = [32, 64, 64, 48]
    Z, B = 40, 3
    n, p = _net(ch, Z, B)
    rng = np.random.default_rng(2)
    x = rng.normal(0, 1, (B, Z, ch[0])).astype(np.float32)
    t = rng.normal(0, 1, (B, Z, ch[-1])).astype(np.float32)
    n.set_data(x, t)
    g, loss = n.gradient()
    gr, lr = R.gradient(p, ch, x, t)
    assert abs(loss - lr) <= 1e-4 * lr
    off = 0
    for l, (ci, co) in enumerate(zip(ch[:-1], ch[1:])):
        nw = co * 5 * ci
        tol = 1e-4 if l == len(ch) - 2 else 1e-2
        assert rel_l2(g[off:off + nw], gr[off:off + nw]) < tol, l
        assert rel_l2(g[off + nw:off + nw + co], gr[off + nw:off + nw + co]) < tol, l
        off += nw + co


def test_training_lowers_the_loss():
    import stratiflow_b200 as sf
    ch = [16, 32, 32, 16]
    Z, B = 32, 4
    n = sf.Net(ch, Z, B, seed=3)
    rng = np.random.default_rng(4)
    x = rng.normal(0, 1, (B, Z, ch[0])).astype(np.float32)
    # a target the network can represent: a fixed smooth map of the input
    t = np.tanh(0.5 * x[:, :, :16] + 0.25 * np.roll(x[:, :, :16], 1, axis=1)).astype(np.float32)
    n.set_data(x, t)
    losses = n.train(300, 3e-3)
    assert losses[-1] < 0.05 * losses[0]
    # the trained parameters reproduce the trained loss on the CPU
    _, lr = R.gradient(n.get_params(), ch, x, t)
    g, lg = n.gradient()
    assert abs(lg - lr) <= 1e-2 * lr


def test_predictor_sized_net_forward():
    """The continuation predictor's own shape: 1024 -> 256 -> 256 -> 256 -> 512
    channels over Z = 256 levels (about 2.3 M parameters)."""
    ch = [1024, 256, 256, 256, 512]
    Z, B = 256, 2
    n, p = _net(ch, Z, B)
    assert n.num_params == sum(co * 5 * ci + co for ci, co in zip(ch[:-1], ch[1:]))
    x = np.random.default_rng(6).normal(0, 1, (B, Z, ch[0])).astype(np.float32)
    y = n.forward(x)
    ref, _ = R.forward(p, ch, x)
    assert rel_l2(y, ref) < 2e-3
