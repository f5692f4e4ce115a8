"""CPU checks of the predictor network's restatement (oracle/net_ref.py),
which the GPU tests use as their reference: BF16 rounding against torch's
(round to nearest even), and the FP64 gradient against central differences."""
import numpy as np
import torch

from oracle import net_ref as R


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(0, 1, 20000), rng.normal(0, 1e-3, 2000), rng.normal(0, 1e4, 2000),
                        [0.0, -0.0, 1.0, -1.0, 1.00390625, 1.01171875]]).astype(np.float32)
    ours = R.bf16_round(x)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours, ref)


def test_fp64_gradient_matches_central_differences():
    ch = [8, 8, 16, 8]
    Z, B = 7, 2
    rng = np.random.default_rng(5)
    p = R.init_params(ch, 7).astype(np.float64)
    x = rng.normal(0, 1, (B, Z, ch[0]))
    t = rng.normal(0, 1, (B, Z, ch[-1]))
    g, loss = R.gradient(p, ch, x, t, bf16=False)
    idx = rng.choice(p.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp = R.gradient(p + e, ch, x, t, bf16=False)[1]
        lm = R.gradient(p - e, ch, x, t, bf16=False)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])
