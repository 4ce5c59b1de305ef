"""The network oracle itself (CPU): its backward pass against central finite differences of its forward pass, and
its BF16 rounding against torch's."""
import numpy as np
import pytest

import nn_oracle as O


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = sum(9 * ci * co + co for ci, co in O.LAYERS) + 2 * (9 * 32 + 1)
    theta = rng.normal(0, 1, n) * 0.2
    x = rng.normal(0, 1, (1, 64, 64, 32))
    out, tape = O.net_forward(theta, x, quantize=False)
    dout = [rng.normal(0, 1, o.shape) for o in out]
    g = O.net_backward(theta, tape, dout)
    live = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())
    checked = 0
    for k in rng.choice(live, 6, replace=False):
        e = 1e-5
        tp, tm = theta.copy(), theta.copy()
        tp[k] += e
        tm[k] -= e
        op, om = O.net_forward(tp, x, False)[0], O.net_forward(tm, x, False)[0]
        fd = sum(((a - b) * d).sum() for a, b, d in zip(op, om, dout)) / (2 * e)
        assert abs(g[k] - fd) <= 1e-5 * abs(fd) + 1e-8
        checked += 1
    assert checked == 6


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-30, 100), [0.0, -0.0, 1.0, 3.0e38]])
    ref = torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(O.bf16(a), ref)
