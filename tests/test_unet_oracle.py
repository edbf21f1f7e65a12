"""The surrogate's oracle (float64 numpy U-Net) pinned on CPU: its analytic
backward pass agrees with central finite differences of its forward pass,
parameter by parameter, for a sample of parameters of every layer."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import unet_oracle as U  # noqa: E402


def test_unet_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    flat = np.concatenate([rng.normal(0, np.sqrt(2.0 / (9 * (1 if k == 'first.w' else s[1]))) if k.endswith('.w')
                                      and k != 'head.w' else 0.1, int(np.prod(s)))
                           for k, s in U.shapes().items()])
    P = U.unflatten(flat)
    x = rng.uniform(0, 1, (1, 16, 16))
    target = rng.normal(0, 1, (1, 16, 16, 6))
    wch = np.array([4.0, 1, 1, 1, 1, 1])
    scale = 1.0 / target.size

    def loss(Pd):
        out, _ = U.forward(Pd, x)
        return U.mse(out, target, wch, scale)[0]
    out, cache = U.forward(P, x)
    _, gout = U.mse(out, target, wch, scale)
    G = U.backward(P, cache, gout)
    for k, s in U.shapes().items():
        assert G[k].shape == tuple(s)
        for idx in [tuple(rng.integers(0, d) for d in s) for _ in range(3)]:
            h = 1e-5
            Pp = {q: v.copy() for q, v in P.items()}
            Pm = {q: v.copy() for q, v in P.items()}
            Pp[k][idx] += h
            Pm[k][idx] -= h
            fd = (loss(Pp) - loss(Pm)) / (2 * h)
            assert G[k][idx] == pytest.approx(fd, rel=1e-4, abs=1e-9), (k, idx)
