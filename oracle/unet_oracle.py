"""TEST INFRASTRUCTURE ONLY -- the oracle of the learned surrogate.

A float64 numpy restatement of the U-Net of clvisc_b200/surrogate.py (the
layer list, the parameter layout, the forward pass and the analytic backward
pass), used by the tests to check the CUDA kernels' forward outputs and
gradients. Its own backward pass is pinned against finite differences in
tests/test_unet_oracle.py. The product never imports it.
"""
import math

import numpy as np
from scipy.special import erf

C1, C2, C3, C4 = 32, 64, 128, 256
K_OUT = 6
LAYERS = [('e1b', C1, C1, 0), ('e2a', C1, C2, 1), ('e2b', C2, C2, 1), ('e3a', C2, C3, 2), ('e3b', C3, C3, 2),
          ('e4a', C3, C4, 3), ('e4b', C4, C4, 3), ('d3a', C4 + C3, C3, 2), ('d3b', C3, C3, 2),
          ('d2a', C3 + C2, C2, 1), ('d2b', C2, C2, 1), ('d1a', C2 + C1, C1, 0), ('d1b', C1, C1, 0)]


def shapes():
    s = {'first.w': (9, C1), 'first.b': (C1,)}
    for name, cin, cout, _ in LAYERS:
        s[name + '.w'] = (9, cin, cout)
        s[name + '.b'] = (cout,)
    s['head.w'] = (C1, K_OUT)
    s['head.b'] = (K_OUT,)
    return s


def unflatten(flat):
    out, n = {}, 0
    for k, s in shapes().items():
        m = int(np.prod(s))
        out[k] = np.asarray(flat[n:n + m], dtype=np.float64).reshape(s)
        n += m
    return out


def flatten(d):
    return np.concatenate([d[k].reshape(-1) for k in shapes()])


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def _shift(x, dy, dx):
    """x[n, h + dy, w + dx, c] with zeros outside the image."""
    N, H, W = x.shape[:3]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)) + ((0, 0),) * (x.ndim - 3))
    return xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv3x3(x, w, b=None):
    """z[p, co] = sum_{tap, ci} x[p + d_tap, ci] w[tap, ci, co] (+ b), zero padding."""
    z = 0.0
    for tap in range(9):
        z = z + _shift(x, tap // 3 - 1, tap % 3 - 1) @ w[tap]
    return z if b is None else z + b


def conv3x3_dgrad(g, w):
    """Gradient wrt x of conv3x3 given g = dL/dz."""
    gx = 0.0
    for tap in range(9):
        gx = gx + _shift(g @ w[tap].T, -(tap // 3 - 1), -(tap % 3 - 1))
    return gx


def conv3x3_wgrad(x, g):
    return np.stack([np.einsum('nhwc,nhwk->ck', _shift(x, tap // 3 - 1, tap % 3 - 1), g) for tap in range(9)])


def first(x, w, b):
    """1-channel image (N, H, W) -> C1 channels."""
    return conv3x3(x[..., None], w[:, None, :], b)


def pool(x):
    N, H, W, C = x.shape
    return x.reshape(N, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def pool_grad(g):
    return np.repeat(np.repeat(g, 2, axis=1), 2, axis=2) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_grad(g):
    N, H, W, C = g.shape
    return g.reshape(N, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def forward(P, x):
    """x (N, H, W) -> output (N, H, W, 6) and the cache of the backward pass."""
    c = {'x': x}
    c['z_first'] = first(x, P['first.w'], P['first.b'])
    c['y_first'] = gelu(c['z_first'])
    inputs = {}

    def layer(name, xin):
        inputs[name] = xin
        c['z_' + name] = conv3x3(xin, P[name + '.w'], P[name + '.b'])
        c['y_' + name] = gelu(c['z_' + name])
        return c['y_' + name]
    y1 = layer('e1b', c['y_first'])
    y2 = layer('e2b', layer('e2a', pool(y1)))
    y3 = layer('e3b', layer('e3a', pool(y2)))
    y4 = layer('e4b', layer('e4a', pool(y3)))
    d3 = layer('d3b', layer('d3a', np.concatenate([up(y4), y3], axis=-1)))
    d2 = layer('d2b', layer('d2a', np.concatenate([up(d3), y2], axis=-1)))
    d1 = layer('d1b', layer('d1a', np.concatenate([up(d2), y1], axis=-1)))
    c['inputs'] = inputs
    out = d1 @ P['head.w'] + P['head.b']
    return out, c


def backward(P, c, gout):
    """Gradients (same keys as P) for dL/d output = gout (N, H, W, 6)."""
    G = {}
    G['head.w'] = np.einsum('nhwc,nhwk->ck', c['y_d1b'], gout)
    G['head.b'] = gout.sum(axis=(0, 1, 2))
    gy = {'d1b': gout @ P['head.w'].T}

    def layer_back(name):
        gz = gy.pop(name) * gelu_grad(c['z_' + name])
        xin = c['inputs'][name]
        G[name + '.w'] = conv3x3_wgrad(xin, gz)
        G[name + '.b'] = gz.sum(axis=(0, 1, 2))
        return conv3x3_dgrad(gz, P[name + '.w'])

    def add(name, g):
        gy[name] = gy.get(name, 0.0) + g
    add('d1a', layer_back('d1b'))
    gcat = layer_back('d1a')
    add('d2b', up_grad(gcat[..., :C2]))
    add('e1b', gcat[..., C2:])
    add('d2a', layer_back('d2b'))
    gcat = layer_back('d2a')
    add('d3b', up_grad(gcat[..., :C3]))
    add('e2b', gcat[..., C3:])
    add('d3a', layer_back('d3b'))
    gcat = layer_back('d3a')
    add('e4b', up_grad(gcat[..., :C4]))
    add('e3b', gcat[..., C4:])
    add('e4a', layer_back('e4b'))
    add('e3b', pool_grad(layer_back('e4a')))
    add('e3a', layer_back('e3b'))
    add('e2b', pool_grad(layer_back('e3a')))
    add('e2a', layer_back('e2b'))
    add('e1b', pool_grad(layer_back('e2a')))
    gfirst_y = layer_back('e1b')
    gz = gfirst_y * gelu_grad(c['z_first'])
    G['first.w'] = conv3x3_wgrad(c['x'][..., None], gz)[:, 0, :]
    G['first.b'] = gz.sum(axis=(0, 1, 2))
    return G


def mse(out, target, wch, scale):
    d = out - target
    return float((wch * d * d).sum() * scale), 2.0 * wch * d * scale
