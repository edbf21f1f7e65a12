"""The surrogate's CUDA kernels (BF16 tensor-core convolutions on tcgen05 with
the accumulator in tensor memory and TMA- or cp.async-staged operands, or on
mma.sync; FP32 accumulation) against the float64 oracle (oracle/unet_oracle.py, itself
checked by finite differences): single layers with channel slices, bias,
GELU and gate; the weight gradient; the whole network's output and every
parameter's gradient; and training that lowers the loss. BF16 activations and
weights bound the agreement to about 1e-2 relative."""
import ctypes
import os
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
import unet_oracle as U  # noqa: E402

pytestmark = pytest.mark.gpu


def _bf(a):
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.fixture(params=[1, 2, 3, 0], ids=['tcgen05', 'tcgen05-noswizzle', 'tcgen05-conv-only', 'mma.sync'])
def conv_path(request, cuda_lib):
    from clvisc_b200 import _lib
    lib = _lib.load()
    _lib.check(lib.clv_unet_set_conv_path(request.param), 'set_conv_path')
    yield request.param
    _lib.check(lib.clv_unet_set_conv_path(1), 'set_conv_path')


def _timeouts(lib):
    n = ctypes.c_int()
    assert lib.clv_unet_timeouts(ctypes.byref(n), 1) == 0
    return n.value


@pytest.mark.parametrize('cin,cout,gelu,gate', [(64, 96, True, False), (96, 64, False, True), (32, 256, True, True),
                                                (384, 128, True, False), (128, 32, False, False)])
def test_conv3x3_layer(cuda_lib, conv_path, cin, cout, gelu, gate):
    from clvisc_b200 import _lib
    from clvisc_b200.surrogate import UnetConv
    lib = _lib.load()
    rng = np.random.default_rng(cin + cout)
    N, H, W = 2, 24, 16
    cs, co = cin + 32, 32  # the input is a slice of a wider buffer
    xb = _bf(rng.normal(0, 1, (N, H, W, cs))).cuda()
    w = _bf(rng.normal(0, 0.1, (9, cin, cout))).cuda()
    bias = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32)).cuda()
    gz = _bf(rng.normal(0, 1, (N, H, W, cout))).cuda() if gate else None
    out = torch.zeros((N, H, W, cout + 2), dtype=torch.bfloat16, device='cuda')
    pre = torch.zeros((N, H, W, cout), dtype=torch.bfloat16, device='cuda')
    a = UnetConv()
    a.in_, a.in_cs, a.in_co = xb.data_ptr(), cs, co
    a.w, a.bias = w.data_ptr(), bias.data_ptr()
    a.out, a.out_cs, a.out_co = out.data_ptr(), cout + 2, 2
    a.pre = pre.data_ptr()
    if gate:
        a.gate, a.gate_cs, a.gate_co = gz.data_ptr(), cout, 0
    a.N, a.H, a.W, a.Cin, a.Cout, a.gelu = N, H, W, cin, cout, int(gelu)
    _lib.check(lib.clv_unet_conv3x3(ctypes.byref(a), None), 'conv')
    torch.cuda.synchronize()
    z = U.conv3x3(_np(xb)[..., co:co + cin], _np(w), _np(bias))
    if gate:
        z = z * U.gelu_grad(_np(gz))
    assert _rel(_np(pre), z) < 1e-2
    y = U.gelu(z) if gelu else z
    assert _rel(_np(out)[..., 2:], y) < 1e-2
    assert (out[..., :2] == 0).all()  # outside the output slice: untouched
    assert _timeouts(lib) == 0


@pytest.mark.parametrize('N,H,W', [(3, 10, 13), (2, 8, 32), (1, 2, 256)])
def test_conv3x3_paths_agree(cuda_lib, N, H, W):
    """The tcgen05 paths and mma.sync give the same convolution up to the
    order of the FP32 accumulation (BF16 outputs: a few units in the last
    place), for every output-channel tile width: on a ragged pixel count (not
    a multiple of the 128-pixel tile: operands by cp.async) and on images that
    tile into 128-pixel blocks of 4 x 32 and 1 x 128 pixels (operands by TMA,
    swizzled and not)."""
    from clvisc_b200 import _lib
    from clvisc_b200.surrogate import UnetConv
    lib = _lib.load()
    rng = np.random.default_rng(3)
    outs = {}
    for cout in (32, 64, 128, 192):
        cin = 64
        xb = _bf(rng.normal(0, 1, (N, H, W, cin))).cuda()
        w = _bf(rng.normal(0, 0.1, (9, cin, cout))).cuda()
        bias = torch.from_numpy(rng.normal(0, 0.1, cout).astype(np.float32)).cuda()
        for path in (1, 2, 0):
            _lib.check(lib.clv_unet_set_conv_path(path), 'set_conv_path')
            out = torch.zeros((N, H, W, cout), dtype=torch.bfloat16, device='cuda')
            a = UnetConv()
            a.in_, a.in_cs, a.in_co = xb.data_ptr(), cin, 0
            a.w, a.bias = w.data_ptr(), bias.data_ptr()
            a.out, a.out_cs, a.out_co = out.data_ptr(), cout, 0
            a.N, a.H, a.W, a.Cin, a.Cout, a.gelu = N, H, W, cin, cout, 1
            _lib.check(lib.clv_unet_conv3x3(ctypes.byref(a), None), 'conv')
            torch.cuda.synchronize()
            outs[(cout, path)] = _np(out)
        _lib.check(lib.clv_unet_set_conv_path(1), 'set_conv_path')
        assert _rel(outs[(cout, 1)], outs[(cout, 0)]) < 4e-3, cout
        assert _rel(outs[(cout, 2)], outs[(cout, 0)]) < 4e-3, cout
    assert _timeouts(lib) == 0


@pytest.mark.parametrize('cin,cout', [(32, 32), (96, 64), (128, 256), (192, 32)])
@pytest.mark.parametrize('N,H,W', [(3, 16, 24), (2, 8, 32), (2, 8, 16), (1, 2, 64)])
def test_wgrad3x3(cuda_lib, conv_path, cin, cout, N, H, W):
    """Weight gradient against the oracle; on the default path, images whose
    pixels tile into 64-pixel blocks (W = 32, 16, 64 here) take the TMA +
    tcgen05 kernel, the others (W = 24) the mma.sync kernel."""
    from clvisc_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(7)
    xb = _bf(rng.normal(0, 1, (N, H, W, cin + 64))).cuda()
    g = _bf(rng.normal(0, 1, (N, H, W, cout))).cuda()
    dw = torch.zeros(9 * cin * cout, device='cuda')
    nbytes = int(lib.clv_unet_wgrad_scratch_bytes(N, H, W, cin, cout))
    scratch = torch.empty(nbytes // 4 + 1, device='cuda')
    _lib.check(lib.clv_unet_wgrad3x3(ctypes.c_void_p(xb.data_ptr()), cin + 64, 64, ctypes.c_void_p(g.data_ptr()),
                                     N, H, W, cin, cout, ctypes.c_void_p(dw.data_ptr()), 0,
                                     ctypes.c_void_p(scratch.data_ptr()), nbytes, None), 'wgrad')
    torch.cuda.synchronize()
    want = U.conv3x3_wgrad(_np(xb)[..., 64:], _np(g))
    assert _rel(dw.cpu().numpy().reshape(9, cin, cout), want) < 1e-5
    assert _timeouts(lib) == 0


@pytest.fixture(scope='module')
def net_and_ref(cuda_lib):
    from clvisc_b200.surrogate import UNet
    net = UNet(2, 32, 32, seed=5)
    rng = np.random.default_rng(11)
    x = rng.uniform(0, 1, (2, 32, 32)).astype(np.float32)
    target = rng.normal(0, 1, (2 * 32 * 32, 6)).astype(np.float32)
    return net, x, target


def test_unet_forward_and_gradients(net_and_ref, conv_path):
    net, x, target = net_and_ref
    wch = torch.tensor([4.0, 1, 1, 1, 1, 1], device='cuda')
    net.forward(torch.from_numpy(x).cuda())
    loss = float(net.loss(torch.from_numpy(target).cuda(), wch))
    net.grads.zero_()
    net.backward()
    torch.cuda.synchronize()
    P = U.unflatten(net.params.cpu().numpy())
    out_ref, cache = U.forward(P, x.astype(np.float64))
    lref, gout = U.mse(out_ref.reshape(-1, 6), target, np.array([4.0, 1, 1, 1, 1, 1]), 1.0 / target.size)
    assert _rel(net.buf['out'].cpu().numpy(), out_ref.reshape(-1, 6)) < 2e-2
    assert loss == pytest.approx(lref, rel=2e-2)
    G = U.backward(P, cache, gout.reshape(out_ref.shape))
    got = U.unflatten(net.grads.cpu().numpy())
    for k in U.shapes():
        a, b = got[k].reshape(-1), G[k].reshape(-1)
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
        assert _rel(a, b) < 6e-2 and cos > 0.998, (k, _rel(a, b), cos)


def test_unet_training_lowers_loss(cuda_lib):
    """Adam on the device fits a smooth map of the input (a blurred and
    squared copy per channel) and lowers the loss by a large factor."""
    from clvisc_b200.surrogate import UNet
    net = UNet(8, 32, 32, seed=2)
    rng = np.random.default_rng(4)
    xs = torch.from_numpy(rng.uniform(0, 1, (64, 32, 32)).astype(np.float32)).cuda()
    k = torch.ones(1, 1, 5, 5, device='cuda') / 25.0
    blur = torch.nn.functional.conv2d(xs[:, None], k, padding=2)[:, 0]
    ys = torch.stack([blur, blur ** 2, xs, -blur, 0.5 * xs, blur * xs], dim=-1).contiguous()
    wch = torch.ones(6, device='cuda')
    losses = []
    for step in range(240):
        i = (step * 8) % 64
        net.forward(xs[i:i + 8])
        losses.append(float(net.loss(ys[i:i + 8].reshape(-1, 6), wch)))
        net.grads.zero_()
        net.backward()
        net.adam(2e-3)
    assert np.mean(losses[-8:]) < 0.05 * np.mean(losses[:8])
