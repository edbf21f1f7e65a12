"""The allocation-free surface finder, clv_hypersf_append_noalloc, for callers
that cannot allocate device memory (an application whose own pool owns the
device, or a loop that cannot afford the device synchronisation a cudaMalloc
may cause). It is called through the C ABI and must append exactly what
clv_hypersf_append appends for the same inputs, over two calls in a row (the
second call reuses the library's fixed scratch array). This file is named so
that pytest collects it last."""
import ctypes

import numpy as np
import pytest
import torch

from parity_util import make_cfg, seeded_ic

pytestmark = pytest.mark.gpu


def _run_finder(lib, v, noalloc, cap):
    """Two appends (steps 0->5 and 5->10 of a viscous run) into fresh buffers."""
    from clvisc_b200 import _lib
    dev = v.device
    dt = v.dtype
    sf = torch.full((cap, 8), float('nan'), dtype=dt, device=dev)
    tx = torch.full((cap, 4), float('nan'), dtype=dt, device=dev)
    pisf = torch.full((cap, 10), float('nan'), dtype=dt, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    snaps = v._snaps
    for (t_old, ev_old, pi_old), (t_new, ev_new, pi_new) in zip(snaps[:-1], snaps[1:]):
        args = [ctypes.byref(v.params), 1, float(t_old), float(t_new), _lib.ptr(ev_old), _lib.ptr(ev_new),
                _lib.ptr(pi_old), _lib.ptr(pi_new), _lib.ptr(sf), _lib.ptr(tx), _lib.ptr(pisf), cap, _lib.ptr(total)]
        if noalloc:
            rc = lib.clv_hypersf_append_noalloc(*args, stream)
        else:
            scratch = torch.empty(int(lib.clv_hypersf_scratch_bytes(ctypes.byref(v.params))), dtype=torch.uint8,
                                  device=dev)
            rc = lib.clv_hypersf_append(*args, _lib.ptr(scratch), scratch.numel(), stream)
        _lib.check(rc, 'hypersf')
    torch.cuda.synchronize()
    n = int(total.item())
    return n, sf[:n].cpu().numpy(), tx[:n].cpu().numpy(), pisf[:n].cpu().numpy()


@pytest.mark.parametrize('use_float32', [True, False])
def test_noalloc_matches_scratch_finder(cuda_lib, use_float32):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(25, 23, 13, use_float32=use_float32, dx=0.8, dz=0.6, dt=0.04, skip=(2, 2, 1))
    v = CLVisc(cfg)
    v.load_ini(seeded_ic(cfg, seed=11, edmax=20.0))
    v._snaps = [(cfg.real(cfg.TAU0), v.ideal.d_ev[1].clone(), v.d_pi[1].clone())]
    for n in range(20):
        v.step(n)
        if (n + 1) % 10 == 0:
            v._snaps.append((v.ideal.tau, v.ideal.d_ev[1].clone(), v.d_pi[1].clone()))
    n_ref, sf_ref, tx_ref, pi_ref = _run_finder(cuda_lib, v, False, 20000)
    n_na, sf_na, tx_na, pi_na = _run_finder(cuda_lib, v, True, 20000)
    assert n_ref > 0 and n_na == n_ref
    np.testing.assert_array_equal(sf_na, sf_ref)
    np.testing.assert_array_equal(tx_na, tx_ref)
    np.testing.assert_array_equal(pi_na, pi_ref)


def test_noalloc_rejects_oversized_grid(cuda_lib):
    """A grid of 512 x 512 x 257 coarse cubes (one over 2^26) is refused on the
    host before anything is launched (the size check precedes every launch in
    clv_noalloc.cu), so the buffers passed can be small: rc == -1 and an
    untouched count show that nothing ran."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(9, 7, 5)
    v = CLVisc(cfg)
    p = type(v.params)()
    ctypes.pointer(p)[0] = v.params
    p.nx, p.ny, p.nz = 512, 512, 257
    p.nxskip = p.nyskip = p.nzskip = 1
    p.ld = p.nx * p.ny * p.nz
    ev = torch.zeros((4, 64), dtype=torch.float32, device=v.device)
    out = torch.zeros(16, dtype=torch.float32, device=v.device)
    total = torch.zeros(1, dtype=torch.int64, device=v.device)
    rc = cuda_lib.clv_hypersf_append_noalloc(ctypes.byref(p), 0, 0.6, 0.7, ev.data_ptr(), ev.data_ptr(), None, None,
                                             out.data_ptr(), out.data_ptr(), None, 0, total.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == -1
    assert b'exceed the limit' in cuda_lib.clv_last_error()
    assert int(total.item()) == 0
