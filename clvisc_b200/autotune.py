"""Autotuner of the fused viscous stage's launch shape for one event.

The tiled stage kernel takes its (y, eta) tile from a compile-time set
(8 x 32, 16 x 16 or 8 x 16, CLV_OPT_TILE) and its x extent per block at run time
(CLV_OPT_CHUNK); the per-cell kernel is the alternative on any grid. Every
variant computes the same bits (in either arithmetic). tune_visc() times each
candidate for a few fused steps on the run's own state, saved before and
restored after each, and leaves the fastest selected for that run only: the
choice goes into the run's own clv_params (opt_* fields), so other CLVisc
objects in the process keep theirs.

    from clvisc_b200.autotune import tune_visc
    v = CLVisc(cfg); v.load_ini(ic)
    best, table = tune_visc(v)
"""
import torch

from . import _lib

DEFAULTS = {'kernel': 0, 'tile': 0, 'chunk': 32, 'blocks': 2}


def _apply(v, c):
    """Select candidate c for the run v (its clv_params opt_* fields)."""
    p = v.params
    p.opt_stage_kernel = c['kernel'] + 1
    p.opt_tile = c['tile'] + 1
    p.opt_chunk = c['chunk']
    p.opt_tiled_blocks = c['blocks']


def candidates(nz, use_float32=True, fast=False):
    """(kernel, tile, chunk, blocks) choices worth timing on a grid with nz
    cells along eta (the 16 x 32 tile exists in the FP32 tolerance build)."""
    out = [dict(DEFAULTS, kernel=1)]
    blocks = (2, 1) if use_float32 else (1,)
    tiles = (0, 1, 2, 3) if (fast and use_float32) else (0, 1, 2)
    for tile in tiles:
        for chunk in (16, 24, 32, 48):
            for b in blocks[:1]:
                out.append({'kernel': 2, 'tile': tile, 'chunk': chunk, 'blocks': b})
    if use_float32:
        out.append({'kernel': 2, 'tile': 0, 'chunk': 32, 'blocks': 1})
    return out


def _state(v):
    ts = list(v.ideal.d_ev) + list(v.d_pi) + [v.d_src, v.d_udiff, v.d_goodcell, v._key]
    return ts


def tune_visc(v, steps=3, cands=None):
    """Time `steps` fused steps of the CLVisc v for each candidate; returns
    (the chosen candidate, {candidate key: ms per step}) and selects it."""
    cands = cands or candidates(v.cfg.NZ, v.cfg.use_float32, bool(v.params.flags & _lib.CLV_FLAG_FAST))
    tensors = _state(v)
    saved = [t.clone() for t in tensors]
    tau = v.ideal.tau
    table = {}
    for c in cands:
        _apply(v, c)
        v.step(0)  # warm-up (and one-time kernel set-up)
        torch.cuda.synchronize(v.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for n in range(1, steps + 1):
            v.step(n)
        e1.record()
        torch.cuda.synchronize(v.device)
        key = 'kernel%d_tile%d_chunk%d_blocks%d' % (c['kernel'], c['tile'], c['chunk'], c['blocks'])
        table[key] = e0.elapsed_time(e1) / steps
        for t, s in zip(tensors, saved):
            t.copy_(s)
        v.ideal.tau = tau
    best_key = min(table, key=table.get)
    best = next(c for c in cands if 'kernel%d_tile%d_chunk%d_blocks%d' % (c['kernel'], c['tile'], c['chunk'],
                                                                            c['blocks']) == best_key)
    _apply(v, best)
    return best, table


def reset(v=None):
    """The run v (if given) back to the process-wide launch choices, and
    those back to the library's defaults."""
    if v is not None:
        p = v.params
        p.opt_stage_kernel = p.opt_tile = p.opt_chunk = p.opt_tiled_blocks = 0
    _lib.set_option(_lib.CLV_OPT_STAGE_KERNEL, DEFAULTS['kernel'])
    _lib.set_option(_lib.CLV_OPT_TILE, DEFAULTS['tile'])
    _lib.set_option(_lib.CLV_OPT_CHUNK, DEFAULTS['chunk'])
    _lib.set_option(_lib.CLV_OPT_TILED_BLOCKS, DEFAULTS['blocks'])
