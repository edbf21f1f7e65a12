"""Shared helpers of the GPU parity tests: configurations, seeded inputs, and
a comparison that reports where two fields differ."""
import numpy as np

from clvisc_b200.config import read_config
from clvisc_b200.initial import glauber_event


def make_cfg(nx, ny, nz, use_float32=True, eos_type='lattice_pce165', dx=0.3, dz=0.3, dt=0.02, etaos=0.08,
             tau0=0.6, ntskip=4, skip=(2, 2, 2), out='/tmp/clv_parity', **extra):
    cfg = read_config([])
    cfg.NX, cfg.NY, cfg.NZ = nx, ny, nz
    cfg.DX = cfg.DY = dx
    cfg.DZ = dz
    cfg.DT = dt
    cfg.TAU0 = tau0
    cfg.eos_type = eos_type
    cfg.use_float32 = use_float32
    cfg.ETAOS_XMIN, cfg.ETAOS_YMIN, cfg.ETAOS_LEFT_SLOP, cfg.ETAOS_RIGHT_SLOP = 0.18, etaos, 0.0, 0.0
    cfg.ntskip = ntskip
    cfg.nxskip, cfg.nyskip, cfg.nzskip = skip
    cfg.fPathOut = out
    for k, v in extra.items():
        setattr(cfg, k, v)
    cfg.BSZ = 64
    # the parity tests compare bit for bit: the reference's arithmetic unless
    # a test asks for the tolerance build
    if 'arithmetic' not in extra:
        cfg.arithmetic = 'exact'
    from clvisc_b200.config import set_real
    return set_real(cfg)


def seeded_ic(cfg, seed=7, b=6.0, edmax=40.0, flow=0.0):
    """Pb+Pb hotspot profile (with optional random initial flow)."""
    ic = glauber_event(cfg.NX, cfg.NY, cfg.NZ, cfg.DX, cfg.DY, cfg.DZ, b=b, seed=seed, edmax=edmax,
                       dtype=np.float64)
    if flow:
        rng = np.random.default_rng(seed + 1)
        v = rng.uniform(-flow, flow, (ic.shape[0], 3))
        ic[:, 1:] = v / np.sqrt(3.0)
    return ic.astype(cfg.real)


def diff_report(name, got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    same = (got == want) | (np.isnan(got) & np.isnan(want))
    if same.all():
        return ''
    bad = np.argwhere(~same)
    d = np.abs(got.astype(np.float64) - want.astype(np.float64))
    scale = np.maximum(np.abs(want.astype(np.float64)), 1e-30)
    rel = (d / scale)[~same]
    first = tuple(bad[0])
    return ('%s: %d/%d differ, max abs %.3e, max rel %.3e, first at %s got %r want %r'
            % (name, (~same).sum(), same.size, d[~same].max(), rel.max(), first, got[first], want[first]))


def assert_same(name, got, want):
    msg = diff_report(name, got, want)
    assert not msg, msg
