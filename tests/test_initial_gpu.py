"""Initial conditions generated on the device.

* Optical Glauber (kernel_glauber.cl): against the oracle's CPU restatement.
  Both evaluate exp and pow, whose last bits differ between CUDA and the host
  C library, so the comparison is within 1e-5 relative in FP32 and 1e-11 in
  FP64 (the tolerance of the hydro path for non-bit-exact outputs).
* Seeded Monte Carlo Glauber hotspots: against initial.glauber_event, the host
  construction in numpy float64; the device sums in double in the same order,
  so the only difference is exp's last bit: 1e-12 relative in FP64, and one
  ulp after rounding to FP32. The batch runner's generator gives the same bits
  as the single-event one.
"""
import numpy as np
import pytest

from clvisc_b200.config import read_config
from parity_util import make_cfg

pytestmark = pytest.mark.gpu


def _glauber_cfg(use_float32, grid=(41, 39, 31), b=7.0):
    cfg = read_config([])
    cfg.NX, cfg.NY, cfg.NZ = grid
    cfg.DX = cfg.DY = 0.3
    cfg.DZ = 0.3
    cfg.use_float32 = use_float32
    cfg.ImpactParameter = b
    cfg.fPathOut = '/tmp/clv_glauber_test'
    from clvisc_b200.config import set_real
    return set_real(cfg)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid,b', [((41, 39, 31), 7.0), ((64, 64, 1), 0.0), ((33, 35, 9), 11.5)])
def test_optical_glauber_matches_oracle(cuda_lib, oracle_mod, use_float32, grid, b):
    from clvisc_b200.visc import CLVisc
    cfg = _glauber_cfg(use_float32, grid, b)
    v = CLVisc(cfg)
    v.optical_glauber_ini()
    got = v.ideal.ev_to_host()
    want = oracle_mod.glauber_ini(cfg)
    rtol = 1e-5 if use_float32 else 1e-11
    scale = np.abs(want[:, 0]).max()
    np.testing.assert_allclose(got[:, 0], want[:, 0], rtol=rtol, atol=rtol * scale * 1e-3)
    assert (got[:, 1:] == 0).all()
    assert want[:, 0].max() > 1.0


@pytest.mark.parametrize('use_float32', [True, False])
def test_glauber_centrality_and_nbinary(cuda_lib, oracle_mod, use_float32, tmp_path):
    """optical_glauber_ini with a centrality class sets the impact parameter to
    weight_mean_b (visc.py:163-167) and saves nbin.dat (glauber.py:94-103)."""
    from clvisc_b200.glauber import weight_mean_b
    from clvisc_b200.visc import CLVisc
    cfg = _glauber_cfg(use_float32, (31, 31, 5))
    cfg.fPathOut = str(tmp_path)
    v = CLVisc(cfg)
    v.optical_glauber_ini('Pb+Pb', 20, 30, save_binary_collisions=True)
    assert cfg.ImpactParameter == weight_mean_b(20, 30, 'Pb+Pb')
    got = np.loadtxt(str(tmp_path / 'nbin.dat')).reshape(-1)
    want = oracle_mod.glauber_nbinary(cfg)
    rtol = 1e-5 if use_float32 else 1e-11
    np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * want.max() * 1e-3)
    np.testing.assert_allclose(v.ideal.ev_to_host(), oracle_mod.glauber_ini(cfg), rtol=rtol,
                               atol=rtol * cfg.Edmax * 1e-3)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid,b,seed', [((61, 57, 1), 8.0, 5), ((45, 43, 21), 3.0, 11), ((121, 121, 1), 11.0, 1033)])
def test_hotspot_event_matches_host(cuda_lib, use_float32, grid, b, seed):
    from clvisc_b200.initial import glauber_event
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32, dx=0.16, dz=0.15)
    v = CLVisc(cfg)
    v.load_hotspot_event(b=b, seed=seed, edmax=50.0)
    got = v.ideal.ev_to_host()
    want = glauber_event(*grid, cfg.DX, cfg.DY, cfg.DZ, b=b, seed=seed, edmax=50.0, dtype=np.float64)
    assert (got[:, 1:] == 0).all()
    if use_float32:
        w32 = want[:, 0].astype(np.float32)
        # at most one ulp apart where exp's last bit rounds the other way
        ulps = np.abs(got[:, 0].view(np.int32).astype(np.int64) - w32.view(np.int32).astype(np.int64))
        assert ulps.max() <= 1
        assert (ulps == 0).mean() > 0.99
    else:
        np.testing.assert_allclose(got[:, 0], want[:, 0], rtol=1e-12, atol=1e-12 * 50.0)
    assert got[:, 0].max() == pytest.approx(50.0, rel=1e-6)


def test_batch_hotspot_matches_single(cuda_lib):
    from clvisc_b200.batch import CLViscBatch
    from clvisc_b200.visc import CLVisc
    grids = [(61, 57, 1), (45, 43, 3), (121, 121, 1)]
    specs = [(8.0, 5), (3.0, 11), (11.0, 1033)]
    cfg = make_cfg(*grids[0], dx=0.16, dz=0.15, etaos=0.16)
    bt = CLViscBatch(cfg, grids)
    for e, (b, seed) in enumerate(specs):
        bt.load_hotspot_event(e, b=b, seed=seed, edmax=50.0)
    for e, (g, (b, seed)) in enumerate(zip(grids, specs)):
        v = CLVisc(make_cfg(*g, dx=0.16, dz=0.15, etaos=0.16))
        v.load_hotspot_event(b=b, seed=seed, edmax=50.0)
        np.testing.assert_array_equal(bt.ev_to_host(e), v.ideal.ev_to_host())
