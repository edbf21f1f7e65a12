"""Bulk viscous pressure Pi on the GPU against the oracle's bulk sector.

The bulk sector is an extension (the reference has none); its oracle is the
CPU restatement of the same specification (tests/test_bulk_oracle.py checks
that one against the Bjorken ODEs). The kernels and the oracle evaluate the
same expressions in the same order, so agreement is bit for bit, like the
rest of the path.
"""
import numpy as np
import pytest

from parity_util import assert_same, make_cfg, seeded_ic

pytestmark = pytest.mark.gpu

BULK = dict(ZETAOS_MAX=0.12, ZETAOS_T0=0.2, ZETAOS_WIDTH=0.05, ZETAOS_SKEW=0.3)


def _compare(v, o, tag):
    assert_same(tag + ' ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
    assert_same(tag + ' pi[1]', v.pi_to_host(1), o.d_pi[1])
    assert_same(tag + ' Pi[1]', v.bulk_to_host(1), o.d_bulk[1])
    assert_same(tag + ' ev[2]', v.ideal.field_to_host(v.ideal.d_ev[2]), o.ideal.d_ev[2])
    assert_same(tag + ' Pi[2]', v.bulk_to_host(2), o.d_bulk[2])
    assert_same(tag + ' udiff', v.ideal.field_to_host(v.d_udiff), o.d_udiff)
    assert_same(tag + ' goodcell', v.d_goodcell[:v.size].cpu().numpy().astype(np.float64),
                o.d_goodcell.astype(np.float64))


def _pair(oracle_mod, grid, use_float32, seed=5, flow=0.2):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32, **BULK)
    ic = seeded_ic(cfg, seed=seed, flow=flow)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    assert v.bulk and o.bulk
    v.load_ini(ic)
    o.load_ini(ic)
    v.IS_initialize()
    o.IS_initialize()
    return v, o


@pytest.mark.parametrize('use_float32', [True, False])
def test_bulk_initialize_parity(cuda_lib, oracle_mod, use_float32):
    v, o = _pair(oracle_mod, (11, 9, 7), use_float32)
    assert_same('Pi[1] from ic', v.bulk_to_host(1), o.d_bulk[1])
    assert (o.d_bulk[1] < 0).any()  # Navier-Stokes Pi = -zeta / tau0 where zeta/s > 0


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(15, 13, 11), (21, 19, 1)])
def test_bulk_parts_parity(cuda_lib, oracle_mod, use_float32, grid):
    """Separate IS_stepUpdate / visc_stepUpdate launches, reference order."""
    v, o = _pair(oracle_mod, grid, use_float32)
    for n in range(4):
        v.d_pi[0].copy_(v.d_pi[1])
        v.ideal.d_ev[0].copy_(v.ideal.d_ev[1])
        v.IS_stepUpdate(1)
        v.visc_stepUpdate(1)
        v.update_time(n)
        v.IS_stepUpdate(2)
        v.visc_stepUpdate(2)
        v.update_udiff(v.ideal.d_ev[0], v.ideal.d_ev[1])
        o.step(n)
        _compare(v, o, 'parts n=%d' % n)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(15, 13, 11), (23, 21, 1), (40, 37, 35), (19, 70, 1)])
@pytest.mark.parametrize('kernel', [0, 1, 3])
def test_bulk_fused_step_parity(cuda_lib, oracle_mod, use_float32, grid, kernel):
    """The fused stage of evolve(); the tiled (3+1)D kernel has no bulk sector,
    so with it selected (0) a bulk run takes the per-cell kernel (1); 3 takes
    the tiled (2+1)D kernel, which has one, on the one-cell eta grids. All
    give the oracle's bits."""
    from clvisc_b200 import _lib
    _lib.set_option(_lib.CLV_OPT_STAGE_KERNEL, kernel)
    try:
        v, o = _pair(oracle_mod, grid, use_float32, seed=9, flow=0.0)
        for n in range(6):
            v.step(n, edmax=True)
            o.step(n)
            _compare(v, o, 'fused n=%d' % n)
            assert v.read_edmax_key() == o.ideal.max_energy_density()
    finally:
        _lib.set_option(_lib.CLV_OPT_STAGE_KERNEL, 0)


@pytest.mark.parametrize('use_float32', [True, False])
def test_bulk_evolve_hypersf_parity(cuda_lib, oracle_mod, use_float32, tmp_path):
    """evolve() to freeze-out with the bulk sector: same history, same state,
    same surface element count."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(19, 17, 9, use_float32=use_float32, dx=0.8, dz=0.6, dt=0.05, out=str(tmp_path), ntskip=3,
                   skip=(1, 1, 1), **BULK)
    ic = seeded_ic(cfg, seed=11, edmax=8.0)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    v.IS_initialize()
    o.IS_initialize()
    v.evolve(max_loops=60, save_hypersf=True, force_run_to_maxloop=True)
    o.evolve(max_loops=60, save_hypersf=True, force_run_to_maxloop=True)
    hv = np.array(v.ideal.history, dtype=np.float64)
    ho = np.array(o.ideal.history, dtype=np.float64)
    np.testing.assert_array_equal(hv, ho)
    assert_same('ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
    assert_same('Pi[1]', v.bulk_to_host(1), o.d_bulk[1])
    sf_o, _, pi_o = o.hypersf()
    n = v.ideal.read_num_of_sf()
    assert n == len(sf_o) and n > 0
    assert_same('hypersf', v.ideal.d_hypersf[:n].cpu().numpy(), sf_o)
    assert_same('pisf', v.d_pi_sf[:n].cpu().numpy(), pi_o)


def test_bulk_edge_stability_to_freezeout(cuda_lib):
    """A peripheral (2+1)D event of the batched workload (229^2 cells of
    0.16 fm, b = 10.5 fm, eta/s = 0.16, zeta/s peak 0.05) evolved to freeze-out
    with the bulk sector: without the regulators (|Pi| <= P, Pi = 0 below
    ZETAOS_TMIN) dilute cells at the edge of the fireball ran away near step
    260. The state must stay finite and the maximum energy density must fall."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from clvisc_b200.initial import glauber_event
    from clvisc_b200.visc import CLVisc
    n, b, seed = bench.batch_event_spec(33)
    cfg = bench.batch_cfg(n)
    v = CLVisc(cfg)
    v.load_ini(glauber_event(n, n, 1, 0.16, 0.16, 0.15, b=b, seed=seed, edmax=50.0))
    v.evolve(save_hypersf=False)
    ev = v.ideal.ev_to_host()
    assert np.isfinite(ev).all() and np.isfinite(v.bulk_to_host()).all()
    h = np.array(v.ideal.history, np.float64)
    assert len(h) > 5 and (np.diff(h[:, 1]) < 0).all()
    assert h[-1, 1] < v.ideal.efrz
