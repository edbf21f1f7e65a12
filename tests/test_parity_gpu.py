"""CUDA kernels (through the C ABI) against the oracle on the same seeded
inputs. The kernels are built without FMA contraction and with IEEE
division/square root, like the oracle, so the expected agreement is exact:
every field bit for bit, and hypersurface element counts equal. The only
transcendental outputs (tau*cosh(eta), tau*sinh(eta) of sf_txyz) are compared
to 4 ulp (rtol 5e-7 FP32, 1e-15 FP64)."""
import numpy as np
import pytest
import torch

from parity_util import assert_same, make_cfg, seeded_ic

pytestmark = pytest.mark.gpu


def _ref_order_step(v, loop):
    """visc.py:527-544 with the separate IS / KT launches."""
    v.d_pi[0].copy_(v.d_pi[1])
    v.ideal.d_ev[0].copy_(v.ideal.d_ev[1])
    v.IS_stepUpdate(1)
    v.visc_stepUpdate(1)
    v.update_time(loop)
    v.IS_stepUpdate(2)
    v.visc_stepUpdate(2)
    v.update_udiff(v.ideal.d_ev[0], v.ideal.d_ev[1])


def _compare_visc(v, o, tag):
    assert_same(tag + ' ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
    assert_same(tag + ' pi[1]', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])
    assert_same(tag + ' ev[2]', v.ideal.field_to_host(v.ideal.d_ev[2]), o.ideal.d_ev[2])
    assert_same(tag + ' pi[2]', v.ideal.field_to_host(v.d_pi[2]), o.d_pi[2])
    assert_same(tag + ' udiff', v.ideal.field_to_host(v.d_udiff), o.d_udiff)
    assert_same(tag + ' goodcell', v.d_goodcell[:v.size].cpu().numpy().astype(np.float64),
                o.d_goodcell.astype(np.float64))


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(13, 11, 9), (17, 15, 1), (1, 9, 12)])
def test_ideal_stage_parity(cuda_lib, oracle_mod, use_float32, grid):
    from clvisc_b200.ideal import CLIdeal
    cfg = make_cfg(*grid, use_float32=use_float32)
    ic = seeded_ic(cfg, seed=3, flow=0.3)
    g = CLIdeal(cfg)
    o = oracle_mod.OracleIdeal(cfg)
    g.load_ini(ic)
    o.load_ini(ic)
    for n in range(6):
        g.stepUpdate(1)
        o.stepUpdate(1)
        assert_same('stage1 ev[2] n=%d' % n, g.field_to_host(g.d_ev[2]), o.d_ev[2])
        assert_same('stage1 src n=%d' % n, g.field_to_host(g.d_Src), o.d_Src)
        g.update_time(n)
        o.update_time(n)
        g.stepUpdate(2)
        o.stepUpdate(2)
        assert_same('stage2 ev[1] n=%d' % n, g.field_to_host(g.d_ev[1]), o.d_ev[1])
    assert g.max_energy_density() == o.max_energy_density()


@pytest.mark.parametrize('use_float32', [True, False])
def test_visc_construction_parity(cuda_lib, oracle_mod, use_float32):
    """IS_initialize on the empty state and the ideal prediction (visc.py:101-102)."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(11, 9, 7, use_float32=use_float32)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    assert_same('pi[1]', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])
    assert_same('ev[2]', v.ideal.field_to_host(v.ideal.d_ev[2]), o.ideal.d_ev[2])
    v.load_ini(seeded_ic(cfg))
    o.load_ini(seeded_ic(cfg))
    v.IS_initialize()
    o.IS_initialize()
    assert_same('pi[1] from ic', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(15, 13, 11), (19, 17, 1), (34, 9, 41)])
def test_visc_parts_parity(cuda_lib, oracle_mod, use_float32, grid, stage_variant):
    """Separate IS_stepUpdate / visc_stepUpdate launches, reference order."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32)
    ic = seeded_ic(cfg, seed=5, flow=0.2)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    v.IS_initialize()
    o.IS_initialize()
    for n in range(4):
        _ref_order_step(v, n)
        o.step(n)
        _compare_visc(v, o, 'parts n=%d' % n)


@pytest.fixture(params=['auto', 'tiled', 'tiled-1blk', 'tiled-chunk5', 'tiled16', 'tiled8x16', 'tiled8x16-1blk',
                        'per-cell', 'tiled2d', 'tiled2d-128-c3'])
def stage_variant(request, cuda_lib):
    """Every viscous-stage kernel variant; restores the default afterwards.
    (tiled2d: the tiled (2+1)D kernel on one-cell eta grids, 64-thread tiles
    of 8 planes; tiled2d-128-c3: 128-thread tiles of 3 planes.)"""
    from clvisc_b200 import _lib
    tiled = (_lib.CLV_OPT_STAGE_KERNEL, 2)  # tiled on every grid, short eta axes included
    opts = {'auto': [], 'tiled': [tiled], 'tiled-1blk': [tiled, (_lib.CLV_OPT_TILED_BLOCKS, 1)],
            'tiled-chunk5': [tiled, (_lib.CLV_OPT_CHUNK, 5)], 'tiled16': [tiled, (_lib.CLV_OPT_TILE, 1)],
            'tiled8x16': [tiled, (_lib.CLV_OPT_TILE, 2)],
            'tiled8x16-1blk': [tiled, (_lib.CLV_OPT_TILE, 2), (_lib.CLV_OPT_TILED_BLOCKS, 1)],
            'per-cell': [(_lib.CLV_OPT_STAGE_KERNEL, 1)], 'tiled2d': [(_lib.CLV_OPT_STAGE_KERNEL, 3)],
            'tiled2d-128-c3': [(_lib.CLV_OPT_STAGE_KERNEL, 3), (_lib.CLV_OPT_TILE2D_ROWS, 128),
                               (_lib.CLV_OPT_CHUNK2D, 3)]}[request.param]
    for o, v in opts:
        _lib.set_option(o, v)
    yield request.param
    _lib.set_option(_lib.CLV_OPT_TILE, 0)
    _lib.set_option(_lib.CLV_OPT_STAGE_KERNEL, 0)
    _lib.set_option(_lib.CLV_OPT_CHUNK, 32)
    _lib.set_option(_lib.CLV_OPT_TILED_BLOCKS, 2)
    _lib.set_option(_lib.CLV_OPT_TILE2D_ROWS, 64)
    _lib.set_option(_lib.CLV_OPT_CHUNK2D, 8)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(15, 13, 11), (21, 19, 1), (9, 1, 13), (40, 37, 35), (23, 131, 1)])
def test_visc_fused_step_parity(cuda_lib, oracle_mod, use_float32, grid, stage_variant):
    """The fused per-stage kernel of evolve() against the reference order."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32)
    ic = seeded_ic(cfg, seed=9)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    for n in range(8):
        v.step(n, edmax=True)
        o.step(n)
        tag = 'fused n=%d' % n
        assert_same(tag + ' ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
        assert_same(tag + ' pi[1]', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])
        assert_same(tag + ' ev[2]', v.ideal.field_to_host(v.ideal.d_ev[2]), o.ideal.d_ev[2])
        assert_same(tag + ' udiff', v.ideal.field_to_host(v.d_udiff), o.d_udiff)
        assert v.read_edmax_key() == o.ideal.max_energy_density()


@pytest.mark.parametrize('use_float32', [True, False])
def test_visc_evolve_hypersf_parity(cuda_lib, oracle_mod, use_float32, tmp_path):
    """evolve() with freeze-out extraction: same history, same state, same
    surface element count and element values."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(25, 23, 13, use_float32=use_float32, dx=0.8, dz=0.6, dt=0.04, ntskip=5, skip=(2, 2, 1),
                   out=str(tmp_path))
    ic = seeded_ic(cfg, seed=11, edmax=20.0)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    v.evolve(max_loops=60, force_run_to_maxloop=True, save_hypersf=True)
    o.evolve(max_loops=60, force_run_to_maxloop=True, save_hypersf=True)
    assert_same('history', np.array(v.ideal.history, np.float64), np.array(o.ideal.history, np.float64))
    assert_same('ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
    sf_o, tx_o, pi_o = o.hypersf()
    n = v.ideal.read_num_of_sf()
    assert n == len(sf_o) and n > 0
    sf_g = v.ideal.d_hypersf[:n].cpu().numpy()
    tx_g = v.ideal.d_sf_txyz[:n].cpu().numpy()
    pi_g = v.d_pi_sf[:n].cpu().numpy()
    assert_same('hypersf', sf_g, sf_o)
    assert_same('pisf', pi_g, pi_o)
    assert_same('sf x, y', tx_g[:, 1:3], tx_o[:, 1:3])
    rtol = 5e-7 if use_float32 else 1e-15
    np.testing.assert_allclose(tx_g[:, [0, 3]], tx_o[:, [0, 3]], rtol=rtol, atol=0)


def test_ideal_config1_parity(cuda_lib, oracle_mod, tmp_path):
    """The (2+1)D ideal case: 101x101x1, dx=0.16, dt=0.02, tau0=0.6, conformal
    EOS, FP64, Gaussian 30*exp(-x^2/8 - y^2/12.5), evolved to tau = 10 fm."""
    from clvisc_b200.ideal import CLIdeal
    from clvisc_b200.initial import gaussian_2d
    cfg = make_cfg(101, 101, 1, use_float32=False, eos_type='ideal_gas', dx=0.16, dt=0.02, ntskip=10,
                   skip=(1, 1, 1), out=str(tmp_path))
    ic = gaussian_2d(101, 101, 0.16, 0.16)
    g = CLIdeal(cfg)
    o = oracle_mod.OracleIdeal(cfg)
    g.load_ini(ic)
    o.load_ini(ic)
    g.evolve(max_loops=470, save_hypersf=True, to_maxloop=True)
    o.evolve(max_loops=470, save_hypersf=True, to_maxloop=True)
    assert_same('history', np.array(g.history, np.float64), np.array(o.history, np.float64))
    assert_same('ev', g.field_to_host(g.d_ev[1]), o.d_ev[1])
    # kernel_hypersf.cl:422 needs (k+1)*nzskip < NZ: a one-cell eta grid has no surface
    assert g.read_num_of_sf() == len(o.hypersf()[0]) == 0


def test_layout_roundtrip_and_max(cuda_lib):
    from clvisc_b200.ideal import CLIdeal
    cfg = make_cfg(7, 5, 3)
    g = CLIdeal(cfg)
    x = np.random.default_rng(1).normal(size=(g.size, 4)).astype(np.float32)
    g.load_ini(x)
    np.testing.assert_array_equal(g.ev_to_host(), x)
    assert g.max_energy_density() == x[:, 0].max()
    x[:, 0] = -np.abs(x[:, 0]) - 1.0
    g.load_ini(x)
    assert g.max_energy_density() == x[:, 0].max()
    torch.cuda.synchronize()


@pytest.mark.parametrize('use_float32', [True, False])
def test_visc_couplings_parity(cuda_lib, oracle_mod, use_float32, stage_variant):
    """PIMUNU_OMEGA_COUPLING and OMEGA_OMEGA_COUPLING (kernel_IS.cl:636-683):
    rational arithmetic only, so bit for bit."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(17, 15, 13, use_float32=use_float32, pimn_omega_coupling=True, omega_omega_coupling=True)
    ic = seeded_ic(cfg, seed=21, flow=0.3)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    for n in range(4):
        v.step(n)
        o.step(n)
    assert_same('ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
    assert_same('pi[1]', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])


@pytest.mark.parametrize('use_float32', [True, False])
def test_visc_gubser_flag_parity(cuda_lib, oracle_mod, use_float32):
    """GUBSER_VISC_TEST terms (kernel_IS.cl:581-590, 629-634) use pow(), whose
    last bit differs between the device and host libraries: fields agree to
    1e-5 (FP32) / 1e-11 (FP64) relative after 4 steps."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(17, 15, 1, use_float32=use_float32, eos_type='ideal_gas', gubser_visc_test=True, LAM1=-10.0,
                   etaos=0.2)
    ic = seeded_ic(cfg, seed=23)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    for n in range(4):
        v.step(n)
        o.step(n)
    rtol = 1e-5 if use_float32 else 1e-11
    for name, g, w in (('ev', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1]),
                       ('pi', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])):
        scale = np.abs(w).max(axis=0, keepdims=True) + 1e-30
        err = np.abs(g.astype(np.float64) - w) / scale
        assert err.max() <= rtol, (name, err.max())


@pytest.mark.parametrize('use_float32', [True, False])
def test_autotune_restores_state(cuda_lib, use_float32):
    """tune_visc times every launch shape on the run's own state and puts it
    back: the following steps are bit for bit those of an untuned run."""
    from clvisc_b200.autotune import reset, tune_visc
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(40, 37, 35, use_float32=use_float32)
    ic = seeded_ic(cfg, seed=9)
    runs = []
    for tuned in (False, True):
        v = CLVisc(cfg)
        v.load_ini(ic)
        v.step(0)
        if tuned:
            best, table = tune_visc(v, steps=2)
            assert len(table) >= 5 and min(table.values()) > 0
        for n in range(1, 4):
            v.step(n)
        runs.append((v.ideal.field_to_host(v.ideal.d_ev[1]), v.ideal.field_to_host(v.d_pi[1])))
    reset()
    assert_same('ev after tuning', runs[1][0], runs[0][0])
    assert_same('pi after tuning', runs[1][1], runs[0][1])


def test_tuned_choice_is_per_run(cuda_lib):
    """A run's own kernel choice (clv_params opt_*) leaves other runs on the
    process-wide setting: a per-cell run and a tiled run of the same input in
    one process, exact arithmetic, give the same bits, and the process-wide
    option is untouched."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(30, 28, 26)
    ic = seeded_ic(cfg, seed=9)
    a, b = CLVisc(cfg), CLVisc(cfg)
    a.params.opt_stage_kernel = 1 + 1  # per-cell for a only
    b.params.opt_stage_kernel = 1 + 2  # tiled for b only
    for v in (a, b):
        v.load_ini(ic)
        for n in range(3):
            v.step(n)
    assert_same('per-run kernels', a.ideal.field_to_host(a.ideal.d_ev[1]), b.ideal.field_to_host(b.ideal.d_ev[1]))
    c = CLVisc(cfg)
    assert c.params.opt_stage_kernel == 0


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(17, 15, 13), (40, 37, 35), (21, 19, 1)])
@pytest.mark.parametrize('eos_type', ['lattice_wb', 'pure_gauge', 'lattice_pce150'])
def test_computed_eos_parity(cuda_lib, oracle_mod, use_float32, grid, eos_type):
    """The Wuppertal-Budapest and the pure-gauge EOS (200 x 1000 images) and
    the regenerated s95p-PCE-v1 table (100 x 1555): fused steps of the exact
    build against the oracle, bit for bit, per-cell and tiled kernels."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32, eos_type=eos_type)
    ic = seeded_ic(cfg, seed=21, flow=0.2)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    for n in range(6):
        v.step(n, edmax=True)
        o.step(n)
        tag = '%s n=%d' % (eos_type, n)
        assert_same(tag + ' ev[1]', v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1])
        assert_same(tag + ' pi[1]', v.ideal.field_to_host(v.d_pi[1]), o.d_pi[1])
        assert v.read_edmax_key() == o.ideal.max_energy_density()
