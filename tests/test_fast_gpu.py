"""The tolerance-arithmetic fused stage (CLV_FLAG_FAST, cfg.arithmetic =
'fast') against the oracle, which follows the reference's arithmetic.

The fast build contracts multiply-adds, divides through reciprocals and
evaluates the limiters in sign-test form, so its fields differ from the
reference's by rounding. The stated tolerance, with tol = 1e-5 in FP32 and
1e-11 in FP64, after the listed numbers of fused time steps:
* energy density:  max_cells |de| <= tol * max_cells e;
* the flow, as the momentum density the step conserves, T^{tau mu} =
  (e + P) u^tau u^mu - P g^{tau mu} (eta component times tau):
  max_cells,mu |dT^{tau mu}| <= tol * max_cells,mu |T^{tau mu}|;
* the shear tensor: max_cells,mu,nu |dpi^{mu nu}| <= tol * max |pi^{mu nu}|.
Each field is scaled by its own largest magnitude, as a whole tensor: single
components that are small against the tensor (pi^{tau tau} = pi^{tau i} v_i
and the eta components of a boost-invariant plateau at early times, v_i in
cells far below freeze-out where e + P is tiny) are dominated by the rounding
of cancelling terms, which any two FP32 evaluations of the reference's
formulas (with or without contracted multiply-adds) share; component by
component they differ by up to 1e-2 of such a component's own maximum after
one step. Each case prints both figures: the tensor-scaled errors checked here,
and the largest per-component one.
"""
import numpy as np
import pytest

from clvisc_b200.eos import Eos
from parity_util import make_cfg, seeded_ic

pytestmark = pytest.mark.gpu

TOL = {True: 1e-5, False: 1e-11}


def scaled_err(got, want):
    """Per-column max |got - want| / max |want| (0 for an all-zero column)."""
    got = np.asarray(got, dtype=np.float64).reshape(want.shape[0], -1)
    want = np.asarray(want, dtype=np.float64).reshape(want.shape[0], -1)
    scale = np.abs(want).max(axis=0)
    d = np.abs(got - want).max(axis=0)
    return np.where(scale > 0, d / np.where(scale > 0, scale, 1.0), d)


def t_tau_mu(ev, eos, tau):
    """T^{tau mu} of (e, v^x, v^y, v^eta) rows, the eta component times tau."""
    ev = np.asarray(ev, dtype=np.float64)
    e = ev[:, 0]
    P = eos.f_P(e)
    v = ev[:, 1:].copy()
    v[:, 2] *= tau
    g2 = 1.0 / np.maximum(1.0 - (v * v).sum(1), 1e-14)
    T = np.empty((ev.shape[0], 4))
    T[:, 0] = (e + P) * g2 - P
    T[:, 1:] = ((e + P) * g2)[:, None] * v
    return T


def field_errors(ev_got, ev_want, pi_got, pi_want, eos, tau):
    """{'e', 'T', 'pi'}: the tensor-scaled errors of the stated tolerance;
    'components': the largest per-component scaled error."""
    def whole(a, b):
        a = np.asarray(a, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    out = {'e': whole(np.asarray(ev_got)[:, 0], np.asarray(ev_want)[:, 0]),
           'T': whole(t_tau_mu(ev_got, eos, tau), t_tau_mu(ev_want, eos, tau)),
           'pi': whole(pi_got, pi_want)}
    out['components'] = float(max(scaled_err(ev_got, ev_want).max(), scaled_err(pi_got, pi_want).max()))
    return out


def compare_fields(v, o, use_float32, tag):
    eos = Eos(v.cfg.eos_type)
    errs = field_errors(v.ideal.field_to_host(v.ideal.d_ev[1]), o.ideal.d_ev[1],
                        v.ideal.field_to_host(v.d_pi[1])[:, :10], o.d_pi[1], eos, float(v.ideal.tau))
    if v.bulk:
        errs['bulk'] = float(np.abs(v.bulk_to_host(1) - o.d_bulk[1]).max() / max(np.abs(o.d_bulk[1]).max(), 1e-300))
    worst = max(v_ for k, v_ in errs.items() if k != 'components')
    print('%s: tensor-scaled errors %s' % (tag, {k: '%.2e' % x for k, x in errs.items()}))
    assert np.isfinite(worst) and worst <= TOL[use_float32], (tag, errs)
    return worst


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid,steps', [((40, 37, 35), 12), ((25, 23, 13), 12), ((41, 39, 1), 20), ((9, 1, 30), 12)])
def test_fast_stage_within_tolerance(cuda_lib, oracle_mod, use_float32, grid, steps):
    """Tiled (3+1)D (40x37x35: eta >= 24 cells), per-cell (short eta, (2+1)D,
    one-cell y) kernels of the fast build against the oracle."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32, arithmetic='fast')
    ic = seeded_ic(cfg, seed=11, flow=0.2)
    v = CLVisc(cfg)
    assert v.params.flags & 32
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    v.IS_initialize()
    o.IS_initialize()
    for n in range(steps):
        v.step(n, edmax=(n == steps - 1))
        o.step(n)
    compare_fields(v, o, use_float32, 'fast %s %s' % (grid, 'fp32' if use_float32 else 'fp64'))
    want = o.ideal.max_energy_density()
    assert abs(v.read_edmax_key() - want) <= TOL[use_float32] * abs(want)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('eos_type', ['lattice_wb', 'pure_gauge'])
def test_fast_computed_eos_within_tolerance(cuda_lib, oracle_mod, use_float32, eos_type):
    """The tolerance build with the Wuppertal-Budapest and the pure-gauge
    EOS."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(40, 37, 35, use_float32=use_float32, arithmetic='fast', eos_type=eos_type)
    ic = seeded_ic(cfg, seed=23, flow=0.2)
    v = CLVisc(cfg)
    o = oracle_mod.OracleVisc(cfg)
    v.load_ini(ic)
    o.load_ini(ic)
    v.IS_initialize()
    o.IS_initialize()
    for n in range(10):
        v.step(n)
        o.step(n)
    compare_fields(v, o, use_float32, 'fast %s %s' % (eos_type, 'fp32' if use_float32 else 'fp64'))


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('bulk', [False, True])
@pytest.mark.parametrize('rows', [64, 128])
def test_fast_tiled2d_within_tolerance(cuda_lib, oracle_mod, use_float32, bulk, rows):
    """The tiled (2+1)D kernel of the fast build for a single event
    (CLV_OPT_STAGE_KERNEL 3 in the run's own options), 64- and 128-thread
    blocks, with and without the bulk sector, against the oracle."""
    from clvisc_b200 import _lib
    from clvisc_b200.visc import CLVisc
    extra = dict(ZETAOS_MAX=0.08, ZETAOS_T0=0.18, ZETAOS_WIDTH=0.03) if bulk else {}
    cfg = make_cfg(61, 67, 1, use_float32=use_float32, arithmetic='fast', **extra)
    ic = seeded_ic(cfg, seed=13, flow=0.2)
    lib = _lib.load()
    assert lib.clv_set_option(_lib.CLV_OPT_TILE2D_ROWS, rows) == 0
    try:
        v = CLVisc(cfg)
        v.params.opt_stage_kernel = 4  # 1 + CLV_OPT_STAGE_KERNEL 3
        o = oracle_mod.OracleVisc(cfg)
        v.load_ini(ic)
        o.load_ini(ic)
        v.IS_initialize()
        o.IS_initialize()
        for n in range(12):
            v.step(n)
            o.step(n)
        compare_fields(v, o, use_float32, 'fast tiled2d rows %d bulk %s %s' % (rows, bulk, 'fp32' if use_float32 else
                                                                             'fp64'))
    finally:
        lib.clv_set_option(_lib.CLV_OPT_TILE2D_ROWS, 64)


@pytest.mark.parametrize('use_float32', [True, False])
def test_fast_bulk_and_gubser_flag(cuda_lib, oracle_mod, use_float32):
    """The fast per-cell instantiations with the bulk sector and with the
    GUBSER_VISC_TEST coupling terms."""
    from clvisc_b200.visc import CLVisc
    bulk = dict(ZETAOS_MAX=0.05, ZETAOS_T0=0.18, ZETAOS_WIDTH=0.02)
    for extra, grid in ((bulk, (19, 17, 9)), (dict(gubser_visc_test=True, LAM1=-10.0), (17, 15, 1))):
        kw = dict(eos_type='ideal_gas') if 'gubser_visc_test' in extra else {}
        cfg = make_cfg(*grid, use_float32=use_float32, arithmetic='fast', **kw, **extra)
        ic = seeded_ic(cfg, seed=4, flow=0.1)
        v = CLVisc(cfg)
        o = oracle_mod.OracleVisc(cfg)
        v.load_ini(ic)
        o.load_ini(ic)
        v.IS_initialize()
        o.IS_initialize()
        for n in range(8):
            v.step(n)
            o.step(n)
        compare_fields(v, o, use_float32, 'fast %s' % sorted(extra))


def test_fast_is_not_exact(cuda_lib):
    """The flag reaches the kernels: fast and exact runs of the same input
    differ (by rounding), exact runs are reproducible bit for bit."""
    from clvisc_b200.visc import CLVisc
    out = {}
    for mode in ('fast', 'exact', 'exact2'):
        cfg = make_cfg(30, 28, 26, arithmetic=mode.rstrip('2'))
        v = CLVisc(cfg)
        v.load_ini(seeded_ic(cfg, seed=2))
        for n in range(4):
            v.step(n)
        out[mode] = v.ideal.field_to_host(v.ideal.d_ev[1])
    assert np.array_equal(out['exact'], out['exact2'])
    assert not np.array_equal(out['fast'], out['exact'])
    assert np.abs(out['fast'][:, 0] - out['exact'][:, 0]).max() < 1e-5 * out['exact'][:, 0].max()
