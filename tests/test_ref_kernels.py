"""The oracle against the reference's own kernels (CPU).

oracle/ref_shim.py compiles the reference's OpenCL kernel sources
(kernel_ideal.cl, kernel_visc.cl, kernel_IS.cl, kernel_hypersf.cl with their
headers) with g++ through an OpenCL C shim, with the compile options the
reference host passes and the reference's launch geometry (work-groups of BSZ
work-items as OpenMP teams). The same orchestration (oracle.OracleIdeal /
OracleVisc, which restates ideal.py / visc.py) then runs once with the
oracle's restated kernels and once with the reference's compiled kernels, and
every field must agree bit for bit: this pins the restatement to the
reference code itself. The freeze-out surface is compared as a set, since the
reference appends elements through atomic_inc in whatever order the threads
reach them.

Skipped where the reference tree is absent (CLVISC_REFERENCE_ROOT).
"""
import numpy as np
import pytest

import ref_shim
from parity_util import diff_report, make_cfg, seeded_ic

pytestmark = pytest.mark.skipif(not ref_shim.available(), reason='reference kernel sources not present')


def _pair(oracle_mod, cfg, visc=True):
    """Two runs of the oracle's orchestration: the oracle's kernels and the
    reference's compiled kernels."""
    cls = oracle_mod.OracleVisc if visc else oracle_mod.OracleIdeal
    o, r = cls(cfg), cls(cfg)
    ideal = r.ideal if visc else r
    rk = ref_shim.RefKernels(r.k, cfg, ideal.meta, ideal.table, ideal.efrz)
    r.k = rk
    if visc:
        r.ideal.k = rk
    return o, r


def _same(tag, got, want):
    msg = diff_report(tag, got, want)
    assert not msg, msg


def _visc_fields(v):
    return {'ev[1]': v.ideal.d_ev[1], 'ev[2]': v.ideal.d_ev[2], 'pi[1]': v.d_pi[1], 'pi[2]': v.d_pi[2],
            'udiff': v.d_udiff, 'udx': v.d_udx, 'udy': v.d_udy, 'udz': v.d_udz, 'IS_src': v.d_IS_src,
            'Src': v.ideal.d_Src, 'goodcell': v.d_goodcell}


def _surface_rows(sf, tx, pi=None):
    a = np.concatenate([sf, tx] + ([pi] if pi is not None else []), axis=1).astype(np.float64)
    return a[np.lexsort(a.T[::-1])]


def test_vector_literal_rewrite():
    f = ref_shim.rewrite_vector_literals
    assert f('r = (real4)(a, (real4)(1, 2, 3, 4).s1, g(b, c), d);') == 'r = real4{a, real4{1, 2, 3, 4}.s1, g(b, c), d};'
    assert f('read_imagef(t, s, (int2)(col, row))') == 'read_imagef(t, s, int2{col, row})'
    assert f('(real) (x)') == '(real) (x)'


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(15, 13, 11), (19, 17, 1), (34, 9, 41)])
def test_visc_steps_match_reference_kernels(oracle_mod, use_float32, grid):
    """IS_initialize, then every step's fields (kernel_IS.cl, kernel_visc.cl)
    bit for bit; grids with a line length above, below and not a multiple of
    the work-group size, and a single η cell."""
    cfg = make_cfg(*grid, use_float32=use_float32)
    o, r = _pair(oracle_mod, cfg)
    ic = seeded_ic(cfg, flow=0.3)
    for v in (o, r):
        v.load_ini(ic)
        v.IS_initialize()
    _same('pi[1] initial', r.d_pi[1], o.d_pi[1])
    for n in range(5):
        o.step(n)
        r.step(n)
        fo, fr = _visc_fields(o), _visc_fields(r)
        for k in fo:
            _same('step %d %s' % (n, k), fr[k], fo[k])
    assert np.abs(r.d_pi[1]).max() > 0.1 and np.abs(r.ideal.d_ev[1] - ic).max() > 1.0


@pytest.mark.parametrize('use_float32', [True, False])
def test_ideal_steps_match_reference_kernels(oracle_mod, use_float32):
    """kernel_ideal.cl's three stages over 6 steps of the ideal evolution."""
    cfg = make_cfg(17, 15, 13, use_float32=use_float32, etaos=0.0)
    o, r = _pair(oracle_mod, cfg, visc=False)
    ic = seeded_ic(cfg, flow=0.2)
    for v in (o, r):
        v.load_ini(ic)
    for n in range(6):
        for v in (o, r):
            v.stepUpdate(1)
            v.update_time(n)
            v.stepUpdate(2)
        for k in (1, 2):
            _same('step %d ev[%d]' % (n, k), r.d_ev[k], o.d_ev[k])
        _same('step %d Src' % n, r.d_Src, o.d_Src)


@pytest.mark.parametrize('extra,kw,grid', [
    (dict(pimn_omega_coupling=True, omega_omega_coupling=True), {}, (17, 15, 13)),
    (dict(pimn_omega_coupling=True), {}, (13, 11, 9)),
    (dict(gubser_visc_test=True, LAM1=-10.0), dict(eos_type='ideal_gas'), (17, 15, 1)),
    (dict(riemann_test=True), {}, (21, 5, 3)),
    ({}, dict(eos_type='lattice_wb'), (15, 13, 11)),
    ({}, dict(eos_type='pure_gauge'), (15, 13, 11)),
    ({}, dict(eos_type='lattice_pce150'), (15, 13, 11)),
])
@pytest.mark.parametrize('use_float32', [True, False])
def test_switches_match_reference_kernels(oracle_mod, use_float32, extra, kw, grid):
    """The compile-time switches (visc.py:110-121): the π-ω and ω-ω
    couplings, GUBSER_VISC_TEST, RIEMANN_TEST; and the Wuppertal-Budapest and
    pure-gauge EOS images (200 x 1000, EOS_NUM_OF_ROWS/COLS of
    eos.py:194-200)."""
    cfg = make_cfg(*grid, use_float32=use_float32, **kw, **extra)
    o, r = _pair(oracle_mod, cfg)
    ic = seeded_ic(cfg, flow=0.3)
    for v in (o, r):
        v.load_ini(ic)
        v.IS_initialize()
    for n in range(3):
        o.step(n)
        r.step(n)
        fo, fr = _visc_fields(o), _visc_fields(r)
        for k in fo:
            _same('%s step %d %s' % (sorted(extra), n, k), fr[k], fo[k])


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('skip,ntskip', [((1, 1, 1), 2), ((2, 2, 2), 4)])
def test_evolve_and_surface_match_reference_kernels(oracle_mod, use_float32, skip, ntskip):
    """evolve() with surface extraction: the history, the final state and the
    freeze-out surface (kernel_hypersf.cl's visc_hypersf: dΣ, velocities,
    η_s, the space-time position and the interpolated π^{μν}) as a set."""
    cfg = make_cfg(31, 29, 21, use_float32=use_float32, ntskip=ntskip, skip=skip)
    o, r = _pair(oracle_mod, cfg)
    ic = seeded_ic(cfg, flow=0.2, edmax=3.0)
    for v in (o, r):
        v.load_ini(ic)
        v.evolve(max_loops=12, force_run_to_maxloop=True)
    _same('history', np.array(r.ideal.history, np.float64), np.array(o.ideal.history, np.float64))
    _same('ev[1]', r.ideal.d_ev[1], o.ideal.d_ev[1])
    so, sr = o.hypersf(), r.hypersf()
    assert len(so[0]) == len(sr[0]) > 100
    _same('surface', _surface_rows(*sr), _surface_rows(*so))


@pytest.mark.parametrize('use_float32', [True, False])
def test_ideal_surface_matches_reference_kernel(oracle_mod, use_float32):
    """kernel_hypersf.cl's get_hypersf (the ideal path's surface)."""
    cfg = make_cfg(25, 23, 17, use_float32=use_float32, etaos=0.0, ntskip=2, skip=(1, 1, 1))
    o, r = _pair(oracle_mod, cfg, visc=False)
    ic = seeded_ic(cfg, edmax=3.0)
    for v in (o, r):
        v.load_ini(ic)
        v.evolve(max_loops=10, to_maxloop=True)
    so, sr = o.hypersf(), r.hypersf()
    assert len(so[0]) == len(sr[0]) > 100
    _same('surface', _surface_rows(*sr), _surface_rows(*so))


@pytest.mark.parametrize('use_float32', [True, False])
def test_reduction_matches_reference_kernel(oracle_mod, use_float32):
    """kernel_reduction.cl's reduction_stage1 with the reference's launch
    (64 work-groups of 256, ideal.py:259-262): the 64 partial maxima equal the
    oracle's, for sizes below one pass, between, and above several passes."""
    cfg = make_cfg(15, 13, 11, use_float32=use_float32)
    o = oracle_mod.OracleVisc(cfg)
    rk = ref_shim.RefKernels(o.k, cfg, o.ideal.meta, o.ideal.table, o.ideal.efrz)
    rng = np.random.default_rng(3)
    for n in (1000, 16384 + 5, 300001):
        ev = rng.uniform(-5.0, 50.0, (n, 4)).astype(o.k.real)
        a, b = np.empty(64, o.k.real), np.empty(64, o.k.real)
        rk.reference_reduction_stage1(ev, a, n)
        o.k.reduction_stage1(ev, b, n)
        _same('semi n=%d' % n, a, b)
        assert a.max() == ev[:, 0].max()


def test_a_planted_difference_shows(oracle_mod):
    """The comparison is not vacuous: one energy density of the oracle run
    changed by one part in 1e7 shows after a step."""
    cfg = make_cfg(15, 13, 11)
    o, r = _pair(oracle_mod, cfg)
    ic = seeded_ic(cfg, flow=0.3)
    for v in (o, r):
        v.load_ini(ic)
        v.IS_initialize()
    o.ideal.d_ev[1][100, 0] *= np.float32(1.0000001)
    o.step(0)
    r.step(0)
    assert diff_report('ev[1]', r.ideal.d_ev[1], o.ideal.d_ev[1])
