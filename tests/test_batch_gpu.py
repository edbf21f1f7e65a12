"""Batched events on the GPU: every event of a CLViscBatch must evolve bit for
bit as a CLVisc object running that event alone (construction, load_ini and
evolve to freeze-out, visc.py:473-560), whatever the other events in the batch,
with or without the CUDA graph, before and after autotuning."""
import numpy as np
import pytest

from parity_util import assert_same, make_cfg, seeded_ic

pytestmark = pytest.mark.gpu

GRIDS = [(21, 19, 1), (33, 29, 1), (17, 15, 5), (27, 31, 1), (9, 9, 1)]
BULK = dict(ZETAOS_MAX=0.08, ZETAOS_T0=0.18, ZETAOS_WIDTH=0.03)


def _cfg(grid, use_float32, bulk, **kw):
    extra = dict(BULK) if bulk else {}
    extra.update(kw)
    return make_cfg(*grid, use_float32=use_float32, dx=0.6, dz=0.6, dt=0.04, ntskip=4, etaos=0.16, **extra)


def _ics(use_float32, bulk):
    out = []
    for e, g in enumerate(GRIDS):
        out.append(seeded_ic(_cfg(g, use_float32, bulk), seed=100 + e, b=2.0 * e, edmax=6.0 + e))
    return out


def _single(grid, ic, use_float32, bulk):
    from clvisc_b200.visc import CLVisc
    v = CLVisc(_cfg(grid, use_float32, bulk))
    v.load_ini(ic)
    v.evolve(save_hypersf=False)
    return v


def _batch(use_float32, bulk, ics, **kw):
    from clvisc_b200.batch import CLViscBatch
    b = CLViscBatch(_cfg(GRIDS[0], use_float32, bulk), GRIDS, **kw)
    for e, ic in enumerate(ics):
        b.load_ini(e, ic)
    return b


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('bulk', [False, True])
def test_batch_events_match_single_runs(cuda_lib, use_float32, bulk):
    ics = _ics(use_float32, bulk)
    b = _batch(use_float32, bulk, ics)
    b.evolve()
    loops = b.loops()
    assert (loops > 0).all()
    assert len(set(loops.tolist())) > 1  # events stop at different steps
    for e, (g, ic) in enumerate(zip(GRIDS, ics)):
        v = _single(g, ic, use_float32, bulk)
        tag = 'event %d %s' % (e, g)
        h = np.array(v.ideal.history, np.float64)
        assert_same(tag + ' history', b.history(e).astype(np.float64), h)
        assert loops[e] == (len(h) - 1) * 4
        assert_same(tag + ' ev[1]', b.ev_to_host(e), v.ideal.field_to_host(v.ideal.d_ev[1]))
        assert_same(tag + ' pi[1]', b.pi_to_host(e), v.pi_to_host(1))
        assert_same(tag + ' Pi[1]', b.bulk_to_host(e), v.bulk_to_host(1))
        assert_same(tag + ' ev[2]', b.ev_to_host(e, slot=2), v.ideal.field_to_host(v.ideal.d_ev[2]))


@pytest.mark.parametrize('use_float32', [True, False])
def test_batch_graph_equals_eager_and_autotune_restores(cuda_lib, use_float32):
    ics = _ics(use_float32, True)
    runs = []
    for mode in ('eager', 'graph', 'tuned'):
        b = _batch(use_float32, True, ics)
        if mode == 'tuned':
            res = b.autotune(steps=3)
            assert len(res) >= 3 and b.launch in res
        steps = b.evolve(use_graph=(mode != 'eager'))
        runs.append((steps, b.loops(), [b.ev_to_host(e) for e in range(len(GRIDS))],
                     [b.bulk_to_host(e) for e in range(len(GRIDS))]))
    for steps, loops, evs, bulks in runs[1:]:
        assert steps == runs[0][0]
        np.testing.assert_array_equal(loops, runs[0][1])
        for e in range(len(GRIDS)):
            assert_same('ev event %d' % e, evs[e], runs[0][2][e])
            assert_same('Pi event %d' % e, bulks[e], runs[0][3][e])


def test_batch_max_loops(cuda_lib):
    """max_loops stops every event after that many steps, as
    CLVisc.evolve(max_loops, force_run_to_maxloop=True) does for one event
    that has not frozen out by then."""
    from clvisc_b200.batch import CLViscBatch
    from clvisc_b200.visc import CLVisc
    ics = _ics(True, False)
    b = CLViscBatch(_cfg(GRIDS[0], True, False), GRIDS, max_loops=10)
    for e, ic in enumerate(ics):
        b.load_ini(e, ic)
    assert b.evolve() == 10
    assert (b.loops() == 10).all()
    for e in (0, 2):
        v = CLVisc(_cfg(GRIDS[e], True, False))
        v.load_ini(ics[e])
        v.evolve(max_loops=10, save_hypersf=False, force_run_to_maxloop=True)
        assert_same('ev event %d' % e, b.ev_to_host(e), v.ideal.field_to_host(v.ideal.d_ev[1]))
        assert_same('history event %d' % e, b.history(e).astype(np.float64),
                    np.array(v.ideal.history, np.float64))


GRIDS_2D = [(21, 19, 1), (33, 29, 1), (9, 9, 1), (27, 131, 1), (64, 5, 1)]


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('bulk', [False, True])
def test_batch_tiled_equals_per_cell(cuda_lib, use_float32, bulk):
    """The tiled (2+1)D batch kernel gives every event the bits of the
    one-thread-per-cell kernel, for 64- and 128-thread tiles, x chunks that do
    and do not divide NX, persistent grids smaller than the tile count, and
    events spanning several tiles along y."""
    from clvisc_b200.batch import CLViscBatch
    ics = [seeded_ic(_cfg(g, use_float32, bulk), seed=200 + e, b=1.5 * e, edmax=7.0 + e)
           for e, g in enumerate(GRIDS_2D)]
    shapes = [('cell', 128, 148, 0), ('tile', 64, 8, None), ('tile', 128, 3, 7), ('tile', 64, 32, 150)]
    runs = []
    for shape in shapes:
        b = CLViscBatch(_cfg(GRIDS_2D[0], use_float32, bulk), GRIDS_2D, max_loops=24, launch=shape)
        for e, ic in enumerate(ics):
            b.load_ini(e, ic)
        assert b.evolve() == 24
        runs.append([(b.ev_to_host(e), b.pi_to_host(e), b.bulk_to_host(e), b.ev_to_host(e, slot=2))
                     for e in range(len(GRIDS_2D))])
    for shape, run in zip(shapes[1:], runs[1:]):
        for e in range(len(GRIDS_2D)):
            for name, got, want in zip(('ev', 'pi', 'Pi', 'ev[2]'), run[e], runs[0][e]):
                assert_same('%s event %d %s' % (name, e, shape), got, want)


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('bulk', [False, True])
def test_fast_batch_tiled_matches_per_cell(cuda_lib, use_float32, bulk):
    """The tiled (2+1)D batch kernel in tolerance arithmetic (the shape the
    batch autotuner picks) against the one-thread-per-cell kernel in the same
    arithmetic, after 24 fixed steps: every event within the fast build's
    tolerance (the two kernels evaluate the same expressions; the compiler may
    contract them differently)."""
    from clvisc_b200.batch import CLViscBatch
    from clvisc_b200.eos import Eos
    from test_fast_gpu import TOL, field_errors
    ics = [seeded_ic(_cfg(g, use_float32, bulk), seed=200 + e, b=1.5 * e, edmax=7.0 + e)
           for e, g in enumerate(GRIDS_2D)]
    cfg0 = _cfg(GRIDS_2D[0], use_float32, bulk, arithmetic='fast')
    runs = []
    for shape in (('cell', 128, 148, 0), ('tile', 64, 8, None), ('tile', 128, 3, 7)):
        b = CLViscBatch(cfg0, GRIDS_2D, max_loops=24, launch=shape)
        assert b.params.flags & 32
        for e, ic in enumerate(ics):
            b.load_ini(e, ic)
        assert b.evolve() == 24
        runs.append([(b.ev_to_host(e), b.pi_to_host(e)) for e in range(len(GRIDS_2D))])
    eos = Eos(cfg0.eos_type)
    for k, run in enumerate(runs[1:], 1):
        for e in range(len(GRIDS_2D)):
            (gev, gpi), (wev, wpi) = run[e], runs[0][e]
            errs = field_errors(gev, wev, np.asarray(gpi)[:, :10], np.asarray(wpi)[:, :10], eos,
                                float(cfg0.TAU0 + 24 * cfg0.DT))
            assert max(errs['e'], errs['T'], errs['pi']) <= TOL[use_float32], (k, e, errs)


@pytest.mark.parametrize('bulk', [False, True])
def test_fast_batch_matches_fast_single_runs(cuda_lib, bulk):
    """The batched stage in tolerance arithmetic (CLV_FLAG_FAST): every event
    stops at the same step as a CLVisc run of it alone in the same arithmetic,
    and its fields agree within the fast build's tolerance (the two evaluate
    the same per-cell function; the check does not rely on the compiler
    contracting it identically in both kernels)."""
    from clvisc_b200.batch import CLViscBatch
    from clvisc_b200.eos import Eos
    from clvisc_b200.visc import CLVisc
    from test_fast_gpu import field_errors
    ics = _ics(True, bulk)
    cfg0 = _cfg(GRIDS[0], True, bulk, arithmetic='fast')
    b = CLViscBatch(cfg0, GRIDS)
    assert b.params.flags & 32
    for e, ic in enumerate(ics):
        b.load_ini(e, ic)
    b.evolve()
    loops = b.loops()
    eos = Eos(cfg0.eos_type)
    bitwise = 0
    for e, (g, ic) in enumerate(zip(GRIDS, ics)):
        v = CLVisc(_cfg(g, True, bulk, arithmetic='fast'))
        v.load_ini(ic)
        v.evolve(save_hypersf=False)
        assert loops[e] == (len(v.ideal.history) - 1) * 4
        got_ev, got_pi = b.ev_to_host(e), b.pi_to_host(e)
        want_ev, want_pi = v.ideal.field_to_host(v.ideal.d_ev[1]), v.pi_to_host(1)
        errs = field_errors(got_ev, want_ev, got_pi, want_pi, eos, float(v.ideal.tau))
        assert max(errs['e'], errs['T'], errs['pi']) <= 1e-5, (e, errs)
        bitwise += int(np.array_equal(got_ev, want_ev) and np.array_equal(got_pi, want_pi))
    print('fast batch: %d of %d events bit for bit equal to their single runs' % (bitwise, len(GRIDS)))


@pytest.mark.parametrize('use_float32', [True, False])
def test_batch_matches_oracle(cuda_lib, oracle_mod, use_float32):
    """The batched stage (exact build, both kernel families of (2+1)D batches
    and the per-cell kernel of a (3+1)D event) against the oracle directly:
    every event's ev and pi after 12 steps, bit for bit, each event run by
    the oracle alone (OracleVisc.evolve, the restatement of visc.py)."""
    from clvisc_b200.batch import CLViscBatch
    grids = [(21, 19, 1), (17, 15, 5), (33, 29, 1)]
    ics = [seeded_ic(_cfg(g, use_float32, False), seed=300 + e, b=1.0 + e, edmax=8.0 + e) for e, g in enumerate(grids)]
    b = CLViscBatch(_cfg(grids[0], use_float32, False), grids, max_loops=12, stop_at_freezeout=False)
    for e, ic in enumerate(ics):
        b.load_ini(e, ic)
    assert b.evolve() == 12
    for e, (g, ic) in enumerate(zip(grids, ics)):
        o = oracle_mod.OracleVisc(_cfg(g, use_float32, False))
        o.load_ini(ic)
        o.evolve(max_loops=12, force_run_to_maxloop=True, save_hypersf=False)
        assert_same('batch event %d ev' % e, b.ev_to_host(e), o.ideal.d_ev[1])
        assert_same('batch event %d pi' % e, b.pi_to_host(e), o.d_pi[1])
