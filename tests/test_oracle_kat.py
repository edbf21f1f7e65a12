"""The oracle pinned against the reference's own known-answer tests and golden
vectors (fixtures generated by tests/golden/make_golden.py)."""
import ctypes
import json
import os

import numpy as np
import pytest

from clvisc_b200.config import read_config
from clvisc_b200.eos import Eos

GOLD = os.path.join(os.path.dirname(__file__), 'golden')


def kat():
    with open(os.path.join(GOLD, 'golden.json')) as f:
        return json.load(f)['kat']


def eosi_consts(O, efrz=0.0):
    c = O.Consts()
    c.NX = c.NY = c.NZ = 1
    c.nxskip = c.nyskip = c.nzskip = 1
    c.eos_kind = 1
    c.EFRZ = efrz
    c.EOS_ED_STEP = 1.0
    c.EOS_NUM_OF_ROWS = c.EOS_NUM_OF_COLS = 1
    return c


@pytest.mark.parametrize('real', [np.float32, np.float64])
def test_minmod4_kat(oracle_mod, real):
    """test_kernel_helper.py:29-54: minmod4(minmod4(a,b),c) = (1, 0, -1, 4)."""
    k = kat()['minmod4']
    sfx = 'f32' if real == np.float32 else 'f64'
    f = getattr(oracle_mod.load(), 'clvo_minmod4_' + sfx)
    a, b, c = (np.array(k[x], real) for x in 'abc')
    ab = np.zeros(4, real)
    out = np.zeros(4, real)
    f(a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p), ab.ctypes.data_as(ctypes.c_void_p))
    f(ab.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_array_equal(out, np.array(k['minmod4(minmod4(a,b),c)'], real))


def _t0m_inputs(n, seed):
    rng = np.random.default_rng(seed)
    ed = rng.uniform(1.0, 10.0, n)
    v = rng.uniform(0.0, 0.999, n)
    th = rng.uniform(0.0, np.pi, n)
    ph = rng.uniform(-np.pi, np.pi, n)
    return ed, np.stack([v * np.cos(th) * np.cos(ph), v * np.cos(th) * np.sin(ph), v * np.sin(th)], 1)


def test_rootfinding_kat(oracle_mod):
    """test_kernel_helper.py:57-119: T^{tau mu} of (e, v) with p = e/3, solved back
    with rootFinding (fixed point), recovers e to 2 decimals."""
    O = oracle_mod
    lib = O.load()
    c = eosi_consts(O)
    ed, v = _t0m_inputs(4000, 11)
    f = lib.clvo_root_fixed_f32
    f.argtypes = [ctypes.POINTER(O.Consts), ctypes.c_float, ctypes.c_float]
    out = np.empty_like(ed)
    for n in range(len(ed)):
        e = np.float32(ed[n])
        vv = v[n].astype(np.float32)
        u0 = np.float32(1.0) / np.sqrt(np.float32(max(1.0 - (vv * vv).sum(), 1e-7)))
        pre = e / np.float32(3.0)
        t00 = (e + pre) * u0 * u0 - pre
        M = np.sqrt((((e + pre) * u0 * u0 * vv) ** 2).sum())
        out[n] = f(ctypes.byref(c), float(t00), float(M))
    np.testing.assert_almost_equal(out, ed, 2)


@pytest.mark.parametrize('real', [np.float32, np.float64])
def test_newton_rootfinding_roundtrip(oracle_mod, real):
    """rootFinding_newton (helper.h:128-167, the solver the update kernels use)
    on the same inputs: within the 1e-5 velocity tolerance it stops at."""
    O = oracle_mod
    lib = O.load()
    c = eosi_consts(O)
    sfx = 'f32' if real == np.float32 else 'f64'
    ct = ctypes.c_float if real == np.float32 else ctypes.c_double
    f = getattr(lib, 'clvo_root_newton_' + sfx)
    f.argtypes = [ctypes.POINTER(O.Consts), ct, ct, ctypes.POINTER(ctypes.c_int)]
    ed, v = _t0m_inputs(3000, 5)
    it = ctypes.c_int()
    for n in range(len(ed)):
        e = ed[n]
        vv = v[n]
        u0 = 1.0 / np.sqrt(1.0 - (vv * vv).sum())
        t00 = (e + e / 3) * u0 * u0 - e / 3
        M = np.sqrt((((e + e / 3) * u0 * u0 * vv) ** 2).sum())
        got = f(ctypes.byref(c), t00, M, ctypes.byref(it))
        assert it.value <= 101
        assert abs(got - e) <= 2e-4 * max(1.0, M), (n, got, e, it.value)


@pytest.mark.parametrize('real', [np.float32, np.float64])
def test_reduction_kat(oracle_mod, real):
    """test_reduction.py:15-53: two-stage max of U(0,1) numbers, and the
    padded case (fewer values than 64*256 work-items)."""
    O = oracle_mod
    rng = np.random.default_rng(3)
    for n in (kat()['reduction']['n'], 777, 1):
        x = np.zeros((n, 4), real)
        x[:, 0] = rng.random(n).astype(real)
        semi = np.empty(64, real)
        k = O.Kernels(eosi_consts(O), real)
        k.reduction_stage1(x, semi, n)
        assert semi.max() == x[:, 0].max()


@pytest.mark.parametrize('real', [np.float32, np.float64])
def test_hypersf_unit_cube_kat(oracle_mod, real):
    """test_hypersf.py:26-59: ed = 3 at tau_old, 2 at tau_new, EFRZ = 2.5 -> a
    flat tau slice of unit volume, dSigma = (1, 0, 0, 0)."""
    O = oracle_mod
    k = kat()['hypersf_unit_cube']
    c = eosi_consts(O, efrz=k['efrz'])
    out = np.zeros(4, real)
    sfx = 'f32' if real == np.float32 else 'f64'
    getattr(O.load(), 'clvo_test_hypersf_' + sfx)(ctypes.byref(c), out.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_allclose(out, k['dSigma'], atol=2e-6)


@pytest.mark.parametrize('use_float32', [True, False])
def test_bjorken_ideal_kat(oracle_mod, use_float32):
    """test_bjorken.py:31-62: a uniform cell expands as ed/ed0 = (tau/tau0)^(-4/3)
    (conformal EOS: the ideal_gas table), 3 decimals over 200 loops."""
    cfg = read_config([])
    cfg.NX = cfg.NY = cfg.NZ = 1
    cfg.eos_type = 'ideal_gas'
    cfg.use_float32 = use_float32
    ideal = oracle_mod.OracleIdeal(cfg)
    ini = np.zeros((1, 4))
    ini[:, 0] = kat()['bjorken_ideal']['ed0']
    ideal.load_ini(ini)
    ideal.evolve(max_loops=kat()['bjorken_ideal']['loops'], save_hypersf=False)
    h = np.array(ideal.history, dtype=np.float64)
    np.testing.assert_almost_equal((h[:, 0] / h[0, 0]) ** (-4.0 / 3.0), h[:, 1] / h[0, 1], 3)


def test_eos_tables_match_reference_construction():
    """The kernels' float32 (cs2, p, T, s) images equal the reference's for
    ideal_gas (eos.py:42-59) and for the regenerated PCE165 grid under the
    reference's own cs2 processing (eos.py:78-100)."""
    g = np.load(os.path.join(GOLD, 'golden.npz'))
    with open(os.path.join(GOLD, 'golden.json')) as f:
        meta = json.load(f)
    t, m = Eos('ideal_gas').create_table(200, 1000)
    np.testing.assert_array_equal(t.reshape(-1, 4)[g['ideal_gas_rows']], g['ideal_gas_table'])
    assert Eos('ideal_gas').f_ed(0.137) == meta['ideal_gas_f_ed_0137']
    t, m = Eos('lattice_pce165').create_table(100, 1555)
    np.testing.assert_array_equal(t.reshape(-1, 4)[g['pce165_rows']], g['pce165_table'])
    assert float(Eos('lattice_pce165').f_ed(0.137)) == meta['pce165_f_ed_0137']


@pytest.mark.parametrize('key,eos_type', [('wb', 'lattice_wb'), ('gb', 'pure_gauge')])
def test_computed_eos_tables_match_reference(key, eos_type):
    """Eos('lattice_wb') (the Wuppertal-Budapest 2014 EOS, eos.py:142-153
    with wb.py) and Eos('pure_gauge') (eos.py:171-182 with glueball.py) give
    the reference's float32 image bit for bit at the golden rows
    (tests/golden/make_golden_eos.py imported the reference), and its
    f_ed(0.137)."""
    g = np.load(os.path.join(GOLD, 'golden_eos.npz'))
    e = Eos(eos_type)
    t, m = e.create_table()
    assert t.shape == (200, 1000, 4) and int(g[key + '_n']) == 200000
    assert m['num_of_ed'] == int(g[key + '_num_of_ed']) and m['ed_step'] == float(g[key + '_ed_step'])
    np.testing.assert_array_equal(t.reshape(-1, 4)[g[key + '_rows']], g[key + '_table'])
    assert float(e.f_ed(0.137)) == float(g[key + '_f_ed_0137'])


@pytest.mark.parametrize('eos_type', ['ideal_gas', 'lattice_pce165', 'lattice_wb', 'pure_gauge'])
def test_oracle_eos_lookup_matches_table(oracle_mod, eos_type):
    """Inside the table the oracle's P() reproduces the tabulated pressure at
    grid points and interpolates linearly between them (eos_table.h:39-71)."""
    O = oracle_mod
    cfg = read_config([])
    cfg.eos_type = eos_type
    e = Eos(eos_type)
    from clvisc_b200.eos import TABLE_SHAPE
    table, meta = e.create_table(*TABLE_SHAPE[eos_type])
    c = O.make_consts(cfg, meta, table, 0.1)
    k = O.Kernels(c, np.float64)
    flat = table.reshape(-1, 4)
    ncol = meta['ncol']
    for i in (1, 17, 999, 1001, 1554, 20001):
        x = np.float32(meta['ed_step']) * np.float64(i)
        assert abs(k.P(x) - flat[i, 1]) <= 1e-6 * max(1.0, abs(flat[i, 1]))
        mid = x + 0.5 * np.float32(meta['ed_step'])
        assert abs(k.P(mid) - 0.5 * (float(flat[i, 1]) + float(flat[i + 1, 1]))) <= 1e-5 * max(1.0, flat[i, 1])
    # At an energy density that lands on a row boundary of the 2-D image from
    # just below, eos_table.h:41-43 computes col == NCOLS; clamp-to-edge then
    # returns the previous row's last texel for both ends of the lerp.
    x = np.float32(meta['ed_step']) * np.float64(ncol)
    row = int(x / (np.float32(meta['ed_step']) * ncol))
    if row == 0:
        assert k.P(x) == flat[ncol - 1, 1]
