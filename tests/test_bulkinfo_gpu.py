"""Bulk-evolution diagnostics on the device against the reference's host-side
formulas (pyvisc/bulkinfo.py:120-340) applied in numpy to the full state.

The slices are copies and must be equal bit for bit (including get_pimn's
own index arithmetic). The sums are taken in double on the device with P(e)
and s(e) from the run's EOS table; the restatement here uses the same table
through the oracle's EOS, so they agree to double rounding (1e-10), and with
the host EOS grid the reference's own code uses, to the table's interpolation
error (1e-4).
"""
import os

import numpy as np
import pytest

from parity_util import make_cfg, seeded_ic

pytestmark = pytest.mark.gpu


def _eccp(ed, vx, vy, vz, P):
    ed = np.maximum(ed, 1.0E-10)  # bulkinfo.py:187 floors in place; the same values
    pre = P(ed)
    vr2 = vx * vx + vy * vy + vz * vz
    vr2 = np.where(vr2 > 1.0, 0.999999, vr2)
    u0 = 1.0 / np.sqrt(1.0 - vr2)
    txx = (ed + pre) * u0 * u0 * vx * vx + pre
    tyy = (ed + pre) * u0 * u0 * vy * vy + pre
    t0x = (ed + pre) * u0 * u0 * vx
    return t0x.sum() / (txx + tyy).sum(), (txx - tyy).sum() / (txx + tyy).sum(), txx, tyy


def _run(oracle_mod, use_float32, grid=(25, 23, 9)):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(*grid, use_float32=use_float32, dx=0.5, dz=0.4, dt=0.04)
    v = CLVisc(cfg)
    v.load_ini(seeded_ic(cfg, seed=21, b=5.0, edmax=20.0))
    for n in range(6):
        v.step(n)
    o = oracle_mod.OracleIdeal(cfg)
    P_tab = np.vectorize(lambda e: float(o.k.P(e)))
    return cfg, v, P_tab


@pytest.mark.parametrize('use_float32', [True, False])
@pytest.mark.parametrize('grid', [(25, 23, 9), (31, 27, 1)])
def test_bulkinfo_slices_and_sums(cuda_lib, oracle_mod, use_float32, grid):
    cfg, v, P_tab = _run(oracle_mod, use_float32, grid)
    NX, NY, NZ = grid
    bi = v.ideal.bulkinfo
    tau = v.ideal.tau
    bi.get(tau, v.ideal.d_ev[1], 7.0, v.d_pi[1])
    ev = v.ideal.field_to_host(v.ideal.d_ev[1]).reshape(NX, NY, NZ, 4)
    pi_flat = v.pi_to_host(1)
    # slices (bulkinfo.py:62-117)
    np.testing.assert_array_equal(bi.ex[-1], ev[:, NY // 2, NZ // 2, 0])
    np.testing.assert_array_equal(bi.ey[-1], ev[NX // 2, :, NZ // 2, 0])
    np.testing.assert_array_equal(bi.ez[-1], ev[NX // 2, NY // 2, :, 0])
    np.testing.assert_array_equal(bi.vx[-1], ev[:, NY // 2, NZ // 2, 1])
    np.testing.assert_array_equal(bi.vy[-1], ev[NX // 2, :, NZ // 2, 2])
    np.testing.assert_array_equal(bi.vz[-1], ev[NX // 2, NY // 2, :, 3])
    np.testing.assert_array_equal(bi.exy[-1], ev[:, :, NZ // 2, 0])
    np.testing.assert_array_equal(bi.vz_xz[-1], ev[:, NY // 2, :, 3])
    i, j = np.meshgrid(np.arange(NX), np.arange(NY), indexing='ij')
    oid = i * NY * (NZ // 2) + j * (NZ // 2) + NZ // 2  # get_pimn's index
    np.testing.assert_array_equal(bi.pixx_xy[-1], pi_flat[oid, 4])
    np.testing.assert_array_equal(bi.piyy_xy[-1], pi_flat[oid, 7])
    np.testing.assert_array_equal(bi.pitx_xy[-1], pi_flat[oid, 1])
    # eccentricity versus eta_s (bulkinfo.py:259-271), table EOS: double rounding
    for k in range(NZ):
        e1, e2, _, _ = _eccp(ev[:, :, k, 0].astype(np.float64), ev[:, :, k, 1].astype(np.float64),
                             ev[:, :, k, 2].astype(np.float64), ev[:, :, k, 3].astype(np.float64), P_tab)
        assert bi.ecc1_vs_rapidity[-1][k] == pytest.approx(e1, rel=1e-10, abs=1e-14)
        assert bi.ecc2_vs_rapidity[-1][k] == pytest.approx(e2, rel=1e-10, abs=1e-14)
    # plane diagnostics with vz = 0 (bulkinfo.py:184-257)
    exy = ev[:, :, NZ // 2, 0].astype(np.float64)
    vx, vy = ev[:, :, NZ // 2, 1].astype(np.float64), ev[:, :, NZ // 2, 2].astype(np.float64)
    e1, e2, txx, tyy = _eccp(exy, vx, vy, 0.0, P_tab)
    assert bi.eccp(0)[1] == pytest.approx(e2, rel=1e-10, abs=1e-14)
    pixx, piyy = bi.pixx_xy[-1].astype(np.float64), bi.piyy_xy[-1].astype(np.float64)
    visc = ((txx - tyy).sum() + (pixx - piyy).sum()) / ((txx + tyy).sum() + (pixx + piyy).sum())
    assert bi.eccp(0, viscous=True)[1] == pytest.approx(visc, rel=1e-10, abs=1e-14)
    ed = np.maximum(exy, 1e-10)
    u0 = 1.0 / np.sqrt(1.0 - np.minimum(vx * vx + vy * vy, 0.999999))
    vr = (u0 * ed * np.sqrt(vx * vx + vy * vy)).sum() / (u0 * ed).sum()
    assert bi.mean_vr(0) == pytest.approx(vr, rel=1e-10)
    # the reference's own host EOS (grid interpolation): within the table's error
    e1h, e2h, _, _ = _eccp(exy, vx, vy, 0.0, v.ideal.eos.f_P)
    assert bi.eccp(0)[1] == pytest.approx(e2h, rel=1e-4, abs=1e-6)
    S_host = (u0 * v.ideal.eos.f_S(ed)).sum() * float(tau) * cfg.DX * cfg.DY
    assert bi.total_entropy(0) == pytest.approx(S_host, rel=1e-4)


@pytest.mark.parametrize('use_float32', [True, False])
def test_bulkinfo_lab_totals(cuda_lib, oracle_mod, use_float32):
    """Lab-frame energy and entropy of kernel_bulkinfo.cl:18-45, summed
    (bulkinfo_h5.py:264-277)."""
    cfg, v, P_tab = _run(oracle_mod, use_float32)
    NX, NY, NZ = 25, 23, 9
    bi = v.ideal.bulkinfo
    tau = v.ideal.tau
    bi.get(tau, v.ideal.d_ev[1], 7.0)
    ev = v.ideal.field_to_host(v.ideal.d_ev[1]).reshape(NX, NY, NZ, 4).astype(np.float64)
    ed, vx, vy, vz = ev[..., 0], ev[..., 1], ev[..., 2], ev[..., 3]
    pr = P_tab(ed)
    u0 = 1.0 / np.sqrt(np.maximum(1.0 - vx * vx - vy * vy - vz * vz, 1e-7 if use_float32 else 1e-14))
    etas = ((np.arange(NZ) - NZ // 2) * np.float32(cfg.DZ))[None, None, :]
    e_lab = (ed + pr) * u0 * u0 * (np.cosh(etas) + vz * np.sinh(etas)) - pr * np.cosh(etas)
    vol = float(tau) * cfg.DX * cfg.DY * cfg.DZ
    rtol = 1e-5 if use_float32 else 1e-10
    assert bi.energy[-1] == pytest.approx(e_lab.sum() * vol, rel=rtol)
    assert bi.entropy_total[-1] > 0


def test_bulkinfo_save_files(cuda_lib, tmp_path):
    """evolve(save_bulk=True) records every ntskip steps and writes the
    reference's files."""
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(21, 19, 5, dx=0.6, dz=0.5, dt=0.05, ntskip=3, out=str(tmp_path))
    v = CLVisc(cfg)
    v.load_ini(seeded_ic(cfg, seed=4, edmax=10.0))
    v.evolve(max_loops=10, save_hypersf=False, save_bulk=True, force_run_to_maxloop=True)
    names = set(os.listdir(str(tmp_path)))
    for f in ('ex.dat', 'ey.dat', 'ez.dat', 'Tx.dat', 'vx.dat', 'ecc1.dat', 'ecc2.dat', 'edxy0.dat', 'Txy3.dat',
              'ed_xz2.dat', 'eccp.dat', 'eccp_visc.dat', 'Tmax.dat', 'edmax.dat', 'vr.dat', 'entropy.dat',
              'energy_entropy_total.dat'):
        assert f in names, f
    assert np.loadtxt(str(tmp_path / 'ex.dat')).shape == (21, 4)  # 4 records: loops 0, 3, 6, 9
    assert np.loadtxt(str(tmp_path / 'ecc2.dat')).shape == (5, 4)
    assert np.loadtxt(str(tmp_path / 'eccp.dat')).shape == (4, 2)
