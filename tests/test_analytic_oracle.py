"""The oracle against the analytic flows of the reference's own tests.

The reference's Gubser and viscous Bjorken tests only plot the solver against
the analytic curves (pyvisc/tests/test_gubser_ideal.py, test_gubser_visc.py,
test_bjorken_visc.py); they state no tolerance. Here the error of the oracle's
step against each analytic solution is measured at two resolutions (FP32, as
the reference's tests compile with USE_SINGLE_PRECISION), and the test asserts
a stated bound at each and that the error falls as the grid is refined. The
bounds are the measured errors with about 30 % headroom; the measured values
are listed beside each bound. Relative L2 errors on the x axis within
|x| <= 4 fm.

These pin the viscous oracle (kernel_IS.cl's shear update, kernel_visc.cl's
viscous KT flux) to something outside this repository: a transcription error
shared by the oracle and the CUDA kernels would show up here.
"""
import numpy as np
import pytest

import analytic_flows as af
from clvisc_b200.eos import Eos
from parity_util import make_cfg


def test_gubser_visc_tensor_is_transverse_and_traceless():
    """u_mu pi^{mu nu} = 0 and g_{mu nu} pi^{mu nu} = 0 for the restated
    second-order Gubser tensor (metric diag(1, -1, -1, -1) on the packed
    components, whose eta-eta entry carries tau^2)."""
    rng = np.random.default_rng(3)
    for tau in (1.0, 1.7, 3.2):
        x = rng.uniform(-6, 6, 200)
        y = rng.uniform(-6, 6, 200)
        ed, u, pi = af.gubser_visc_fields(tau, x, y, 2.0, -10.0)
        P = np.zeros((200, 4, 4))
        for n, (a, b) in enumerate([(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]):
            P[:, a, b] = P[:, b, a] = pi[:, n]
        g = np.array([1.0, -1.0, -1.0, -1.0])
        ulow = u * g
        scale = np.abs(P).max(axis=(1, 2))
        assert np.max(np.abs(np.einsum('na,nab->nb', ulow, P)) / scale[:, None]) < 1e-12
        assert np.max(np.abs(np.einsum('a,naa->n', g, P)) / scale) < 1e-12
        # u is normalised and pi^{eta eta} tau^2 = 2 e / lambda1
        assert np.max(np.abs(np.einsum('na,na->n', ulow, u) - 1.0)) < 1e-12
        np.testing.assert_allclose(pi[:, 9], 2.0 * ed / -10.0, rtol=1e-14)


def test_gubser_ideal_oracle(oracle_mod):
    """Ideal Gubser flow, q = 0.25, tau 0.6 -> 2.6 fm, x in [-8, 8] fm.
    Measured: dx 0.32 / dt 0.04: e 2.24 %, v_r 1.23 %; dx 0.16 / dt 0.02:
    e 0.89 %, v_r 0.26 %."""
    tau, c = af.run_gubser_ideal(oracle_mod.OracleIdeal, make_cfg, 0.32, 0.04, 2.6)
    _, f = af.run_gubser_ideal(oracle_mod.OracleIdeal, make_cfg, 0.16, 0.02, 2.6)
    assert tau == pytest.approx(2.6, abs=1e-5)
    assert c['e'] < 0.029 and c['vr'] < 0.016, c
    assert f['e'] < 0.012 and f['vr'] < 0.0035, f
    assert f['e'] < 0.6 * c['e'] and f['vr'] < 0.5 * c['vr'], (c, f)


def test_gubser_visc_oracle(oracle_mod):
    """Second-order viscous Gubser flow (L = 2 fm, lambda1 = -10, eta/s = 0.2,
    tau 1 -> 2 fm, x in [-10, 10] fm). Measured: dx 0.16 / dt 0.02: e 1.06 %,
    v_r 0.60 %, tau^2 pi^{eta eta} 2.06 %, pi^{xx} 2.74 %; dx 0.08 / dt 0.01:
    e 0.54 %, v_r 0.14 %, pi^{eta eta} 1.67 %, pi^{xx} 1.35 %. The
    pi^{eta eta} error falls slowly (1.53 % at dx 0.04 / dt 0.005, the GPU
    test's finest grid): the reference's discretised equations approach this
    solution more slowly in that component than in the others."""
    tau, c = af.run_gubser_visc(oracle_mod.OracleVisc, make_cfg, 0.16, 0.02, 2.0)
    _, f = af.run_gubser_visc(oracle_mod.OracleVisc, make_cfg, 0.08, 0.01, 2.0)
    assert tau == pytest.approx(2.0, abs=1e-5)
    bound_c = {'e': 0.014, 'vr': 0.008, 'pizz': 0.027, 'pixx': 0.036}
    bound_f = {'e': 0.007, 'vr': 0.0019, 'pizz': 0.022, 'pixx': 0.0175}
    for k in bound_c:
        assert c[k] < bound_c[k], (k, c)
        assert f[k] < bound_f[k], (k, f)
    assert f['e'] < 0.6 * c['e'] and f['vr'] < 0.4 * c['vr'] and f['pixx'] < 0.6 * c['pixx'], (c, f)
    assert f['pizz'] < 0.9 * c['pizz'], (c, f)


def test_bjorken_visc_oracle(oracle_mod):
    """Viscous Bjorken flow (e0 = 30 GeV/fm^3, tau0 = 0.6 fm, eta/s = 0.08,
    tau to 6.6 fm). Against the Israel-Stewart equations the step integrates
    (LSODA): measured max relative error of e 5.2e-3 (dt 0.02) and 2.6e-3
    (dt 0.01): first order in dt; of pi, 3.7e-2 and 2.0e-2 of its largest
    value. Against the reference's own first-order check
    (test_bjorken_visc.py:72-80, left as a commented-out 2-decimal assertion
    there): T/T0 within 3.9e-3 of a^{1/3} (1 + 2/3 b) from tau0 + 1 fm on."""
    eos = Eos('ideal_gas')
    T0 = float(eos.f_T(30.0))
    errs = []
    for dt in (0.02, 0.01):
        taus, eds, pis = af.run_bjorken_visc(oracle_mod.OracleVisc, make_cfg, eos, dt, 6.6)
        eo, po = af.bjorken_is_ode(eos, taus, 30.0, pis[0], 0.08)
        e_err = np.max(np.abs(eds / eo - 1.0))
        p_err = np.max(np.abs(pis - po)) / np.max(np.abs(po))
        late = taus > 1.6
        ref_form = np.max(np.abs(eds[late] ** 0.25 / 30.0 ** 0.25 - af.bjorken_first_order_T(taus[late], 0.6, T0, 0.08)
                                 / T0))
        errs.append((e_err, p_err))
        assert ref_form < 5e-3, (dt, ref_form)
    (ec, pc), (ef, pf) = errs
    assert ec < 6.8e-3 and ef < 3.4e-3, errs
    assert pc < 0.048 and pf < 0.026, errs
    assert 1.8 < ec / ef < 2.2 and pf < 0.6 * pc, errs
