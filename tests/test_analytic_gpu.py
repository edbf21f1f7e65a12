"""The CUDA classes against the analytic flows (Gubser ideal and viscous,
viscous Bjorken), in both arithmetic builds, at three resolutions each.

Bounds are the measured errors with about 30 % headroom (FP32, relative L2 on
the x axis within |x| <= 4 fm); the exact build reproduces the oracle's
numbers (test_analytic_oracle.py) bit for bit, and the tolerance build must
meet the same bounds and the same convergence. Measured (exact build):
* ideal Gubser, q = 0.25, tau 0.6 -> 3.6 fm, x in [-12, 12] fm:
  e 1.35 % / 0.77 % / 0.40 %, v_r 0.29 % / 0.064 % / 0.026 % at
  dx 0.16 / 0.08 / 0.04 fm (dt = dx / 8);
* viscous Gubser (L = 2 fm, lambda1 = -10, eta/s = 0.2), tau 1 -> 2 fm,
  x in [-10, 10] fm: e 1.06 / 0.54 / 0.42 %, v_r 0.60 / 0.14 / 0.077 %,
  tau^2 pi^{eta eta} 2.06 / 1.67 / 1.53 %, pi^{xx} 2.74 / 1.35 / 1.03 %;
* viscous Bjorken (e0 = 30 GeV/fm^3, eta/s = 0.08) against its
  Israel-Stewart equations: e 5.2e-3 / 2.6e-3 / 1.3e-3 at dt 0.02 / 0.01 /
  0.005 fm.
"""
import numpy as np
import pytest

import analytic_flows as af
from clvisc_b200.eos import Eos
from parity_util import make_cfg

pytestmark = pytest.mark.gpu

MODES = ['exact', 'fast']


def _cfg_maker(mode):
    def mk(*a, **k):
        return make_cfg(*a, arithmetic=mode, **k)
    return mk


@pytest.mark.parametrize('mode', MODES)
def test_gubser_ideal_gpu(cuda_lib, mode):
    from clvisc_b200.ideal import CLIdeal
    res = [af.run_gubser_ideal(CLIdeal, make_cfg, dx, dx / 8.0, 3.6, half_width=12.0)[1]
           for dx in (0.16, 0.08, 0.04)]
    print('ideal Gubser', mode, res)
    bounds = [(0.0176, 0.0038), (0.0100, 0.00084), (0.0052, 0.00034)]
    for r, (be, bv) in zip(res, bounds):
        assert r['e'] < be and r['vr'] < bv, res
    for a, b in zip(res, res[1:]):
        assert b['e'] < 0.65 * a['e'] and b['vr'] < 0.5 * a['vr'], res


@pytest.mark.parametrize('mode', MODES)
def test_gubser_visc_gpu(cuda_lib, mode):
    from clvisc_b200.visc import CLVisc
    res = [af.run_gubser_visc(CLVisc, _cfg_maker(mode), dx, dx / 8.0, 2.0)[1] for dx in (0.16, 0.08, 0.04)]
    print('viscous Gubser', mode, res)
    bounds = [{'e': 0.014, 'vr': 0.008, 'pizz': 0.027, 'pixx': 0.036},
              {'e': 0.007, 'vr': 0.0019, 'pizz': 0.022, 'pixx': 0.0175},
              {'e': 0.0055, 'vr': 0.0010, 'pizz': 0.020, 'pixx': 0.0134}]
    for r, b in zip(res, bounds):
        for k in b:
            assert r[k] < b[k], (k, res)
    for a, b in zip(res, res[1:]):
        for k in ('e', 'vr', 'pixx'):
            assert b[k] < 0.8 * a[k], (k, res)
        assert b['pizz'] < 0.95 * a['pizz'], res


@pytest.mark.parametrize('mode', MODES)
def test_gubser_visc_reference_grid_gpu(cuda_lib, mode):
    """The reference's own set-up (test_gubser_visc.py:82-107: 501 x 501,
    dx = 0.04 fm, dt = 0.005 fm) run to tau = 3 fm: e 1.2 %, v_r 0.27 %,
    pi^{eta eta} 3.9 %, pi^{xx} 2.8 % (measured on the oracle)."""
    from clvisc_b200.visc import CLVisc
    tau, r = af.run_gubser_visc(CLVisc, _cfg_maker(mode), 0.04, 0.005, 3.0)
    print('viscous Gubser 501x501 tau=3', mode, r)
    assert tau == pytest.approx(3.0, abs=1e-5)
    assert r['e'] < 0.016 and r['vr'] < 0.0036 and r['pizz'] < 0.051 and r['pixx'] < 0.037, r


@pytest.mark.parametrize('mode', MODES)
def test_bjorken_visc_gpu(cuda_lib, mode):
    from clvisc_b200.visc import CLVisc
    eos = Eos('ideal_gas')
    T0 = float(eos.f_T(30.0))
    errs = []
    for dt in (0.02, 0.01, 0.005):
        taus, eds, pis = af.run_bjorken_visc(CLVisc, _cfg_maker(mode), eos, dt, 6.6)
        eo, po = af.bjorken_is_ode(eos, taus, 30.0, pis[0], 0.08)
        late = taus > 1.6
        ref_form = np.max(np.abs(eds[late] ** 0.25 / 30.0 ** 0.25
                                 - af.bjorken_first_order_T(taus[late], 0.6, T0, 0.08) / T0))
        assert ref_form < 5e-3, (dt, ref_form)
        errs.append(float(np.max(np.abs(eds / eo - 1.0))))
    print('viscous Bjorken', mode, errs)
    assert errs[0] < 6.8e-3 and errs[1] < 3.4e-3 and errs[2] < 1.7e-3, errs
    assert 1.8 < errs[0] / errs[1] < 2.2 and 1.8 < errs[1] / errs[2] < 2.2, errs
