"""The optical Glauber restatement (oracle, CPU) and the impact-parameter
average, pinned without a GPU:
* weight_mean_b() equals the reference's own glauber.py weight_mean_b() on the
  centrality classes of its __main__ (golden values, tests/golden/);
* the Woods-Saxon thickness function of kernel_glauber.cl:10-32 integrates to
  the nucleon number of its density (the 3-D integral of
  Ro0 / (1 + exp((r - R) / a))), so the 10 x 5-point Gauss-Legendre
  quadrature and the 5R cut are restated correctly;
* the energy density peaks at Edmax for a head-on collision and has the
  plateau-with-Gaussian-tails profile along eta_s.
"""
import json
import os

import numpy as np
import pytest
from scipy.integrate import quad

from clvisc_b200.config import read_config
from clvisc_b200.glauber import weight_mean_b

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_weight_mean_b_matches_reference():
    with open(os.path.join(GOLD, 'golden.json')) as f:
        g = json.load(f)['weight_mean_b']
    for system in ('Au+Au', 'Pb+Pb'):
        got = [weight_mean_b(a, b, system) for a, b in g['classes']]
        np.testing.assert_allclose(got, g[system], rtol=1e-12)


def test_thickness_integrates_to_nucleon_number(oracle_mod):
    cfg = read_config([])
    R, a, rho0 = cfg.Ra, cfg.Eta, cfg.NucleonDensity
    total = 4.0 * np.pi * quad(lambda r: r * r * rho0 / (1.0 + np.exp((r - R) / a)), 0.0, 5.0 * R)[0]
    h = 0.25
    xs = np.arange(-3.0 * R, 3.0 * R + h / 2, h)
    t = np.array([[oracle_mod.thickness(cfg, x, y) for y in xs] for x in xs])
    assert t.sum() * h * h == pytest.approx(total, rel=2e-3)
    assert oracle_mod.thickness(cfg, 0.0, 0.0) == pytest.approx(
        2.0 * quad(lambda z: rho0 / (1.0 + np.exp((abs(z) - R) / a)), 0.0, 5.0 * R)[0], rel=1e-5)


@pytest.mark.parametrize('use_float32', [True, False])
def test_glauber_ini_profile(oracle_mod, use_float32):
    cfg = read_config([])
    cfg.NX, cfg.NY, cfg.NZ = 41, 39, 31
    cfg.DX = cfg.DY = 0.3
    cfg.DZ = 0.3
    cfg.use_float32 = use_float32
    cfg.ImpactParameter = 0.0
    ev = oracle_mod.glauber_ini(cfg).reshape(41, 39, 31, 4)
    assert (ev[..., 1:] == 0).all()
    # centre of a head-on collision: Edmax (kFactor normalises at T(0, 0))
    assert ev[20, 19, 15, 0] == pytest.approx(cfg.Edmax, rel=1e-6)
    eta = (np.arange(31) - 15) * 0.3
    h = np.where(np.abs(eta) > cfg.Eta_flat, np.exp(-(np.abs(eta) - cfg.Eta_flat) ** 2 / (2 * cfg.Eta_gw ** 2)), 1.0)
    np.testing.assert_allclose(ev[20, 19, :, 0], cfg.Edmax * h, rtol=2e-5)
