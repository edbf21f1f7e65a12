"""Cooper-Frye restatement (oracle, CPU), pinned by a closed form.

A boost-invariant source at rest on a constant-tau surface, elements
dSigma_mu = (tau A d eta, 0, 0, 0) at eta_s on a fine grid, has for
Boltzmann statistics (fermi_boson = 0)
    dN/(dY pt dpt dphi) = g/(2 pi)^3 tau A * 2 mt K1(mt / T),
independent of Y and phi; for Bose statistics the sum over n of
K1(n mt / T) (Juttner series). A chemical potential mu multiplies the n-th
term by exp(n mu / T) (kernel_spec.cl:52 subtracts mu from u.p). The grid helpers reproduce Spec::InitGrid.
"""
import numpy as np
import pytest
from scipy.special import k1

from clvisc_b200.spectra import momentum_grid


def _bjorken_surface(n=4001, etamax=12.0, tau=1.0, area=2.0):
    eta = np.linspace(-etamax, etamax, n)
    deta = eta[1] - eta[0]
    sf = np.zeros((n, 8))
    sf[:, 0] = tau * area * deta
    sf[:, 7] = eta
    return sf, tau * area


def test_momentum_grid_matches_reference_construction():
    y, pt, phi = momentum_grid()
    assert len(y) == 41 and y[0] == -8.0 and y[-1] == 8.0 and y[20] == pytest.approx(0.0, abs=1e-15)
    assert pt[0] == pytest.approx(0.093307812017 / 12.0, rel=1e-11)  # gala15x[0] / 12 (Int.h)
    assert phi[0] == pytest.approx(np.pi * (1.0 - 0.998771007252426118601), rel=1e-13)
    assert phi[-1] == pytest.approx(np.pi * (1.0 + 0.998771007252426118601), rel=1e-15)
    assert (np.diff(phi) > 0).all()


@pytest.mark.parametrize('use_float32', [False, True])
@pytest.mark.parametrize('fb', [0.0, -1.0])
@pytest.mark.parametrize('mu', [0.0, 0.0456])
def test_static_bjorken_source(oracle_mod, use_float32, fb, mu):
    sf, ta = _bjorken_surface()
    y, pt, phi = momentum_grid(ny=5, ylo=-2.0, yhi=2.0, npt=15, nphi=8)
    T, m, g = 0.15, 0.13957, 1.0
    spec = oracle_mod.spectra(sf, None, m, g, fb, mu, T, 0.0, y, pt, phi, use_float32)
    mt = np.sqrt(m * m + pt * pt)
    nmax = 1 if fb == 0.0 else 40
    series = sum(np.exp(n * mu / T) * k1(n * mt / T) for n in range(1, nmax + 1))
    want = g / (2 * np.pi) ** 3 * ta * 2.0 * mt * series
    rtol = 2e-4 if use_float32 else 1e-7
    for k in range(5):
        for q in range(8):
            np.testing.assert_allclose(spec[k, :, q], want, rtol=rtol)
