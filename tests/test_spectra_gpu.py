"""Cooper-Frye spectra on the device against the oracle's restatement of
kernel_spec.cl / kernel_spec_csc.cl, on the analytic boost-invariant source and
on the freeze-out surface of a viscous run (with and without delta f). Both
sum each momentum point in double; the per-term arithmetic calls exp, cosh and
sinh, whose last bits differ between CUDA and the host library, so the
agreement is to 1e-5 (FP32) and 1e-11 (FP64) of the largest value."""
import os

import numpy as np
import pytest

from parity_util import make_cfg, seeded_ic

pytestmark = pytest.mark.gpu


def _close(got, want, use_float32):
    tol = 1e-5 if use_float32 else 1e-11
    np.testing.assert_allclose(got, want, rtol=tol, atol=tol * np.abs(want).max())


@pytest.mark.parametrize('use_float32', [True, False])
def test_spectra_bjorken_source(cuda_lib, oracle_mod, use_float32):
    from scipy.special import k1
    from clvisc_b200.spectra import SmoothSpec
    n = 4001
    eta = np.linspace(-12.0, 12.0, n)
    sf = np.zeros((n, 8))
    sf[:, 0] = 2.0 * (eta[1] - eta[0])
    sf[:, 7] = eta
    s = SmoothSpec(sf, 0.15, use_float32=use_float32)
    got = s.calc(211, 0.13957, 1.0, 0.0)
    want = oracle_mod.spectra(sf, None, 0.13957, 1.0, 0.0, 0.0, 0.15, 0.0, s.y, s.pt, s.phi, use_float32)
    _close(got, want, use_float32)
    mt = np.sqrt(0.13957 ** 2 + s.pt ** 2)
    analytic = 2.0 * 2.0 * mt * k1(mt / 0.15) / (2 * np.pi) ** 3
    np.testing.assert_allclose(got[20, :, 0], analytic, rtol=2e-4 if use_float32 else 1e-7)


@pytest.fixture(scope='module', params=[True, False], ids=['fp32', 'fp64'])
def surface(request, tmp_path_factory, cuda_lib):
    from clvisc_b200.visc import CLVisc
    use_float32 = request.param
    out = str(tmp_path_factory.mktemp('sf'))
    cfg = make_cfg(25, 23, 11, use_float32=use_float32, dx=0.8, dz=0.6, dt=0.05, ntskip=4, skip=(1, 1, 1), out=out)
    v = CLVisc(cfg)
    v.load_ini(seeded_ic(cfg, seed=8, edmax=12.0))
    v.evolve(max_loops=400, save_hypersf=True)
    n = v.ideal.read_num_of_sf()
    assert n > 100
    return (use_float32, out, v.ideal.d_hypersf[:n].clone(), v.d_pi_sf[:n].clone(), cfg,
            v.ideal.eos.f_P(v.ideal.efrz), v.ideal.efrz)


@pytest.mark.parametrize('viscous', [False, True])
@pytest.mark.parametrize('pid', [211, 2212])
def test_spectra_on_hydro_surface(oracle_mod, surface, viscous, pid):
    from clvisc_b200.spectra import HADRONS, SmoothSpec
    use_float32, out, sf, pisf, cfg, pr, ed = surface
    T = cfg.TFRZ
    coeff = 1.0 / (2.0 * T * T * (ed + pr))
    s = SmoothSpec(sf, T, pisf if viscous else None, coeff, use_float32=use_float32)
    got = s.calc(pid)
    m, g, fb = HADRONS[pid]
    want = oracle_mod.spectra(sf.cpu().numpy(), pisf.cpu().numpy() if viscous else None, m, g, fb, 0.0, T,
                              coeff, s.y, s.pt, s.phi, use_float32)
    _close(got, want, use_float32)
    assert got[20, 0, 0] > 0


def test_spectra_from_files_and_write(surface, tmp_path):
    """From hypersf.dat / pimnsf.dat as written by the run; the text's six
    significant digits bound the difference to the device buffers."""
    from clvisc_b200.spectra import SmoothSpec
    use_float32, out, sf, pisf, cfg, pr, ed = surface
    a = SmoothSpec.from_files(out, viscous_on=True, use_float32=use_float32)
    b = SmoothSpec(sf, a.tfrz, pisf, a.tcoeff, use_float32=use_float32, mu=a.mu)
    sa, sb = a.calc(211), b.calc(211)
    np.testing.assert_allclose(sa, sb, rtol=1e-3, atol=1e-4 * np.abs(sb).max())
    a.write(str(tmp_path))
    vals = open(str(tmp_path / 'dNdYPtdPtdPhi_211.dat')).read().split()
    assert len(vals) == 41 * 15 * 48
    assert os.path.exists(str(tmp_path / 'dNdEtaPtdPtdPhi_211.dat'))


@pytest.mark.parametrize('pid', [211, 2212])
def test_spectra_with_chemical_potential(oracle_mod, surface, pid):
    """The run wrote chemical_potential.dat at construction (ideal.py:65);
    from_files reads it and calc() subtracts each hadron's mu from u.p
    (kernel_spec.cl:28,52), against the oracle at the same nonzero mu."""
    from clvisc_b200.spectra import HADRONS, SmoothSpec
    use_float32, out, sf, pisf, cfg, pr, ed = surface
    a = SmoothSpec.from_files(out, viscous_on=False, use_float32=use_float32)
    mu = a.mu[pid]
    assert mu > 0.03
    b = SmoothSpec(sf, cfg.TFRZ, use_float32=use_float32)
    got = b.calc(pid, mu=mu)
    m, g, fb = HADRONS[pid]
    want = oracle_mod.spectra(sf.cpu().numpy(), None, m, g, fb, mu, cfg.TFRZ, 0.0, b.y, b.pt, b.phi, use_float32)
    _close(got, want, use_float32)
    zero = b.calc(pid, mu=0.0)
    ratio = got[20, 0, 0] / zero[20, 0, 0]
    # at least the Boltzmann factor exp(mu/T) at the lowest p_T (Bose-Einstein
    # enhances it further for pions)
    assert ratio > 0.99 * np.exp(mu / cfg.TFRZ), ratio
