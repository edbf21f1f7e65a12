"""Bulk viscous pressure Pi: the oracle's bulk sector on CPU.

The reference has no bulk viscosity (kernel_visc.cl:31-33 keeps a zero
placeholder for it), so nothing of the reference pins this sector. It is
checked here against physics instead:

* Bjorken flow: a uniform cell obeys the two ordinary differential equations
      de/dtau  = -(e + P + Pi) / tau
      dPi/dtau = -(Pi - Pi_NS) / tau_Pi - (2/3) Pi / tau,   Pi_NS = -zeta / tau
  (no shear: eta/s = 0), which scipy integrates to high accuracy with the same
  EOS and zeta/s(T); the solver's RK2 step must follow within its
  discretisation error, and that error must fall as dtau halves;
* zeta/s(T) has the stated skewed-Cauchy shape;
* with ZETAOS_MAX = 0 the sector is off and every field is identical to a
  run without it.
"""
import numpy as np
import pytest

from clvisc_b200.eos import Eos
from parity_util import make_cfg

HBARC = 0.19733


def bjorken_bulk_oracle(oracle_mod, dt, tau_end, e0, zmax, use_float32=False):
    cfg = make_cfg(1, 1, 1, use_float32=use_float32, dt=dt, etaos=0.0, tau0=0.6, ZETAOS_MAX=zmax,
                   ZETAOS_T0=0.18, ZETAOS_WIDTH=0.02, ZETAOS_SKEW=0.0)
    v = oracle_mod.OracleVisc(cfg)
    ini = np.zeros((1, 4))
    ini[0, 0] = e0
    v.load_ini(ini)
    v.IS_initialize()  # Pi(tau0) = Pi_NS at the loaded energy density
    v.ideal.stepUpdate(1)
    nsteps = int(round((tau_end - 0.6) / dt))
    taus, eds, bulks = [0.6], [float(v.ideal.d_ev[1][0, 0])], [float(v.d_bulk[1][0]) if v.bulk else 0.0]
    for n in range(nsteps):
        v.step(n)
        taus.append(float(v.ideal.tau))
        eds.append(float(v.ideal.d_ev[1][0, 0]))
        bulks.append(float(v.d_bulk[1][0]) if v.bulk else 0.0)
    return np.array(taus), np.array(eds), np.array(bulks), v


def bjorken_bulk_ode(taus, e0, zmax, t0=0.18, w=0.02):
    from scipy.integrate import solve_ivp
    eos = Eos('lattice_pce165')

    def zetaos(T):
        return zmax * w * w / (w * w + (T - t0) ** 2)

    def rhs(tau, y):
        e, pi = y
        P, T, s, cs2 = (float(eos.f_P(e)), float(eos.f_T(e)), float(eos.f_S(e)), float(eos.f_cs2(e)))
        zs = zetaos(T)
        zeta = zs * s * HBARC
        rate = 14.55 * (1.0 / 3.0 - cs2) ** 2 * T / (zs * HBARC)
        return [-(e + P + pi) / tau, -(pi + zeta / tau) * rate - 2.0 / 3.0 * pi / tau]

    T0 = float(eos.f_T(e0))
    pi0 = -zetaos(T0) * float(eos.f_S(e0)) * HBARC / taus[0]
    sol = solve_ivp(rhs, (taus[0], taus[-1]), [e0, pi0], t_eval=taus, rtol=1e-10, atol=1e-12, method='LSODA')
    return sol.y[0], sol.y[1]


def test_zetaos_shape(oracle_mod):
    cfg = make_cfg(1, 1, 1, use_float32=False, ZETAOS_MAX=0.05, ZETAOS_T0=0.18, ZETAOS_WIDTH=0.02,
                   ZETAOS_SKEW=0.5)
    v = oracle_mod.OracleVisc(cfg)
    k = v.k
    f32 = lambda x: float(np.float32(x))
    assert k.zetaos(f32(0.18)) == pytest.approx(0.05, rel=1e-6)  # the peak
    # half maximum one (skewed) width from the peak: w (1 + skew) above, w (1 - skew) below
    assert k.zetaos(f32(0.18) + f32(0.02) * 1.5) == pytest.approx(0.025, rel=1e-5)
    assert k.zetaos(f32(0.18) - f32(0.02) * 0.5) == pytest.approx(0.025, rel=1e-5)
    assert k.zetaos(0.5) < 0.05 * 0.01


def test_bjorken_bulk_follows_ode(oracle_mod):
    """The RK2 + implicit-relaxation step follows the Bjorken ODEs, and its
    error falls as dtau halves."""
    e0, zmax, tau_end = 4.0, 0.2, 4.6
    errs = []
    for dt in (0.04, 0.02):
        taus, eds, bulks, v = bjorken_bulk_oracle(oracle_mod, dt, tau_end, e0, zmax)
        assert v.bulk
        e_ode, pi_ode = bjorken_bulk_ode(taus, e0, zmax)
        # the bulk pressure is a sizeable fraction of P near the zeta/s peak
        eos = Eos('lattice_pce165')
        assert np.max(np.abs(pi_ode) / eos.f_P(e_ode)) > 0.05
        err_e = np.max(np.abs(eds - e_ode) / e_ode)
        err_pi = np.max(np.abs(bulks - pi_ode)) / np.max(np.abs(pi_ode))
        errs.append((err_e, err_pi))
    # stated discretisation error at dtau = 0.02 fm: 0.5 % in e, 2 % of the
    # largest |Pi| (measured 0.31 % and 1.2 %)
    assert errs[1][0] < 5e-3, errs
    assert errs[1][1] < 2e-2, errs
    # first-order convergence: the relaxation term is taken implicitly
    # (backward Euler), as in the reference's shear update (kernel_IS.cl:689-690),
    # so halving dtau halves the error
    assert 0.4 < errs[1][0] / errs[0][0] < 0.6, errs
    assert 0.4 < errs[1][1] / errs[0][1] < 0.6, errs


def test_bulk_changes_cooling(oracle_mod):
    """A negative bulk pressure slows the Bjorken cooling: e(tau) lies above
    the zeta = 0 solution."""
    _, e_bulk, pi, _ = bjorken_bulk_oracle(oracle_mod, 0.02, 3.0, 4.0, 0.2)
    _, e_none, _, _ = bjorken_bulk_oracle(oracle_mod, 0.02, 3.0, 4.0, 0.0)
    assert (pi[1:] < 0).all()
    assert e_bulk[-1] > e_none[-1] * 1.005


@pytest.mark.parametrize('use_float32', [True, False])
def test_bulk_off_is_bitwise_unchanged(oracle_mod, use_float32):
    """ZETAOS_MAX = 0 (the default) leaves the bulk buffers unallocated and
    every field equal to the same run with the keys absent."""
    from parity_util import seeded_ic
    base = make_cfg(9, 8, 5, use_float32=use_float32)
    off = make_cfg(9, 8, 5, use_float32=use_float32, ZETAOS_MAX=0.0, ZETAOS_T0=0.2, ZETAOS_WIDTH=0.05)
    del base.ZETAOS_MAX
    ic = seeded_ic(base, seed=3)
    runs = []
    for cfg in (base, off):
        v = oracle_mod.OracleVisc(cfg)
        v.load_ini(ic)
        v.IS_initialize()
        v.ideal.stepUpdate(1)
        for n in range(3):
            v.step(n)
        assert not v.bulk
        runs.append((v.ideal.d_ev[1].copy(), v.d_pi[1].copy()))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_bulk_held_at_zero_below_tmin(oracle_mod):
    """Cells colder than ZETAOS_TMIN carry no bulk pressure: with the cut above
    every temperature of the run, Pi stays 0 and e(tau) is bit for bit the
    run without the bulk sector (P + 0 = P)."""
    def run(zmax, tmin):
        cfg = make_cfg(1, 1, 1, use_float32=True, dt=0.02, etaos=0.08, ZETAOS_MAX=zmax, ZETAOS_TMIN=tmin)
        v = oracle_mod.OracleVisc(cfg)
        ini = np.zeros((1, 4))
        ini[0, 0] = 4.0
        v.load_ini(ini)
        v.IS_initialize()
        v.ideal.stepUpdate(1)
        for n in range(60):
            v.step(n)
            if zmax > 0:
                assert v.d_bulk[1][0] == 0.0
        return v.ideal.d_ev[1].copy(), v.d_pi[1].copy()
    e_cut, pi_cut = run(0.2, 5.0)
    e_off, pi_off = run(0.0, 5.0)
    np.testing.assert_array_equal(e_cut, e_off)
    np.testing.assert_array_equal(pi_cut, pi_off)


def test_bulk_bounded_by_pressure(oracle_mod):
    """A large zeta/s drives the Navier-Stokes value -zeta theta below -P; the
    bulk pressure is held at -P of the energy density the update reads (the
    Runge-Kutta predictor in d_ev[2]), so P + Pi stays >= 0 there."""
    cfg = make_cfg(1, 1, 1, use_float32=False, dt=0.02, etaos=0.0, ZETAOS_MAX=20.0, ZETAOS_T0=0.18,
                   ZETAOS_WIDTH=0.02)
    v = oracle_mod.OracleVisc(cfg)
    ini = np.zeros((1, 4))
    ini[0, 0] = 4.0
    v.load_ini(ini)
    v.IS_initialize()
    v.ideal.stepUpdate(1)
    at_bound = 0
    for n in range(70):
        v.step(n)
        pb = v.k.P(v.ideal.d_ev[2][0, 0])
        assert -pb <= v.d_bulk[1][0] <= pb
        at_bound += v.d_bulk[1][0] == -pb
    assert at_bound > 50
