"""Analytic flows that pin the hydro step: Gubser flow (ideal and second-order
viscous) and viscous Bjorken flow, with runners that drive either the oracle
(OracleIdeal / OracleVisc) or the CUDA classes (CLIdeal / CLVisc) through the
same sequence of calls.

The formulas restate the reference's own tests:
* ideal Gubser flow, pyvisc/tests/test_gubser_ideal.py:22-26 (energy density
  and radial velocity, q = 0.25) with the initial state of :43-63
  (x = (i - NX/2) DX in floating point, zero eta velocity);
* second-order viscous Gubser flow with the conformal transport coefficients
  of the GUBSER_VISC_TEST branch (kernel_IS.cl:581-590), pyvisc/tests/
  test_gubser_visc.py:11-26 (e, v_r, pi^{eta eta}, pi^{xx}) and the initial
  state of pyvisc/kernel/kernel_gubser_visc.cl (all ten pi components at tau0
  and tau0 + DT, x = (i - NX/2) DX with integer NX/2), set up as in
  test_gubser_visc.py:82-107 (L = 2 fm, lambda1 = -10, eta/s = 0.2, tau0 = 1);
* viscous Bjorken flow, pyvisc/tests/test_bjorken_visc.py:41-80: a uniform
  e = 30 GeV/fm^3 at tau0 = 0.6 fm, eta/s = 0.08, and its first-order
  (Navier-Stokes) temperature T/T0 = a^{1/3} (1 + 2/3 b),
  a = tau0/tau, b = eta/s hbarc (1 - a^{2/3}) / (tau0 T0).

The reference's Gubser tests name IEOS = 0, the conformal ideal gas
(p = e/3) of the older configuration; the runs here use eos_type ideal_gas.

The viscous Gubser tensor is written in the singularity-free form that the
reference's expressions reduce to with C = cosh^2(rho) =
1 + (L^2 - tau^2 + r^2)^2 / (4 L^2 tau^2), D = (L^2 + tau^2 + r^2)^2 and
W = D - 4 tau^2 r^2 (W is the reference's 4L^2 r^2 + (L^2 + tau^2 - r^2)^2):
e = C^p / tau^4 with p = 1/lambda1 - 4/3, and e.g.
pi^{xx} = -4 L^2 C^{p+1} (D - 4 tau^2 y^2) / (lambda1 tau^2 W^2);
test_analytic_oracle.py checks that the tensor is transverse to u and
traceless, which pins these forms independently of how they were reduced.
"""
import numpy as np

HBARC = 0.19733


# ------------------------------------------------------------ ideal Gubser
def gubser_ideal_ed(tau, r, q):
    """test_gubser_ideal.py:22-23."""
    return (2.0 * q) ** (8.0 / 3.0) / (tau * (1.0 + 2.0 * q * q * (tau * tau + r * r)
                                              + q ** 4 * (tau * tau - r * r) ** 2)) ** (4.0 / 3.0)


def gubser_ideal_vr(tau, r, q):
    """test_gubser_ideal.py:25-26 (also the viscous solution's, q = 1/L)."""
    return 2.0 * q * q * tau * r / (1.0 + q * q * tau * tau + q * q * r * r)


def gubser_ideal_state(cfg, tau, q):
    """(cells, 4) initial state of test_gubser_ideal.py:43-63."""
    i = np.arange(cfg.NX)[:, None]
    j = np.arange(cfg.NY)[None, :]
    x = (i - 0.5 * cfg.NX) * cfg.DX
    y = (j - 0.5 * cfg.NY) * cfg.DY
    r = np.sqrt(x * x + y * y)
    ed = gubser_ideal_ed(tau, r, q)
    den = 1.0 + q * q * tau * tau + q * q * r * r
    vx = 2.0 * q * q * tau * x / den
    vy = 2.0 * q * q * tau * y / den
    out = np.zeros((cfg.NX, cfg.NY, cfg.NZ, 4))
    out[..., 0] = ed[..., None]
    out[..., 1] = vx[..., None]
    out[..., 2] = vy[..., None]
    return out.reshape(-1, 4)


# ---------------------------------------------------------- viscous Gubser
def gubser_visc_fields(tau, x, y, L, lam1):
    """e, u^mu and the ten packed pi^{mu nu} (tt, tx, ty, teta, xx, xy, xeta,
    yy, yeta, tau^2 eta-eta) of the second-order Gubser solution at (tau, x, y),
    as kernel_gubser_visc.cl evaluates them; returns (e, u[4], pi[10])."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    A = L * L
    t2 = tau * tau
    R2 = x * x + y * y
    C = 1.0 + (A - t2 + R2) ** 2 / (4.0 * A * t2)
    D = (A + t2 + R2) ** 2
    W = D - 4.0 * t2 * R2
    p = 1.0 / lam1 - 4.0 / 3.0
    ed = C ** p / tau ** 4
    ut = np.sqrt(D / W)
    ux = 2.0 * tau * x / np.sqrt(W)
    uy = 2.0 * tau * y / np.sqrt(W)
    K = 4.0 * A * C ** (p + 1.0) / (lam1 * W * W)  # common factor
    pi = np.zeros(np.broadcast(x, y).shape + (10,))
    pi[..., 0] = -4.0 * K * R2                               # pitt
    pi[..., 1] = -2.0 * K * x * (A + t2 + R2) / tau          # pitx
    pi[..., 2] = -2.0 * K * y * (A + t2 + R2) / tau          # pity
    pi[..., 4] = -K * (D - 4.0 * t2 * y * y) / t2            # pixx
    pi[..., 5] = -4.0 * K * x * y                             # pixy
    pi[..., 7] = -K * (D - 4.0 * t2 * x * x) / t2            # piyy
    pi[..., 9] = 2.0 * ed / lam1                              # tau^2 pi^{eta eta}
    return ed, np.stack([ut, ux, uy, np.zeros_like(ut)], axis=-1), pi


def gubser_visc_state(cfg, tau, L, lam1):
    """(ev (cells, 4), pi (cells, 10)) of kernel_gubser_visc.cl's CreateIniCond."""
    i = np.arange(cfg.NX)[:, None]
    j = np.arange(cfg.NY)[None, :]
    x = (i - cfg.NX // 2) * cfg.DX
    y = (j - cfg.NY // 2) * cfg.DY
    ed, u, pi = gubser_visc_fields(tau, x, y, L, lam1)
    ev = np.zeros((cfg.NX, cfg.NY, cfg.NZ, 4))
    ev[..., 0] = ed[..., None]
    ev[..., 1] = (u[..., 1] / u[..., 0])[..., None]
    ev[..., 2] = (u[..., 2] / u[..., 0])[..., None]
    pim = np.broadcast_to(pi[:, :, None, :], (cfg.NX, cfg.NY, cfg.NZ, 10))
    return ev.reshape(-1, 4), np.ascontiguousarray(pim).reshape(-1, 10)


def gubser_visc_cfg(make_cfg, dx, dt, half_width=10.0, tau0=1.0, L=2.0, lam1=-10.0, etaos=0.2, use_float32=True):
    """The configuration of test_gubser_visc.py:82-101 at grid spacing dx
    (NX = NY odd, x in [-half_width, half_width])."""
    n = 2 * int(round(half_width / dx)) + 1
    cfg = make_cfg(n, n, 1, use_float32=use_float32, eos_type='ideal_gas', dx=dx, dt=dt, etaos=etaos, tau0=tau0,
                   ntskip=100, gubser_visc_test=True, LAM1=lam1)
    cfg.ETAOS_XMIN, cfg.ETAOS_LEFT_SLOP, cfg.ETAOS_RIGHT_SLOP = 0.0, 0.0, 0.0
    return cfg


# ------------------------------------------------------------ Bjorken flow
def bjorken_first_order_T(tau, tau0, T0, etaos):
    """Navier-Stokes Bjorken temperature, test_bjorken_visc.py:74-76."""
    a = tau0 / tau
    b = etaos / tau0 / T0 * HBARC * (1.0 - a ** (2.0 / 3.0))
    return T0 * a ** (1.0 / 3.0) * (1.0 + 2.0 / 3.0 * b)


def bjorken_is_ode(eos, taus, e0, pi0, etaos):
    """The Israel-Stewart equations the step integrates for a uniform cell at
    rest (theta = 1/tau, no gradients): with pi = tau^2 pi^{eta eta},
        de/dtau  = -(e + P + pi) / tau
        dpi/dtau = -(pi - pi_NS) / tau_pi - 4/3 pi / tau,
        pi_NS = -4/3 eta/s s hbarc / tau,  tau_pi = 3 eta/s hbarc / T
    (kernel_visc.cl:24-50, kernel_IS.cl:560-690); solved by LSODA at tight
    tolerances with the EOS that the step reads."""
    from scipy.integrate import solve_ivp

    def rhs(tau, yv):
        e, pi = yv
        P, T, s = float(eos.f_P(e)), float(eos.f_T(e)), float(eos.f_S(e))
        pins = -4.0 / 3.0 * etaos * s * HBARC / tau
        rate = T / (3.0 * etaos * HBARC)
        return [-(e + P + pi) / tau, -(pi - pins) * rate - 4.0 / 3.0 * pi / tau]

    sol = solve_ivp(rhs, (taus[0], taus[-1]), [e0, pi0], t_eval=taus, rtol=1e-11, atol=1e-13, method='LSODA')
    return sol.y[0], sol.y[1]


# ---------------------------------------------------------------- runners
def x_axis(cfg, f, centred_int=True):
    """Values of a (cells,) field on the x axis (j = NY/2, k = 0) and their x."""
    f = np.asarray(f).reshape(cfg.NX, cfg.NY, cfg.NZ)
    j = cfg.NY // 2
    if centred_int:
        x = (np.arange(cfg.NX) - cfg.NX // 2) * cfg.DX
    else:
        x = (np.arange(cfg.NX) - 0.5 * cfg.NX) * cfg.DX
    return x, f[:, j, 0].astype(np.float64)


def rel_err(got, want):
    """max |got - want| / max |want|."""
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def _put(solver_ideal, field, arr):
    if hasattr(solver_ideal, 'field_from_host'):  # CLIdeal: SoA device planes
        solver_ideal.field_from_host(field, arr)
    else:                                         # oracle: (cells, w) numpy
        field[...] = np.asarray(arr, dtype=field.dtype)


def _get(solver_ideal, field):
    if hasattr(solver_ideal, 'field_to_host'):
        return solver_ideal.field_to_host(field)
    return np.array(field)


def run_gubser_ideal(Ideal, make_cfg, dx, dt, tau_end, half_width=8.0, q=0.25, use_float32=True, region=4.0):
    """test_gubser_ideal.py:35-78 on an NX = NY = 2 half_width / dx grid:
    returns (tau, {'e': .., 'vr': ..}) with the relative L2 errors of e and
    v_x = v_r on the x axis within |x| <= region."""
    n = 2 * int(round(half_width / dx))
    cfg = make_cfg(n, n, 1, use_float32=use_float32, eos_type='ideal_gas', dx=dx, dt=dt, etaos=0.0, tau0=0.6)
    s = Ideal(cfg)
    s.load_ini(gubser_ideal_state(cfg, cfg.TAU0, q))
    for k in range(int(round((tau_end - cfg.TAU0) / dt))):
        s.stepUpdate(1)
        s.update_time(k)
        s.stepUpdate(2)
    tau = float(s.tau)
    ev = _get(s, s.d_ev[1])
    x, e = x_axis(cfg, ev[:, 0], centred_int=False)
    _, vx = x_axis(cfg, ev[:, 1], centred_int=False)
    m = np.abs(x) <= region + 1e-9
    return tau, {'e': rel_l2(e[m], gubser_ideal_ed(tau, np.abs(x[m]), q)),
                 'vr': rel_l2(vx[m], gubser_ideal_vr(tau, x[m], q))}


def run_gubser_visc(Visc, make_cfg, dx, dt, tau_end, half_width=10.0, L=2.0, lam1=-10.0, use_float32=True,
                    region=4.0, setup=None):
    """test_gubser_visc.py:82-107: the analytic state at tau0 into d_ev[1],
    d_pi[1] and at tau0 + DT into d_ev[2], d_pi[2], udiff between them, then
    evolve to tau_end; returns (tau, relative L2 errors of e, v_r, tau^2
    pi^{eta eta} and pi^{xx} on the x axis within |x| <= region)."""
    cfg = gubser_visc_cfg(make_cfg, dx, dt, half_width=half_width, L=L, lam1=lam1, use_float32=use_float32)
    v = Visc(cfg)
    if setup is not None:
        setup(v)
    ev1, pi1 = gubser_visc_state(cfg, cfg.TAU0, L, lam1)
    ev2, pi2 = gubser_visc_state(cfg, cfg.TAU0 + cfg.DT, L, lam1)
    _put(v.ideal, v.ideal.d_ev[1], ev1)
    _put(v.ideal, v.ideal.d_ev[2], ev2)
    _put(v.ideal, v.d_pi[1], pi1)
    _put(v.ideal, v.d_pi[2], pi2)
    v.update_udiff(v.ideal.d_ev[1], v.ideal.d_ev[2])
    v.evolve(max_loops=int(round((tau_end - cfg.TAU0) / dt)), save_hypersf=False, force_run_to_maxloop=True)
    tau = float(v.ideal.tau)
    ev = _get(v.ideal, v.ideal.d_ev[1])
    pi = _get(v.ideal, v.d_pi[1])[:, :10]
    x, e = x_axis(cfg, ev[:, 0])
    _, vx = x_axis(cfg, ev[:, 1])
    _, pz = x_axis(cfg, pi[:, 9])
    _, pxx = x_axis(cfg, pi[:, 4])
    m = np.abs(x) <= region + 1e-9
    ea, ua, pia = gubser_visc_fields(tau, x[m], 0.0 * x[m], L, lam1)
    return tau, {'e': rel_l2(e[m], ea), 'vr': rel_l2(vx[m], ua[:, 1] / ua[:, 0]),
                 'pizz': rel_l2(pz[m], pia[:, 9]), 'pixx': rel_l2(pxx[m], pia[:, 4])}


def run_bjorken_visc(Visc, make_cfg, eos, dt, tau_end, e0=30.0, etaos=0.08, use_float32=True, setup=None):
    """test_bjorken_visc.py:22-80 (8 x 8 x 1 cells, uniform e0 at rest,
    tau0 = 0.6 fm): returns (tau, e, pi = tau^2 pi^{eta eta}) of cell 0 after
    every step, with the initial values first."""
    cfg = make_cfg(8, 8, 1, use_float32=use_float32, eos_type='ideal_gas', dx=0.3, dt=dt, etaos=etaos, tau0=0.6,
                   ntskip=20)
    cfg.ETAOS_XMIN, cfg.ETAOS_LEFT_SLOP, cfg.ETAOS_RIGHT_SLOP = 0.0, 0.0, 0.0
    v = Visc(cfg)
    if setup is not None:
        setup(v)
    ini = np.zeros((cfg.NX * cfg.NY * cfg.NZ, 4))
    ini[:, 0] = e0
    v.load_ini(ini)

    def cell0():
        return float(_get(v.ideal, v.ideal.d_ev[1])[0, 0]), float(_get(v.ideal, v.d_pi[1])[0, 9])

    taus, eds, pis = [float(v.ideal.tau)], [], []
    e, p = cell0()
    eds.append(e)
    pis.append(p)
    for k in range(int(round((tau_end - cfg.TAU0) / dt))):
        v.step(k)
        taus.append(float(v.ideal.tau))
        e, p = cell0()
        eds.append(e)
        pis.append(p)
    return np.array(taus), np.array(eds), np.array(pis)


def rel_l2(got, want):
    """||got - want||_2 / ||want||_2."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    return float(np.sqrt(np.sum((got - want) ** 2) / np.sum(want ** 2)))
