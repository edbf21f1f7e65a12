"""TEST INFRASTRUCTURE ONLY -- the oracle's Python driver.

Restates the orchestration of pyvisc/ideal.py (CLIdeal, ideal.py:28-349) and
pyvisc/visc.py (CLVisc, visc.py:20-560) over numpy buffers in the reference's
own layout -- d_ev[k] is (cells, 4), d_pi[k] is (cells, 10), d_Src (cells, 4),
d_IS_src (cells, 10) -- and calls the C++ restatement of each OpenCL kernel
(clv_oracle.cpp) in the reference's launch order. Used by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker and
the timed CPU baseline; the product package never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_build', 'liboracle_clvisc.so')


class Consts(ctypes.Structure):
    _fields_ = [
        ('NX', ctypes.c_int), ('NY', ctypes.c_int), ('NZ', ctypes.c_int),
        ('DT', ctypes.c_float), ('DX', ctypes.c_float), ('DY', ctypes.c_float), ('DZ', ctypes.c_float),
        ('TAU0', ctypes.c_float),
        ('ETAOS_XMIN', ctypes.c_float), ('ETAOS_YMIN', ctypes.c_float), ('ETAOS_LEFT_SLOP', ctypes.c_float),
        ('ETAOS_RIGHT_SLOP', ctypes.c_float), ('LAM1', ctypes.c_float),
        ('EFRZ', ctypes.c_float),
        ('nxskip', ctypes.c_int), ('nyskip', ctypes.c_int), ('nzskip', ctypes.c_int),
        ('eos_kind', ctypes.c_int),
        ('EOS_ED_START', ctypes.c_float), ('EOS_ED_STEP', ctypes.c_float),
        ('EOS_NUM_ED', ctypes.c_int), ('EOS_NUM_OF_ROWS', ctypes.c_int), ('EOS_NUM_OF_COLS', ctypes.c_int),
        ('eos_table', ctypes.c_void_p),
        ('riemann_test', ctypes.c_int), ('gubser_visc_test', ctypes.c_int),
        ('pimn_omega_coupling', ctypes.c_int), ('omega_omega_coupling', ctypes.c_int),
        ('bulk', ctypes.c_int),
        ('ZETAOS_MAX', ctypes.c_float), ('ZETAOS_T0', ctypes.c_float), ('ZETAOS_WIDTH', ctypes.c_float),
        ('ZETAOS_SKEW', ctypes.c_float), ('ZETAOS_TMIN', ctypes.c_float),
    ]


class GlauberC(ctypes.Structure):  # the -D literals of glauber.py:79-90
    _fields_ = [(n, ctypes.c_float) for n in ('NumOfNucleons', 'SQRTS', 'Ro0', 'R', 'Eta', 'Si0', 'ImpactParameter',
                                                'Edmax', 'Hwn', 'Eta_flat', 'Eta_gw')]


def glauber_consts(cfg):
    """Constants as glauber.py emits them: '-D KEY=%ff' of each entry."""
    from clvisc_b200.config import float_literal as fl
    g = GlauberC()
    for field, key in (('NumOfNucleons', 'NumOfNucleons'), ('SQRTS', 'SQRTS'), ('Ro0', 'NucleonDensity'),
                       ('R', 'Ra'), ('Eta', 'Eta'), ('Si0', 'Si0'), ('ImpactParameter', 'ImpactParameter'),
                       ('Edmax', 'Edmax'), ('Hwn', 'Hwn'), ('Eta_flat', 'Eta_flat'), ('Eta_gw', 'Eta_gw')):
        setattr(g, field, fl('%f' % float(getattr(cfg, key))))
    return g


def glauber_ini(cfg, consts=None):
    """kernel_glauber.cl glauber_ini on the CPU: (cells, 4) array."""
    lib = load()
    from clvisc_b200.config import set_real
    set_real(cfg)
    real = cfg.real
    if consts is None:
        consts = make_consts(cfg, {'ed_start': 0, 'ed_step': 1, 'num_of_ed': 1, 'nrow': 1, 'ncol': 1}, None, 0.0)
    ev = np.zeros((cfg.NX * cfg.NY * cfg.NZ, 4), real)
    g = glauber_consts(cfg)
    f = lib.clvo_glauber_ini_f32 if real == np.float32 else lib.clvo_glauber_ini_f64
    f(ctypes.byref(consts), ctypes.byref(g), _p(ev))
    return ev


def glauber_nbinary(cfg, xlow=-9.75, ylow=-9.75, dx=0.3, dy=0.3, nx=66, ny=66):
    lib = load()
    real = np.float32 if cfg.use_float32 else np.float64
    R = ctypes.c_float if real == np.float32 else ctypes.c_double
    out = np.zeros(nx * ny, real)
    f = lib.clvo_glauber_nbinary_f32 if real == np.float32 else lib.clvo_glauber_nbinary_f64
    f(ctypes.byref(glauber_consts(cfg)), _p(out), R(real(xlow)), R(real(ylow)), R(real(dx)), R(real(dy)),
      ctypes.c_int(nx), ctypes.c_int(ny))
    return out


def thickness(cfg, x, y, use_float32=False):
    lib = load()
    f = lib.clvo_thickness_f32 if use_float32 else lib.clvo_thickness_f64
    R = ctypes.c_float if use_float32 else ctypes.c_double
    f.restype = R
    return f(ctypes.byref(glauber_consts(cfg)), R(x), R(y))


def spectra(sf, pisf, mass, gspin, fb, mu, tfrz, tcoeff, y, pt, phi, use_float32=True):
    """kernel_spec.cl / kernel_spec_csc.cl on the CPU: (ny, npt, nphi)."""
    lib = load()
    real = np.float32 if use_float32 else np.float64
    sfx = 'f32' if use_float32 else 'f64'
    a = lambda x: np.ascontiguousarray(x, dtype=real)
    sf, y, pt = a(sf), a(y), a(pt)
    cphi, sphi = a(np.cos(phi)), a(np.sin(phi))
    pis = None if pisf is None else a(pisf)
    out = np.zeros((len(y), len(pt), len(phi)), real)
    D = ctypes.c_double
    getattr(lib, 'clvo_spectra_' + sfx)(_p(sf), _p(pis), ctypes.c_long(sf.shape[0]), D(mass), D(gspin), D(fb), D(mu),
                                        D(tfrz), D(tcoeff), _p(y), _p(pt), _p(cphi), _p(sphi), ctypes.c_int(len(y)),
                                        ctypes.c_int(len(pt)), ctypes.c_int(len(phi)), _p(out))
    return out


_lib = None


def build():
    """Compile the oracle library (make in oracle/)."""
    subprocess.check_call(['make', '-s', '-C', HERE])
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
                os.path.getmtime(os.path.join(HERE, f)) for f in ('clv_oracle.cpp', 'clv_oracle.hpp')):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.clvo_hypersf_f32.restype = ctypes.c_long
        _lib.clvo_hypersf_f64.restype = ctypes.c_long
        for sfx, rt in (('f32', ctypes.c_float), ('f64', ctypes.c_double)):
            for fn in ('P', 'T', 'S', 'CS2', 'root_fixed', 'root_newton', 'zetaos'):
                getattr(_lib, 'clvo_%s_%s' % (fn, sfx)).restype = rt
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Kernels(object):
    """The reference's kernels at one precision, over numpy arrays."""

    def __init__(self, consts, real):
        self.lib = load()
        self.c = consts
        self.real = real
        self.sfx = 'f32' if real == np.float32 else 'f64'
        self.R = ctypes.c_float if real == np.float32 else ctypes.c_double

    def f(self, name):
        return getattr(self.lib, 'clvo_%s_%s' % (name, self.sfx))

    def r(self, x):
        return self.R(float(x))

    # kernel_ideal.cl
    def ideal_christoffel(self, Src, ev, tau, step):
        self.f('ideal_christoffel')(ctypes.byref(self.c), _p(Src), _p(ev), self.r(tau), int(step))

    def ideal_along(self, axis, Src, ev, tau):
        self.f('ideal_along')(ctypes.byref(self.c), int(axis), _p(Src), _p(ev), self.r(tau))

    def ideal_update_ev(self, evnew, ev1, Src, tau, step):
        self.f('ideal_update_ev')(ctypes.byref(self.c), _p(evnew), _p(ev1), _p(Src), self.r(tau), int(step))

    # kernel_visc.cl
    # the bulk arguments are None (NULL) without the bulk sector
    def visc_christoffel(self, Src, ev, pi, tau, step, bulk=None):
        self.f('visc_christoffel')(ctypes.byref(self.c), _p(Src), _p(ev), _p(pi), self.r(tau), int(step), _p(bulk))

    def visc_along(self, axis, Src, ev, pi, tau, bulk=None):
        self.f('visc_along')(ctypes.byref(self.c), int(axis), _p(Src), _p(ev), _p(pi), self.r(tau), _p(bulk))

    def visc_update_ev(self, evnew, ev1, pi1, pi2, Src, tau, step, bulk1=None, bulk2=None):
        self.f('visc_update_ev')(ctypes.byref(self.c), _p(evnew), _p(ev1), _p(pi1), _p(pi2), _p(Src), self.r(tau),
                                 int(step), _p(bulk1), _p(bulk2))

    # kernel_IS.cl
    def visc_initialize(self, pi1, goodcell, udiff, ev, tau, bulk1=None):
        self.f('visc_initialize')(ctypes.byref(self.c), _p(pi1), _p(goodcell), _p(udiff), _p(ev), self.r(tau),
                                  _p(bulk1))

    def visc_src_christoffel(self, Src, pi1, ev, tau, step, SrcB=None):
        self.f('visc_src_christoffel')(ctypes.byref(self.c), _p(Src), _p(pi1), _p(ev), self.r(tau), int(step),
                                       _p(SrcB))

    def visc_src_along(self, axis, Src, ud, pi1, ev, tau, SrcB=None, bulk1=None):
        self.f('visc_src_along')(ctypes.byref(self.c), int(axis), _p(Src), _p(ud), _p(pi1), _p(ev), self.r(tau),
                                 _p(SrcB), _p(bulk1))

    def update_pimn(self, pinew, goodcell, pi1, pistep, ev1, ev2, udiff, udx, udy, udz, Src, tau, step,
                    bulknew=None, bulk1=None, bulkstep=None, SrcB=None):
        self.f('update_pimn')(ctypes.byref(self.c), _p(pinew), _p(goodcell), _p(pi1), _p(pistep), _p(ev1), _p(ev2),
                              _p(udiff), _p(udx), _p(udy), _p(udz), _p(Src), self.r(tau), int(step),
                              _p(bulknew), _p(bulk1), _p(bulkstep), _p(SrcB))

    def zetaos(self, T):
        return self.f('zetaos')(ctypes.byref(self.c), self.r(T))

    def get_udiff(self, udiff, ev0, ev1):
        self.f('get_udiff')(ctypes.byref(self.c), _p(udiff), _p(ev0), _p(ev1))

    def reduction_stage1(self, ev, semi, size):
        self.f('reduction_stage1')(_p(ev), _p(semi), int(size))

    def hypersf(self, ev_old, ev_new, pi_old, pi_new, t_old, t_new, visc, sf, txyz, pisf, capacity):
        return int(self.f('hypersf')(ctypes.byref(self.c), _p(ev_old), _p(ev_new), _p(pi_old), _p(pi_new),
                                     self.r(t_old), self.r(t_new), int(visc), _p(sf), _p(txyz), _p(pisf),
                                     ctypes.c_long(capacity)))

    def P(self, e):
        return self.f('P')(ctypes.byref(self.c), self.r(e))


def make_consts(cfg, meta, table, efrz, eos_kind=0):
    """Kernel constants as the reference host emits them (float literals)."""
    from clvisc_b200.config import float_literal as fl
    c = Consts()
    c.NX, c.NY, c.NZ = cfg.NX, cfg.NY, cfg.NZ
    c.DT, c.DX, c.DY, c.DZ, c.TAU0 = fl(cfg.DT), fl(cfg.DX), fl(cfg.DY), fl(cfg.DZ), fl(cfg.TAU0)
    c.ETAOS_XMIN, c.ETAOS_YMIN = fl(cfg.ETAOS_XMIN), fl(cfg.ETAOS_YMIN)
    c.ETAOS_LEFT_SLOP, c.ETAOS_RIGHT_SLOP = fl(cfg.ETAOS_LEFT_SLOP), fl(cfg.ETAOS_RIGHT_SLOP)
    c.LAM1 = fl(cfg.LAM1)
    c.EFRZ = fl(efrz)
    c.nxskip, c.nyskip, c.nzskip = cfg.nxskip, cfg.nyskip, cfg.nzskip
    c.eos_kind = eos_kind
    c.EOS_ED_START, c.EOS_ED_STEP = fl(meta['ed_start']), fl(meta['ed_step'])
    c.EOS_NUM_ED, c.EOS_NUM_OF_ROWS, c.EOS_NUM_OF_COLS = int(meta['num_of_ed']), int(meta['nrow']), int(meta['ncol'])
    c.eos_table = table.ctypes.data_as(ctypes.c_void_p).value if table is not None else None
    c.riemann_test = int(bool(getattr(cfg, 'riemann_test', False)))
    c.gubser_visc_test = int(bool(getattr(cfg, 'gubser_visc_test', False)))
    c.pimn_omega_coupling = int(bool(getattr(cfg, 'pimn_omega_coupling', False)))
    c.omega_omega_coupling = int(bool(getattr(cfg, 'omega_omega_coupling', False)))
    c.ZETAOS_MAX = fl(getattr(cfg, 'ZETAOS_MAX', 0.0))
    c.ZETAOS_T0 = fl(getattr(cfg, 'ZETAOS_T0', 0.18))
    c.ZETAOS_WIDTH = fl(getattr(cfg, 'ZETAOS_WIDTH', 0.02))
    c.ZETAOS_SKEW = fl(getattr(cfg, 'ZETAOS_SKEW', 0.0))
    c.ZETAOS_TMIN = fl(getattr(cfg, 'ZETAOS_TMIN', 0.1))
    c.bulk = int(float(getattr(cfg, 'ZETAOS_MAX', 0.0)) > 0.0)
    return c


class OracleIdeal(object):
    """CPU restatement of CLIdeal (ideal.py:28-349)."""

    def __init__(self, cfg, handcrafted_eos=None):
        from clvisc_b200.eos import Eos, TABLE_SHAPE
        from clvisc_b200.config import set_real
        self.cfg = set_real(cfg)
        real = cfg.real
        self.eos = Eos(cfg.eos_type) if handcrafted_eos is None else handcrafted_eos
        if handcrafted_eos is None:
            self.table, meta = self.eos.create_table(*TABLE_SHAPE[cfg.eos_type])
        else:
            self.table, meta = self.eos.create_table()
        self.efrz = self.eos.f_ed(cfg.TFRZ)
        self.meta = meta
        self.consts = make_consts(cfg, meta, self.table, self.efrz)
        self.k = Kernels(self.consts, real)
        self.size = cfg.NX * cfg.NY * cfg.NZ
        self.tau = real(cfg.TAU0)
        z = lambda w: np.zeros((self.size, w), real)
        self.d_ev = [z(4), z(4), z(4)]
        self.d_Src = z(4)
        self.d_ev_old = z(4)
        self.history = []
        self.edmax = None
        self.sf, self.txyz = [], []
        self.tau_old = cfg.TAU0

    def load_ini(self, dat):
        self.d_ev[1][...] = np.asarray(dat, self.cfg.real).reshape(self.size, 4)

    def stepUpdate(self, step):  # ideal.py:211-255
        k, ev = self.k, self.d_ev
        k.ideal_christoffel(self.d_Src, ev[step], self.tau, step)
        for axis in range(3):
            k.ideal_along(axis, self.d_Src, ev[step], self.tau)
        k.ideal_update_ev(ev[3 - step], ev[1], self.d_Src, self.tau, step)

    def max_energy_density(self):  # ideal.py:257-262
        semi = np.empty(64, self.cfg.real)
        self.k.reduction_stage1(self.d_ev[1], semi, self.size)
        return semi.max()

    def update_time(self, loop):
        self.tau = self.cfg.real(self.cfg.TAU0 + (loop + 1) * self.cfg.DT)

    def _hypersf(self, visc, t_old, t_new, ev_old, ev_new, pi_old=None, pi_new=None):
        real = self.cfg.real
        cap = 1 << 16
        while True:
            sf = np.empty((cap, 8), real)
            txyz = np.empty((cap, 4), real)
            pisf = np.empty((cap, 10), real) if visc else None
            n = self.k.hypersf(ev_old, ev_new, pi_old, pi_new, t_old, t_new, visc, sf, txyz, pisf, cap)
            if n <= cap:
                return sf[:n], txyz[:n], (pisf[:n] if visc else None)
            cap = n

    def get_hypersf(self, n, ntskip):  # ideal.py:269-293
        is_finished = self.edmax < self.efrz
        if n == 0:
            self.d_ev_old[...] = self.d_ev[1]
            self.tau_old = self.cfg.TAU0
        elif (n % ntskip == 0) or is_finished:
            tau_new = self.tau
            sf, txyz, _ = self._hypersf(0, self.cfg.real(self.tau_old), self.cfg.real(tau_new), self.d_ev_old,
                                        self.d_ev[1])
            self.sf.append(sf)
            self.txyz.append(txyz)
            self.d_ev_old[...] = self.d_ev[1]
            self.tau_old = tau_new
        return is_finished

    def hypersf(self):
        real = self.cfg.real
        sf = np.concatenate(self.sf) if self.sf else np.zeros((0, 8), real)
        tx = np.concatenate(self.txyz) if self.txyz else np.zeros((0, 4), real)
        return sf, tx

    def evolve(self, max_loops=2000, save_hypersf=True, to_maxloop=False):  # ideal.py:322-349
        for n in range(max_loops):
            self.edmax = self.max_energy_density()
            self.history.append([self.tau, self.edmax])
            is_finished = False
            if save_hypersf:
                is_finished = self.get_hypersf(n, self.cfg.ntskip)
            if is_finished and not to_maxloop:
                break
            self.stepUpdate(1)
            self.update_time(n)
            self.stepUpdate(2)


class OracleVisc(object):
    """CPU restatement of CLVisc (visc.py:20-560)."""

    def __init__(self, cfg, handcrafted_eos=None):
        self.ideal = OracleIdeal(cfg, handcrafted_eos)
        self.cfg = cfg
        real = cfg.real
        self.k = self.ideal.k
        self.size = self.ideal.size
        z = lambda w: np.zeros((self.size, w), real)
        self.d_pi = [z(10), z(10), z(10)]
        self.d_IS_src = z(10)
        self.d_udx, self.d_udy, self.d_udz = z(4), z(4), z(4)
        self.d_udiff = z(4)
        self.d_goodcell = np.ones(self.size, real)
        self.d_pi_old = z(10)
        self.pisf = []
        # bulk sector (no counterpart in the reference): Pi per cell in three
        # slots like d_pi, and its IS source
        self.bulk = bool(self.ideal.consts.bulk)
        zb = lambda: np.zeros(self.size, real) if self.bulk else None
        self.d_bulk = [zb(), zb(), zb()]
        self.d_bulk_src = zb()
        self.IS_initialize()
        self.ideal_predict_for_first_step()

    def IS_initialize(self):  # visc.py:143-149
        self.k.visc_initialize(self.d_pi[1], self.d_goodcell, self.d_udiff, self.ideal.d_ev[1], self.ideal.tau,
                               self.d_bulk[1])

    def ideal_predict_for_first_step(self):  # visc.py:468-470
        self.ideal.stepUpdate(1)

    def load_ini(self, dat):
        self.ideal.load_ini(dat)

    def visc_stepUpdate(self, step):  # visc.py:232-283
        k, ev, pi, bp = self.k, self.ideal.d_ev, self.d_pi, self.d_bulk
        tau = self.ideal.tau
        k.visc_christoffel(self.ideal.d_Src, ev[step], pi[step], tau, step, bp[step])
        for axis in range(3):
            k.visc_along(axis, self.ideal.d_Src, ev[step], pi[step], tau, bp[step])
        k.visc_update_ev(ev[3 - step], ev[1], pi[0], pi[3 - step], self.ideal.d_Src, tau, step, bp[0], bp[3 - step])

    def IS_stepUpdate(self, step):  # visc.py:287-314
        k, ev, pi, bp = self.k, self.ideal.d_ev, self.d_pi, self.d_bulk
        tau = self.ideal.tau
        k.visc_src_christoffel(self.d_IS_src, pi[step], ev[step], tau, step, self.d_bulk_src)
        for axis, ud in enumerate((self.d_udx, self.d_udy, self.d_udz)):
            k.visc_src_along(axis, self.d_IS_src, ud, pi[step], ev[step], tau, self.d_bulk_src, bp[step])
        k.update_pimn(pi[3 - step], self.d_goodcell, pi[1], pi[step], ev[1], ev[2], self.d_udiff, self.d_udx,
                      self.d_udy, self.d_udz, self.d_IS_src, tau, step, bp[3 - step], bp[1], bp[step],
                      self.d_bulk_src)

    def update_udiff(self, ev0, ev1):
        self.k.get_udiff(self.d_udiff, ev0, ev1)

    def update_time(self, loop):
        self.ideal.update_time(loop)

    def step(self, loop):  # visc.py:527-544
        ev = self.ideal.d_ev
        self.d_pi[0][...] = self.d_pi[1]
        if self.bulk:
            self.d_bulk[0][...] = self.d_bulk[1]
        ev[0][...] = ev[1]
        self.IS_stepUpdate(1)
        self.visc_stepUpdate(1)
        self.update_time(loop)
        self.IS_stepUpdate(2)
        self.visc_stepUpdate(2)
        self.update_udiff(ev[0], ev[1])

    def get_hypersf(self, n, ntskip, is_finished):  # visc.py:359-397
        if n == 0:
            self.ideal.d_ev_old[...] = self.ideal.d_ev[1]
            self.d_pi_old[...] = self.d_pi[1]
            self.tau_old = self.cfg.TAU0
        elif (n % ntskip == 0) or is_finished:
            tau_new = self.ideal.tau
            sf, txyz, pisf = self.ideal._hypersf(1, self.cfg.real(self.tau_old), self.cfg.real(tau_new),
                                                 self.ideal.d_ev_old, self.ideal.d_ev[1], self.d_pi_old, self.d_pi[1])
            self.ideal.sf.append(sf)
            self.ideal.txyz.append(txyz)
            self.pisf.append(pisf)
            self.ideal.d_ev_old[...] = self.ideal.d_ev[1]
            self.d_pi_old[...] = self.d_pi[1]
            self.tau_old = tau_new

    def hypersf(self):
        sf, tx = self.ideal.hypersf()
        pisf = np.concatenate(self.pisf) if self.pisf else np.zeros((0, 10), self.cfg.real)
        return sf, tx, pisf

    def evolve(self, max_loops=1000, save_hypersf=True, force_run_to_maxloop=False):  # visc.py:473-560
        c = self.cfg
        if (c.ETAOS_YMIN < 1.0E-6 and c.ETAOS_LEFT_SLOP < 1.0E-6 and c.ETAOS_RIGHT_SLOP < 1.0E-6
                and not self.bulk):
            self.ideal.evolve(max_loops, save_hypersf, force_run_to_maxloop)
            return
        loop = 0
        while True:
            if force_run_to_maxloop and loop == max_loops:
                break
            if loop % c.ntskip == 0:
                self.ideal.edmax = self.ideal.max_energy_density()
                self.ideal.history.append([self.ideal.tau, self.ideal.edmax])
            is_finished = self.ideal.edmax < self.ideal.efrz
            if save_hypersf:
                self.get_hypersf(loop, c.ntskip, is_finished)
            if is_finished and not force_run_to_maxloop:
                break
            self.step(loop)
            loop += 1
