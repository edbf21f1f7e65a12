"""CLIdeal: ideal (3+1)D hydro on one GPU, the drop-in for pyvisc/ideal.py.

Same constructor, attributes and methods as the reference class
(ideal.py:28-349): d_ev[0..2] (d_ev[1] is the state and the target of the
initial condition), d_Src, tau, edmax, efrz, history, num_of_sf, eos, h_ev1;
load_ini, stepUpdate, max_energy_density, ev_to_host, get_hypersf, save,
update_time, evolve. Device buffers are torch tensors holding
structure-of-arrays planes (shape (components, ld)); the arrays exchanged with
the host keep the reference's (cells, 4) layout. All arithmetic runs in the
CUDA library libclvisc_b200.so.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib
from .config import float_literal, set_real
from .eos import Eos, TABLE_SHAPE

HYPERSF_CAPACITY = 1500000  # elements, as the reference allocates (ideal.py:113-115)


def plane_stride(n):
    """Plane stride: n rounded up to 64 elements (256-byte aligned planes)."""
    return ((n + 63) // 64) * 64


def make_params(c, meta, eos_table, efrz, nx, ny, nz, ld):
    """clv_params of a run: the grid, and the constants the reference passes
    to its kernels as -D float literals (ideal.py:146-171, eos.py:194-201)."""
    p = _lib.ClvParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.ld = ld
    p.precision = 4 if c.use_float32 else 8
    for key in ('dt', 'dx', 'dy', 'dz', 'tau0'):
        setattr(p, key, float_literal(getattr(c, key.upper())))
    p.etaos_xmin = float_literal(c.ETAOS_XMIN)
    p.etaos_ymin = float_literal(c.ETAOS_YMIN)
    p.etaos_left_slop = float_literal(c.ETAOS_LEFT_SLOP)
    p.etaos_right_slop = float_literal(c.ETAOS_RIGHT_SLOP)
    p.lam1 = float_literal(c.LAM1)
    p.efrz = float_literal(efrz)
    p.nxskip, p.nyskip, p.nzskip = c.nxskip, c.nyskip, c.nzskip
    p.eos_ed_start = float_literal(meta['ed_start'])
    p.eos_ed_step = float_literal(meta['ed_step'])
    p.eos_num_ed = int(meta['num_of_ed'])
    p.eos_nrow, p.eos_ncol = int(meta['nrow']), int(meta['ncol'])
    p.eos_table = eos_table.data_ptr()
    # pressure pairs (p[t], p[t+1]) for the tolerance build's one-read lookup,
    # kept alive with the struct
    pr = eos_table.view(-1, 4)[:, 1]
    p._eos_p2 = torch.stack([pr, torch.cat([pr[1:], pr[-1:]])], dim=1).contiguous()
    p.eos_p2 = p._eos_p2.data_ptr()
    flags = 0
    if getattr(c, 'riemann_test', False):
        flags |= _lib.CLV_FLAG_RIEMANN_TEST
    p.flags = flags
    return p


def add_visc_params(c, p):
    """The viscous run's flags (visc.py:111-121) and bulk-sector constants on
    top of make_params(); returns whether the bulk sector is on."""
    flags = p.flags
    if getattr(c, 'gubser_visc_test', False):
        flags |= _lib.CLV_FLAG_GUBSER_VISC_TEST
    if getattr(c, 'pimn_omega_coupling', False):
        flags |= _lib.CLV_FLAG_PIMN_OMEGA_COUPLING
    if getattr(c, 'omega_omega_coupling', False):
        flags |= _lib.CLV_FLAG_OMEGA_OMEGA_COUPLING
    bulk = float(getattr(c, 'ZETAOS_MAX', 0.0)) > 0.0
    p.zetaos_max = float_literal(getattr(c, 'ZETAOS_MAX', 0.0))
    p.zetaos_t0 = float_literal(getattr(c, 'ZETAOS_T0', 0.18))
    p.zetaos_width = float_literal(getattr(c, 'ZETAOS_WIDTH', 0.02))
    p.zetaos_skew = float_literal(getattr(c, 'ZETAOS_SKEW', 0.0))
    p.zetaos_tmin = float_literal(getattr(c, 'ZETAOS_TMIN', 0.1))
    if bulk:
        flags |= _lib.CLV_FLAG_BULK
    if fast_arithmetic(c):
        flags |= _lib.CLV_FLAG_FAST
    p.flags = flags
    return bulk


def fast_arithmetic(c):
    """Whether the fused viscous stage runs in the tolerance arithmetic
    (CLV_FLAG_FAST): cfg.arithmetic 'fast' (the default) or 'auto'; 'exact'
    keeps the reference's arithmetic bit for bit."""
    mode = str(getattr(c, 'arithmetic', 'fast')).lower()
    if mode not in ('auto', 'fast', 'exact'):
        raise ValueError("cfg.arithmetic must be 'fast' or 'exact' ('auto' = 'fast'), not %r" % mode)
    return mode != 'exact'


def load_eos(cfg, handcrafted_eos, device):
    """(Eos object, device float32 table, table metadata, freeze-out energy density)."""
    eos = Eos(cfg.eos_type) if handcrafted_eos is None else handcrafted_eos
    if handcrafted_eos is None:
        table, meta = eos.create_table(*TABLE_SHAPE[cfg.eos_type])
    else:
        table, meta = eos.create_table()
    return eos, torch.from_numpy(table.reshape(-1)).to(device), meta, eos.f_ed(cfg.TFRZ)


class CLIdeal(object):
    """Ideal hydro (pyvisc/ideal.py:28)."""

    def __init__(self, configs, handcrafted_eos=None, gpu_id=0, hypersf_capacity=HYPERSF_CAPACITY):
        self.cfg = configs
        os.makedirs(self.cfg.fPathOut, exist_ok=True)
        set_real(self.cfg)
        if not torch.cuda.is_available():
            raise RuntimeError('CLIdeal needs a CUDA device; there is no CPU path')
        self.lib = _lib.load()
        self.device = torch.device('cuda', gpu_id)
        torch.cuda.set_device(self.device)
        self.dtype = torch.float32 if self.cfg.use_float32 else torch.float64
        self.size = self.cfg.NX * self.cfg.NY * self.cfg.NZ
        self.ld = plane_stride(self.size)
        self.tau = self.cfg.real(self.cfg.TAU0)

        self.eos, self.eos_table, meta, self.efrz = load_eos(self.cfg, handcrafted_eos, self.device)
        # effective chemical potentials on the freeze-out surface (ideal.py:65)
        from .chempot import write_chemical_potential
        self.chemical_potential = write_chemical_potential(self.eos.f_ed(self.cfg.TFRZ), self.cfg.fPathOut,
                                                           eos_type=self.cfg.eos_type)
        self.params = self._make_params(meta)
        from .bulkinfo import BulkInfo
        self.bulkinfo = BulkInfo(self.cfg, self.lib, self.params, self.eos, self.device)

        z = lambda w: torch.zeros((w, self.ld), dtype=self.dtype, device=self.device)
        self.h_ev1 = np.zeros((self.size, 4), self.cfg.real)
        self.d_ev = [z(4), z(4), z(4)]
        self.d_Src = z(4)
        self.d_ev_old = z(4)
        self.hypersf_capacity = int(hypersf_capacity)
        self.d_hypersf = torch.zeros((self.hypersf_capacity, 8), dtype=self.dtype, device=self.device)
        self.d_sf_txyz = torch.zeros((self.hypersf_capacity, 4), dtype=self.dtype, device=self.device)
        self.d_num_of_sf = torch.zeros(1, dtype=torch.int64, device=self.device)
        self._hsf_scratch = torch.empty(int(self.lib.clv_hypersf_scratch_bytes(ctypes.byref(self.params))),
                                        dtype=torch.uint8, device=self.device)
        self._key = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.history = []
        self.edmax = None
        self.num_of_sf = 0
        self.tau_old = self.cfg.TAU0

    # ------------------------------------------------------------ helpers
    def _make_params(self, meta):
        return make_params(self.cfg, meta, self.eos_table, self.efrz, self.cfg.NX, self.cfg.NY, self.cfg.NZ, self.ld)

    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _call(self, name, *args):
        _lib.check(getattr(self.lib, name)(ctypes.byref(self.params), *args), name)

    # ------------------------------------------------------------- API
    def load_ini(self, dat):
        """Copy an (NX*NY*NZ, 4) array of (ed, vx, vy, veta) into d_ev[1]
        (ideal.py:138-144). A pinned torch tensor is copied without staging."""
        if isinstance(dat, torch.Tensor) and dat.device.type == 'cpu' and dat.is_pinned() \
                and dat.dtype == self.dtype and dat.is_contiguous():
            host = dat.reshape(self.size, 4)
        else:
            self.h_ev1 = np.ascontiguousarray(dat, dtype=self.cfg.real).reshape(self.size, 4)
            host = torch.from_numpy(self.h_ev1).pin_memory()
        dev = host.to(self.device, non_blocking=True)
        self._call('clv_aos_to_soa', _lib.ptr(dev), _lib.ptr(self.d_ev[1]), self.size, 4, self.stream)
        torch.cuda.current_stream(self.device).synchronize()

    def optical_glauber_ini(self, system='Au+Au', cent_min=None, cent_max=None, save_binary_collisions=False):
        """d_ev[1] from the optical Glauber model on the device
        (visc.py:151-172, kernel_glauber.cl:86-102); with a centrality class the
        impact parameter is its weighted mean (glauber.py:14-57) and is written
        into the configuration, as in the reference."""
        from .glauber import glauber_consts, weight_mean_b
        if cent_min is not None and cent_max is not None:
            self.cfg.ImpactParameter = weight_mean_b(cent_min, cent_max, system)
        g = glauber_consts(self.cfg)
        self._call('clv_glauber_ini', ctypes.byref(g), _lib.ptr(self.d_ev[1]), self.stream)
        if save_binary_collisions:
            self.save_nbinary()

    def save_nbinary(self, dx=0.3, dy=0.3, xlow=-9.75, ylow=-9.75, nx=66, ny=66):
        """Binary collisions on a (66, 66) grid into fPathOut/nbin.dat (glauber.py:94-103)."""
        from .glauber import glauber_consts
        g = glauber_consts(self.cfg)
        out = torch.empty(nx * ny, dtype=self.dtype, device=self.device)
        self._call('clv_glauber_nbinary', ctypes.byref(g), _lib.ptr(out), float(self.cfg.real(xlow)),
                   float(self.cfg.real(ylow)), float(self.cfg.real(dx)), float(self.cfg.real(dy)), nx, ny, self.stream)
        np.savetxt(os.path.join(self.cfg.fPathOut, 'nbin.dat'), out.cpu().numpy().reshape(nx, ny))

    def load_hotspot_event(self, b=8.0, seed=5, edmax=50.0):
        """d_ev[1] = initial.glauber_event(NX, NY, NZ, DX, DY, DZ, b, seed,
        edmax), with the participants sampled on the host and the energy density
        summed on the device."""
        from .initial import hotspot_ini, hotspot_table
        c = self.cfg
        keep = hotspot_ini(self.lib, self.params, self.d_ev[1], hotspot_table(b, seed), c.DX, c.DY, c.DZ,
                           edmax=edmax, stream=self.stream)
        torch.cuda.current_stream(self.device).synchronize()
        del keep

    def load_ini_device(self, dev_aos):
        """load_ini from a device tensor of shape (NX*NY*NZ, 4)."""
        dev_aos = dev_aos.to(self.device, self.dtype).contiguous()
        self._call('clv_aos_to_soa', _lib.ptr(dev_aos), _lib.ptr(self.d_ev[1]), self.size, 4, self.stream)

    def ev_to_host(self, out=None):
        """d_ev[1] -> h_ev1 as (cells, 4) (ideal.py:265-267). `out`: an
        optional pinned host tensor of that shape and the run's dtype, filled
        by one direct copy (no pageable staging)."""
        self.h_ev1 = self.field_to_host(self.d_ev[1], out=out)
        return self.h_ev1

    def field_to_host(self, t, w=None, out=None):
        """Any SoA field -> numpy (cells, w); into the pinned host tensor
        `out` when one is given."""
        w = t.shape[0] if w is None else w
        aos = torch.empty((self.size, w), dtype=self.dtype, device=self.device)
        self._call('clv_soa_to_aos', _lib.ptr(t), _lib.ptr(aos), self.size, w, self.stream)
        if out is not None:
            if tuple(out.shape) != (self.size, w) or out.dtype != self.dtype or not out.is_pinned():
                raise ValueError('out must be a pinned (%d, %d) %s tensor' % (self.size, w, self.dtype))
            out.copy_(aos, non_blocking=True)
            torch.cuda.current_stream(self.device).synchronize()
            return out.numpy()
        return aos.cpu().numpy()

    def field_from_host(self, t, arr):
        """numpy (cells, w) -> the first w planes of an SoA field (the inverse
        of field_to_host), e.g. d_ev[2] or d_pi[1] for a test's initial state."""
        w = int(np.asarray(arr).shape[1])
        if w > t.shape[0]:
            raise ValueError('field has %d planes, array has %d columns' % (t.shape[0], w))
        host = torch.from_numpy(np.ascontiguousarray(arr, dtype=self.cfg.real).reshape(self.size, w))
        dev = host.to(self.device)
        self._call('clv_aos_to_soa', _lib.ptr(dev), _lib.ptr(t), self.size, w, self.stream)
        torch.cuda.current_stream(self.device).synchronize()

    def stepUpdate(self, step, jet_eloss_src=None):
        """One Runge-Kutta stage (ideal.py:211-255): d_ev[3-step] from
        d_ev[step], with d_Src zeroed at step 1 and accumulated at step 2."""
        if jet_eloss_src is not None and jet_eloss_src.get('switch_on', False):
            raise NotImplementedError('jet energy-loss sources are not part of this backend')
        self._call('clv_ideal_stage', int(step), float(self.tau), _lib.ptr(self.d_ev[step]), _lib.ptr(self.d_ev[1]),
                   _lib.ptr(self.d_ev[3 - step]), _lib.ptr(self.d_Src), 1, None, self.stream)

    def max_energy_density(self):
        """Maximum energy density of d_ev[1] (ideal.py:257-262)."""
        self._call('clv_max_ed_reset', _lib.ptr(self._key), self.stream)
        self._call('clv_max_ed', _lib.ptr(self.d_ev[1]), _lib.ptr(self._key), self.stream)
        out = ctypes.c_double()
        self._call('clv_max_ed_read', _lib.ptr(self._key), ctypes.byref(out), self.stream)
        return self.cfg.real(out.value)

    def _hypersf(self, visc, tau_old, tau_new, ev_old, ev_new, pi_old=None, pi_new=None, pisf=None):
        self._call('clv_hypersf_append', int(visc), float(tau_old), float(tau_new), _lib.ptr(ev_old), _lib.ptr(ev_new),
                   _lib.ptr(pi_old), _lib.ptr(pi_new), _lib.ptr(self.d_hypersf), _lib.ptr(self.d_sf_txyz),
                   _lib.ptr(pisf), self.hypersf_capacity, _lib.ptr(self.d_num_of_sf), _lib.ptr(self._hsf_scratch),
                   self._hsf_scratch.numel(), self.stream)

    def get_hypersf(self, n, ntskip):
        """Freeze-out surface between d_ev_old and d_ev[1] (ideal.py:269-293)."""
        is_finished = self.edmax < self.efrz
        if n == 0:
            self.d_ev_old.copy_(self.d_ev[1])
            self.tau_old = self.cfg.TAU0
        elif (n % ntskip == 0) or is_finished:
            tau_new = self.tau
            self._hypersf(0, self.cfg.real(self.tau_old), self.cfg.real(tau_new), self.d_ev_old, self.d_ev[1])
            self.d_ev_old.copy_(self.d_ev[1])
            self.tau_old = tau_new
        return is_finished

    def read_num_of_sf(self):
        n = int(self.d_num_of_sf.item())
        if n > self.hypersf_capacity:
            raise RuntimeError('freeze-out surface has %d elements, capacity %d: raise hypersf_capacity'
                               % (n, self.hypersf_capacity))
        return n

    def hypersf_to_host(self):
        n = self.read_num_of_sf()
        return self.d_hypersf[:n].cpu().numpy(), self.d_sf_txyz[:n].cpu().numpy()

    def save(self, save_hypersf=True, save_bulk=False, viscous_on=False):
        """Write hypersf.dat and sf_txyz.dat, and the bulk diagnostics
        (ideal.py:295-315)."""
        self.num_of_sf = self.read_num_of_sf()
        if save_hypersf:
            hypersf, sf_txyz = self.hypersf_to_host()
            _lib.write_table(os.path.join(self.cfg.fPathOut, 'hypersf.dat'),
                             'Tfrz=%.6e ; other rows: dS0, dS1, dS2, dS3, vx, vy, veta, etas' % self.cfg.TFRZ, hypersf)
            _lib.write_table(os.path.join(self.cfg.fPathOut, 'sf_txyz.dat'),
                             '(t, x, y, z) the time-space coordinates of hypersf elements', sf_txyz)
        if save_bulk:
            self.bulkinfo.save(viscous_on=viscous_on)

    def update_time(self, loop):
        """tau = TAU0 + (loop+1)*DT in the run precision (ideal.py:317-320)."""
        self.tau = self.cfg.real(self.cfg.TAU0 + (loop + 1) * self.cfg.DT)

    def evolve(self, max_loops=2000, save_hypersf=True, save_bulk=True, plot_bulk=True, to_maxloop=False,
               jet_eloss_src=None):
        """Main loop (ideal.py:322-349)."""
        for n in range(max_loops):
            self.edmax = self.max_energy_density()
            self.history.append([self.tau, self.edmax])
            is_finished = False
            if save_hypersf:
                is_finished = self.get_hypersf(n, self.cfg.ntskip)
            if is_finished and not to_maxloop:
                break
            if (save_bulk or plot_bulk) and n % self.cfg.ntskip == 0:
                self.bulkinfo.get(self.tau, self.d_ev[1], self.edmax)
            self.stepUpdate(step=1)
            self.update_time(loop=n)
            self.stepUpdate(step=2, jet_eloss_src=jet_eloss_src)
        self.save(save_hypersf=save_hypersf, save_bulk=save_bulk)
