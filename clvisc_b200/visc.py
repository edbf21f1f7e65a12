"""CLVisc: viscous (3+1)D hydro on one GPU, the drop-in for pyvisc/visc.py.

Same constructor, attributes and methods as the reference class
(visc.py:20-560): ideal (the CLIdeal it wraps), d_pi[0..2], d_udiff,
d_goodcell; IS_initialize, visc_stepUpdate, IS_stepUpdate, update_udiff,
get_hypersf, save_pimn_sf, save, update_time, evolve. The construction
sequence is the reference's: pi is initialised from the still-empty state and
an ideal stage is run on it (visc.py:101-102), so the first time step sees the
same pi and d_ev[2] as the reference's.

Bulk viscosity is an extension (the reference has none): with ZETAOS_MAX > 0
the pi buffers carry an eleventh plane, the bulk pressure Pi, which the same
kernels advance (14-moment relaxation, P + Pi in T^{mu nu}); bulk_to_host()
reads it. ZETAOS_MAX = 0 (the default) leaves every result unchanged.

IS_stepUpdate and visc_stepUpdate launch the two halves of a Runge-Kutta
stage separately, as the reference does. evolve() launches one fused kernel
per stage that does both halves in one pass over memory; it skips the
reference's per-step copies d_pi[0] <- d_pi[1] and d_ev[0] <- d_ev[1]
(visc.py:527-532) because the fused kernel reads those values before it
overwrites them, so after evolve() d_pi[0] and d_ev[0] are not updated.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib
from .ideal import CLIdeal, add_visc_params


class CLVisc(object):
    """Viscous hydro (pyvisc/visc.py:20)."""

    def __init__(self, configs, handcrafted_eos=None, gpu_id=0, hypersf_capacity=None):
        kw = {} if hypersf_capacity is None else {'hypersf_capacity': hypersf_capacity}
        self.ideal = CLIdeal(configs, handcrafted_eos, gpu_id, **kw)
        self.cfg = configs
        self.lib = self.ideal.lib
        self.size = self.ideal.size
        self.ld = self.ideal.ld
        self.device = self.ideal.device
        self.dtype = self.ideal.dtype
        self.bulk = add_visc_params(self.cfg, self.ideal.params)
        self.params = self.ideal.params

        z = lambda w: torch.zeros((w, self.ld), dtype=self.dtype, device=self.device)
        npi = 11 if self.bulk else 10  # plane 10: the bulk pressure
        self.d_pi = [z(npi), z(npi), z(npi)]
        self.d_src = z(4 + npi)   # d_Src (planes 0..3), d_IS_src (planes 4..13), bulk source (14)
        self.d_udiff = z(4)
        self.d_goodcell = torch.ones(self.ld, dtype=torch.uint8, device=self.device)
        self.d_pi_old = z(npi)
        self.d_pi_sf = torch.zeros((self.ideal.hypersf_capacity, 10), dtype=self.dtype, device=self.device)
        self._key = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.IS_initialize()
        self.ideal_predict_for_first_step()

    @property
    def stream(self):
        return self.ideal.stream

    def _call(self, name, *args):
        _lib.check(getattr(self.lib, name)(ctypes.byref(self.params), *args), name)

    def IS_initialize(self):
        """Navier-Stokes pi from d_ev[1] (visc.py:143-149)."""
        self._call('clv_visc_initialize', _lib.ptr(self.d_pi[1]), _lib.ptr(self.d_goodcell), _lib.ptr(self.d_udiff),
                   _lib.ptr(self.ideal.d_ev[1]), float(self.ideal.tau), self.stream)

    def ideal_predict_for_first_step(self):
        """visc.py:468-470."""
        self.ideal.stepUpdate(step=1)

    def load_ini(self, dat):
        self.ideal.load_ini(dat)

    def optical_glauber_ini(self, system='Au+Au', cent_min=None, cent_max=None, save_binary_collisions=False):
        """visc.py:151-172: the optical Glauber initial condition into d_ev[1]."""
        self.ideal.optical_glauber_ini(system, cent_min, cent_max, save_binary_collisions)

    def load_hotspot_event(self, b=8.0, seed=5, edmax=50.0):
        """The seeded Pb+Pb event of initial.glauber_event, generated on the device."""
        self.ideal.load_hotspot_event(b, seed, edmax)

    def _buffers(self, step, parts, fused=False, edmax=False):
        e, pi = self.ideal.d_ev, self.d_pi
        b = _lib.ClvViscBuffers()
        b.ev_st = e[step].data_ptr()
        b.pi_st = pi[step].data_ptr()
        b.ev1 = e[1].data_ptr()
        b.ev2_ed = e[2].data_ptr()
        b.pi1 = pi[1].data_ptr()
        b.pi_n = (pi[1] if fused else pi[0]).data_ptr()
        b.pi_new_in = pi[3 - step].data_ptr()
        b.ev_new = e[3 - step].data_ptr()
        b.pi_new = pi[3 - step].data_ptr()
        b.src = self.d_src.data_ptr()
        b.udiff = self.d_udiff.data_ptr()
        b.goodcell = self.d_goodcell.data_ptr()
        b.edmax_key = self._key.data_ptr() if edmax else None
        b.write_src = 1 if (step == 1 or not fused) else 0
        b.write_udiff = 1 if (fused and step == 2) else 0
        return b

    def _stage(self, step, parts, fused=False, edmax=False):
        b = self._buffers(step, parts, fused, edmax)
        _lib.check(self.lib.clv_visc_stage(ctypes.byref(self.params), int(step), float(self.ideal.tau), int(parts),
                                           ctypes.byref(b), self.stream), 'clv_visc_stage')

    def visc_stepUpdate(self, step, jet_eloss_src=None):
        """T^{tau mu} half of a stage (visc.py:232-283): d_ev[3-step]."""
        if jet_eloss_src is not None and jet_eloss_src.get('switch_on', False):
            raise NotImplementedError('jet energy-loss sources are not part of this backend')
        self._stage(step, _lib.CLV_PART_KT)

    def IS_stepUpdate(self, step):
        """pi^{mu nu} half of a stage (visc.py:287-314): d_pi[3-step]."""
        self._stage(step, _lib.CLV_PART_IS)

    def update_udiff(self, d_ev0, d_ev1):
        """d_udiff = u(d_ev1) - u(d_ev0) (visc.py:352-357)."""
        self._call('clv_get_udiff', _lib.ptr(self.d_udiff), _lib.ptr(d_ev0), _lib.ptr(d_ev1), self.stream)

    def update_time(self, loop):
        self.ideal.update_time(loop)

    def step(self, loop, edmax=False):
        """One fused time step: both Runge-Kutta stages, pi and T^{tau mu}
        together (visc.py:527-544)."""
        both = _lib.CLV_PART_IS | _lib.CLV_PART_KT
        self._stage(1, both, fused=True)
        self.update_time(loop)
        if edmax:
            self._call('clv_max_ed_reset', _lib.ptr(self._key), self.stream)
        self._stage(2, both, fused=True, edmax=edmax)

    def read_edmax_key(self):
        out = ctypes.c_double()
        self._call('clv_max_ed_read', _lib.ptr(self._key), ctypes.byref(out), self.stream)
        return self.cfg.real(out.value)

    def get_hypersf(self, n, ntskip, is_finished):
        """Freeze-out surface between (d_ev_old, d_pi_old) and (d_ev[1], d_pi[1])
        (visc.py:359-397)."""
        if n == 0:
            self.ideal.d_ev_old.copy_(self.ideal.d_ev[1])
            self.d_pi_old.copy_(self.d_pi[1])
            self.tau_old = self.cfg.TAU0
        elif (n % ntskip == 0) or is_finished:
            tau_new = self.ideal.tau
            self.ideal._hypersf(1, self.cfg.real(self.tau_old), self.cfg.real(tau_new), self.ideal.d_ev_old,
                                self.ideal.d_ev[1], self.d_pi_old, self.d_pi[1], self.d_pi_sf)
            self.ideal.d_ev_old.copy_(self.ideal.d_ev[1])
            self.d_pi_old.copy_(self.d_pi[1])
            self.tau_old = tau_new

    def save_pimn_sf(self, set_to_zero=False):
        """pimnsf.dat (visc.py:400-419)."""
        num_of_sf = self.ideal.num_of_sf
        ed = self.ideal.efrz
        pr = self.ideal.eos.f_P(ed)
        T = self.cfg.TFRZ
        const_for_deltaf = 1.0 / (2.0 * T ** 2 * (ed + pr))
        pi_onsf = np.zeros((num_of_sf, 10), dtype=self.cfg.real)
        if not set_to_zero:
            pi_onsf = self.d_pi_sf[:num_of_sf].cpu().numpy()
        out_path = os.path.join(self.cfg.fPathOut, 'pimnsf.dat')
        comment_line = 'one_o_2TsqrEplusP=%.6e ' % const_for_deltaf + 'pi00 01 02 03 11 12 13 22 23 33'
        _lib.write_table(out_path, comment_line, pi_onsf.reshape(num_of_sf, 10))

    def save(self, save_hypersf=True, save_bulk=False, save_pi=False, save_vorticity=False):
        """visc.py:423-462 (vorticity output is not part of this backend)."""
        self.ideal.save(save_hypersf, save_bulk, viscous_on=True)
        if save_hypersf:
            self.save_pimn_sf()

    def status(self, slot=1):
        """Health of d_ev[slot], d_pi[slot] after a step (clv_status): a dict
        with the non-finite values of the fields ('nan'), the cells whose pi
        was reset by the bad-cell test ('bad_cells', kernel_IS.cl:697-708) and
        the surface elements found beyond the capacity ('sf_overflow')."""
        counts = torch.zeros(3, dtype=torch.int64, device=self.device)
        host = (ctypes.c_longlong * 3)()
        self._call('clv_status', _lib.ptr(self.ideal.d_ev[slot]), _lib.ptr(self.d_pi[slot]),
                   int(self.d_pi[slot].shape[0]), _lib.ptr(self.d_goodcell), _lib.ptr(self.ideal.d_num_of_sf),
                   int(self.ideal.hypersf_capacity), _lib.ptr(counts), ctypes.cast(host, ctypes.c_void_p),
                   self.stream)
        return {'nan': int(host[0]), 'bad_cells': int(host[1]), 'sf_overflow': int(host[2])}

    def pi_to_host(self, slot=1):
        """d_pi[slot] as (cells, 10)."""
        return self.ideal.field_to_host(self.d_pi[slot][:10])

    def bulk_to_host(self, slot=1):
        """The bulk pressure Pi of d_pi[slot] as (cells,); zeros without the
        bulk sector."""
        if not self.bulk:
            return np.zeros(self.size, self.cfg.real)
        return self.d_pi[slot][10, :self.size].cpu().numpy()

    def evolve(self, max_loops=1000, save_hypersf=True, save_bulk=False, plot_bulk=False, save_pi=True,
               force_run_to_maxloop=False, save_vorticity=False, jet_eloss_src=None, debug=False):
        """Main loop (visc.py:473-560)."""
        if save_vorticity:
            raise NotImplementedError('vorticity output is not part of this backend')
        c = self.cfg
        if (c.ETAOS_YMIN < 1.0E-6 and c.ETAOS_LEFT_SLOP < 1.0E-6 and c.ETAOS_RIGHT_SLOP < 1.0E-6
                and not self.bulk):
            # visc.py:483-489: ideal evolution when eta/s vanishes
            self.ideal.evolve(max_loops, save_hypersf, save_bulk, plot_bulk, force_run_to_maxloop, jet_eloss_src)
            self.save_pimn_sf(set_to_zero=True)
            return
        loop = 0
        edmax_pending = False
        while True:
            if force_run_to_maxloop and loop == max_loops:
                break
            if loop % c.ntskip == 0:
                self.ideal.edmax = self.read_edmax_key() if edmax_pending else self.ideal.max_energy_density()
                self.ideal.history.append([self.ideal.tau, self.ideal.edmax])
            is_finished = self.ideal.edmax < self.ideal.efrz
            if save_hypersf:
                self.get_hypersf(loop, c.ntskip, is_finished)
            if (plot_bulk or save_bulk) and loop % c.ntskip == 0:
                self.ideal.bulkinfo.get(self.ideal.tau, self.ideal.d_ev[1], self.ideal.edmax, self.d_pi[1])
            if is_finished and not force_run_to_maxloop:
                break
            edmax_pending = ((loop + 1) % c.ntskip == 0)
            self.step(loop, edmax=edmax_pending)
            loop = loop + 1
        self.save(save_hypersf=save_hypersf, save_bulk=save_bulk, save_pi=save_pi, save_vorticity=save_vorticity)
