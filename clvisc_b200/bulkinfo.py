"""BulkInfo: evolution diagnostics of a run (pyvisc/bulkinfo.py), computed on
the device.

The reference copies slices of the state to the host every ntskip steps and,
for the momentum eccentricity versus rapidity, the whole state
(bulkinfo.py:120-271); the sums behind every diagnostic are then taken with
numpy. Here the slices are gathered by a kernel and the sums are reduced on
the device (clv_bulk_slices, clv_bulk_sums, clv_bulk_lab_totals), so a call
moves a few slices and a few numbers to the host. The attributes, get() and
save() and the files save() writes are the reference's; the only difference in
the numbers is that the device evaluates P(e) and s(e) from the run's EOS
table where the reference's host code interpolates the EOS grid. The lab-frame
total energy and entropy of bulkinfo_h5.py are recorded too (energy,
entropy_total; written to energy_entropy_total.dat).
"""
import ctypes
import os
from math import floor

import numpy as np
import torch

from . import _lib


class BulkInfo(object):
    """Bulk information of one run: ed, T, v along x, y, eta_s and in planes,
    momentum eccentricities, <v_r>, entropy (pyvisc/bulkinfo.py:25)."""

    def __init__(self, cfg, lib, params, eos, device):
        self.cfg = cfg
        self.lib = lib
        self.params = params
        self.eos = eos
        self.device = device
        NX, NY, NZ = cfg.NX, cfg.NY, cfg.NZ
        self.ex, self.ey, self.ez = [], [], []
        self.vx, self.vy, self.vz = [], [], []
        self.exy, self.vx_xy, self.vy_xy, self.vz_xy = [], [], [], []
        self.pixx_xy, self.piyy_xy, self.pitx_xy = [], [], []
        self.exz, self.vx_xz, self.vy_xz, self.vz_xz = [], [], [], []
        self.ecc2_vs_rapidity = []
        self.ecc1_vs_rapidity = []
        self.time = []
        self.edmax = []
        self.plane_sums = []
        self.energy, self.entropy_total = [], []
        self.x = np.linspace(-floor(NX / 2) * cfg.DX, floor(NX / 2) * cfg.DX, NX, endpoint=True)
        self.y = np.linspace(-floor(NY / 2) * cfg.DY, floor(NY / 2) * cfg.DY, NY, endpoint=True)
        self.z = np.linspace(-floor(NZ / 2) * cfg.DZ, floor(NZ / 2) * cfg.DZ, NZ, endpoint=True)
        dtype = torch.float32 if cfg.use_float32 else torch.float64
        n = int(lib.clv_bulk_slices_size(ctypes.byref(params)))
        self._slices = torch.zeros(n, dtype=dtype, device=device)
        self._sums = torch.zeros(3 * NZ + 8, dtype=torch.float64, device=device)
        self._lab = torch.zeros(2, dtype=torch.float64, device=device)
        self._lab_scratch = torch.zeros(int(lib.clv_bulk_lab_scratch_bytes()) // 8 + 1, dtype=torch.float64,
                                        device=device)

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _call(self, name, *args):
        _lib.check(getattr(self.lib, name)(ctypes.byref(self.params), *args), name)

    def get(self, tau, d_ev1, edmax, d_pi=None):
        """Record the diagnostics of the state d_ev1 (and d_pi) at tau
        (bulkinfo.py:120-182)."""
        c = self.cfg
        NX, NY, NZ = c.NX, c.NY, c.NZ
        self.time.append(tau)
        self.edmax.append(edmax)
        s = self._stream()
        self._call('clv_bulk_slices', _lib.ptr(d_ev1), _lib.ptr(d_pi), _lib.ptr(self._slices), s)
        self._call('clv_bulk_sums', _lib.ptr(d_ev1), _lib.ptr(d_pi), _lib.ptr(self._sums), s)
        volume = float(tau) * c.DX * c.DY * c.DZ
        self._call('clv_bulk_lab_totals', _lib.ptr(d_ev1), float(tau), volume, _lib.ptr(self._lab),
                   _lib.ptr(self._lab_scratch), self._lab_scratch.numel() * 8, s)
        h = self._slices.cpu().numpy()
        sums = self._sums.cpu().numpy()
        lab = self._lab.cpu().numpy()
        o = 0

        def take(n, w):
            nonlocal o
            a = h[o:o + n * w].reshape(n, w) if w > 1 else h[o:o + n]
            o += n * w
            return a
        evx0, evy0, evz0 = take(NX, 4), take(NY, 4), take(NZ, 4)
        evxy, evxz = take(NX * NY, 4), take(NX * NZ, 4)
        take(NY * NZ, 4)
        self.ex.append(evx0[:, 0].copy())
        self.ey.append(evy0[:, 0].copy())
        self.ez.append(evz0[:, 0].copy())
        self.vx.append(evx0[:, 1].copy())
        self.vy.append(evy0[:, 2].copy())
        self.vz.append(evz0[:, 3].copy())
        self.exy.append(evxy[:, 0].reshape(NX, NY).copy())
        self.vx_xy.append(evxy[:, 1].reshape(NX, NY).copy())
        self.vy_xy.append(evxy[:, 2].reshape(NX, NY).copy())
        self.exz.append(evxz[:, 0].reshape(NX, NZ).copy())
        self.vx_xz.append(evxz[:, 1].reshape(NX, NZ).copy())
        self.vy_xz.append(evxz[:, 2].reshape(NX, NZ).copy())
        self.vz_xz.append(evxz[:, 3].reshape(NX, NZ).copy())
        if d_pi is not None:
            self.pixx_xy.append(take(NX * NY, 1).reshape(NX, NY).copy())
            self.piyy_xy.append(take(NX * NY, 1).reshape(NX, NY).copy())
            self.pitx_xy.append(take(NX * NY, 1).reshape(NX, NY).copy())
        # momentum eccentricities per eta_s slice (bulkinfo.py:259-271)
        per = sums[:3 * NZ].reshape(NZ, 3)
        self.ecc1_vs_rapidity.append(per[:, 2] / (per[:, 0] + per[:, 1]))
        self.ecc2_vs_rapidity.append((per[:, 0] - per[:, 1]) / (per[:, 0] + per[:, 1]))
        self.plane_sums.append(sums[3 * NZ:].copy())
        self.energy.append(float(lab[0]))
        self.entropy_total.append(float(lab[1]))

    # the plane diagnostics of bulkinfo.py:184-257 from the device sums
    def eccp(self, idx, viscous=False):
        txx, tyy, t0x, _, _, _, pi_sum, pi_dif = self.plane_sums[idx]
        v1 = t0x / (txx + tyy)
        v2 = ((txx - tyy) + pi_dif) / ((txx + tyy) + pi_sum) if viscous else (txx - tyy) / (txx + tyy)
        return v1, v2

    def mean_vr(self, idx):
        s = self.plane_sums[idx]
        return s[3] / s[4]

    def total_entropy(self, idx):
        return self.plane_sums[idx][5] * self.time[idx] * self.cfg.DX * self.cfg.DY

    def save(self, viscous_on=False):
        """Write the recorded diagnostics to fPathOut (bulkinfo.py:273-340)."""
        path_out = os.path.abspath(self.cfg.fPathOut)
        os.makedirs(path_out, exist_ok=True)
        f_T = self.eos.f_T
        np.savetxt(path_out + '/ex.dat', np.array(self.ex).T)
        np.savetxt(path_out + '/ey.dat', np.array(self.ey).T)
        np.savetxt(path_out + '/ez.dat', np.array(self.ez).T)
        np.savetxt(path_out + '/Tx.dat', f_T(np.array(self.ex)).T)
        np.savetxt(path_out + '/Ty.dat', f_T(np.array(self.ey)).T)
        np.savetxt(path_out + '/Tz.dat', f_T(np.array(self.ez)).T)
        np.savetxt(path_out + '/vx.dat', np.array(self.vx).T)
        np.savetxt(path_out + '/vy.dat', np.array(self.vy).T)
        np.savetxt(path_out + '/vz.dat', np.array(self.vz).T)
        if len(self.ecc2_vs_rapidity) != 0:
            np.savetxt(path_out + '/ecc2.dat', np.array(self.ecc2_vs_rapidity).T)
            np.savetxt(path_out + '/ecc1.dat', np.array(self.ecc1_vs_rapidity).T)
        entropy, vr, ecc2, ecc2_visc = [], [], [], []
        for idx, exy in enumerate(self.exy):
            np.savetxt(path_out + '/edxy%d.dat' % idx, exy)
            np.savetxt(path_out + '/Txy%d.dat' % idx, f_T(exy))
            np.savetxt(path_out + '/vx_xy%d.dat' % idx, self.vx_xy[idx])
            np.savetxt(path_out + '/vy_xy%d.dat' % idx, self.vy_xy[idx])
            ecc2.append(self.eccp(idx)[1])
            vr.append(self.mean_vr(idx))
            entropy.append(self.total_entropy(idx))
            if viscous_on:
                ecc2_visc.append(self.eccp(idx, viscous=True)[1])
        for idx, exz in enumerate(self.exz):
            np.savetxt(path_out + '/ed_xz%d.dat' % idx, exz)
            np.savetxt(path_out + '/vx_xz%d.dat' % idx, self.vx_xz[idx])
            np.savetxt(path_out + '/vy_xz%d.dat' % idx, self.vy_xz[idx])
            np.savetxt(path_out + '/vz_xz%d.dat' % idx, self.vz_xz[idx])
            np.savetxt(path_out + '/T_xz%d.dat' % idx, f_T(exz))
        np.savetxt(path_out + '/eccp.dat', np.array(list(zip(self.time, ecc2))), header='tau  eccp')
        if viscous_on:
            np.savetxt(path_out + '/eccp_visc.dat', np.array(list(zip(self.time, ecc2_visc))),
                       header='tau  eccp_visc')
        np.savetxt(path_out + '/Tmax.dat', np.array(list(zip(self.time, f_T(np.array(self.edmax))))),
                   header='tau, Tmax')
        np.savetxt(path_out + '/edmax.dat', np.array(list(zip(self.time, self.edmax))), header='tau, edmax')
        np.savetxt(path_out + '/vr.dat', np.array(list(zip(self.time, vr))), header='tau <vr>')
        np.savetxt(path_out + '/entropy.dat', np.array(list(zip(self.time, entropy))), header='tau  entropy')
        np.savetxt(path_out + '/energy_entropy_total.dat',
                   np.array(list(zip(self.time, self.energy, self.entropy_total))),
                   header='tau  lab-frame energy  entropy (all cells, tau DX DY DZ per cell)')
