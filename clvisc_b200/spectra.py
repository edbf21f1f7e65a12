"""SmoothSpec: Cooper-Frye smooth hadron spectra from the freeze-out surface
(CLSmoothSpec/src/cl_spec.cpp, kernel_spec.cl, kernel_spec_csc.cl), on the
device.

The surface may be the device buffers of a finished CLVisc / CLIdeal run
(d_hypersf, d_pi_sf) or the hypersf.dat / pimnsf.dat files they write. The
momentum grid is the reference's (Spec::InitGrid, cl_spec.cpp:150-182): NY
rapidities evenly spaced in [YLO, YHI], NPT transverse momenta at the 15-point
Gauss-Laguerre nodes scaled by 1/12 GeV, NPHI azimuths at the 48-point
Gauss-Legendre nodes mapped onto [0, 2 pi] (nodes computed with numpy rather
than read from a table). Resonance decays (kernel_decay.cl) are not part of
this module; with decays off the reference also computes only the direct
spectra of pi+, K+ and p (cl_spec.cpp:531-534).
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib

# mass [GeV], 2J+1, +1 baryon (Fermi-Dirac) / -1 meson (Bose-Einstein) of the
# hadrons whose direct spectra the reference writes without decays
HADRONS = {211: (0.13957, 1.0, -1.0), 321: (0.493677, 1.0, -1.0), 2212: (0.938272, 2.0, 1.0)}


class SpectraArgs(ctypes.Structure):  # clv_spectra_args
    _fields_ = [('precision', ctypes.c_int), ('sf', ctypes.c_void_p), ('pisf', ctypes.c_void_p),
                ('n', ctypes.c_longlong), ('mass', ctypes.c_double), ('gspin', ctypes.c_double),
                ('fermi_boson', ctypes.c_double), ('mu', ctypes.c_double), ('tfrz', ctypes.c_double),
                ('tcoeff', ctypes.c_double), ('y', ctypes.c_void_p), ('pt', ctypes.c_void_p),
                ('cphi', ctypes.c_void_p), ('sphi', ctypes.c_void_p), ('ny', ctypes.c_int), ('npt', ctypes.c_int),
                ('nphi', ctypes.c_int)]


def momentum_grid(ny=41, ylo=-8.0, yhi=8.0, npt=15, nphi=48, invslope=1.0 / 12.0):
    """(Y, Pt, Phi) of Spec::InitGrid (cl_spec.cpp:150-182)."""
    dy = (yhi - ylo) / (ny - 1.0)
    y = np.array([ylo + i * dy for i in range(ny)])
    x, _ = np.polynomial.legendre.leggauss(nphi)
    pgauss = x[nphi // 2:][::-1]  # positive nodes, largest first
    phi = np.empty(nphi)
    for i in range(nphi // 2):
        phi[nphi - 1 - i] = np.pi * (pgauss[i] + 1.0)
        phi[i] = np.pi * (1.0 - pgauss[i])
    xl, _ = np.polynomial.laguerre.laggauss(npt)
    pt = invslope * xl + 0.0
    return y, pt, phi


def read_hypersf(path):
    """hypersf.dat -> (n, 8) array and Tfrz (Spec::ReadHyperSF, cl_spec.cpp:205-233:
    elements with a NaN in dSigma are zeroed)."""
    with open(path) as f:
        head = f.readline()
    tfrz = float(head.split('Tfrz=')[1].split(';')[0])
    sf = np.loadtxt(path, ndmin=2)
    bad = np.isnan(sf[:, :4]).any(1)
    sf[bad] = 0.0
    return sf, tfrz


def read_pimnsf(path):
    """pimnsf.dat -> (n, 10) array and 1/(2 T^2 (e+P)) from its header."""
    with open(path) as f:
        head = f.readline()
    coeff = float(head.split('one_o_2TsqrEplusP=')[1].split()[0])
    return np.loadtxt(path, ndmin=2), coeff


class SmoothSpec(object):
    """Direct Cooper-Frye spectra on a freeze-out surface (Spec, cl_spec.h)."""

    def __init__(self, sf, tfrz, pisf=None, one_o_2TsqrEplusP=0.0, use_float32=True, device=None,
                 ny=41, ylo=-8.0, yhi=8.0, npt=15, nphi=48, mu=None):
        if not torch.cuda.is_available():
            raise RuntimeError('SmoothSpec needs a CUDA device; there is no CPU path')
        self.lib = _lib.load()
        self.device = torch.device('cuda', 0) if device is None else torch.device(device)
        self.dtype = torch.float32 if use_float32 else torch.float64
        self.real = np.float32 if use_float32 else np.float64
        self.sf = torch.as_tensor(sf).to(self.device, self.dtype).reshape(-1, 8).contiguous()
        self.pisf = None if pisf is None else torch.as_tensor(pisf).to(self.device, self.dtype).reshape(-1, 10)
        self.tfrz = float(tfrz)
        self.tcoeff = float(one_o_2TsqrEplusP)
        # effective chemical potential of each hadron by PDG id (the
        # chemical_potential.dat of the run; cl_spec.cpp:56-58, 183-200)
        self.mu = dict(mu or {})
        self.y, self.pt, self.phi = momentum_grid(ny, ylo, yhi, npt, nphi)
        self.ylo, self.yhi = ylo, yhi
        as_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=self.real)).to(self.device)
        self.d_y, self.d_pt = as_dev(self.y), as_dev(self.pt)
        self.d_cphi, self.d_sphi = as_dev(np.cos(self.phi)), as_dev(np.sin(self.phi))
        self.spec = {}

    @classmethod
    def from_files(cls, path, viscous_on=False, **kw):
        """hypersf.dat (and pimnsf.dat) of a run, with the effective chemical
        potentials of its chemical_potential.dat (cl_spec.cpp:56-58)."""
        from .chempot import read_chemical_potential
        sf, tfrz = read_hypersf(os.path.join(path, 'hypersf.dat'))
        pisf, coeff = (None, 0.0)
        if viscous_on:
            pisf, coeff = read_pimnsf(os.path.join(path, 'pimnsf.dat'))
        kw.setdefault('mu', read_chemical_potential(path))
        return cls(sf, tfrz, pisf, coeff, **kw)

    def calc(self, pid, mass=None, gspin=None, fermi_boson=None, mu=None):
        """dN/(dY pt dpt dphi) of one species as (ny, npt, nphi); the hadron
        is one of HADRONS by its PDG id, or given explicitly. mu defaults to
        the hadron's effective chemical potential (0 without one), which the
        kernel subtracts from u.p as kernel_spec.cl:28,52 does."""
        if mass is None:
            mass, gspin, fermi_boson = HADRONS[pid]
        if mu is None:
            mu = self.mu.get(int(pid), 0.0)
        ny, npt, nphi = len(self.y), len(self.pt), len(self.phi)
        out = torch.empty(ny * npt * nphi, dtype=self.dtype, device=self.device)
        n = self.sf.shape[0]
        nbytes = int(self.lib.clv_spectra_scratch_bytes(n, ny, npt, nphi))
        scratch = torch.empty(max(nbytes, 8) // 8 + 1, dtype=torch.float64, device=self.device)
        a = SpectraArgs()
        a.precision = 4 if self.dtype == torch.float32 else 8
        a.sf = self.sf.data_ptr()
        a.pisf = None if self.pisf is None else self.pisf.data_ptr()
        a.n = n
        a.mass, a.gspin, a.fermi_boson, a.mu = float(mass), float(gspin), float(fermi_boson), float(mu)
        a.tfrz, a.tcoeff = self.tfrz, self.tcoeff
        a.y, a.pt, a.cphi, a.sphi = (self.d_y.data_ptr(), self.d_pt.data_ptr(), self.d_cphi.data_ptr(),
                                      self.d_sphi.data_ptr())
        a.ny, a.npt, a.nphi = ny, npt, nphi
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(self.lib.clv_spectra(ctypes.byref(a), ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(scratch.data_ptr()), nbytes, stream), 'clv_spectra')
        spec = out.cpu().numpy().reshape(ny, npt, nphi)
        self.spec[pid] = (float(mass), spec)
        return spec

    def dNdEta(self, mass, spec):
        """dN/(deta pt dpt dphi) by the Jacobian and linear interpolation in Y
        (Spec::get_dNdEtaPtdPtdPhi, cl_spec.cpp:1001-1036)."""
        ny, npt = len(self.y), len(self.pt)
        out = np.empty_like(spec)
        for k in range(ny):
            eta = self.y[k]
            for i in range(npt):
                pt = self.pt[i]
                ptce = pt * np.cosh(eta)
                dYdEta = ptce / np.sqrt(mass * mass + ptce * ptce)
                Y = np.arctanh(dYdEta * np.tanh(eta))
                Y = min(max(Y, self.ylo), self.yhi)
                IY = 1
                while Y > self.y[IY] and IY < ny - 1:
                    IY += 1
                Y1, Y2 = self.y[IY - 1], self.y[IY]
                a = (Y - Y1) / (Y2 - Y1)
                out[k, i, :] = ((1.0 - a) * spec[IY - 1, i, :] + a * spec[IY, i, :]) * dYdEta
        return out

    def write(self, path):
        """dNdYPtdPtdPhi_<pid>.dat and dNdEtaPtdPtdPhi_<pid>.dat, values
        separated by spaces in (Y, pt, phi) order (cl_spec.cpp:494-503, 627-636)."""
        os.makedirs(path, exist_ok=True)
        for pid, (mass, spec) in self.spec.items():
            for name, arr in (('dNdYPtdPtdPhi', spec), ('dNdEtaPtdPtdPhi', self.dNdEta(mass, spec))):
                with open(os.path.join(path, '%s_%d.dat' % (name, pid)), 'w') as f:
                    f.write(' '.join('%g' % v for v in arr.reshape(-1)) + ' ')
