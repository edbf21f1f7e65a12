"""Build recipe and binding of the reference's own hydro kernels on the CPU
(test infrastructure: they check the oracle's restatement, oracle.Kernels,
against the reference code itself).

The reference is OpenCL C (pyvisc/kernel/*.cl), not C or C++, and its host
needs pyopencl, which is absent. Its kernel sources are plain C apart from
vector types, address-space qualifiers, work-item functions and one image
read, so they compile with g++ through refshim/cl_shim.hpp once the vector
literals (real4)(a, b, c, d) are rewritten as braced lists real4{a, b, c, d}. This recipe
copies kernel_ideal.cl, kernel_visc.cl, kernel_IS.cl, kernel_hypersf.cl,
kernel_reduction.cl, helper.h, eos_table.h, real_type.h and
kernel_vorticity.h from the reference
tree into oracle/_ref/<configuration>/, applies that one rewrite, and
compiles refshim/ref_driver.cpp with the -D constants the reference host
would pass (ideal.py:146-171 and 190-194, visc.py:107-121, eos.py:194-200)
into a library per configuration. Nothing here is copied into
the repository; the reference tree is read from CLVISC_REFERENCE_ROOT
(default /root/reference) at build time, and available() is False where it
is absent (the GPU box), so the tests that use it skip there.
"""
import ctypes
import hashlib
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get('CLVISC_REFERENCE_ROOT', '/root/reference')
KDIR = os.path.join(REF_ROOT, 'pyvisc', 'kernel')
SOURCES = ('kernel_ideal.cl', 'kernel_visc.cl', 'kernel_IS.cl', 'kernel_hypersf.cl', 'kernel_reduction.cl',
           'helper.h', 'eos_table.h', 'real_type.h', 'kernel_vorticity.h')
_VEC = re.compile(r'\((real[0-9]|float[0-9]|double[0-9]|int[0-9])\)\s*\(')


def rewrite_vector_literals(src):
    """(real4)(a, b, c, d) -> real4{a, b, c, d}: a braced list, whose
    elements C++ evaluates left to right, as clang-based OpenCL compilers
    evaluate a vector literal's (kernel_hypersf.cl:148-151 draws four random
    numbers in one literal; argument lists have no order in C++)."""
    out, pos = [], 0
    for m in _VEC.finditer(src):
        if m.start() < pos:  # inside a literal already rewritten
            continue
        depth, i = 1, m.end()
        while depth:
            c = src[i]
            depth += (c == '(') - (c == ')')
            i += 1
        inner = src[m.end():i - 1]
        out.append(src[pos:m.start()])
        out.append('%s{%s}' % (m.group(1), rewrite_vector_literals(inner)))
        pos = i
    out.append(src[pos:])
    return ''.join(out)


def available():
    return all(os.path.exists(os.path.join(KDIR, f)) for f in SOURCES)


def defines(cfg, meta, efrz, bsz=8):
    """The reference's compile options for this run: '-D KEY=%sf' of the float
    constants (ideal.py:147-150), the grid, BSZ and precision, EOS_TABLE with
    its table constants (eos.py:194-200), the viscous test switches
    (visc.py:110-121), and the surface finder's skips and EFRZ
    (ideal.py:190-194). One translation unit takes them all; none of the
    hydro kernels names the surface finder's constants."""
    d = []
    for key in ('TAU0', 'DT', 'DX', 'DY', 'DZ', 'ETAOS_XMIN', 'ETAOS_YMIN', 'ETAOS_LEFT_SLOP', 'ETAOS_RIGHT_SLOP',
                'LAM1'):
        d.append('-D%s=%sf' % (key, getattr(cfg, key)))
    d += ['-DNX=%d' % cfg.NX, '-DNY=%d' % cfg.NY, '-DNZ=%d' % cfg.NZ, '-DSIZE=%d' % (cfg.NX * cfg.NY * cfg.NZ),
          '-DBSZ=%d' % bsz]
    if cfg.use_float32:
        d.append('-DUSE_SINGLE_PRECISION')
    if getattr(cfg, 'riemann_test', False):
        d.append('-DRIEMANN_TEST')
    d.append('-DEOS_TABLE')
    if getattr(cfg, 'gubser_visc_test', False):
        d.append('-DGUBSER_VISC_TEST')
    if getattr(cfg, 'pimn_omega_coupling', False):
        d.append('-DPIMUNU_OMEGA_COUPLING')
    if getattr(cfg, 'omega_omega_coupling', False):
        d.append('-DOMEGA_OMEGA_COUPLING')
    d += ['-DEOS_ED_START=%sf' % meta['ed_start'], '-DEOS_ED_STEP=%sf' % meta['ed_step'],
          '-DEOS_NUM_ED=%d' % int(meta['num_of_ed']), '-DEOS_NUM_OF_ROWS=%d' % int(meta['nrow']),
          '-DEOS_NUM_OF_COLS=%d' % int(meta['ncol'])]
    d += ['-Dnxskip=%d' % cfg.nxskip, '-Dnyskip=%d' % cfg.nyskip, '-Dnzskip=%d' % cfg.nzskip, '-DEFRZ=%sf' % efrz]
    return d


def build(cfg, meta, efrz, bsz=8):
    """Path of the reference kernels' library for this configuration."""
    defs = defines(cfg, meta, efrz, bsz)
    h = hashlib.sha1(' '.join(defs).encode())
    for f in [os.path.join(KDIR, f) for f in SOURCES] + [os.path.abspath(__file__)] + \
            [os.path.join(HERE, 'refshim', f) for f in sorted(os.listdir(os.path.join(HERE, 'refshim')))]:
        with open(f, 'rb') as fi:
            h.update(fi.read())
    key = h.hexdigest()[:16]
    out = os.path.join(HERE, '_ref', key)
    lib = os.path.join(out, 'libref_kernels.so')
    if os.path.exists(lib):
        return lib
    os.makedirs(out, exist_ok=True)
    for f in SOURCES:
        src = open(os.path.join(KDIR, f)).read()
        dst = f + '.i' if f.endswith('.cl') else f
        with open(os.path.join(out, dst), 'w') as fo:
            fo.write(rewrite_vector_literals(src))
    cmd = ['g++', '-O2', '-std=c++17', '-fopenmp', '-ffp-contract=off', '-fno-fast-math', '-fwrapv', '-fPIC', '-shared', '-w', '-Wno-narrowing',
           '-I', out, '-I', os.path.join(HERE, 'refshim')] + defs + \
          [os.path.join(HERE, 'refshim', 'ref_driver.cpp'), '-o', lib + '.tmp']
    subprocess.check_call(cmd)
    os.replace(lib + '.tmp', lib)
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class RefKernels(object):
    """oracle.Kernels' interface over the reference's compiled kernels (the
    hydro stages and the surface finder; the max reduction as
    reference_reduction_stage1); the other methods (reduction_stage1, the
    bulk sector, which the reference lacks) are the oracle's."""

    def __init__(self, oracle_kernels, cfg, meta, table, efrz):
        self.o = oracle_kernels
        self.cfg = cfg
        self.lib = ctypes.CDLL(build(cfg, meta, efrz))
        self.real = oracle_kernels.real
        self.R = ctypes.c_float if self.real == np.float32 else ctypes.c_double
        assert self.lib.ref_real_size() == np.dtype(self.real).itemsize
        self.table = np.ascontiguousarray(table, dtype=np.float32)
        self.lib.ref_set_eos(_p(self.table), int(meta['ncol']), int(meta['nrow']))

    def __getattr__(self, name):  # the oracle's own methods for the rest
        return getattr(self.o, name)

    def _r(self, x):
        return self.R(float(x))

    def _check(self):
        assert self.lib.ref_team_error() == 0, 'work-group team smaller than BSZ'

    def ideal_christoffel(self, Src, ev, tau, step):
        self.lib.ref_ideal_christoffel(_p(Src), _p(ev), self._r(tau), int(step))

    def ideal_along(self, axis, Src, ev, tau):
        self.lib.ref_ideal_along(int(axis), _p(Src), _p(ev), self._r(tau))
        self._check()

    def ideal_update_ev(self, evnew, ev1, Src, tau, step):
        self.lib.ref_ideal_update_ev(_p(evnew), _p(ev1), _p(Src), self._r(tau), int(step))

    def visc_christoffel(self, Src, ev, pi, tau, step, bulk=None):
        assert bulk is None
        self.lib.ref_visc_christoffel(_p(Src), _p(ev), _p(pi), self._r(tau), int(step))

    def visc_along(self, axis, Src, ev, pi, tau, bulk=None):
        assert bulk is None
        self.lib.ref_visc_along(int(axis), _p(Src), _p(ev), _p(pi), self._r(tau))
        self._check()

    def visc_update_ev(self, evnew, ev1, pi1, pi2, Src, tau, step, bulk1=None, bulk2=None):
        assert bulk1 is None and bulk2 is None
        self.lib.ref_visc_update_ev(_p(evnew), _p(ev1), _p(pi1), _p(pi2), _p(Src), self._r(tau), int(step))

    def visc_initialize(self, pi1, goodcell, udiff, ev, tau, bulk1=None):
        assert bulk1 is None
        self.lib.ref_visc_initialize(_p(pi1), _p(goodcell), _p(udiff), _p(ev), self._r(tau))

    def visc_src_christoffel(self, Src, pi1, ev, tau, step, SrcB=None):
        self.lib.ref_visc_src_christoffel(_p(Src), _p(pi1), _p(ev), self._r(tau), int(step))

    def visc_src_along(self, axis, Src, ud, pi1, ev, tau, SrcB=None, bulk1=None):
        self.lib.ref_visc_src_along(int(axis), _p(Src), _p(ud), _p(pi1), _p(ev), self._r(tau))
        self._check()

    def update_pimn(self, pinew, goodcell, pi1, pistep, ev1, ev2, udiff, udx, udy, udz, Src, tau, step,
                    bulknew=None, bulk1=None, bulkstep=None, SrcB=None):
        self.lib.ref_update_pimn(_p(pinew), _p(goodcell), _p(pi1), _p(pistep), _p(ev1), _p(ev2), _p(udiff),
                                 _p(udx), _p(udy), _p(udz), _p(Src), self._r(tau), int(step))

    def get_udiff(self, udiff, ev0, ev1):
        self.lib.ref_get_udiff(_p(udiff), _p(ev0), _p(ev1))

    def reference_reduction_stage1(self, ev, semi, size):
        """kernel_reduction.cl's reduction_stage1 into semi[64] (64
        work-groups of 256 work-items, each a team of 256 threads here: about
        2 s a call on a few cores, so the orchestration keeps the oracle's
        reduction_stage1, which a test checks against this one)."""
        assert semi.shape[0] >= 64
        self.lib.ref_reduction_stage1(_p(ev), _p(semi), int(size))
        self._check()

    def hypersf(self, ev_old, ev_new, pi_old, pi_new, t_old, t_new, visc, sf, txyz, pisf, capacity):
        """The reference's get_hypersf / visc_hypersf into buffers of one
        element per cube (the kernels have no capacity check), the first
        `capacity` elements copied out, the count returned; the order is
        that of the threads' atomic_inc. The vorticity inputs are zero."""
        c = self.cfg
        cubes = ((c.NX - 1) // c.nxskip + 1) * ((c.NY - 1) // c.nyskip + 1) * ((c.NZ - 1) // c.nzskip + 1)
        real = self.real
        sf_all = np.zeros((cubes, 8), real)
        tx_all = np.zeros((cubes, 4), real)
        if visc:
            size = c.NX * c.NY * c.NZ
            pi_all = np.zeros((cubes, 10), real)
            om = [(np.zeros((cubes, w), real), np.zeros((size, w), real), np.zeros((size, w), real))
                  for w in (6, 16, 4, 6)]
            args = [_p(a) for trio in om for a in trio]
            n = self.lib.ref_visc_hypersf(_p(sf_all), _p(tx_all), _p(pi_all), _p(ev_old), _p(ev_new), _p(pi_old),
                                          _p(pi_new), *args, self._r(t_old), self._r(t_new))
        else:
            n = self.lib.ref_get_hypersf(_p(sf_all), _p(tx_all), _p(ev_old), _p(ev_new), self._r(t_old),
                                         self._r(t_new))
        m = min(n, capacity)
        sf[:m] = sf_all[:m]
        txyz[:m] = tx_all[:m]
        if visc:
            pisf[:m] = pi_all[:m]
        return n
