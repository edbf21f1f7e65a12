"""Equation-of-state tables, mirroring pyvisc/eos/eos.py (class Eos).

An Eos carries the tabulated (cs2, p, T, s) on a uniform energy-density grid
(ed_start, ed_step, num_of_ed) plus the host-side functions f_P, f_T, f_S,
f_ed, f_cs2 the reference exposes. create_table() returns the float32 image
the kernels read (the reference's RGBA image2d, eos.py:184-203): nrow x ncol
texels of (cs2, p, T, s), read with clamp-to-edge nearest sampling and a
manual linear interpolation (eos_table.h:39-62).

Supported eos_type values: 'ideal_gas' (eos.py:42-59, computed here),
'lattice_pce165' and 'lattice_pce150' (eos.py:102-127; the tables are
regenerated from the s95p source grids by eos_tables/make_pce165.py because
EOS_PST.dat is absent from the reference snapshot), 'lattice_wb' (eos.py:142-153 with wb.py: the
Wuppertal-Budapest 2014 parametrisation, computed once a process by
eos_tables/wb.py, on the 200 x 1000 image of eos.py:184) and 'pure_gauge'
(eos.py:171-182 with glueball.py: the SU(3) gauge EOS with its first-order
transition, from the reference's glueball_v2.dat extracted by
eos_tables/make_glueball.py). A user-built table can be passed as a
handcrafted_eos object with the same attributes (ideal.py:60-69).
"""
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# (nrow, ncol) that CLIdeal passes to create_table per eos_type (ideal.py:67-83)
TABLE_SHAPE = {
    'ideal_gas': (200, 1000),
    'lattice_pce165': (100, 1555),
    'lattice_pce150': (100, 1555),
    # the reference's CLIdeal asks for 4 x 1001 here (ideal.py:79-81), which
    # cannot hold the 200 000 entries; create_table's default shape does
    'lattice_wb': (200, 1000),
    'pure_gauge': (200, 1000),
}


class Eos(object):
    """EOS table and host-side thermodynamic functions (pyvisc/eos/eos.py:20)."""

    def __init__(self, eos_type='ideal_gas'):
        self.eos_type = eos_type
        if eos_type == 'ideal_gas':
            self.ideal_gas()
        elif eos_type == 'lattice_pce165':
            self.lattice_pce165()
        elif eos_type == 'lattice_pce150':
            self.lattice_pce150()
        elif eos_type == 'lattice_wb':
            self.lattice_wb()
        elif eos_type == 'pure_gauge':
            self.pure_gauge()
        else:
            raise ValueError('unsupported eos_type %r (supported: %s)'
                             % (eos_type, ', '.join(sorted(TABLE_SHAPE))))

    def ideal_gas(self):
        """Conformal gas p = e/3 with 169/4 degrees of freedom (eos.py:42-59)."""
        hbarc = 0.1973269
        dof = 169.0 / 4.0
        coef = np.pi * np.pi / 30.0
        self.f_P = lambda ed: np.array(ed) / 3.0
        self.f_T = lambda ed: hbarc * (1.0 / (dof * coef) * np.array(ed) / hbarc) ** 0.25 + 1.0E-10
        self.f_S = lambda ed: (np.array(ed) + self.f_P(ed)) / self.f_T(ed)
        self.f_ed = lambda T: dof * coef * hbarc * (np.array(T) / hbarc) ** 4.0
        self.f_cs2 = lambda ed: 1.0 / 3.0 * np.ones_like(ed)
        self.ed = np.linspace(0, 1999.99, 200000)
        self.pr = self.f_P(self.ed)
        self.T = self.f_T(self.ed)
        self.s = self.f_S(self.ed)
        self.cs2 = self.f_cs2(self.ed)
        self.ed_start = 0.0
        self.ed_step = 0.01
        self.num_of_ed = 200000

    def lattice_pce165(self, name='lattice_pce165'):
        """s95p-PCE165-v0 lattice + partial-chemical-equilibrium HRG EOS."""
        d = np.load(os.path.join(_HERE, 'eos_tables', name + '.npz'))
        self.ed_start = float(d['ed_start'])
        self.ed_step = float(d['ed_step'])
        self.num_of_ed = int(d['num_of_ed'])
        self.ed = np.arange(self.num_of_ed) * self.ed_step
        e = d['src_e']
        self.pr = np.interp(self.ed, e, d['src_p'])
        self.s = np.interp(self.ed, e, d['src_s'])
        self.T = np.interp(self.ed, e, d['src_T'])
        self.cs2 = d['cs2'].astype(np.float64)
        self._from_arrays()

    def lattice_pce150(self):
        """s95p-PCE-v1 lattice + partial-chemical-equilibrium HRG EOS with
        chemical freeze-out at 150 MeV (eos.py:116-127), regenerated like
        PCE165 (eos_tables/make_pce165.py)."""
        self.lattice_pce165('lattice_pce150')

    def lattice_wb(self):
        """Wuppertal-Budapest 2014 lattice EOS in chemical equilibrium
        (eos.py:142-153, lattice_ce)."""
        from .eos_tables.wb import ED_START, ED_STEP, NUM_ED, wb_arrays
        ed, pr, T, s, cs2 = wb_arrays()
        self.ed, self.pr, self.T, self.s, self.cs2 = ed, pr, T, s, cs2.copy()
        self.ed_start, self.ed_step, self.num_of_ed = ED_START, ED_STEP, NUM_ED
        self._from_arrays()

    def pure_gauge(self):
        """Pure SU(3) gauge EOS (eos.py:171-182, pure_su3): the glueball
        table linearly interpolated onto e = 0, 0.01, .., 1999.99 GeV/fm^3
        (glueball.py:34-40), s = (e + p) / (T + 1e-10), cs2 from p(e)."""
        from scipy import interpolate
        from .eos_tables.make_pce165 import cs2_from_pressure
        d = np.load(os.path.join(_HERE, 'eos_tables', 'glueball.npz'))
        ed = np.linspace(0.0, 2000, 200000, endpoint=False)
        T = interpolate.interp1d(d['ed'], d['T'])(ed)
        pr = interpolate.interp1d(d['ed'], d['pr'])(ed)
        self.ed, self.pr, self.T = ed, pr, T
        self.s = (ed + pr) / (T + 1.0E-10)
        self.ed_start, self.ed_step, self.num_of_ed = 0.0, 0.01, 200000
        self.cs2 = cs2_from_pressure(ed, pr.copy(), self.ed_step)
        self._from_arrays()

    def _from_arrays(self):
        """Linear (k=1) interpolants as eos.py:78-83 builds them, with the
        same scipy spline (linear extrapolation outside the table)."""
        from scipy.interpolate import InterpolatedUnivariateSpline as Spline
        ed, pr, T, s = self.ed, self.pr, self.T, self.s

        def wrap(f):
            def g(x):
                y = f(np.asarray(x, dtype=np.float64))
                return y[()] if np.ndim(y) == 0 else y
            return g

        self.f_ed = wrap(Spline(T, ed, k=1, ext=0))
        self.f_T = wrap(Spline(ed, T, k=1, ext=0))
        self.f_P = wrap(Spline(ed, pr, k=1, ext=0))
        self.f_S = wrap(Spline(ed, s, k=1, ext=0))
        self.f_cs2 = wrap(Spline(ed, self.cs2, k=1, ext=0))

    def create_table(self, nrow=None, ncol=None):
        """Return (table, meta): the float32 (nrow, ncol, 4) image of
        (cs2, p, T, s) and the constants the kernels use (eos.py:184-203)."""
        if nrow is None or ncol is None:
            nrow, ncol = TABLE_SHAPE.get(self.eos_type, (200, 1000))
        src = np.stack([np.asarray(self.cs2, np.float64), self.pr, self.T, self.s], axis=1).astype(np.float32)
        if src.shape[0] != nrow * ncol:
            raise ValueError('EOS table has %d rows, image is %dx%d' % (src.shape[0], nrow, ncol))
        src = np.ascontiguousarray(src.reshape(nrow, ncol, 4))
        meta = dict(ed_start=self.ed_start, ed_step=self.ed_step, num_of_ed=self.num_of_ed,
                    nrow=nrow, ncol=ncol)
        return src, meta
