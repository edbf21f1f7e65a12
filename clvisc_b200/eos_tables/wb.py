"""The 2+1-flavour lattice QCD EOS of the Wuppertal-Budapest collaboration
(Borsanyi et al., Phys. Lett. B 730 (2014) 99) in chemical equilibrium, on
the uniform energy-density grid the reference's Eos('lattice_wb') uses
(pyvisc/eos/wb.py, eos.py:142-153). eos.Eos('lattice_wb') computes it once a
process (about 2 s) through wb_arrays().

The published parametrisation of the trace anomaly, with t = T / 0.2 GeV,
    I(T)/T^4 = exp(-h1/t - h2/t^2) (h0 + f0 (tanh(f1 t + f2) + 1) / (1 + g1 t + g2 t^2)),
h0 = 0.1396, h1 = -0.18, h2 = 0.035, f0 = 1.05, f1 = 6.39, f2 = -4.72,
g1 = -0.92, g2 = 0.57, gives the pressure by integration from T* = 0.214 GeV,
where p/T^4 = 1.842:
    p/T^4 = 1.842 + int_{T*}^{T} I(T')/T'^5 dT',   e = I + 3 p.
The steps follow wb.py:80-106 so that the table has the reference's values:
e(T) and p/e on 2000 temperatures from 0.03 to 1.13 GeV (adaptive
quadrature), cubic interpolating splines of T(e) and (p/e)(e) evaluated on
e = 0.01 .. 1999.99 GeV/fm^3 (199 999 points), the point e = 0 prepended
(T = 0.001 GeV, p/e extrapolated linearly), p = e (p/e). eos.py:145-154 then
takes s = (e + p) / (T + 1e-10) and the speed of sound from p(e)
(cs2_from_pressure, eos.py:85-100). 200 000 entries: a 200 x 1000 image.
"""
import math

import numpy as np
from scipy import interpolate
from scipy.integrate import quad

from .make_pce165 import cs2_from_pressure

HBARC = 0.19732          # GeV fm (wb.py:15)
T_STAR = 0.214           # GeV
P_OVER_T4_STAR = 1.842
ED_START, ED_STEP, NUM_ED = 0.0, 0.01, 200000


def trace_anomaly(T):
    """I(T)/T^4 of the published fit."""
    h0, h1, h2 = 0.1396, -0.18, 0.035
    f0, f1, f2 = 1.05, 6.39, -4.72
    g1, g2 = -0.92, 0.57
    t = T / 0.2
    return math.exp(-h1 / t - h2 / (t * t)) * (h0 + f0 * (math.tanh(f1 * t + f2) + 1.0) / (1.0 + g1 * t + g2 * t * t))


def p_over_t4(T):
    return quad(lambda x: trace_anomaly(x) / x, T_STAR, T)[0] + P_OVER_T4_STAR


def table():
    """(ed, pr, T): the uniform grid, pressure and temperature."""
    T_grid = np.linspace(0.03, 1.13, 2000)
    ed_grid = np.empty_like(T_grid)
    p_over_e = np.empty_like(T_grid)
    for i, T in enumerate(T_grid):
        pt4 = p_over_t4(T)
        et4 = 3 * pt4 + trace_anomaly(T)
        ed_grid[i] = et4 * T ** 4 / HBARC ** 3
        p_over_e[i] = pt4 / et4
    ed = np.linspace(0.01, 1999.99, 199999)
    T = interpolate.splev(ed, interpolate.splrep(ed_grid, T_grid, s=0), der=0)
    ratio = interpolate.splev(ed, interpolate.splrep(ed_grid, p_over_e, s=0), der=0)
    ratio0 = -(ratio[1] - ratio[0]) / (ed[1] - ed[0]) * ed[0] + ratio[0]
    ed = np.insert(ed, 0, 0.0)
    T = np.insert(T, 0, 0.001)
    ratio = np.insert(ratio, 0, ratio0)
    return ed, ed * ratio, T


_CACHE = {}


def wb_arrays():
    """(ed, pr, T, s, cs2) of the 200 000-entry table, computed once."""
    if 'wb' not in _CACHE:
        ed, pr, T = table()
        s = (ed + pr) / (T + 1.0E-10)
        cs2 = cs2_from_pressure(ed, pr.copy(), ED_STEP)
        _CACHE['wb'] = (ed, pr, T, s, cs2)
    return _CACHE['wb']
