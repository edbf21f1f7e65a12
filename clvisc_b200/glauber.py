"""Optical Glauber initial condition (pyvisc/glauber.py), on the device.

glauber_consts() gives the kernel constants the reference emits as
'-D KEY=%ff' literals (glauber.py:79-90): the float value of each configuration
entry printed with six decimals. weight_mean_b() restates glauber.py:14-57
(the impact parameter averaged over a centrality class with N_part-weighted
b^2 dN/db, from the tabulated centrality, N_part and b of Au+Au 200 GeV and
Pb+Pb 2.76 TeV).
"""
import numpy as np

from . import _lib
from .config import float_literal


def glauber_consts(cfg):
    g = _lib.ClvGlauber()
    for field, key in (('num_of_nucleons', 'NumOfNucleons'), ('sqrts', 'SQRTS'), ('ro0', 'NucleonDensity'),
                       ('r', 'Ra'), ('eta', 'Eta'), ('si0', 'Si0'), ('impact_parameter', 'ImpactParameter'),
                       ('edmax', 'Edmax'), ('hwn', 'Hwn'), ('eta_flat', 'Eta_flat'), ('eta_gw', 'Eta_gw')):
        setattr(g, field, float_literal('%f' % float(getattr(cfg, key))))
    return g


# glauber.py:22-42: centrality [%], wounded nucleons, impact parameter [fm]
_TABLES = {
    'Au+Au': ([0, 5, 10, 15, 20, 30, 40, 50, 60, 70, 80, 90],
              [393.0, 327.0, 278.0, 237.0, 202.0, 144.0, 99.0, 65.0, 44.0, 22.0, 11.0, 4.0],
              [0.0, 3.3, 4.7, 5.8, 6.7, 8.2, 9.4, 10.6, 11.6, 12.5, 13.4, 14.3]),
    'Pb+Pb': ([0, 5, 10, 15, 20, 30, 40, 50, 60, 70, 80, 90],
              [416.0, 357.0, 305.0, 261.0, 216.0, 159.0, 110.0, 70.0, 42.0, 23.0, 11.0, 4.0],
              [0.0, 3.54, 5.00, 6.13, 7.08, 8.67, 10.01, 11.19, 12.26, 13.24, 14.16, 15.07]),
}


def weight_mean_b(cent_low, cent_high, system='Au+Au'):
    """<b> of the centrality class [cent_low, cent_high] (glauber.py:14-57)."""
    from scipy.integrate import quad
    from scipy.interpolate import interp1d
    if system not in _TABLES:
        raise ValueError('collisions system must be Au+Au or Pb+Pb')
    cent, nwn, bimp = (np.array(v, dtype=float) for v in _TABLES[system])
    bimp_vs_cent = interp1d(cent, bimp, kind='cubic')
    nwn_vs_b = interp1d(bimp, nwn, kind='cubic')
    f1 = lambda b: b * (b * b) * nwn_vs_b(b)
    f2 = lambda b: (b * b) * nwn_vs_b(b)
    bmin = bimp_vs_cent(cent_low)
    bmax = bimp_vs_cent(cent_high)
    return quad(f1, bmin, bmax)[0] / quad(f2, bmin, bmax)[0]
