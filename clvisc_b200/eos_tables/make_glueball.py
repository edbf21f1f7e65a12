"""Extract the pure-SU(3) gauge (glueball) EOS data the reference's
Eos('pure_gauge') reads (pyvisc/eos/glueball.py:16-32 with
pyvisc/eos/glueball_v2.dat: columns T/Tc, s/T^3, e/T^4, p/T^4, T [MeV],
cs^2) into glueball.npz: T [GeV], e, p in GeV/fm^3 (x T^4 / hbarc^3 with
hbarc = 0.19732 GeV fm, glueball.py:13,27-29), the numbers unchanged
otherwise. Run from the repository root:

    python clvisc_b200/eos_tables/make_glueball.py REFERENCE_ROOT
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HBARC = 0.19732


def main(refroot):
    dat = np.loadtxt(os.path.join(refroot, 'pyvisc', 'eos', 'glueball_v2.dat'))
    T = 1.0E-3 * dat[:, 4]
    hbarc3 = HBARC ** 3
    ed = dat[:, 2] * T ** 4 / hbarc3
    pr = dat[:, 3] * T ** 4 / hbarc3
    out = os.path.join(HERE, 'glueball.npz')
    np.savez_compressed(out, T=T, ed=ed, pr=pr)
    print(out, dat.shape)


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: make_glueball.py REFERENCE_ROOT')
    main(sys.argv[1])
