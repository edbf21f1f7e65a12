"""Golden rows of the reference's Eos('lattice_wb') image (pyvisc/eos/eos.py
lattice_ce with pyvisc/eos/wb.py), generated by importing the reference:

    python tests/golden/make_golden_wb.py /path/to/reference

Records into golden_wb.npz the float32 (cs2, p, T, s) rows of the image the
reference builds (eos.py:190-191) at a fixed set of indices, and its
f_ed(0.137), num_of_ed and ed_step. eos.py is loaded as a module of a
stand-in package so that its `from . import wb` finds wb.py beside it.
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref_eos_package(refroot):
    eosdir = os.path.join(refroot, 'pyvisc', 'eos')
    pkg = types.ModuleType('ref_eos_pkg')
    pkg.__path__ = [eosdir]
    sys.modules['ref_eos_pkg'] = pkg
    spec = importlib.util.spec_from_file_location('ref_eos_pkg.eos', os.path.join(eosdir, 'eos.py'))
    mod = importlib.util.module_from_spec(spec)
    sys.modules['ref_eos_pkg.eos'] = mod
    spec.loader.exec_module(mod)
    return mod


def main(refroot):
    sys.path.insert(0, HERE)
    from make_golden import sample_rows
    ref = load_ref_eos_package(refroot)
    e = ref.Eos('lattice_wb')
    img = np.array(list(zip(e.cs2, e.pr, e.T, e.s)), dtype=np.float32)
    rows = sample_rows(img.shape[0])
    np.savez_compressed(os.path.join(HERE, 'golden_wb.npz'), rows=rows, table=img[rows],
                        f_ed_0137=np.float64(e.f_ed(0.137)), num_of_ed=np.int64(e.num_of_ed),
                        ed_step=np.float64(e.ed_step), n=np.int64(img.shape[0]))
    print('rows', len(rows), 'f_ed(0.137)', float(e.f_ed(0.137)))


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: make_golden_wb.py REFERENCE_ROOT')
    main(sys.argv[1])
