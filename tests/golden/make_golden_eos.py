"""Golden rows of the reference's Eos('lattice_wb') and Eos('pure_gauge')
images (pyvisc/eos/eos.py lattice_ce with wb.py, pure_su3 with glueball.py),
generated by importing the reference:

    python tests/golden/make_golden_eos.py /path/to/reference

Records into golden_eos.npz, per type, the float32 (cs2, p, T, s) rows of
the image the reference builds (eos.py:190-191) at a fixed set of indices,
and its f_ed(0.137), num_of_ed and ed_step. eos.py is loaded as a module of
a stand-in package so that its `from . import wb` finds wb.py beside it, and
with its directory on sys.path for its `import glueball`.
"""
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_ref_eos_package(refroot):
    eosdir = os.path.join(refroot, 'pyvisc', 'eos')
    sys.path.insert(0, eosdir)
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
    out = {}
    for key, eos_type in (('wb', 'lattice_wb'), ('gb', 'pure_gauge')):
        e = ref.Eos(eos_type)
        img = np.array(list(zip(e.cs2, e.pr, e.T, e.s)), dtype=np.float32)
        rows = sample_rows(img.shape[0])
        out.update({key + '_rows': rows, key + '_table': img[rows], key + '_f_ed_0137': np.float64(e.f_ed(0.137)),
                    key + '_num_of_ed': np.int64(e.num_of_ed), key + '_ed_step': np.float64(e.ed_step),
                    key + '_n': np.int64(img.shape[0])})
        print(eos_type, 'rows', len(rows), 'f_ed(0.137)', float(e.f_ed(0.137)))
    np.savez_compressed(os.path.join(HERE, 'golden_eos.npz'), **out)


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: make_golden_eos.py REFERENCE_ROOT')
    main(sys.argv[1])
