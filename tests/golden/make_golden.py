"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root while the reference source tree is available:

    python tests/golden/make_golden.py /path/to/reference

What it records (all into golden.npz / golden.json):
  * eos_ideal_gas: rows of the float32 (cs2, p, T, s) image that the
    reference's pyvisc/eos/eos.py Eos('ideal_gas') builds (eos.py:42-59,
    190-191), at a fixed set of row indices, and its f_ed(0.137);
  * eos_pce165_cs2: the reference's own cs2 post-processing
    (Eos.eos_func_from_interp1d, eos.py:78-100) applied to the regenerated
    s95p-PCE165 (e, p, s, T) grid, sampled at the same kind of indices, and its
    f_ed(0.137);
  * weight_mean_b: the reference's pyvisc/glauber.py weight_mean_b() for the
    centrality classes its own __main__ lists (glauber.py:106-123), Au+Au and
    Pb+Pb (glauber.py is imported with its pyopencl import stubbed: the
    function itself is numpy/scipy);
  * kat: the known-answer vectors the reference's tests hold for this path
    (pyvisc/tests/test_kernel_helper.py:29-54, test_reduction.py:15-53,
    test_hypersf.py:26-59, test_bjorken.py:31-62).
The reference's eos.py is imported on its own (its package __init__ pulls in
plotting code that is not installed here).
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def load_ref_eos(refroot):
    path = os.path.join(refroot, 'pyvisc', 'eos', 'eos.py')
    spec = importlib.util.spec_from_file_location('ref_eos', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_ref_glauber(refroot):
    import types
    for name in ('pyopencl', 'pyopencl.array'):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules['pyopencl'].array = sys.modules['pyopencl.array']
    path = os.path.join(refroot, 'pyvisc', 'glauber.py')
    spec = importlib.util.spec_from_file_location('ref_glauber', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def sample_rows(n):
    idx = set(range(0, 8)) | set(range(n - 4, n))
    idx |= set(range(0, n, max(1, n // 400)))
    idx |= {n // 2, n // 3, 999, 1000, 1001, 1554, 1555, 1556, 63728 % n}
    return np.array(sorted(i for i in idx if 0 <= i < n), np.int64)


def main(refroot):
    ref = load_ref_eos(refroot)
    out = {}
    # ideal gas table exactly as the reference builds its image
    e = ref.Eos('ideal_gas')
    img = np.array(list(zip(e.cs2, e.pr, e.T, e.s)), dtype=np.float32)
    rows = sample_rows(img.shape[0])
    out['ideal_gas_rows'] = rows
    out['ideal_gas_table'] = img[rows]
    meta = {'ideal_gas_f_ed_0137': float(e.f_ed(0.137)), 'ideal_gas_num_of_ed': int(e.num_of_ed),
            'ideal_gas_ed_step': float(e.ed_step)}

    # reference cs2 post-processing on the regenerated PCE165 grid
    from clvisc_b200.eos_tables.make_pce165 import regenerate
    ed, pr, sd, Td = regenerate(refroot)

    class Bare(object):
        pass
    b = Bare()
    b.ed, b.pr, b.s, b.T = ed, pr.copy(), sd, Td
    b.ed_step = 0.002
    ref.Eos.eos_func_from_interp1d(b)
    img2 = np.stack([b.cs2, pr, Td, sd], axis=1).astype(np.float32)
    rows2 = sample_rows(img2.shape[0])
    out['pce165_rows'] = rows2
    out['pce165_table'] = img2[rows2]
    meta['pce165_f_ed_0137'] = float(b.f_ed(0.137))

    np.savez_compressed(os.path.join(HERE, 'golden.npz'), **out)
    kat = {
        'minmod4': {'source': 'pyvisc/tests/test_kernel_helper.py:29-54',
                    'a': [1.0, -2.0, -1.0, 4.0], 'b': [2.0, 0.0, -2.0, 4.0], 'c': [3.0, 2.0, -3.0, 4.0],
                    'minmod4(minmod4(a,b),c)': [1.0, 0.0, -1.0, 4.0]},
        'rootfinding': {'source': 'pyvisc/tests/test_kernel_helper.py:93-117',
                        'ed_range': [1.0, 10.0], 'v_range': [0.0, 0.999], 'decimals': 2, 'eos': 'EOSI'},
        'reduction': {'source': 'pyvisc/tests/test_reduction.py:15-53', 'n': 50000},
        'hypersf_unit_cube': {'source': 'pyvisc/tests/test_hypersf.py:26-59 (value derived: flat tau slice)',
                              'ed_old': 3.0, 'ed_new': 2.0, 'efrz': 2.5, 'dSigma': [1.0, 0.0, 0.0, 0.0]},
        'bjorken_ideal': {'source': 'pyvisc/tests/test_bjorken.py:31-62', 'ed0': 30.0, 'loops': 200,
                          'decimals': 3, 'law': 'ed/ed0 = (tau/tau0)^(-4/3)'},
    }
    meta['kat'] = kat
    g = load_ref_glauber(refroot)
    classes = list(zip([0, 5, 0, 10, 20, 10, 30, 50, 0], [5, 10, 10, 15, 30, 30, 50, 80, 80]))
    meta['weight_mean_b'] = {'source': 'pyvisc/glauber.py:14-57, classes of glauber.py:106-123',
                             'classes': classes,
                             'Au+Au': [float(g.weight_mean_b(a, b, 'Au+Au')) for a, b in classes],
                             'Pb+Pb': [float(g.weight_mean_b(a, b, 'Pb+Pb')) for a, b in classes]}
    with open(os.path.join(HERE, 'golden.json'), 'w') as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print('wrote golden.npz, golden.json')


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('CLVISC_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: make_golden.py REFERENCE_ROOT (or set CLVISC_REFERENCE_ROOT): '
                 'the directory that holds the reference project (pyvisc/)')
    main(root)
