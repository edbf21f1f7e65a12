"""Regenerate the s95p-PCE165-v0 and s95p-PCE-v1 equation-of-state tables
used by eos_type 'lattice_pce165' and 'lattice_pce150'.

The reference loads this EOS from pyvisc/eos/eos_table/s95p-PCE165-v0/EOS_PST.dat
(pyvisc/eos/eos.py:102-113), a file that is not present in the reference
snapshot. Its raw inputs are present: s95p-PCE165-v0_dens{1..4}.dat (e, p, s,
nb, plasma fraction) and _par{1..4}.dat (T, mu...), four descending grids
0.001..1.001 (step 0.002), ..11.001 (0.02), ..61.001 (0.1), ..311.001 (0.5)
(format: eos_table/s95p-PCE165-v0/README).

This script builds what eos.py:102-113 expects, a uniform table of
num_of_ed = 155500 rows at e_k = 0.002*k (ed_start 0.0, ed_step 0.002):
  * the four grids are merged in ascending order, duplicated end points
    dropped, and the point (e, p, s, T) = (0, 0, 0, 0) prepended, as eos.py
    inserts a zero row;
  * p, s and T are linearly interpolated onto e_k (numpy.interp);
  * cs2 is post-processed exactly as Eos.eos_func_from_interp1d
    (eos.py:78-100): numpy.gradient(p, 0.002), a minmod repair of entries with
    |cs2| > 0.34, and a least-squares fit cs2 = a/(exp(b/e) + c) for e >= 30.
lattice_pce165.npz next to this file holds the merged source grid (float64)
and cs2 (float32); clvisc_b200.eos rebuilds the uniform p, s, T columns from
the source grid with the same numpy.interp call at load time. The
s95p-PCE-v1 table behind 'lattice_pce150' (eos.py:116-127, EOS_PST.dat of
s95p-PCE-v1, also absent) has the same four grids and is regenerated the same
way into lattice_pce150.npz. Run it from the repository root:

    python clvisc_b200/eos_tables/make_pce165.py /path/to/reference [lattice_pce150]
"""
import os
import sys

import numpy as np
from scipy.optimize import curve_fit

NUM_ED = 155500
ED_STEP = 0.002


def _read_grid(path):
    with open(path) as f:
        lines = f.read().split('\n')
    e0 = float(lines[0].split()[0])
    de, ne = lines[1].split()[:2]
    rows = np.array([[float(x) for x in ln.split()] for ln in lines[2:] if ln.strip()])
    assert rows.shape[0] == int(ne), (path, rows.shape, ne)
    return e0, float(de), rows[::-1]  # ascending


def _minmod(a, b):
    if a > 0 and b > 0:
        return min(a, b)
    elif a < 0 and b < 0:
        return max(a, b)
    return 0


def cs2_from_pressure(ed, pr, ed_step):
    """Speed of sound squared as eos.py:85-100 derives it from p(e)."""
    cs2 = np.gradient(pr, ed_step)
    for i, c in enumerate(cs2):
        if abs(c) > 0.34:
            cs2[i] = _minmod(cs2[i - 1], _minmod(c, cs2[i + 1]))
    mask = ed >= 30.
    def exp_func(x, a, b, c):
        return a / (np.exp(b / x) + c)
    popt, _ = curve_fit(exp_func, ed[mask], cs2[mask])
    cs2[mask] = exp_func(ed[mask], *popt)
    return cs2


TABLES = {'lattice_pce165': 's95p-PCE165-v0', 'lattice_pce150': 's95p-PCE-v1'}


def source_grid(refroot, eos_type='lattice_pce165'):
    """Merged ascending (e, p, s, T) points of the four s95p grids, with the
    zero row prepended."""
    name = TABLES[eos_type]
    d = os.path.join(refroot, 'pyvisc', 'eos', 'eos_table', name)
    es, ps, ss, ts = [], [], [], []
    for n in range(1, 5):
        _, _, dens = _read_grid(os.path.join(d, '%s_dens%d.dat' % (name, n)))
        _, _, par = _read_grid(os.path.join(d, '%s_par%d.dat' % (name, n)))
        es.append(dens[:, 0]); ps.append(dens[:, 1]); ss.append(dens[:, 2]); ts.append(par[:, 0])
    e = np.concatenate(es); p = np.concatenate(ps); s = np.concatenate(ss); T = np.concatenate(ts)
    order = np.argsort(e, kind='stable')
    e, p, s, T = e[order], p[order], s[order], T[order]
    keep = np.concatenate([[True], np.diff(e) > 1e-9])
    e, p, s, T = e[keep], p[keep], s[keep], T[keep]
    e = np.insert(e, 0, 0.0); p = np.insert(p, 0, 0.0); s = np.insert(s, 0, 0.0); T = np.insert(T, 0, 0.0)
    return e, p, s, T


def uniform(e, p, s, T):
    """(ed, p, s, T) on the uniform 155500-row grid, float64."""
    ed = np.arange(NUM_ED) * ED_STEP
    return ed, np.interp(ed, e, p), np.interp(ed, e, s), np.interp(ed, e, T)


def regenerate(refroot, eos_type='lattice_pce165'):
    return uniform(*source_grid(refroot, eos_type))


def build(refroot, eos_type='lattice_pce165'):
    src = source_grid(refroot, eos_type)
    ed, pr, sd, Td = uniform(*src)
    cs2 = cs2_from_pressure(ed, pr.copy(), ED_STEP)
    return src, cs2


if __name__ == '__main__':
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('CLVISC_REFERENCE_ROOT')
    if not ref:
        sys.exit('usage: make_pce165.py REFERENCE_ROOT [lattice_pce165|lattice_pce150] (or set '
                 'CLVISC_REFERENCE_ROOT): the directory that holds the reference project (pyvisc/, eos tables)')
    eos_type = sys.argv[2] if len(sys.argv) > 2 else 'lattice_pce165'
    (e, p, s, T), cs2 = build(ref, eos_type)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), '%s.npz' % eos_type)
    np.savez_compressed(out, src_e=e, src_p=p, src_s=s, src_T=T, cs2=cs2.astype(np.float32),
                        ed_start=np.float64(0.0), ed_step=np.float64(ED_STEP), num_of_ed=np.int64(NUM_ED))
    print('wrote', out, e.shape, os.path.getsize(out), 'bytes')
