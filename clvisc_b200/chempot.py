"""Effective chemical potentials of the hadrons on the freeze-out surface
(chemical_potential.dat), the drop-in for pyvisc/eos/chemical_potential.py.

With a partial-chemical-equilibrium EOS (lattice_pce165) the stable species
carry chemical potentials that keep their yields fixed below chemical
freeze-out. At the freeze-out energy density efrz they are interpolated
linearly in the EOS's own table (chemical_potential.py:61-93: the row index
floor((efrz - e0)/de), zero for an index above 500), and each hadron's
potential is the branching-ratio-weighted sum of its daughters' potentials,
mu_i = sum_channels BR sum_daughters mu_d, in the order of the decay table, so
that daughters come first (chemical_potential.py:95-133). Gamma has mu = 0.
Other EOS types write 0.0 for every hadron (chemical_potential.py:99-102,
128-133). The file has one line 'pid mu' per hadron, written as Python's
print() writes them.

The tables (eos_tables/pce165_chem.npz, pce165_decays.json) are the
reference's s95p-PCE165-v0 files, extracted by eos_tables/make_chempot.py.
"""
import json
import math
import os

import numpy as np

_HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'eos_tables')
PCE_TYPES = ('lattice_pce165', 'lattice_pce150')


def _tables(eos_type='lattice_pce165'):
    """The stable species' chemical-potential table and the decay table of
    the EOS's data set: s95p-PCE-v1 for lattice_pce150, s95p-PCE165-v0
    otherwise (chemical_potential.py:33-36, 62-64)."""
    tag = 'pce150' if eos_type == 'lattice_pce150' else 'pce165'
    t = np.load(os.path.join(_HERE, '%s_chem.npz' % tag))
    with open(os.path.join(_HERE, '%s_decays.json' % tag)) as f:
        d = json.load(f)
    return t, d['stable'], d['hadrons']


def mu_for_stable(efrz, tab=None):
    """Chemical potentials of the stable species (28 in s95p-PCE165-v0, 35 in
    s95p-PCE-v1) at efrz (chemical_potential.py:61-93)."""
    if tab is None:
        tab = _tables()[0]
    e0, de, ne = float(tab['e0']), float(tab['de']), int(tab['ne'])
    table = tab['table']
    energy_density = np.array([e0 + i * de for i in range(ne)])
    idx = int(math.floor((efrz - e0) / de))
    if idx > 500:
        return np.zeros_like(table[0])
    ed0, ed1 = energy_density[idx], energy_density[idx + 1]
    mu0, mu1 = table[idx], table[idx + 1]
    w0 = (efrz - ed0) / de
    w1 = (ed1 - efrz) / de
    return w0 * mu1 + w1 * mu0


def chemical_potentials(efrz, eos_type='lattice_pce165'):
    """[(pid, mu)] for every hadron of the decay table, in its order."""
    tab, stable, hadrons = _tables(eos_type)
    mu_s = mu_for_stable(efrz, tab)
    mu = {pid: mu_s[i] for i, pid in enumerate(stable)}
    mu['22'] = 0.0
    out = []
    for pid, channels in hadrons:
        m = 0.0
        for br, daughters in channels:
            for dpid in daughters:
                m += br * mu[dpid]
        mu[pid] = m
        out.append((pid, m))
    if eos_type not in PCE_TYPES:
        out = [(pid, 0.0) for pid, _ in out]
    return out


def write_chemical_potential(efrz, path, eos_type='lattice_pce165'):
    """chemical_potential.dat in `path` (ideal.py:65, chemical_potential.py:
    135-154); returns {int pid: mu}."""
    rows = chemical_potentials(efrz, eos_type)
    os.makedirs(path, exist_ok=True)
    with open(os.path.join(path, 'chemical_potential.dat'), 'w') as fout:
        for pid, m in rows:
            print(pid, m, file=fout)
    return {int(pid): float(m) for pid, m in rows}


def read_chemical_potential(path):
    """{int pid: mu} from a chemical_potential.dat (the reader of
    CLSmoothSpec/src/cl_spec.cpp:183-200); empty if there is none."""
    fname = os.path.join(path, 'chemical_potential.dat')
    out = {}
    if not os.path.exists(fname):
        return out
    for line in open(fname):
        f = line.split()
        if len(f) >= 2:
            out[int(f[0])] = float(f[1])
    return out
