"""Extract the data behind chemical_potential.dat for the s95p-PCE165-v0
(lattice_pce165) and s95p-PCE-v1 (lattice_pce150) equations of state.

The reference computes effective chemical potentials of every hadron at the
freeze-out energy density when CLIdeal is constructed
(pyvisc/ideal.py:65 -> pyvisc/eos/chemical_potential.py:146-169), from three
files of its EOS directory (eos_table/s95p-PCE165-v0/):
  * s95p-PCE165-v0_pichem1.dat: e0, (de, ne), nstable, then ne rows of the 28
    stable species' chemical potentials, highest energy density first;
  * particles.dat: the stable species (last column 'Stable' or '********'),
    Gamma excluded;
  * pdg05.dat: every hadron with its decay channels (branching ratio and
    daughters), lighter states first.
This script copies those numbers, unchanged, into pce165_chem.npz (the
chemical-potential table, reversed as the reference reads it) and
pce165_decays.json (the stable ids and, in file order, each hadron's id with
its decay channels), which clvisc_b200.chempot reads. Run it from the
repository root (lattice_pce150: pce150_chem.npz, pce150_decays.json from the
s95p-PCE-v1 files):

    python clvisc_b200/eos_tables/make_chempot.py REFERENCE_ROOT [lattice_pce150]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


# eos_type -> (table directory, output tag): chemical_potential.py:33-36, 62-64
SOURCES = {'lattice_pce165': ('s95p-PCE165-v0', 'pce165'), 'lattice_pce150': ('s95p-PCE-v1', 'pce150')}


def extract(refroot, eos_type='lattice_pce165'):
    name = SOURCES[eos_type][0]
    d = os.path.join(refroot, 'pyvisc', 'eos', 'eos_table', name)
    with open(os.path.join(d, '%s_pichem1.dat' % name)) as f:
        e0 = float(f.readline())
        de, ne = f.readline().split()
        de, ne = float(de), int(ne)
        nstable = int(f.readline())
    table = np.loadtxt(os.path.join(d, '%s_pichem1.dat' % name), skiprows=3)[::-1]
    stables = []
    for line in open(os.path.join(d, 'particles.dat')):
        info = line.split()
        if info and (info[-1] == 'Stable' or info[-1] == '********') and info[1] != 'Gamma':
            stables.append(info[1])
    hadrons = []
    lines = open(os.path.join(d, 'pdg05.dat')).readlines()
    i = 0
    while i < len(lines):
        head = lines[i].split()
        ndecays = int(head[-1])
        channels = []
        for j in range(ndecays):
            dec = lines[i + j + 1].split()
            nd = int(dec[1])
            channels.append([float(dec[2]), dec[3:3 + nd]])
        hadrons.append([head[0], channels])
        i += ndecays + 1
    return dict(e0=e0, de=de, ne=ne, nstable=nstable, table=np.ascontiguousarray(table)), stables, hadrons


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('CLVISC_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: make_chempot.py REFERENCE_ROOT [lattice_pce165|lattice_pce150] (or set '
                 'CLVISC_REFERENCE_ROOT): the directory that holds the reference project (pyvisc/)')
    eos_type = sys.argv[2] if len(sys.argv) > 2 else 'lattice_pce165'
    tag = SOURCES[eos_type][1]
    tab, stables, hadrons = extract(root, eos_type)
    np.savez_compressed(os.path.join(HERE, '%s_chem.npz' % tag), **tab)
    with open(os.path.join(HERE, '%s_decays.json' % tag), 'w') as f:
        json.dump({'stable': stables, 'hadrons': hadrons}, f, separators=(',', ':'))
    print('wrote %s_chem.npz' % tag, tab['table'].shape, 'and %s_decays.json,' % tag, len(hadrons), 'hadrons,',
          len(stables), 'stable')
