"""Generate the chemical_potential.dat fixtures from the reference itself.

    python tests/golden/make_golden_chempot.py REFERENCE_ROOT

Imports the reference's pyvisc/eos/chemical_potential.py on its own (numpy
only) and runs ChemicalPotential(efrz, eos_type).get_chemical_potential_for_
resonance (chemical_potential.py:95-133), the work create_table does before it
copies the file into the reference's own tree (:146-169), for
eos_type lattice_pce165 and ideal_gas, and lattice_pce150 (s95p-PCE-v1
data). efrz is the freeze-out energy density at T = 0.137 GeV of this
repository's lattice_pce165 (lattice_pce150) table (the reference's Eos of
those types needs EOS_PST.dat, which its snapshot lacks), also recorded in
the fixtures' efrz files.
"""
import importlib.util
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(refroot):
    from clvisc_b200.eos import Eos
    path = os.path.join(refroot, 'pyvisc', 'eos', 'chemical_potential.py')
    spec = importlib.util.spec_from_file_location('ref_chempot', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    efrz = float(Eos('lattice_pce165').f_ed(0.137))
    for eos_type in ('lattice_pce165', 'ideal_gas'):
        tmp = tempfile.mkdtemp()
        mod.ChemicalPotential(efrz, eos_type=eos_type).get_chemical_potential_for_resonance(tmp)
        shutil.copy(os.path.join(tmp, 'chemical_potential.dat'),
                    os.path.join(HERE, 'chemical_potential_%s.dat' % eos_type))
        shutil.rmtree(tmp)
    with open(os.path.join(HERE, 'chemical_potential_efrz.txt'), 'w') as f:
        f.write(repr(efrz) + '\n')
    # lattice_pce150 (s95p-PCE-v1 data) at its own table's T = 0.137 GeV
    efrz150 = float(Eos('lattice_pce150').f_ed(0.137))
    tmp = tempfile.mkdtemp()
    mod.ChemicalPotential(efrz150, eos_type='lattice_pce150').get_chemical_potential_for_resonance(tmp)
    shutil.copy(os.path.join(tmp, 'chemical_potential.dat'), os.path.join(HERE, 'chemical_potential_lattice_pce150.dat'))
    shutil.rmtree(tmp)
    with open(os.path.join(HERE, 'chemical_potential_efrz_pce150.txt'), 'w') as f:
        f.write(repr(efrz150) + '\n')
    print('wrote chemical_potential_{lattice_pce165,ideal_gas}.dat at efrz', efrz,
          'and chemical_potential_lattice_pce150.dat at efrz', efrz150)


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('CLVISC_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: make_golden_chempot.py REFERENCE_ROOT (or set CLVISC_REFERENCE_ROOT)')
    main(root)
