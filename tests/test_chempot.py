"""chemical_potential.dat (pyvisc/ideal.py:65, eos/chemical_potential.py)
against the file the reference's own module writes for the same freeze-out
energy density (tests/golden/make_golden_chempot.py): byte for byte."""
import filecmp
import os

import pytest

from clvisc_b200 import chempot

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_pce150_chemical_potential_file_matches_reference(tmp_path):
    """lattice_pce150: the s95p-PCE-v1 data (35 stable species), at the
    freeze-out energy density of the regenerated PCE150 table."""
    from clvisc_b200.eos import Eos
    efrz = float(open(os.path.join(GOLDEN, 'chemical_potential_efrz_pce150.txt')).read())
    assert efrz == float(Eos('lattice_pce150').f_ed(0.137))
    mu = chempot.write_chemical_potential(efrz, str(tmp_path), 'lattice_pce150')
    assert filecmp.cmp(str(tmp_path / 'chemical_potential.dat'),
                       os.path.join(GOLDEN, 'chemical_potential_lattice_pce150.dat'), shallow=False)
    assert len(mu) == 217 and mu[22] == 0.0 and mu[211] > 0.0
    tab, stable, _ = chempot._tables('lattice_pce150')
    assert len(stable) == 35 and tab['table'].shape == (501, 35)


@pytest.mark.parametrize('eos_type', ['lattice_pce165', 'ideal_gas'])
def test_chemical_potential_file_matches_reference(tmp_path, eos_type):
    efrz = float(open(os.path.join(GOLDEN, 'chemical_potential_efrz.txt')).read())
    mu = chempot.write_chemical_potential(efrz, str(tmp_path), eos_type)
    assert filecmp.cmp(str(tmp_path / 'chemical_potential.dat'),
                       os.path.join(GOLDEN, 'chemical_potential_%s.dat' % eos_type), shallow=False)
    assert len(mu) == 217
    if eos_type == 'lattice_pce165':
        assert 0.04 < mu[211] < 0.05 and mu[22] == 0.0 and mu[2212] > mu[211]
    else:
        assert set(mu.values()) == {0.0}
    assert chempot.read_chemical_potential(str(tmp_path)) == mu


def test_stable_interpolation_edges():
    """The row index floor((e - e0)/de); zeros above row 500."""
    tab, stable, _ = chempot._tables()
    assert len(stable) == 28 and tab['table'].shape == (501, 28)
    e0, de = float(tab['e0']), float(tab['de'])
    assert (chempot.mu_for_stable(e0 + 501.5 * de, tab) == 0).all()
    row = chempot.mu_for_stable(e0 + 10 * de, tab)
    assert abs(row - tab['table'][10]).max() < 1e-12
