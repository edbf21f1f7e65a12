"""clv_status after a step: non-finite values, bad cells, surface overflow.
Each fault is made on the host (a NaN in the initial condition, a surface
buffer too small for the event); no kernel is made to fault."""
import numpy as np
import pytest

from parity_util import make_cfg, seeded_ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('arithmetic', ['exact', 'fast'])
def test_status_clean_run(cuda_lib, arithmetic):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(31, 29, 27, arithmetic=arithmetic)
    v = CLVisc(cfg)
    v.load_ini(seeded_ic(cfg, seed=3))
    for n in range(4):
        v.step(n)
    st = v.status()
    bad = int((v.d_goodcell[:v.size] == 0).sum().item())
    assert st == {'nan': 0, 'bad_cells': bad, 'sf_overflow': 0}, st


def test_status_counts_nan_from_initial_condition(cuda_lib):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(21, 19, 17)
    ic = seeded_ic(cfg, seed=3)
    ic[(10 * 19 + 9) * 17 + 8, 0] = np.nan
    v = CLVisc(cfg)
    v.load_ini(ic)
    assert v.status()['nan'] == 1  # before any step: the loaded NaN itself
    v.step(0)
    st = v.status()
    ev = v.ideal.field_to_host(v.ideal.d_ev[1])
    pi = v.ideal.field_to_host(v.d_pi[1])
    assert st['nan'] == int(np.count_nonzero(~np.isfinite(ev)) + np.count_nonzero(~np.isfinite(pi))) > 1, st


def test_status_reports_surface_overflow(cuda_lib, tmp_path):
    from clvisc_b200.visc import CLVisc
    cfg = make_cfg(25, 23, 13, dx=0.8, dz=0.6, dt=0.04, ntskip=5, skip=(2, 2, 1), out=str(tmp_path))
    v = CLVisc(cfg, hypersf_capacity=16)
    v.load_ini(seeded_ic(cfg, seed=11, edmax=20.0))
    with pytest.raises(RuntimeError, match='capacity'):
        v.evolve(max_loops=30, force_run_to_maxloop=True, save_hypersf=True)
    st = v.status()
    total = int(v.ideal.d_num_of_sf.item())
    assert total > 16 and st['sf_overflow'] == total - 16, (st, total)
