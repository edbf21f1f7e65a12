"""Parity at the sizes the headline metric is quoted on.

* 201 x 201 x 105 (dx = dy = 0.16 fm, d_eta = 0.15, dtau = 0.02 fm, eta/s =
  0.08, lattice PCE165 EOS, FP32, seeded Pb+Pb at b = 8 fm, seed 2): 20 fused
  steps, then the freeze-out surface between the initial and the final state;
* 385 x 385 x 115 (dx = dy = 0.08 fm, dtau = 0.01 fm, seed 5): 3 fused steps
  in FP32 and in FP64.

The exact build must equal the oracle bit for bit (every field, the surface
element count and every element); the tolerance build must stay within 1e-5
(FP32) / 1e-11 (FP64) of each field's largest magnitude, each field scaled as
a whole tensor (test_fast_gpu.py states the measure). Each case prints its
errors. The oracle runs on every host core (OpenMP).
"""
import numpy as np
import pytest

from parity_util import assert_same, make_cfg, seeded_ic
from clvisc_b200.eos import Eos
from test_fast_gpu import TOL, field_errors

pytestmark = pytest.mark.gpu


def _run(cfg, ic, steps, oracle_mod=None):
    from clvisc_b200.visc import CLVisc
    if oracle_mod is not None:
        v = oracle_mod.OracleVisc(cfg)
    else:
        v = CLVisc(cfg)
    v.load_ini(ic)
    for n in range(steps):
        v.step(n)
    return v


def _host(v):
    if hasattr(v.ideal, 'field_to_host'):
        return (v.ideal.field_to_host(v.ideal.d_ev[1]), v.ideal.field_to_host(v.d_pi[1]),
                v.ideal.field_to_host(v.ideal.d_ev[2]), v.ideal.field_to_host(v.d_udiff))
    return v.ideal.d_ev[1], v.d_pi[1], v.ideal.d_ev[2], v.d_udiff


def _check(grid, dx, dt, seed, steps, use_float32, oracle_mod, hypersf=False):
    kw = dict(use_float32=use_float32, dx=dx, dz=0.15, dt=dt, etaos=0.08, tau0=0.6, skip=(2, 2, 2))
    cfg_exact = make_cfg(*grid, arithmetic='exact', **kw)
    ic = seeded_ic(cfg_exact, seed=seed, b=8.0, edmax=50.0)
    o = _run(cfg_exact, ic, steps, oracle_mod)
    want = _host(o)
    g = _run(cfg_exact, ic, steps)
    got = _host(g)
    for name, a, b in zip(('ev[1]', 'pi[1]', 'ev[2]', 'udiff'), got, want):
        assert_same('%s exact %s' % (grid, name), a, b)
    print('%s %s exact: every field bit for bit after %d steps' % (grid, 'fp32' if use_float32 else 'fp64', steps))
    if hypersf:
        _check_hypersf(cfg_exact, g, o, ic)
    del g
    f = _run(make_cfg(*grid, arithmetic='fast', **kw), ic, steps)
    fast = _host(f)
    errs = field_errors(fast[0], want[0], fast[1], want[1], Eos(cfg_exact.eos_type), float(f.ideal.tau))
    worst = max(v for k, v in errs.items() if k != 'components')
    print('%s %s fast after %d steps (bound %.0e): %s' % (grid, 'fp32' if use_float32 else 'fp64', steps,
                                                         TOL[use_float32], {k: '%.2e' % x for k, x in errs.items()}))
    assert worst <= TOL[use_float32], errs


def _check_hypersf(cfg, g, o, ic):
    """Surface between the initial state and the state after the steps, from
    the same inputs on both sides: element count and elements exact."""
    import torch
    ev0 = g.ideal.d_ev_old
    g.ideal.field_from_host(ev0, ic)
    pi0 = torch.zeros_like(g.d_pi[1])
    tau_new = cfg.real(g.ideal.tau)
    tau_old = cfg.real(cfg.TAU0)
    g.ideal.d_num_of_sf.zero_()
    g.ideal._hypersf(1, tau_old, tau_new, ev0, g.ideal.d_ev[1], pi0, g.d_pi[1], g.d_pi_sf)
    n = g.ideal.read_num_of_sf()
    sf_o, tx_o, pi_o = o.ideal._hypersf(1, tau_old, tau_new, np.asarray(ic, cfg.real), o.ideal.d_ev[1],
                                        np.zeros_like(o.d_pi[1]), o.d_pi[1])
    assert n == len(sf_o) and n > 1000, (n, len(sf_o))
    assert_same('hypersf', g.ideal.d_hypersf[:n].cpu().numpy(), sf_o)
    assert_same('pisf', g.d_pi_sf[:n].cpu().numpy(), pi_o)
    tx_g = g.ideal.d_sf_txyz[:n].cpu().numpy()
    assert_same('sf x, y', tx_g[:, 1:3], tx_o[:, 1:3])
    np.testing.assert_allclose(tx_g[:, [0, 3]], tx_o[:, [0, 3]], rtol=5e-7, atol=0)
    print('surface: %d elements, count and elements exact' % n)


def test_config2_parity(cuda_lib, oracle_mod):
    _check((201, 201, 105), 0.16, 0.02, 2, 20, True, oracle_mod, hypersf=True)


@pytest.mark.parametrize('use_float32', [True, False])
def test_config5_parity(cuda_lib, oracle_mod, use_float32):
    _check((385, 385, 115), 0.08, 0.01, 5, 3, use_float32, oracle_mod)
