"""The learned surrogate end to end on a small case: events from the batched
solver (64 x 64 (2+1)D events, 100 steps), training with the library's own
kernels, evaluation against the solver on held-out seeds. The trained network
must beat the method without it (Bjorken cooling of the initial profile) by a
wide margin on the relative L2 error of e, and answer faster than the solver
(the full-size comparison with fallbacks is bench.py's surrogate leg)."""
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_gains_over_no_network(cuda_lib):
    from clvisc_b200.surrogate import run_experiment
    r = run_experiment(n_train=512, n_test=64, epochs=10, batch=32, n=64, steps=100, gen_batch=256, lr=2e-3,
                       log=lambda m: None)
    assert r['rel_l2_e_network_only']['mean'] < 0.5 * r['rel_l2_e_without_network']['mean'], r
    assert r['loss_history'][-1] < 0.3 * r['loss_history'][0], r
    # at this size the solver is quick and a fallback batch costs mostly its
    # set-up; the network's own answer must still be faster than the solver's
    assert r['inference_s'] < r['solver_s'], r
