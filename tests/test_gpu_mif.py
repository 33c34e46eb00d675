"""Iterated filtering on the GPU against the oracle's restatement of one MIF
iteration (FP64, the same Philox draws on both sides)."""

import numpy as np
import pytest

import models
from plomgpu import mif, native

pytestmark = pytest.mark.gpu


def _setup(name, J, R, precision=64):
    eng = models.engine(name)
    p = models.make_problem(name, J=J, dt=1.0, precision=precision, seed=3)
    sd = {'r0': 0.2, 'v': 0.1, 'rep': 0.1, 'sto': 0.3, 'phi': 0.1}
    names = [n for n in sd if n in p.model.par_proc + p.model.par_obs]
    run = mif.Mif(eng, p, n_runs=R, names=names, sd_transf=sd, a=0.95, b=2.0)
    return eng, p, run


@pytest.mark.parametrize('name,J,R', [('sir_short', 400, 3), ('seir3', 256, 2), ('noise', 300, 2)])
def test_mif_iteration_matches_oracle(name, J, R):
    """noise: r0 (process) and phi (observation) are fitted per group, one component each."""
    eng, p, run = _setup(name, J, R)
    orc = models.build_oracle(name)
    rng = np.random.default_rng(1)
    run.theta_hat = run.theta_hat + 0.05 * rng.standard_normal(run.theta_hat.shape)
    for m in (1, 7):
        freeze, sd_init, sd_mut, vt_add = run.schedules(m)
        seed = 4242 + m
        g = run.plan.iteration(run.theta_hat, sd_init, sd_mut, vt_add, seed)
        o = orc.mif_iteration(p, run.holder, run.theta_hat, sd_init, sd_mut, vt_add, seed)
        np.testing.assert_allclose(g[0], o[0], rtol=1e-9)
        np.testing.assert_array_equal(g[1], o[1])
        rows = np.nonzero(run.has_data)[0]
        np.testing.assert_allclose(g[2][:, rows], o[2][:, rows], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(g[3][:, rows], o[3][:, rows], rtol=1e-7, atol=1e-12)
    run.close()


def test_mif_runs_improve_likelihood_fp32():
    """A few iterations from a perturbed start raise the log-likelihood of every run."""
    eng, p, run = _setup('sir', 2000, 4, precision=32)
    run.theta_hat = run.theta_hat + np.array([0.3 if c['name'] == 'r0' else 0.0 for c in run.comp])
    trace = run.run(12, seed=5)
    first = trace[0]['loglik']
    last = np.mean([t['loglik'] for t in trace[-3:]], axis=0)
    assert np.all(np.isfinite(last))
    assert np.mean(last) > np.mean(first)
    run.close()


FLS_CASES = [
    # noise: S fitted per population (2 groups), I fitted once, remainder R: the proposals of the
    # initial proportions are redrawn until they sum to at most 1 in every population
    ('noise', 300, 2, {'S': 0.1, 'I': 0.3, 'r0': 0.2, 'phi': 0.1}),
    # drift: r0 is drifted (its start value is a fixed-lag component, one per population), its
    # volatility a random-walk component read by the drift of every particle
    ('drift', 256, 2, {'S': 0.1, 'I': 0.2, 'r0': 0.2, 'vol': 0.3, 'rep': 0.1}),
]


@pytest.mark.parametrize('prior', [False, True])
@pytest.mark.parametrize('name,J,R,sd', FLS_CASES)
def test_mif_fixed_lag_and_prior_match_oracle(name, J, R, sd, prior):
    """Initial conditions and drift start values fitted by fixed-lag smoothing, with and without
    the --prior patch: GPU iteration = oracle restatement (FP64, same Philox draws) for the
    log-likelihood, the filtered moments and the fixed-lag means at interval L."""
    from plomgpu.best import Best
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=J, dt=1.0, precision=64, seed=3)
    best = Best(p.model, p.theta, is_bayesian=True) if prior else None
    lag = p.n_obs // 2
    run = mif.Mif(eng, p, n_runs=R, names=list(sd), sd_transf=sd, a=0.95, b=2.0, lag=lag, prior=best)
    fls = run.fls.astype(bool)
    assert fls.any() and (~fls).any()
    rng = np.random.default_rng(2)
    run.theta_hat = run.theta_hat + 0.02 * rng.standard_normal(run.theta_hat.shape)
    for m in (1, 3):
        freeze, sd_init, sd_mut, vt_add = run.schedules(m)
        seed = 777 + m
        g = run.plan.iteration(run.theta_hat, sd_init, sd_mut, vt_add, seed)
        o = orc.mif_iteration(p, run.holder, run.theta_hat, sd_init, sd_mut, vt_add, seed)
        np.testing.assert_allclose(g[0], o[0], rtol=1e-9)
        np.testing.assert_array_equal(g[1], o[1])
        rows = np.nonzero(run.has_data)[0]
        np.testing.assert_allclose(g[2][:, rows], o[2][:, rows], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(g[3][:, rows], o[3][:, rows], rtol=1e-7, atol=1e-12)
        means, updated = run.plan.fls_means()
        assert updated
        np.testing.assert_allclose(means[:, fls], orc.last_fls_means[:, fls], rtol=1e-9, atol=1e-12)
        assert np.all(np.isnan(means[:, ~fls]))
        run.update(m, g[2], g[3], means)
        np.testing.assert_array_equal(run.theta_hat[:, fls], means[:, fls])
    run.close()


def test_mif_fixed_lag_fp32_moves_initial_conditions():
    """FP32 production: starting from a wrong initial infected proportion, the fixed-lag means
    move it towards the value the data were simulated with."""
    eng = models.engine('sir')
    p = models.make_problem('sir', J=4000, dt=1.0, precision=32, seed=4)
    run = mif.Mif(eng, p, n_runs=4, names=['I', 'r0'], sd_transf={'I': 0.5, 'r0': 0.05}, a=0.9, b=2.0, lag=20)
    q = [k for k, c in enumerate(run.comp) if c['name'] == 'I'][0]
    truth = run.theta_hat[0, q]
    run.theta_hat[:, q] = truth + 1.0  # logit scale
    run.run(8, seed=9)
    assert np.all(np.abs(run.theta_hat[:, q] - truth) < 0.8)
    run.close()
