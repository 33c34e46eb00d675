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
