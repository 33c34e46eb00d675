"""The command-line drivers end to end on the GPU, in a model directory made
by pmbuilder: smc (trace / hat / pred_res / X / .done), pmcmc (trace, X
trajectories, acceptance, covariance), mif (trace), and the sampled
trajectory against a restatement of sample_traj_and_print on the same
genealogy."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

import models

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'iterated-inference-pipeline_b200')


def _model_dir(tmp_path_factory, name):
    from plomgpu import build
    c, p, l, th = models.files(name)
    if name == 'sir':  # fit r0 and v
        for k in ('r0', 'v'):
            th['parameter'][k]['sd_transf'] = 0.1
    d = str(tmp_path_factory.mktemp('cli') / name)
    build.build_model_dir(c, p, l, d, name=name, shared_lib=True)
    with open(os.path.join(d, 'theta.json'), 'w') as f:
        f.write(json.dumps(th) + '\n')
    return d


@pytest.fixture(scope='module')
def model_dir(tmp_path_factory):
    return _model_dir(tmp_path_factory, 'noise')


@pytest.fixture(scope='module')
def sir_dir(tmp_path_factory):
    return _model_dir(tmp_path_factory, 'sir')


def _run(d, cmd, *args):
    env = dict(os.environ, PYTHONPATH=PKG + os.pathsep + os.environ.get('PYTHONPATH', ''))
    with open(os.path.join(d, 'theta.json')) as f:
        r = subprocess.run([sys.executable, '-m', 'plomgpu', cmd] + list(args), stdin=f, cwd=d, env=env,
                           capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _csv(path):
    with open(path) as f:
        lines = f.read().splitlines()
    return lines[0].split(','), [l.split(',') for l in lines[1:]]


def test_smc_cli_outputs(model_dir):
    d = model_dir
    out = _run(d, 'smc', 'sde', '-J', '500', '-s', '1', '--precision', '64', '-r')
    assert 'logV:' in out and 'clean up...' in out
    head, rows = _csv(os.path.join(d, 'trace_0.csv'))
    assert head[0] == 'index' and head[-1] == 'log_like' and len(rows) == 1
    ll_cli = float(rows[0][-1])
    # the same filter through the library
    p = models.make_problem('noise', J=500, dt=1.0, precision=64, seed=2)
    eng = models.engine('noise')
    g = eng.smc(p)
    assert ll_cli == pytest.approx(g.loglik, rel=1e-5)
    head, rows = _csv(os.path.join(d, 'hat_0.csv'))
    assert len(rows) == p.n_obs + 1 and all(len(r) == len(head) for r in rows)
    head, rows = _csv(os.path.join(d, 'pred_res_0.csv'))
    assert head[-1] == 'ess' and len(rows) == int(np.sum(~np.all(np.isnan(p.data), axis=1)))
    head, rows = _csv(os.path.join(d, 'X_0.csv'))
    assert len(rows) == (p.n_obs + 1) * 500 and all(len(r) == len(head) for r in rows[:1000])
    done = json.load(open(os.path.join(d, '.done_0.json')))
    assert 'parameter' in done
    # the reference's default implementation (psr) and the deterministic skeleton (ode)
    out = _run(d, 'smc', '-J', '300', '-s', '1', '-i', '5')
    assert 'logV:' in out
    head, rows = _csv(os.path.join(d, 'trace_5.csv'))
    assert np.isfinite(float(rows[0][-1]))
    out = _run(d, 'smc', 'ode', '-J', '1', '-i', '6')
    head, rows = _csv(os.path.join(d, 'hat_6.csv'))
    assert all(r[1] == r[2] == r[3] for r in rows[1:])  # one deterministic path: the interval collapses
    # -P: theta on stdout, no .done file
    out = _run(d, 'smc', 'sde', '-J', '200', '-s', '1', '-P', '-i', '4', '-b', '-e', '-d')
    assert json.loads(out)['parameter']
    assert not os.path.exists(os.path.join(d, '.done_4.json'))


def test_pmcmc_cli_outputs(model_dir):
    d = model_dir
    out = _run(d, 'pmcmc', 'sde', '-J', '200', '-s', '1', '-M', '12', '--acc', '-i', '7')
    assert 'acceptance rate(s)' in out
    head, rows = _csv(os.path.join(d, 'trace_7.csv'))
    assert head[-1] == 'log_like' and len(rows) >= 2
    head, rows = _csv(os.path.join(d, 'X_7.csv'))
    assert head[0] == 'index' and len(rows) > 0 and all(len(r) == len(head) for r in rows)
    assert os.path.exists(os.path.join(d, 'acc_7.csv'))
    assert os.path.exists(os.path.join(d, 'covariance_7.csv'))
    assert json.load(open(os.path.join(d, '.done_7.json')))['parameter']


def test_mif_cli_outputs(sir_dir):
    """MIF fits parameters that take one value for every population (the SIR workload)."""
    d = sir_dir
    _run(d, 'mif', 'sde', '-J', '300', '-s', '1', '-M', '3', '-i', '9', '-r')
    head, rows = _csv(os.path.join(d, 'trace_9.csv'))
    assert len(rows) == 4 and rows[0][-1] == 'nan'
    assert all(np.isfinite(float(r[-1])) for r in rows[1:])
    head, rows = _csv(os.path.join(d, 'mif_9.csv'))
    assert head[:2] == ['index', 'time'] and head[-1] == 'ess'


def _walk(weights, u, anc, x_pred, x0, weigh):
    """sample_traj_and_print (model_builder/C/core/print.c:715-784) on a genealogy: rows in
    print order as (time row, state)."""
    J = len(weights)
    c, j = weights[0], 0
    while c < u and j < J - 1:
        j += 1
        c += weights[j]
    T = anc.shape[0]
    D = [n for n in range(T) if weigh[n]]

    def post(n, jj):
        return (0, x0) if n < 0 else (n + 1, x_pred[n][:, anc[n][jj]])
    rows = [post(T - 1, j)]
    for nn in range(D[-1] - 1, D[-2], -1):
        rows.append(post(nn, j))
    for k in range(len(D) - 2, 0, -1):
        indn = D[k]
        j = anc[indn][j]
        rows.append(post(indn, j))
        for nn in range(indn - 1, D[k - 1], -1):
            rows.append(post(nn, j))
    j = anc[D[0]][j]
    for nn in range(D[0], -2, -1):
        rows.append(post(nn, j))
    return rows


@pytest.mark.parametrize('precision', [64, 32])
def test_sampled_trajectory_follows_the_genealogy(precision):
    from plomgpu.native import Plan
    eng = models.engine('sir')
    p = models.make_problem('sir', J=700, dt=1.0, precision=precision, seed=21)
    plan = Plan(eng, p, traj=True)
    plan.update(p.par_cac, p.par_ts, p.x0, 21)
    plan.launch()
    out = plan.results(ancestors=True, x_pred=True)
    # weights of the last weighted interval, from the engine's own x_pred + the oracle's likelihood
    orc = models.build_oracle('sir')
    weigh = ~np.all(np.isnan(p.data), axis=1)
    last = np.nonzero(weigh)[0][-1]
    ll = np.array([orc.obs_loglik(p, out.x_pred[last][:, j], last) for j in range(p.J)])
    w = np.exp(ll - ll.max())
    fail = np.exp(ll) <= p.like_min ** eng.info.n_ts
    w[fail] = 0.0
    w /= w.sum()
    x0 = p.x0.copy()
    x0[eng.info.off_inc:] = 0.0
    # u away from multiples of 1/J: with equal weights the crossing index would hinge on rounding
    for u in (0.0123, 0.3777, 0.9191):
        rows_t, states = plan.sample_traj(u)
        ref = _walk(w, u, out.ancestors, out.x_pred, x0, weigh)
        assert list(rows_t) == [r[0] for r in ref]
        np.testing.assert_allclose(states, np.array([r[1] for r in ref]), rtol=1e-12)
    plan.close()
