"""Host side of the command-line drivers (no GPU): option parsing, the
parameter vector, output formats, and the pMCMC logic driven by a stand-in
likelihood."""

import io
import json
import math

import numpy as np
import pytest

import models
from plomgpu import best as best_mod, cli, drivers


def _noise():
    c, p, l, th = models.files('noise')
    from plomgpu.model import PlomModel
    m = PlomModel(c, p, l)
    return m, m.settings(), th


def test_smc_options_match_the_reference():
    a = cli.smc_parser().parse_args(['sde', '-J', '100', '--no_dem_sto', '-y', '-s', '0.5', '-l', '1e-20', '-i', '3',
                                     '-o', '12', '-g', '7', '-t', '-r', '-b', '-e', '-d', '-q', '-P', '--prior'])
    assert a.implementation == 'sde' and a.J == 100 and a.DT == 0.5 and a.LIKE_MIN == 1e-20 and a.id == 3
    assert a.nb_obs == 12 and a.freeze_forcing == 7.0
    assert a.no_filter and a.traj and a.no_trace and a.no_hat and a.no_pred_res and a.quiet and a.pipe and a.prior
    assert cli.noises_off_of(a) == 3
    assert cli.smc_parser().parse_args([]).implementation == 'psr'  # the reference's default
    assert cli.noises_off_of(cli.smc_parser().parse_args(['ode'])) == 7


def test_trace_and_done_formats():
    m, s, th = _noise()
    b = best_mod.Best(m, th)
    head = b.trace_header()
    assert head.startswith('index,') and head.endswith(',log_like\n')
    names = [x.split(':')[0] for x in head.strip().split(',')[1:-1]]
    # par_sv, then par_proc, then par_obs (build_routers order)
    order = m.par_sv + m.par_proc + m.par_obs
    assert [order.index(n) for n in names] == sorted(order.index(n) for n in names)
    row = b.trace_row(0, -123.5)
    vals = row.strip().split(',')
    assert vals[0] == '0' and vals[-1] == '-123.5'
    # the trace shows the guesses (f_inv of the transformed guesses)
    for k, v in zip(b.visible(), vals[1:-1]):
        assert float(v) == pytest.approx(b.entries[k]['guess'], rel=1e-5)
    done = b.theta_with()
    for k in b.visible():
        e = b.entries[k]
        if not e['follower']:
            assert done['parameter'][e['name']]['group'][e['group']]['guess']['value'] == pytest.approx(e['guess'])


def test_priors_known_answers():
    assert best_mod.flat_prior(0.5, 0.0, 2.0) == 0.5
    assert best_mod.flat_prior(2.0, 0.0, 2.0) == 0.0
    assert best_mod.normal_prior(1.0, 0.0, 2.0) == pytest.approx(1.0 / (math.sqrt(2 * math.pi) * 0.5))
    # pseudo-uniform: flat in the middle, continuous at the edges of the ramps
    lo, hi = 0.0, 1.0
    mid = best_mod.pseudo_unif_prior(0.5, lo, hi)
    assert mid == pytest.approx(1.0 / (1.0 - 2.0 / 3.0 * 0.01))
    assert best_mod.pseudo_unif_prior(0.0, lo, hi) == 0.0
    d = 0.01
    assert best_mod.pseudo_unif_prior(lo + d - 1e-12, lo, hi) == pytest.approx(mid, rel=1e-6)


def test_log_prob_prior_counts_estimated_only():
    m, s, th = _noise()
    b = best_mod.Best(m, th, is_bayesian=True)
    lp, err = b.log_prob_prior()
    assert not err
    exp = 0.0
    for k in np.nonzero(b.is_estimated)[0]:
        e = b.entries[k]
        fn = best_mod.PRIORS.get(e['prior'], best_mod.flat_prior)
        exp += math.log(max(fn(e['guess'], e['min'], e['max']), 1e-17))
    assert lp == pytest.approx(exp, rel=1e-9)


def test_f_inv_derivatives():
    # d/dx exp(x), logistic, logit_ab; identity keeps the reference's f_id (returns x)
    assert drivers.f_inv_derivative('log', 0.3, 0, 0) == pytest.approx(math.exp(0.3))
    s = 1.0 / (1.0 + math.exp(-0.7))
    assert drivers.f_inv_derivative('logit', 0.7, 0, 0) == pytest.approx(s * (1 - s))
    assert drivers.f_inv_derivative('logit_ab', -0.2, 1.0, 3.0) == pytest.approx(
        2.0 * math.exp(-0.2) / (1 + math.exp(-0.2)) ** 2)
    assert drivers.f_inv_derivative('identity', 4.0, 0, 0) == 4.0


def test_hat_and_pred_res_formats():
    m, s, th = _noise()
    from plomgpu.problem import Problem
    p = Problem(m, s, th, J=10, dt=1.0, precision=64)
    head = cli.header_hat(m, p)
    cols = head.strip().split(',')
    n_state = len(m.par_sv) * m.N_CAC + (m.N_CAC if m.remainder else 0)
    assert cols[0] == 'time'
    assert len(cols) == 1 + 3 * (n_state + m.N_TS)
    assert cols[1].startswith('low95:') and cols[3].startswith('high95:')
    n_hat = n_state + m.N_TS
    hat = np.arange((p.n_obs + 1) * n_hat * 3, dtype=float).reshape(p.n_obs + 1, n_hat, 3)
    rows = cli.hat_rows(m, p, hat)
    assert len(rows) == p.n_obs + 1
    assert all(len(r.strip().split(',')) == len(cols) for r in rows)
    assert rows[0].startswith('0,0,1,2,')
    pr = np.zeros((p.n_obs, m.N_TS, 2))
    ess = np.ones(p.n_obs)
    rows = cli.pred_res_rows(p, pr, ess)
    n_data = int(np.sum(~np.all(np.isnan(p.data), axis=1)))
    assert len(rows) == n_data
    assert cli.header_pred_res(m).strip().split(',')[-1] == 'ess'


def test_fmt_g_spells_non_finite_like_printf():
    assert best_mod.fmt_g(float('nan')) == 'nan'
    assert best_mod.fmt_g(float('inf')) == 'inf'
    assert best_mod.fmt_g(1e-17) == '1e-17'
    assert best_mod.fmt_g(123456789.0) == '1.23457e+08'


class _FakePlan(object):
    """Stand-in filter: the log-likelihood of a Gaussian centred on a target vector."""

    def __init__(self, engine, problem, traj=False):
        self.problem = problem
        self.calls = 0

    def update(self, par_cac, par_ts, x0, seed):
        self.par = np.concatenate([np.ravel(par_cac), np.ravel(par_ts)])

    def update_drift(self, v):
        pass

    def launch(self):
        self.calls += 1

    def results(self):
        class R(object):
            pass
        r = R()
        r.loglik = -0.5 * float(np.sum(((self.par - self.target) / self.scale) ** 2))
        return r

    def close(self):
        pass


def test_pmcmc_chain_logic_with_stand_in_likelihood(tmp_path):
    """Sequential and full updates: the chain moves, accepts at a sane rate, writes trace,
    acceptance and covariance files in the reference's layout."""
    m, s, th = _noise()
    for full in (False, True):
        args = drivers.pmcmc_parser().parse_args(
            ['sde', '-M', '60', '-J', '10', '-n', '0', '-q', '--acc', '-p', str(tmp_path) + '/', '-i', '1']
            + (['--full'] if full else []))
        plans = []

        def factory(engine, problem, traj=False):
            pl = _FakePlan(engine, problem, traj)
            pl.target = np.concatenate([np.ravel(problem.par_cac), np.ravel(problem.par_ts)]) * 1.05
            pl.scale = np.maximum(np.abs(pl.target) * 0.1, 1e-6)
            plans.append(pl)
            return pl

        chain = drivers.Pmcmc(None, m, s, th, args, plan_factory=factory)
        chain.run()
        assert plans[0].calls == 60
        trace = open(str(tmp_path) + '/trace_1.csv').read().splitlines()
        assert trace[0] == chain.best.trace_header().strip()
        ne = len(chain.best.to_be_estimated)
        n_rows = 1 + (59 if full else 59 // ne)
        assert len(trace) == 1 + n_rows
        acc = open(str(tmp_path) + '/acc_1.csv').read().splitlines()
        assert acc[0].startswith('index,epsilon,global_ar')
        assert 0.0 < chain.state.global_acceptance_rate < 1.0
        cov = open(str(tmp_path) + '/covariance_1.csv').read().splitlines()
        assert len(cov) == 1 + len(chain.best.visible())
        assert np.all(np.diag(chain.var_sampling) >= 0.0)


def test_model_directory_and_cli_reach_the_engine(tmp_path, capsys):
    """pmbuilder writes the model directory; smc parses theta, opens its outputs and fails
    loudly at the engine when no GPU is present (no CPU fallback)."""
    from plomgpu import build
    c, p, l, th = models.files('noise')
    d = str(tmp_path / 'model')
    build.build_model_dir(c, p, l, d, name='noise', shared_lib=True)
    man = json.load(open(d + '/.plomgpu.json'))
    assert man['name'] == 'noise'
    assert json.load(open(d + '/.settings.json'))['orders']['par_sv']
    import os
    assert os.access(d + '/smc', os.X_OK)
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    rc = cli.main(['smc', 'sde', '-J', '50', '-q'])
    assert rc == 1  # no model directory in the cwd
    cwd = os.getcwd()
    os.chdir(d)
    try:
        old = cli.sys.stdin
        cli.sys.stdin = io.StringIO(json.dumps(th) + '\n')
        try:
            rc = cli.main(['smc', 'sde', '-J', '50', '-q'])
        finally:
            cli.sys.stdin = old
    finally:
        os.chdir(cwd)
    assert rc == 1
    assert 'no CUDA device' in capsys.readouterr().err


def test_mif_components_fixed_lag_tables():
    """Initial conditions and drift start values become fixed-lag components placed on their
    state words; a drifted parameter is not a random-walk component; volatilities map to the
    drift groups."""
    import numpy as np
    import models
    from plomgpu import mif
    p = models.make_problem('drift', J=8, dt=1.0)
    m = p.model
    comp = mif.components(p, names=['S', 'I', 'r0', 'vol'])
    kinds = sorted(set((c['name'], c['kind']) for c in comp))
    assert kinds == [('I', 'sv'), ('S', 'sv'), ('r0', 'drift'), ('vol', 'proc')]
    slots = mif.x0_slots(m, comp)
    assert len(slots) == len(m.par_sv) * m.N_CAC + len(m.drift_par_proc) * m.N_CAC
    for q, c in enumerate(comp):
        if c['kind'] == 'sv':
            for cac in c['members']:
                assert slots[m.par_sv.index(c['name']) * m.N_CAC + cac] == q
        if c['kind'] == 'drift':
            assert slots[len(m.par_sv) * m.N_CAC + c['g']] == q
    assert np.all(slots >= 0)
    vol = mif.vol_slots(p, comp)
    qv = [q for q, c in enumerate(comp) if c['name'] == 'vol']
    assert set(vol[0][:p.params.routers['r0'].n_gp].tolist()) <= set(qv)
