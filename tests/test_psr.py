"""The "psr" implementation (Poisson system with stochastic rates).

CPU: the emitted step against the reference generator's own psr code
(model_builder/Ccoder.py:155-322, recorded in the golden fixture), the
samplers against their distributions, and the oracle filter.  GPU: engine
against oracle with the same Philox draws (FP64), and FP32 statistics.
"""

import math
import re

import numpy as np
import pytest
from scipy import stats

import models


def _emitted_psr(name):
    from plomgpu import build
    path, _ = build.write_header(models.plom_model(name), models.lib_name(name))
    text = open(path).read()
    return text[text.index('static void psr_cac'):text.index('static void step_psr')]


def _norm_ref_update(line, par_sv, remainder):
    # X[ORDER_S*N_CAC+cac] = p_calc->inc[ORDER_S][cac][2] + p_calc->inc[ORDER_U][cac][0];
    lhs, rhs = line.split('=', 1)
    tgt = re.search(r'ORDER_(\w+)\*N_CAC', lhs).group(1)
    terms = []
    for t in re.findall(r'p_calc->inc\[ORDER_(\w+)\]\[cac\]\[(\d+)\]', rhs):
        terms.append((t[0], int(t[1])))
    for t in re.findall(r'X\[ORDER_(\w+)\*N_CAC\+cac\]', rhs):
        terms.append((t, 'x'))
    return tgt, sorted(terms, key=str)


def _norm_mine_update(line, par_sv):
    # x[0*N_CAC+cac] = (T)(inc_S[2] + inc_U[0]);  or  (T)(xo_R + inc_I[0]);
    i = int(re.search(r'x\[(\d+)\*N_CAC\+cac\]', line).group(1))
    rhs = line.split('=', 1)[1]
    terms = []
    for t in re.findall(r'inc_(\w+?)\[(\d+)\]', rhs):
        name = t[0][4:] if t[0].startswith('rem_') else t[0]
        terms.append((name, int(t[1])))
    for t in re.findall(r'\bxo_(\w+)', rhs):
        terms.append((t, 'x'))
    return par_sv[i], sorted(terms, key=str)


@pytest.mark.parametrize('name', ['noise', 'drift', 'sir', 'seir_local'])
def test_psr_structure_matches_reference_generator(name):
    g = models.golden()['models'][name]
    ref = g['psr']
    m = models.plom_model(name)
    code = _emitted_psr(name)
    # multinomial splits: one per compartment with exits, exits + stay categories
    mine_multi = re.findall(r'plomrt::multinomial<(\d+)>\(rs, xs > T\(0\) \? floor\(xs\) : T\(0\), p, inc_(\w+)\)', code)
    assert sorted((s, int(k)) for k, s in mine_multi) == sorted((d['state'], d['nb_exit']) for d in ref['multinomial'])
    # Poisson arrivals: as many as the reference draws, from the same sources
    ref_pois = [re.search(r'inc\[ORDER_(\w+)\]\[cac\]\[(\d+)\]', p_).groups() for p_ in ref['poisson']]
    mine_pois = re.findall(r'inc_(\w+)\[(\d+)\] = plomrt::poisson', code)
    norm = lambda n: n[4:] if n.startswith('rem_') else n
    assert sorted((norm(a), int(b)) for a, b in mine_pois) == sorted((a, int(b)) for a, b in ref_pois)
    # the new contents of every compartment
    ref_upd = dict(_norm_ref_update(l, m.par_sv, m.remainder) for l in ref['update'].strip().splitlines())
    mine_upd = dict(_norm_mine_update(l, m.par_sv) for l in code.splitlines() if re.search(r'x\[\d+\*N_CAC\+cac\] =', l))
    assert mine_upd == ref_upd
    # incidence of the observed flows
    ref_inc = [sorted(re.findall(r'inc\[ORDER_(\w+)\]\[cac\]\[(\d+)\]', d['right_hand_side'])) for d in ref['obs_inc']]
    mine_inc = []
    for o in range(len(ref_inc)):
        mm = re.search(r'if \(o == %d\) inc_acc\.add\(w, (.*)\);' % o, code)
        mine_inc.append(sorted((norm(a), b) for a, b in re.findall(r'inc_(\w+?)\[(\d+)\]', mm.group(1))))
    assert mine_inc == ref_inc


@pytest.mark.parametrize('precision', [64, 32])
@pytest.mark.parametrize('n,p', [(7, 0.3), (40, 0.2), (100, 0.3), (1000, 0.035), (1000, 0.05), (100000, 0.3),
                                 (2_000_000, 0.9), (50, 0.97), (80, 0.5),
                                 (10_000_000, 1e-6), (10_000_000, 2e-6), (8_000_000, 1e-3)])
def test_binomial_sampler(n, p, precision):
    orc = models.build_oracle('sir')
    x = orc.psr_samples('binomial', n, p, seed=n, count=40000, precision=precision)
    assert np.all(x == np.floor(x)) and x.min() >= 0 and x.max() <= n
    mu, var = n * p, n * p * (1 - p)
    assert abs(x.mean() - mu) < 5 * math.sqrt(var / len(x))
    assert abs(x.var() / var - 1.0) < 0.05
    if n <= 1000:
        k = np.arange(n + 1)
        obs = np.bincount(x.astype(int), minlength=n + 1)
        exp = stats.binom.pmf(k, n, p) * len(x)
        keep = exp > 5
        chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
        assert stats.chi2.sf(chi, keep.sum() - 1) > 1e-4


@pytest.mark.parametrize('precision', [64, 32])
@pytest.mark.parametrize('mu', [0.3, 4.0, 9.99, 10.0, 37.5, 39.9, 40.0, 55.0, 2e4, 3e6])
def test_poisson_sampler(mu, precision):
    orc = models.build_oracle('sir')
    x = orc.psr_samples('poisson', mu, seed=int(mu * 100) + 1, count=40000, precision=precision)
    assert np.all(x == np.floor(x)) and x.min() >= 0
    assert abs(x.mean() - mu) < 5 * math.sqrt(mu / len(x))
    assert abs(x.var() / mu - 1.0) < 0.05
    if mu < 100:
        k = np.arange(int(mu * 4 + 20))
        obs = np.bincount(x.astype(int), minlength=len(k))[:len(k)]
        exp = stats.poisson.pmf(k, mu) * len(x)
        keep = exp > 5
        chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
        assert stats.chi2.sf(chi, keep.sum() - 1) > 1e-4


@pytest.mark.parametrize('precision', [64, 32])
@pytest.mark.parametrize('a,theta', [(0.3, 2.0), (1.0, 1.0), (100.0, 0.01), (7.0, 3.0)])
def test_gamma_sampler(a, theta, precision):
    orc = models.build_oracle('sir')
    x = orc.psr_samples('gamma', a, theta, seed=int(a * 10) + 3, count=40000, precision=precision)
    assert x.min() > 0
    ks = stats.kstest(x, stats.gamma(a, scale=theta).cdf)
    assert ks.pvalue > 1e-4


def test_psr_oracle_filter_keeps_integer_states():
    orc = models.build_oracle('sir')
    p = models.make_problem('sir', J=500, dt=1.0, precision=64, seed=3, psr=True, nb_obs=20)
    out = orc.smc(p, x_pred=True)
    assert np.isfinite(out.loglik)
    S = orc.info.n_par_sv * orc.info.n_cac
    xs = out.x_pred[:, :S, :]
    assert np.all(xs == np.floor(xs)) and np.all(xs >= 0)
    # without white noise and with a small step the Euler-multinomial chain's mean path
    # approaches the deterministic skeleton of the same rates (exit probabilities
    # 1 - exp(-r dt) -> r dt)
    q = models.make_problem('sir', J=2000, dt=1.0 / 64, precision=64, seed=3, psr=True, nb_obs=3, noises_off=2,
                            filter=False)
    a = orc.smc(q, x_pred=True).x_pred[:, :S, :].mean(axis=2)
    det = models.make_problem('sir', J=1, dt=1.0, precision=64, seed=3, nb_obs=3, ode=True, filter=False,
                              eps_abs=1e-9, eps_rel=1e-9)
    b = orc.smc(det, x_pred=True).x_pred[:, :S, 0]
    np.testing.assert_allclose(a, b, rtol=0.05)


@pytest.mark.gpu
@pytest.mark.parametrize('name,noises_off', [('sir', 0), ('noise', 0), ('drift', 0), ('noise', 2), ('seir3', 0)])
def test_psr_gpu_matches_oracle(name, noises_off):
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=400, dt=1.0, precision=64, seed=7, psr=True, noises_off=noises_off, nb_obs=25)
    g = eng.smc(p, ancestors=True, x_pred=True)
    o = orc.smc(p, ancestors=True, x_pred=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    np.testing.assert_allclose(g.x_pred, o.x_pred, rtol=1e-9, atol=1e-9)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize('name,J,R', [('sir', 1000, 40), ('seir3', 500, 24)])
def test_psr_gpu_fp32_statistics(name, J, R):
    """FP32 state (single-precision samplers): the psr log-likelihood estimator over replicates has the FP64
    oracle's mean."""
    eng = models.engine(name)
    orc = models.build_oracle(name)
    g = [eng.smc(models.make_problem(name, J=J, dt=1.0, precision=32, seed=100 + r, psr=True)).loglik
         for r in range(R)]
    o = [orc.smc(models.make_problem(name, J=J, dt=1.0, precision=64, seed=500 + r, psr=True)).loglik
         for r in range(R)]
    se = math.sqrt(np.var(g) / R + np.var(o) / R)
    assert abs(np.mean(g) - np.mean(o)) < 4 * se + 0.5
