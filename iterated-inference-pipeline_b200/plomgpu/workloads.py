"""Seeded synthetic workloads in plom's JSON model format.

* ``sir`` -- one population SIR diffusion: N = 1e6 (constant covariate),
  no remainder, R0 = 2.5, recovery 1/(5 days), births = deaths = 1/(50 yr),
  environmental noise sd 0.1 on transmission, weekly incidence of I -> R
  reported with rho = 0.6, overdispersion phi = 0.1; dt = 1 day, 52 weeks.
  Initial state S0 = N/R0, I0 = 1e-4 N, R0 = rest.
* ``seir20x2`` -- SEIR with 20 populations x 2 age classes, seasonal forcing
  beta(t) = beta0 (1 + 0.3 cos(2 pi t / 364)) (t in days, 52-week period),
  N_c ~ LogUniform(1e5, 1e7), force of infection mixed across populations
  (gravity kernel, coupling 1e-3) and age classes, 520 weekly observations,
  one incidence series per population (both age classes).

Observations are drawn from the discretised normal observation model along
one simulated path (Euler-Maruyama with demographic and environmental
noise, numpy Philox generator seeded per workload).  The simulator evaluates
the same rate expressions through sympy.
"""

import copy
import datetime
import math

import numpy as np
import sympy

from .model import PlomModel, tokenize, UNIVERSE
from .problem import Problem, substep_times, round_dt

T0 = datetime.date(2000, 1, 1)


def _date(days):
    return str(T0 + datetime.timedelta(days=int(days)))


def _context(pops, series, n_obs, metadata, coupling=None, period=7):
    ctx = {'name': 'synthetic', 'description': 'seeded synthetic workload',
           'population': [{'id': p} for p in pops],
           'time_series': [{'id': ts, 'population_id': pids} for ts, pids in series],
           'data': {'source': {}},
           'metadata': metadata}
    for ts, _ in series:
        ctx['data']['source'][ts] = {'t0': _date(0),
                                     'value': [[_date((k + 1) * period), None] for k in range(n_obs)]}
    if coupling is not None:
        ctx['coupling'] = coupling
    return ctx


def _const_meta(mid, ids, values, n_days):
    return {'id': mid, 'source': dict((i, {'value': [[_date(0), float(v)], [_date(n_days), float(v)]]})
                                      for i, v in zip(ids, values))}


def _obs_link(series_ids, inc_def):
    return {'name': 'discretized normal reporting',
            'observed': [{'id': 'inc', 'definition': inc_def, 'time_series_id': series_ids,
                          'observation_id': 'common'}],
            'observation': [{'id': 'common',
                             'parameter': [{'id': 'rep'}, {'id': 'phi'}, {'id': 'prop'}],
                             'model': {'distribution': 'discretized_normal',
                                       'mean': 'rep*prop*x',
                                       'var': 'rep*(1.0-rep)*prop*x + (rep*phi*prop*x)**2'}}]}


def _fixed(v, transformation='log', **kw):
    d = {'partition_id': 'identical_population', 'transformation': transformation,
         'min': v, 'guess': v, 'max': v, 'sd_transf': 0.0}
    d.update(kw)
    return d


def sir(n_obs=52, N=1e6, r0=2.5):
    """cfg0 model files (data filled by :func:`with_data`)."""
    pops = ['city1__all']
    series = [('city1__CDC__inc', pops)]
    process = {
        'name': 'SIR', 'description': 'SIR with births and deaths, white noise on transmission',
        'state': [{'id': 'S'}, {'id': 'I'}, {'id': 'R'}],
        'parameter': [{'id': 'r0'}, {'id': 'v'}, {'id': 'sto'}, {'id': 'mu_b'}, {'id': 'mu_d'}],
        'model': [
            {'from': 'U', 'to': 'S', 'rate': 'mu_b*N'},
            {'from': 'S', 'to': 'I', 'rate': 'r0/N*v*I'},
            {'from': 'I', 'to': 'R', 'rate': 'correct_rate(v)'},
            {'from': 'S', 'to': 'U', 'rate': 'mu_d'},
            {'from': 'I', 'to': 'U', 'rate': 'mu_d'},
            {'from': 'R', 'to': 'U', 'rate': 'mu_d'}],
        'white_noise': [{'reaction': [{'from': 'S', 'to': 'I'}], 'sd': 'sto'}]}
    link = _obs_link(['city1__CDC__inc'], [{'from': 'I', 'to': 'R'}])
    days = 7 * (n_obs + 1)
    ctx = _context(pops, series, n_obs, [_const_meta('N', pops, [N], days),
                                         _const_meta('prop', ['city1__CDC__inc'], [1.0], days)])
    S0 = 1.0 / r0
    I0 = 1e-4
    theta = {'name': 'sir', 'parameter': {
        'S': _fixed(S0, 'logit'), 'I': _fixed(I0, 'logit'), 'R': _fixed(1.0 - S0 - I0, 'logit'),
        'r0': _fixed(r0), 'v': _fixed(5.0, unit='D', type='rate_as_duration'), 'sto': _fixed(0.1),
        'mu_b': _fixed(0.02, unit='Y'), 'mu_d': _fixed(0.02, unit='Y'),
        'rep': dict(_fixed(0.6, 'logit'), partition_id='identical_time_series'),
        'phi': dict(_fixed(0.1), partition_id='identical_time_series')}}
    return ctx, process, link, theta


def gravity_coupling(n_pop, sizes, g, rng, age_mix):
    """Row-stochastic-like cac x cac mixing: (1-g) within population + g x gravity, times age mixing."""
    xy = rng.uniform(0.0, 1.0, size=(n_pop, 2))
    K = np.zeros((n_pop, n_pop))
    for a in range(n_pop):
        for b in range(n_pop):
            if a != b:
                d2 = float(np.sum((xy[a] - xy[b]) ** 2)) + 1e-3
                K[a, b] = math.sqrt(sizes[a] * sizes[b]) / d2
        K[a] /= K[a].sum()
    G = (1.0 - g) * np.eye(n_pop) + g * K
    nac = len(age_mix)
    W = np.zeros((n_pop * nac, n_pop * nac))
    for c in range(n_pop):
        for a in range(nac):
            for c2 in range(n_pop):
                for a2 in range(nac):
                    W[c * nac + a, c2 * nac + a2] = G[c, c2] * age_mix[a][a2]
    return W


def seir20x2(n_obs=520, n_pop=20, r0=2.5, seed=1, coupling=1e-3):
    """cfg1 model files (data filled by :func:`with_data`)."""
    rng = np.random.Generator(np.random.Philox(seed))
    sizes = np.exp(rng.uniform(math.log(1e5), math.log(1e7), size=n_pop))
    ages = ['young', 'old']
    age_frac = [0.25, 0.75]
    pops = ['pop%02d__%s' % (c, a) for c in range(n_pop) for a in ages]
    series = [('pop%02d__CDC__inc' % c, ['pop%02d__%s' % (c, a) for a in ages]) for c in range(n_pop)]
    age_mix = [[1.2, 0.4], [0.4, 0.8]]
    W = gravity_coupling(n_pop, sizes, coupling, rng, age_mix)
    process = {
        'name': 'SEIR20x2', 'description': 'SEIR, 20 populations x 2 age classes, seasonal forcing, gravity coupling',
        'state': [{'id': 'S'}, {'id': 'E'}, {'id': 'I'}, {'id': 'R'}],
        'parameter': [{'id': 'r0'}, {'id': 'v'}, {'id': 'eps'}, {'id': 'sto'}, {'id': 'mu_b'}, {'id': 'mu_d'}],
        'model': [
            {'from': 'U', 'to': 'S', 'rate': 'mu_b*N'},
            {'from': 'S', 'to': 'E', 'rate': 'r0*v*(1+0.3*cos(2*pi*t/364))*foi(I)'},
            {'from': 'E', 'to': 'I', 'rate': 'eps'},
            {'from': 'I', 'to': 'R', 'rate': 'v'},
            {'from': 'S', 'to': 'U', 'rate': 'mu_d'},
            {'from': 'E', 'to': 'U', 'rate': 'mu_d'},
            {'from': 'I', 'to': 'U', 'rate': 'mu_d'},
            {'from': 'R', 'to': 'U', 'rate': 'mu_d'}],
        'white_noise': [{'reaction': [{'from': 'S', 'to': 'E'}], 'sd': 'sto'}]}
    sids = [s for s, _ in series]
    link = _obs_link(sids, [{'from': 'I', 'to': 'R'}])
    days = 7 * (n_obs + 1)
    Ncac = [sizes[c] * age_frac[a] for c in range(n_pop) for a in range(len(ages))]
    ctx = _context(pops, series, n_obs, [_const_meta('N', pops, Ncac, days),
                                         _const_meta('prop', sids, [1.0] * len(sids), days)],
                   coupling=W.tolist())
    S0, E0, I0 = 1.0 / r0, 5e-5, 1e-4
    theta = {'name': 'seir20x2', 'parameter': {
        'S': _fixed(S0, 'logit'), 'E': _fixed(E0, 'logit'), 'I': _fixed(I0, 'logit'),
        'R': _fixed(1.0 - S0 - E0 - I0, 'logit'),
        'r0': _fixed(r0), 'v': _fixed(5.0, unit='D', type='rate_as_duration'),
        'eps': _fixed(8.0, unit='D', type='rate_as_duration'), 'sto': _fixed(0.1),
        'mu_b': _fixed(0.02, unit='Y'), 'mu_d': _fixed(0.02, unit='Y'),
        'rep': dict(_fixed(0.6, 'logit'), partition_id='identical_time_series'),
        'phi': dict(_fixed(0.1), partition_id='identical_time_series')}}
    return ctx, process, link, theta


# ---------------------------------------------------------------- simulation
def _rate_functions(model):
    names = model.par_sv + model.par_proc + [p for p in model.par_fixed] + ['t']
    syms = dict((n, sympy.Symbol('plom___' + n)) for n in names)
    funcs = []
    for r in model.proc_model:
        toks = tokenize(r['rate'])
        out = []
        i = 0
        while i < len(toks):
            t = toks[i]
            if t == 'correct_rate':
                i += 1
                continue
            if t == 'foi':
                out.append('plom___foi_' + toks[i + 2])
                i += 4
                continue
            out.append('plom___' + t if t in syms else t)
            i += 1
        expr = sympy.sympify(''.join(out), locals=dict(
            [('plom___' + n, s) for n, s in syms.items()] +
            [('plom___foi_' + s, sympy.Symbol('plom___foi_' + s)) for s in model.par_sv]))
        args = [syms[n] for n in names] + [sympy.Symbol('plom___foi_' + s) for s in model.par_sv]
        funcs.append(sympy.lambdify(args, expr, 'numpy'))
    return names, funcs


def simulate_path(problem, rng):
    """One Euler-Maruyama path (full noise) of the problem's model; returns weekly incidence [n_obs][N_TS_INC_UNIQUE]."""
    m = problem.model
    names, funcs = _rate_functions(m)
    nsv = len(m.par_sv)
    X = problem.x0[:nsv * m.N_CAC].reshape(nsv, m.N_CAC).copy()
    par = dict((p, problem.par_cac[k]) for k, p in enumerate(m.par_proc))
    cov_names = [p for p in m.par_fixed if p not in m.par_fixed_obs]
    W = problem.coupling
    univ = (UNIVERSE, m.remainder)
    inc_cacs = []
    for o in range(m.N_OBS_INC):
        info = m.obs2ts[o]
        for u in range(info['n_ts_unique']):
            inc_cacs.append((o, [c * m.N_AC + a for (c, a) in info['cac'][u]]))
    inc_reac = []
    for defs in m.obs_var_def:
        if isinstance(defs[0], dict):
            inc_reac.append([i for i, r in enumerate(m.proc_model) for d in defs
                             if r['from'] == d['from'] and r['to'] == d['to'] and r['rate'] == d['rate']])
    dt = problem.dt
    out = np.zeros((problem.n_obs, len(inc_cacs)))
    sub = 0
    for n in range(problem.n_obs):
        inc = np.zeros(len(inc_cacs))
        for k in range(int(problem.n_sub[n])):
            t = problem.t_sub[sub]
            cov = problem.cov_cac[sub]
            sub += 1
            env = {}
            for i, s in enumerate(m.par_sv):
                env[s] = X[i]
            for p in m.par_proc:
                env[p] = par[p]
            for kk, p in enumerate(cov_names):
                env[p] = cov[kk]
            env['t'] = t
            npop = X.sum(axis=0) if m.remainder is None else env.get('N')
            foi = {}
            for i, s in enumerate(m.par_sv):
                foi[s] = (W @ (X[i] / npop)) if W is not None else np.zeros(m.N_CAC)
            args = [env.get(nm, 0.0) for nm in names] + [foi[s] for s in m.par_sv]
            flows = []
            for ri, r in enumerate(m.proc_model):
                rate = np.broadcast_to(np.asarray(funcs[ri](*args), dtype=float), (m.N_CAC,))
                base = rate if r['from'] in univ else rate * X[m.par_sv.index(r['from'])]
                base = np.maximum(base, 0.0)
                f = base * dt + np.sqrt(base * dt) * rng.standard_normal(m.N_CAC)
                if 'white_noise' in r:
                    sd = par[r['white_noise']['sd']]
                    f = f + base * sd * math.sqrt(dt) * rng.standard_normal(m.N_CAC)
                flows.append(f)
            newX = X.copy()
            for ri, r in enumerate(m.proc_model):
                if r['from'] not in univ:
                    newX[m.par_sv.index(r['from'])] -= flows[ri]
                if r['to'] not in univ:
                    newX[m.par_sv.index(r['to'])] += flows[ri]
            for w, (o, cacs) in enumerate(inc_cacs):
                inc[w] = max(inc[w] + sum(flows[ri][cacs].sum() for ri in inc_reac[o]), 0.0)
            X = np.maximum(newX, 0.0)
        out[n] = inc
    return out


def draw_observations(problem, inc, rng):
    """Discretised-normal draws around rho*prop*x, rounded, >= 0 (the reference's observation())."""
    m = problem.model
    ts_word = []
    w = 0
    for o in range(m.N_OBS_INC):
        info = m.obs2ts[o]
        for u in range(info['n_ts_unique']):
            ts_word.extend([w] * info['n_stream'][u])
            w += 1
    rep = problem.par_ts[m.par_obs.index('rep')]
    phi = problem.par_ts[m.par_obs.index('phi')]
    y = np.zeros((problem.n_obs, m.N_TS))
    for n in range(problem.n_obs):
        for ts in range(m.N_TS):
            x = inc[n, ts_word[ts]]
            mu = rep[ts] * x
            var = rep[ts] * (1.0 - rep[ts]) * x + (rep[ts] * phi[ts] * x) ** 2
            v = mu + math.sqrt(max(var, 0.0)) * rng.standard_normal()
            y[n, ts] = float(max(round(v), 0.0))
    return y


def with_data(files, seed=0, dt=1.0):
    """Simulates one path and writes its observations into the context's data."""
    ctx, process, link, theta = files
    m = PlomModel(ctx, process, link)
    prob = Problem(m, m.settings(), theta, J=1, dt=dt)
    rng = np.random.Generator(np.random.Philox(seed))
    inc = simulate_path(prob, rng)
    y = draw_observations(prob, inc, rng)
    # write back in the context's own series order
    for k, ts in enumerate(m.ts_id):
        vals = ctx['data']['source'][ts]['value']
        for n in range(len(vals)):
            vals[n][1] = y[n, k]
    return ctx, process, link, theta


def load(name, n_obs=None):
    """(context, process, link, theta) of a named workload with data."""
    if name == 'sir':
        return with_data(sir(n_obs=n_obs or 52), seed=0)
    if name == 'seir20x2':
        return with_data(seir20x2(n_obs=n_obs or 520), seed=0)
    raise KeyError(name)


# ---------------------------------------------------------------- batches of parameter sets
def simulate_paths(problem, par_cac, x0, rng):
    """Euler-Maruyama paths of many parameter sets at once.

    par_cac: [n][N_PAR_PROC][N_CAC], x0: [n][S]; returns incidence [n][n_obs][words].
    """
    m = problem.model
    names, funcs = _rate_functions(m)
    n = par_cac.shape[0]
    nsv = len(m.par_sv)
    X = np.array([x0[i][:nsv * m.N_CAC].reshape(nsv, m.N_CAC) for i in range(n)]).transpose(1, 0, 2)  # [sv][n][cac]
    par = dict((p, par_cac[:, k, :]) for k, p in enumerate(m.par_proc))
    cov_names = [p for p in m.par_fixed if p not in m.par_fixed_obs]
    W = problem.coupling
    univ = (UNIVERSE, m.remainder)
    words = []
    for o in range(m.N_OBS_INC):
        info = m.obs2ts[o]
        for u in range(info['n_ts_unique']):
            words.append((o, [c * m.N_AC + a for (c, a) in info['cac'][u]]))
    inc_reac = []
    for defs in m.obs_var_def:
        if isinstance(defs[0], dict):
            inc_reac.append([i for i, r in enumerate(m.proc_model) for d in defs
                             if r['from'] == d['from'] and r['to'] == d['to'] and r['rate'] == d['rate']])
    dt = problem.dt
    out = np.zeros((n, problem.n_obs, len(words)))
    sub = 0
    for k_obs in range(problem.n_obs):
        inc = np.zeros((n, len(words)))
        for _k in range(int(problem.n_sub[k_obs])):
            t = problem.t_sub[sub]
            cov = problem.cov_cac[sub]
            sub += 1
            env = {'t': t}
            for i, s in enumerate(m.par_sv):
                env[s] = X[i]
            env.update(par)
            for kk, p in enumerate(cov_names):
                env[p] = np.broadcast_to(cov[kk], (n, m.N_CAC))
            npop = X.sum(axis=0) if m.remainder is None else env['N']
            foi = {}
            for i, s in enumerate(m.par_sv):
                foi[s] = (X[i] / npop) @ W.T if W is not None else np.zeros((n, m.N_CAC))
            args = [env.get(nm, 0.0) for nm in names] + [foi[s] for s in m.par_sv]
            flows = []
            for ri, r in enumerate(m.proc_model):
                rate = np.broadcast_to(np.asarray(funcs[ri](*args), dtype=float), (n, m.N_CAC))
                base = rate if r['from'] in univ else rate * X[m.par_sv.index(r['from'])]
                base = np.maximum(base, 0.0)
                f = base * dt + np.sqrt(base * dt) * rng.standard_normal((n, m.N_CAC))
                if 'white_noise' in r:
                    sd = par[r['white_noise']['sd']]
                    f = f + base * sd * math.sqrt(dt) * rng.standard_normal((n, m.N_CAC))
                flows.append(f)
            newX = X.copy()
            for ri, r in enumerate(m.proc_model):
                if r['from'] not in univ:
                    newX[m.par_sv.index(r['from'])] -= flows[ri]
                if r['to'] not in univ:
                    newX[m.par_sv.index(r['to'])] += flows[ri]
            for w, (o, cacs) in enumerate(words):
                inc[:, w] = np.maximum(inc[:, w] + sum(flows[ri][:, cacs].sum(axis=1) for ri in inc_reac[o]), 0.0)
            X = np.maximum(newX, 0.0)
        out[:, k_obs] = inc
    return out


def sir_batch(n_sets=4096, seed=2, J_range=(256, 16384), T_range=(52, 520), sd=0.1):
    """cfg2: parameter sets of the SIR workload around its values (relative sd 0.1),
    uneven particle counts and series lengths, data simulated under each set.

    Returns (base Problem with the longest time grid, thetas, J, T, data, seeds)."""
    from .batch import BatchProblem
    rng = np.random.Generator(np.random.Philox(seed))
    files = sir(n_obs=T_range[1])
    ctx, process, link, theta0 = files
    base_model = PlomModel(ctx, process, link)
    base = Problem(base_model, base_model.settings(), theta0, J=1, dt=1.0)
    thetas = []
    keys = ['r0', 'v', 'sto', 'mu_b', 'mu_d', 'rep', 'phi']
    for i in range(n_sets):
        th = copy.deepcopy(theta0)
        for k in keys:
            p = th['parameter'][k]
            v = p['guess'] * (1.0 + sd * rng.standard_normal())
            if k == 'rep':
                v = min(max(v, 0.05), 0.95)
            v = max(v, 1e-3 * p['guess'])
            p['guess'] = p['min'] = p['max'] = v
        r0 = th['parameter']['r0']['guess']
        S0, I0 = 1.0 / r0, 1e-4
        for s, val in (('S', S0), ('I', I0), ('R', 1.0 - S0 - I0)):
            q = th['parameter'][s]
            q['guess'] = q['min'] = q['max'] = val
        thetas.append(th)
    J = rng.integers(J_range[0], J_range[1] + 1, size=n_sets)
    T = rng.integers(T_range[0], T_range[1] + 1, size=n_sets)
    from .theta import Parameters
    pc = np.array([Parameters(base_model, th).par_cac() for th in thetas])
    pt = np.array([Parameters(base_model, th).par_ts() for th in thetas])
    x0 = np.array([Parameters(base_model, th).x0(base.pop_size_t0) for th in thetas])
    inc = simulate_paths(base, pc, x0, rng)
    m = base_model
    data = []
    for i in range(n_sets):
        y = np.zeros((int(T[i]), m.N_TS))
        rep = pt[i][m.par_obs.index('rep')]
        phi = pt[i][m.par_obs.index('phi')]
        for n in range(int(T[i])):
            for ts in range(m.N_TS):
                x = inc[i, n, 0]
                mu = rep[ts] * x
                var = rep[ts] * (1.0 - rep[ts]) * x + (rep[ts] * phi[ts] * x) ** 2
                y[n, ts] = float(max(round(mu + math.sqrt(max(var, 0.0)) * rng.standard_normal()), 0.0))
        data.append(y)
    seeds = np.arange(n_sets, dtype=np.uint64) * 7919 + 17
    return BatchProblem(base, thetas, J, T, data, seeds)
