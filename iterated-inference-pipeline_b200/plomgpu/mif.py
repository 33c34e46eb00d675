"""Iterated filtering (MIF, Ionides et al. 2006) driven from the host.

The per-iteration work (proposal, filtering with per-particle parameters,
filtered moments, resampling + random walk) runs on the GPU for all runs at
once (plomgpu_mif_*).  This module restates the host part of the reference's
``mif`` binary:

* perturbation variances: sd_transf squared and rescaled by 1/nb_obs
  (rescale_covariance_mif, model_builder/C/mif/methods.c:28-72);
* cooling FREEZE = a^(m-1) (model_builder/C/mif/mif.h:25), initial proposal
  sd b * FREEZE * sqrt(var) (mif.c:119-121), random-walk sd
  FREEZE * sqrt(delta_t) * sqrt(var) where delta_t accumulates the time since
  the previous observation with data (mif.c:138-191);
* the theta-hat update: the mean of the filtered means for the first
  ``switch`` iterations (update_theta_best_stable_mif, methods.c:394-420),
  then the Ionides 2006 formula (update_theta_best_king_mif, methods.c:429-467).

* initial conditions and the start values of drifted parameters are fitted
  by fixed-lag smoothing: proposed with the others at the start of an
  iteration, resampled but never perturbed, and set at interval L to the
  weighted mean of the resampled components (resample_and_mut_theta_mif,
  update_fixed_lag_smoothing, methods.c:261-392); their proposal variance is
  sd_transf squared, not rescaled (rescale_covariance_mif rescales the
  random-walk block only);
* with ``prior`` the weights are multiplied by prior^(1/nb_obs) for the
  random-walk components and prior^(1/L) for the fixed-lag ones while n < L
  (patch_likelihood_prior, methods.c:469-520), and the transformations of the
  bounded parameters are those of the Bayesian routers (build.c: the
  uniform priors map to logit_ab).

A parameter fitted per group contributes one component per group (the
populations or series of the group read it).
"""

import math

import numpy as np

from .native import MifDescHolder, MifPlan


class MifError(Exception):
    pass


FLS_KINDS = ('sv', 'drift')


def components(problem, names=None, params=None):
    """theta components: one per group of every estimated (sd_transf > 0 in some group) parameter:
    process and observation parameters fitted by the random walk ('proc', 'obs'; drifted
    parameters excluded, as p_it_par_proc_par_obs_no_drift), initial conditions ('sv') and
    drift start values ('drift') fitted by fixed-lag smoothing (p_it_par_sv_and_drift)."""
    m = problem.model
    params = params or problem.params
    drifted = set(m.drift_par_proc)
    out = []
    lists = (('proc', [x for x in m.par_proc if x not in drifted], m.par_proc), ('obs', m.par_obs, m.par_obs),
             ('sv', m.par_sv, m.par_sv), ('drift', m.drift_par_proc, m.drift_par_proc))
    for kind, plist, index_list in lists:
        for name in plist:
            idx = index_list.index(name)
            r = params.routers[name]
            if names is not None and name not in names:
                continue
            sds = _sd_transf(problem, name, r)
            if names is None and not max(sds) > 0.0:
                continue
            for g in range(r.n_gp):
                members = None if (r.n_gp == 1 and kind in ('proc', 'obs')) else \
                    [c for c in range(len(r.map)) if r.map[c] == g]
                out.append({'name': name, 'kind': kind, 'index': idx, 'g': g, 'bt': r.bt(g), 'sd_transf': sds[g],
                            'theta0': r.transformed_guess(g), 'members': members, 'router': r,
                            'fls': kind in FLS_KINDS})
    if not out:
        raise MifError('no parameter to fit (sd_transf > 0)')
    if len(out) > 16:
        raise MifError('%d components to fit; the engine takes at most 16' % len(out))
    return out


def _sd_transf(problem, name, router):
    from .theta import adapt_theta
    th = adapt_theta(problem.theta, problem.model)
    par = th['parameter'][name]
    if 'follow' in par:
        par = th['parameter'][par['follow']]
    g = par['group']
    return [float(g[gid].get('sd_transf', {}).get('value', 0.0)) for gid in router.group_name]


PRIOR_KINDS = {'normal': 1, 'pseudo_uniform': 2}


def x0_slots(m, comp):
    """[off_inc] component of every initial state word (-1: the problem's x0): compartment s of
    every cac of group g for an 'sv' component, drift word g of the parameter for a 'drift' one
    (the words the reference loads from theta, prop2Xpop_size / theta_driftIC2Xdrift)."""
    off_inc = len(m.par_sv) * m.N_CAC + len(m.drift_par_proc) * m.N_CAC
    x0_slot = np.full(off_inc, -1, dtype=np.int32)
    for q, c in enumerate(comp):
        if c['kind'] == 'sv':
            for cac in c['members']:
                x0_slot[c['index'] * m.N_CAC + cac] = q
        elif c['kind'] == 'drift':
            x0_slot[len(m.par_sv) * m.N_CAC + c['index'] * m.N_CAC + c['g']] = q
    return x0_slot


def vol_slots(problem, comp):
    """[n_drift][n_cac] component of the volatility of drift i, group g (-1: the problem's table);
    the volatility of group g is the volatility parameter's group min(g, n_groups - 1), as the
    drift tables index it."""
    m = problem.model
    vol = np.full((len(m.drift_par_proc), m.N_CAC), -1, dtype=np.int32)
    for i, (dp, vp) in enumerate(zip(m.drift_par_proc, m.vol_par_proc)):
        n_gp = problem.params.routers[dp].n_gp
        for q, c in enumerate(comp):
            if c['kind'] == 'proc' and c['name'] == vp:
                n_gp_v = c['router'].n_gp
                for g in range(n_gp):
                    if min(g, n_gp_v - 1) == c['g']:
                        vol[i, g] = q
    return vol


class Mif(object):
    """``lag``: L, the interval of the fixed-lag means (default floor(0.75 n_data), as mif -L 0.75);
    ``prior``: the --prior patch (a Best of the theta gives the priors)."""

    def __init__(self, engine, problem, n_runs=1, names=None, a=0.975, b=2.0, switch=5, sd_transf=None,
                 precision=None, lag=None, prior=None):
        self.problem = problem
        m = problem.model
        params = None
        if prior is not None:
            from .theta import Parameters
            params = Parameters(m, problem.theta, is_bayesian=True)
        self.comp = components(problem, names, params)
        if sd_transf is not None:
            for c in self.comp:
                c['sd_transf'] = float(sd_transf.get(c['name'], c['sd_transf'])) if isinstance(sd_transf, dict) \
                    else float(sd_transf)
        self.R = int(n_runs)
        self.Q = len(self.comp)
        self.a, self.b, self.switch = float(a), float(b), int(switch)
        n_data = problem.n_obs
        self.lag = int(math.floor(0.75 * n_data)) if lag is None else int(lag)
        if self.lag < 0 or self.lag > n_data:
            raise MifError('L > N_DATA (%d > %d). Please choose a L <= %d' % (self.lag, n_data, n_data))
        rw = [c for c in self.comp if not c['fls']]
        self.holder = MifDescHolder(self.R, [(c['kind'], c['index'], c['bt'], c['sd_transf'] > 0, c['members'])
                                             for c in rw] +
                                    [('fls', 0, c['bt'], c['sd_transf'] > 0, None) for c in self.comp if c['fls']],
                                    len(m.par_proc), len(m.par_obs), m.N_CAC, m.N_TS)
        # components in the order of the holder: random-walk first, then fixed-lag
        self.comp = rw + [c for c in self.comp if c['fls']]
        self.fls = np.array([1 if c['fls'] else 0 for c in self.comp], dtype=np.int32)
        self.holder.set_fixed_lag(self.fls, x0_slots(m, self.comp), problem.pop_size_t0, self.lag)
        if m.drift_par_proc:
            self.holder.set_vol_slot(vol_slots(problem, self.comp))
        if prior is not None:
            kinds, lo, hi, finv = [], [], [], []
            index = dict(((e['name'], e['g']), e) for e in prior.entries)
            for c in self.comp:
                e = index[(c['name'], c['g'])]
                r = c['router']
                kinds.append(PRIOR_KINDS.get(e['prior'], 0))
                lo.append(e['min'])
                hi.append(e['max'])
                finv.append((r._finv_code(c['g']), 0, 0, r.min[c['g']], r.max[c['g']], 1.0))
            self.holder.set_prior(kinds, lo, hi, finv, self.lag)
        self.plan = MifPlan(engine, problem, self.holder, precision=precision)
        # random-walk components: sd_transf^2 / nb_obs (rescale_covariance_mif); fixed-lag: sd_transf^2
        self.var = np.array([c['sd_transf'] ** 2 / (1.0 if c['fls'] else n_data) for c in self.comp])
        self.theta_hat = np.tile(np.array([c['theta0'] for c in self.comp]), (self.R, 1))
        # delta_t of every interval: time since the previous interval with data
        has = ~np.all(np.isnan(problem.data), axis=1) if problem.filter else np.zeros(problem.n_obs, bool)
        t_prev = np.concatenate([[0.0], problem.t_obs[:-1]])
        lengths = problem.t_obs - t_prev
        self.delta_t = np.zeros(problem.n_obs)
        acc = 0.0
        for n in range(problem.n_obs):
            acc += lengths[n]
            self.delta_t[n] = acc
            if has[n]:
                acc = 0.0
        self.has_data = has
        self.t0 = 0.0

    def schedules(self, m):
        freeze = self.a ** (m - 1)
        sd_init = self.b * freeze * np.sqrt(self.var)
        sd_mut = freeze * np.sqrt(self.delta_t)[:, None] * np.sqrt(self.var)[None, :]
        vt_add = self.delta_t[:, None] * freeze ** 2 * self.var[None, :]
        return freeze, sd_init, sd_mut, vt_add

    def update(self, m, bart, vt, fls_means=None):
        """theta-hat update of every run: the random-walk components from the filtered means /
        variances, the fixed-lag components from their means at interval L (when it was reached)."""
        freeze = self.a ** (m - 1)
        rw = self.fls == 0
        idx = np.nonzero(self.has_data)[0]
        new = self.theta_hat.copy()
        if len(idx):
            if m <= self.switch:
                new = bart[:, idx, :].mean(axis=1)
            else:
                tmp = (bart[:, idx[0], :] - self.theta_hat) / vt[:, idx[0], :]
                for k in range(1, len(idx)):
                    tmp += (bart[:, idx[k], :] - bart[:, idx[k - 1], :]) / vt[:, idx[k], :]
                new = self.theta_hat + (self.t0 + self.b * self.b) * freeze ** 2 * self.var[None, :] * tmp
        out = self.theta_hat.copy()
        out[:, rw] = new[:, rw]
        if fls_means is not None:
            out[:, ~rw] = fls_means[:, ~rw]
        self.theta_hat = out

    def fixed_lag_means(self):
        """Fixed-lag means of the last iteration, None when there are none (no fixed-lag component,
        or interval L not reached)."""
        if not np.any(self.fls):
            return None
        means, updated = self.plan.fls_means()
        return means if updated else None

    def run(self, iterations, seed=1):
        trace = []
        for m in range(1, iterations + 1):
            freeze, sd_init, sd_mut, vt_add = self.schedules(m)
            ll, nf, bart, vt = self.plan.iteration(self.theta_hat, sd_init, sd_mut, vt_add, seed + 1000003 * m)
            self.update(m, bart, vt, self.fixed_lag_means())
            trace.append({'m': m, 'loglik': ll.copy(), 'n_all_fail': nf.copy(), 'theta_hat': self.theta_hat.copy()})
        return trace

    def close(self):
        self.plan.close()
