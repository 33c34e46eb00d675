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

A parameter fitted per group contributes one component per group (the
populations or series of the group read it); initial conditions are not
fitted (no fixed-lag smoothing).
"""

import numpy as np

from .native import MifDescHolder, MifPlan


class MifError(Exception):
    pass


def components(problem, names=None):
    """theta components: one per group of every estimated (sd_transf > 0 in some group) process
    and observation parameter."""
    m = problem.model
    params = problem.params
    out = []
    for kind, plist in (('proc', m.par_proc), ('obs', m.par_obs)):
        for idx, name in enumerate(plist):
            r = params.routers[name]
            if names is not None and name not in names:
                continue
            sds = _sd_transf(problem, name, r)
            if names is None and not max(sds) > 0.0:
                continue
            for g in range(r.n_gp):
                members = None if r.n_gp == 1 else [c for c in range(len(r.map)) if r.map[c] == g]
                out.append({'name': name, 'kind': kind, 'index': idx, 'g': g, 'bt': r.bt(g), 'sd_transf': sds[g],
                            'theta0': r.transformed_guess(g), 'members': members})
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


class Mif(object):
    def __init__(self, engine, problem, n_runs=1, names=None, a=0.975, b=2.0, switch=5, sd_transf=None,
                 precision=None):
        self.problem = problem
        self.comp = components(problem, names)
        if sd_transf is not None:
            for c in self.comp:
                c['sd_transf'] = float(sd_transf.get(c['name'], c['sd_transf'])) if isinstance(sd_transf, dict) \
                    else float(sd_transf)
        m = problem.model
        self.R = int(n_runs)
        self.Q = len(self.comp)
        self.a, self.b, self.switch = float(a), float(b), int(switch)
        self.holder = MifDescHolder(self.R, [(c['kind'], c['index'], c['bt'], c['sd_transf'] > 0, c['members'])
                                             for c in self.comp], len(m.par_proc), len(m.par_obs), m.N_CAC, m.N_TS)
        self.plan = MifPlan(engine, problem, self.holder, precision=precision)
        n_data = problem.n_obs
        self.var = np.array([c['sd_transf'] ** 2 / n_data for c in self.comp])
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

    def update(self, m, bart, vt):
        """theta-hat update of every run from the filtered means / variances."""
        freeze = self.a ** (m - 1)
        idx = np.nonzero(self.has_data)[0]
        if len(idx) == 0:
            return
        if m <= self.switch:
            self.theta_hat = bart[:, idx, :].mean(axis=1)
        else:
            tmp = (bart[:, idx[0], :] - self.theta_hat) / vt[:, idx[0], :]
            for k in range(1, len(idx)):
                tmp += (bart[:, idx[k], :] - bart[:, idx[k - 1], :]) / vt[:, idx[k], :]
            self.theta_hat = self.theta_hat + (self.t0 + self.b * self.b) * freeze ** 2 * self.var[None, :] * tmp

    def run(self, iterations, seed=1):
        trace = []
        for m in range(1, iterations + 1):
            freeze, sd_init, sd_mut, vt_add = self.schedules(m)
            ll, nf, bart, vt = self.plan.iteration(self.theta_hat, sd_init, sd_mut, vt_add, seed + 1000003 * m)
            self.update(m, bart, vt)
            trace.append({'m': m, 'loglik': ll.copy(), 'n_all_fail': nf.copy(), 'theta_hat': self.theta_hat.copy()})
        return trace

    def close(self):
        self.plan.close()
