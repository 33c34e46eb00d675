"""The parameter vector of the reference's drivers (``struct s_best``).

One entry per (parameter, group) in the order of ``p_it_all``: the state
variables, then the process parameters, then the observation parameters
(build_routers, model_builder/C/core/build.c:400-470), each with its groups.
Restates:

* load_best (model_builder/C/core/load.c:304-374): guess, sd_transf on the
  diagonal of the proposal covariance (zero for followers), prior kind and
  its (min, max) bounds;
* transform_theta (model_builder/C/core/transform.c:494-514): guesses to the
  transformed scale, sd_transf squared unless theta carries a covariance;
* update_to_be_estimated (model_builder/C/core/func.c:171-187);
* log_prob_prior and the priors (model_builder/C/core/metropolis_hastings_prior.c:64-133);
* the "theta remainder": a state variable absent from theta when the
  population size is the sum of the states gets a logit parameter in
  [0, 1] with guess 0 (plom_theta_remainder_new, model_builder/C/core/json.c:405-424),
  excluded from the trace and from .done (``p_it_all_no_theta_remainder``,
  build.c:72-93).
"""

import copy
import math

import numpy as np

from .theta import Router, adapt_theta, back_transform, f_forward

LIKE_MIN_DEFAULT = 1e-17


def _plain_finv(kind_code, x, a, b):
    """router->f_inv (no scale, unit or duration: those belong to back_transform_x)."""
    return back_transform(x, (kind_code, 0, 0, a, b, 1.0))


def normal_prior(x, lo, hi):
    mean = (hi + lo) / 2.0
    sd = (hi - lo) / 4.0
    z = (x - mean) / sd
    return math.exp(-0.5 * z * z) / (math.sqrt(2.0 * math.pi) * sd)


def pseudo_unif_prior(x, lo, hi):
    delta = 0.01 * (hi - lo)
    alpha = 1.0 / (hi - lo - 2.0 / 3.0 * delta)
    a = -alpha / (delta ** 2)
    b = -2.0 * (lo + delta) * a
    c = alpha + a * (lo + delta) ** 2
    if x <= lo or x >= hi:
        return 0.0
    if x < lo + delta:
        return a * x * x + b * x + c
    if x < hi - delta:
        return alpha
    y = x - (hi - lo - 2.0 * delta)
    return a * y * y + b * y + c


def flat_prior(x, lo, hi):
    """gsl_ran_flat_pdf: 1/(hi-lo) on [lo, hi), 0 elsewhere."""
    return 1.0 / (hi - lo) if lo <= x < hi else 0.0


PRIORS = {'normal': normal_prior, 'pseudo_uniform': pseudo_unif_prior}


class Best(object):
    """Transformed parameter vector + proposal covariance + priors of one theta."""

    def __init__(self, model, theta, u_data='D', is_bayesian=False):
        self.model = model
        self.theta = copy.deepcopy(theta)
        th = adapt_theta(theta, model)
        self.adapted = th
        parts = th['partition']
        P = th['parameter']
        self.entries = []      # dicts: name, group, router, g, kind ('sv', 'proc', 'obs')
        self.routers = []
        self.theta_remainder = None
        for kind, names, order, link in (('sv', model.par_sv, model.cac_id, 'population_id'),
                                         ('proc', model.par_proc, model.cac_id, 'population_id'),
                                         ('obs', model.par_obs, model.ts_id, 'time_series_id')):
            for name in names:
                par = P.get(name)
                follow = None
                if par is None:
                    # theta remainder (json.c:405-424)
                    self.theta_remainder = len(self.routers)
                    grp = dict((g['id'], {'min': {'value': 0.0}, 'max': {'value': 1.0}, 'guess': {'value': 0.0},
                                          'sd_transf': {'value': 0.0}, 'prior': {'value': 'uniform'}})
                               for g in parts['variable_population']['group'])
                    par = {'partition_id': 'variable_population', 'transformation': 'logit', 'group': grp}
                elif 'follow' in par:
                    follow = par['follow']
                    par = P[follow]
                r = Router(name, par, parts[par['partition_id']], order, link, u_data, is_bayesian)
                self.routers.append(r)
                for g in range(r.n_gp):
                    gid = r.group_name[g]
                    pg = par['group'][gid]
                    self.entries.append({
                        'name': name, 'group': gid, 'router': r, 'g': g, 'kind': kind,
                        'follower': follow is not None, 'follow': follow,
                        'prior': pg.get('prior', {}).get('value', 'uniform'),
                        'min': float(pg['min']['value']), 'max': float(pg['max']['value']),
                        'guess': float(pg['guess']['value']),
                        'sd_transf': 0.0 if follow is not None else float(pg.get('sd_transf', {}).get('value', 0.0)),
                        'remainder': self.theta_remainder == len(self.routers) - 1,
                    })
        n = len(self.entries)
        self.n = n
        self.mean = np.array([self._f(e, e['guess']) for e in self.entries])
        cov = theta.get('covariance')
        self.var = np.zeros((n, n))
        if cov is not None:
            c = np.asarray(cov, dtype=float)
            if c.shape != (n, n):
                raise ValueError('theta covariance has shape %r, expected %r' % (c.shape, (n, n)))
            self.var[:] = c
            for k, e in enumerate(self.entries):
                self.var[k, k] = 0.0 if e['follower'] else c[k, k]
        else:
            for k, e in enumerate(self.entries):
                sd = e['sd_transf']
                self.var[k, k] = sd * sd if sd > 0.0 else 0.0
        self.update_to_be_estimated()

    @staticmethod
    def _f(e, x):
        r, g = e['router'], e['g']
        k = r.f_inv[g]
        if k == 'scale_pow10_neg_bounded':
            k = 'logit_ab'
        return f_forward(k, x, r.min[g], r.max[g])

    def update_to_be_estimated(self):
        self.is_estimated = np.zeros(self.n, bool)
        for k, e in enumerate(self.entries):
            if self.var[k, k] > 0.0 and not e['follower']:
                self.is_estimated[k] = True
            else:
                self.var[k, k] = 0.0
        self.to_be_estimated = np.nonzero(self.is_estimated)[0]

    def f_inv(self, x=None):
        """Entries back on the scale of theta (router f_inv of the transformed values)."""
        x = self.mean if x is None else x
        out = np.zeros(self.n)
        for k, e in enumerate(self.entries):
            r, g = e['router'], e['g']
            out[k] = _plain_finv(r._finv_code(g), x[k], r.min[g], r.max[g])
        return out

    def log_prob_prior(self, x=None, like_min=LIKE_MIN_DEFAULT):
        """(log prior over the estimated entries, error flag), as log_prob_prior."""
        x = self.mean if x is None else x
        nat = self.f_inv(x)
        lp, err = 0.0, False
        for k, e in enumerate(self.entries):
            if not self.is_estimated[k]:
                continue
            fn = PRIORS.get(e['prior'], flat_prior)
            p = fn(nat[k], e['min'], e['max'])
            if math.isnan(p) or math.isinf(p) or p < 0.0:
                err = True
                p = like_min
            else:
                p = like_min if p <= like_min else p
            lp += math.log(p)
        return lp, err

    def visible(self):
        """Indices of ``p_it_all_no_theta_remainder``."""
        return [k for k, e in enumerate(self.entries) if not e['remainder']]

    def trace_header(self):
        return 'index,' + ''.join('%s:%s,' % (self.entries[k]['name'], self.entries[k]['group'])
                                  for k in self.visible()) + 'log_like\n'

    def trace_row(self, index, log_like, x=None):
        nat = self.f_inv(x)
        return '%d,' % index + ''.join('%s,' % fmt_g(nat[k]) for k in self.visible()) + '%s\n' % fmt_g(log_like)

    def theta_with(self, x=None):
        """theta.json with every visible guess replaced by f_inv of the vector (plom_print_done,
        model_builder/C/core/print.c:33-58); groups are written in the adapted form."""
        nat = self.f_inv(x)
        out = copy.deepcopy(self.theta)
        params = out.setdefault('parameter', {})
        for k in self.visible():
            e = self.entries[k]
            if e['follower']:
                continue
            par = params.setdefault(e['name'], {})
            grp = par.setdefault('group', {}).setdefault(e['group'], {})
            grp['guess'] = {'value': float(nat[k])}
        return out

    def theta_for(self, x):
        """theta.json whose guesses are the (transformed) vector x, for a new filter."""
        out = copy.deepcopy(self.adapted)
        nat = self.f_inv(x)
        for k, e in enumerate(self.entries):
            if e['remainder'] or e['follower']:
                continue
            out['parameter'][e['name']]['group'][e['group']]['guess'] = {'value': float(nat[k])}
        return out


def fmt_g(x):
    """printf("%g") of a double, including the C spelling of non-finite values."""
    if x != x:
        return '-nan' if math.copysign(1.0, x) < 0 else 'nan'
    if x == float('inf'):
        return 'inf'
    if x == float('-inf'):
        return '-inf'
    return '%g' % x
