"""Parameters: theta.json -> natural-scale tables for the engine.

Restates the host-side parameter machinery of the reference's C core:

* routers: groups of a parameter and the map cac -> group or ts -> group
  (``build_router``, model_builder/C/core/build.c:267-374);
* transformations and their inverses (``set_f_trans``, ``f_log`` ...,
  model_builder/C/core/transform.c:23-111, 332-415), unit multipliers
  (``get_multiplier`` / ``u_duration_par2u_data``, transform.c:185-305) and
  durations turned into rates (``back_transform_x``, transform.c:462-481);
* ``transform_theta`` of the guesses (transform.c:494-514) followed by
  ``back_transform_theta2par`` (transform.c:447-460);
* initial conditions: ``linearize_and_repeat`` + ``prop2Xpop_size`` +
  ``theta_driftIC2Xdrift`` (model_builder/C/core/prediction_util.c:82-131).

The C side of the reference reads an *adapted* theta.json (per-parameter
``group`` objects whose fields are ``{"value": ...}`` and explicit partitions,
model_builder/C/core/build.c:285-362, load.c:304-347).  The tool that turned
the user form shipped with the examples into that form is not part of the
reference; :func:`adapt_theta` defines the conversion used here.
"""

import copy
import math

import numpy as np

ZERO_LOG = 1e-17          # model_builder/C/core/plom.h:93
ONE_LOGIT = 0.999999999   # model_builder/C/core/plom.h:94

FINV = {'identity': 0, 'log': 1, 'logit': 2, 'logit_ab': 3,
        'scale_pow10': 0, 'scale_pow10_bounded': 3, 'scale_pow10_neg': 1}
SCALE = {'scale_pow10': 1, 'scale_pow10_bounded': 1, 'scale_pow10_neg': 2}

_UNITS = {  # u_duration_par2u_data(u_par, u_data), transform.c:185-250
    ('D', 'D'): 1.0, ('D', 'W'): 1.0 / 7.0, ('D', 'B'): 1.0 / 14.0, ('D', 'M'): 12.0 / 365.0, ('D', 'Y'): 1.0 / 365.0,
    ('W', 'D'): 7.0, ('W', 'W'): 1.0, ('W', 'B'): 0.5, ('W', 'M'): 84.0 / 365.0, ('W', 'Y'): 7.0 / 365.0,
    ('B', 'D'): 14.0, ('B', 'W'): 2.0, ('B', 'B'): 1.0, ('B', 'M'): 84.0 / 365.0, ('B', 'Y'): 7.0 / 365.0,
    ('M', 'D'): 365.0 / 12.0, ('M', 'W'): 365.0 / 84.0, ('M', 'B'): 365.0 / 168.0, ('M', 'M'): 1.0, ('M', 'Y'): 1.0 / 12.0,
    ('Y', 'D'): 365.0, ('Y', 'W'): 365.0 / 7.0, ('Y', 'B'): 365.0 / 14.0, ('Y', 'M'): 12.0, ('Y', 'Y'): 1.0,
}


class ThetaError(Exception):
    pass


def u_duration_par2u_data(u_par, u_data):
    try:
        return _UNITS[(u_par, u_data)]
    except KeyError:
        raise ThetaError('invalid units %r -> %r' % (u_par, u_data))


def get_multiplier(u_data, par, direction=0):
    unit = par.get('unit')
    if unit is None:
        return 1.0
    if unit not in ('D', 'B', 'W', 'M', 'Y'):
        raise ThetaError('not a valid unit: %r' % unit)
    typ = par.get('type')
    if typ is not None:
        if typ != 'rate_as_duration':
            raise ThetaError('not a valid type: %r' % typ)
        return u_duration_par2u_data(u_data, unit) if direction else u_duration_par2u_data(unit, u_data)
    return u_duration_par2u_data(unit, u_data) if direction else u_duration_par2u_data(u_data, unit)


def is_duration(par):
    return par.get('unit') is not None and par.get('type') == 'rate_as_duration'


# forward transforms (transform.c:23-76) -----------------------------------
def f_forward(kind, x, a, b):
    if kind in ('identity', 'scale_pow10'):
        return x
    if kind in ('log', 'scale_pow10_neg'):
        return math.log(x if x > ZERO_LOG else ZERO_LOG)
    if kind == 'logit':
        s = x if x > ZERO_LOG else ZERO_LOG
        s = s if s < ONE_LOGIT else ONE_LOGIT
        return math.log(s / (1.0 - s))
    if kind in ('logit_ab', 'scale_pow10_bounded'):
        if a == b:
            return x
        ratio = (x - a) / (b - x)
        ratio = min(max(ratio, ZERO_LOG), 1.0 / ZERO_LOG)
        return math.log(ratio)
    raise ThetaError('unknown transformation %r' % kind)


def back_transform(x, bt):
    """Host twin of plomrt::back_transform (back_transform_x, transform.c:462-481)."""
    f_inv, scale, dur, a, b, mult = bt
    if f_inv == 1:
        v = math.exp(x)
    elif f_inv == 2:
        v = 1.0 / (1.0 + math.exp(-x)) if x > 0 else math.exp(x) / (1.0 + math.exp(x))
    elif f_inv == 3:
        if a == b:
            v = x
        elif x < 0:
            v = (b * math.exp(x) + a) / (1.0 + math.exp(x))
        else:
            v = (b + a * math.exp(-x)) / (1.0 + math.exp(-x))
    else:
        v = x
    if scale == 1:
        v = math.pow(10.0, v)
    elif scale == 2:
        v = math.pow(10.0, -v)
    v *= mult
    if dur:
        v = 1.0 / (0.00001 + v)
    return v


# adapter -------------------------------------------------------------------
_GROUP_FIELDS = ('min', 'max', 'guess', 'sd_transf', 'prior')


def is_adapted(theta):
    for p in theta.get('parameter', {}).values():
        g = p.get('group')
        if isinstance(g, dict):
            for v in g.values():
                return isinstance(v.get('guess'), dict)
    return False


def adapt_theta(theta, model):
    """User-form theta.json -> adapted form read by the C side.

    Built-in partitions: ``identical_population`` (one group ``all``),
    ``variable_population`` (one group per population), and the
    ``*_time_series`` twins for observation parameters; other partitions come
    from ``theta["partition"]`` (groups with ``population_id`` or
    ``time_series_id`` lists).  An already adapted document passes through
    unchanged (its group fields are ``{"value": ...}`` objects), and documents
    mixing both forms, as the reference's examples do, are accepted.  Parameter values given at the top level apply
    to every group; ``{"group": {gid: {...}}}`` gives them per group, as
    plain numbers or ``{"value": ...}``.  ``prior`` defaults to ``uniform``.
    """
    out = copy.deepcopy(theta)
    parts = copy.deepcopy(theta.get('partition', {}))
    parts.setdefault('identical_population', {'group': [{'id': 'all', 'population_id': list(model.cac_id)}]})
    parts.setdefault('variable_population', {'group': [{'id': c, 'population_id': [c]} for c in model.cac_id]})
    parts.setdefault('identical_time_series', {'group': [{'id': 'all', 'time_series_id': list(model.ts_id)}]})
    parts.setdefault('variable_time_series', {'group': [{'id': t, 'time_series_id': [t]} for t in model.ts_id]})
    out['partition'] = parts
    params = {}
    for name, p in theta.get('parameter', {}).items():
        q = dict((k, v) for k, v in p.items() if k not in _GROUP_FIELDS + ('group',))
        pid = p.get('partition_id')
        if pid is None:
            raise ThetaError('parameter %r has no partition_id' % name)
        if pid not in parts:
            raise ThetaError('unknown partition %r for %r' % (pid, name))
        groups = {}
        user_groups = p.get('group', {})
        for g in parts[pid]['group']:
            gid = g['id']
            src = user_groups.get(gid, {})
            fields = {}
            for f in _GROUP_FIELDS:
                if f in src:
                    v = src[f]
                    fields[f] = v if isinstance(v, dict) else {'value': v}
                elif f in p:
                    fields[f] = {'value': p[f]}
            fields.setdefault('prior', {'value': 'uniform'})
            for f in ('min', 'max', 'guess'):
                if f not in fields:
                    raise ThetaError('parameter %r group %r has no %s' % (name, gid, f))
            fields.setdefault('sd_transf', {'value': 0.0})
            groups[gid] = fields
        q['group'] = groups
        params[name] = q
    out['parameter'] = params
    return out


class Router(object):
    """Groups of one parameter (build_router, build.c:267-374)."""

    def __init__(self, name, par, partition, order, link_key, u_data='D', is_bayesian=False):
        self.name = name
        groups = partition['group']
        self.n_gp = len(groups)
        self.p = len(order)
        self.map = [0] * self.p
        self.group_name = []
        self.min = []
        self.max = []
        self.guess = []
        self.transf = par.get('transformation', 'identity')
        self.is_duration = is_duration(par)
        self.multiplier = get_multiplier(u_data, par, 0)
        self.f_inv = []
        self.scale = []
        pgroups = par['group']
        for g, grp in enumerate(groups):
            gid = grp['id']
            pg = pgroups[gid]
            self.group_name.append(gid)
            self.min.append(float(pg['min']['value']))
            self.max.append(float(pg['max']['value']))
            self.guess.append(float(pg['guess']['value']))
            prior = pg.get('prior', {}).get('value', 'uniform')
            kind = self.transf
            if is_bayesian and prior in ('uniform', 'pseudo_uniform'):
                kind = {'scale_pow10': 'scale_pow10_bounded', 'scale_pow10_bounded': 'scale_pow10_bounded',
                        'scale_pow10_neg': 'scale_pow10_neg_bounded'}.get(self.transf, 'logit_ab')
            self.f_inv.append(kind)
            self.scale.append(SCALE.get(self.transf, 0))
            for e in grp.get(link_key, []):
                if e not in order:
                    raise ThetaError("could not find element %r in array %r" % (e, link_key))
                self.map[order.index(e)] = g

    def _finv_code(self, g):
        k = self.f_inv[g]
        if k == 'scale_pow10_neg_bounded':
            return 3
        return FINV[k]

    def bt(self, g):
        return (self._finv_code(g), self.scale[g], 1 if self.is_duration else 0,
                self.min[g], self.max[g], self.multiplier)

    def transformed_guess(self, g):
        k = self.f_inv[g]
        if k == 'scale_pow10_neg_bounded':
            k = 'logit_ab'
        return f_forward(k, self.guess[g], self.min[g], self.max[g])

    def natural(self, g, x=None):
        return back_transform(self.transformed_guess(g) if x is None else x, self.bt(g))


class Parameters(object):
    """Natural parameters of one theta for one model + settings."""

    def __init__(self, model, theta, u_data='D', is_bayesian=False):
        th = adapt_theta(theta, model)
        self.model = model
        parts = th['partition']
        P = th['parameter']
        self.routers = {}
        for name in model.par_sv + model.par_proc:
            self.routers[name] = self._router(name, P, parts, model.cac_id, 'population_id', u_data, is_bayesian)
        for name in model.par_obs:
            self.routers[name] = self._router(name, P, parts, model.ts_id, 'time_series_id', u_data, is_bayesian)

    @staticmethod
    def _router(name, P, parts, order, link_key, u_data, is_bayesian):
        if name not in P:
            raise ThetaError('theta has no parameter %r' % name)
        par = P[name]
        if 'follow' in par:
            par = dict(P[par['follow']], **{'partition_id': P[par['follow']]['partition_id']})
        pid = par['partition_id']
        return Router(name, par, parts[pid], order, link_key, u_data, is_bayesian)

    def natural_cac(self, name):
        r = self.routers[name]
        return [r.natural(r.map[c]) for c in range(len(self.model.cac_id))]

    def natural_ts(self, name):
        r = self.routers[name]
        return [r.natural(r.map[t]) for t in range(len(self.model.ts_id))]

    def par_cac(self):
        m = self.model
        out = np.zeros((len(m.par_proc), m.N_CAC))
        for k, p in enumerate(m.par_proc):
            out[k] = self.natural_cac(p)
        return out

    def par_ts(self):
        m = self.model
        out = np.zeros((len(m.par_obs), m.N_TS))
        for k, p in enumerate(m.par_obs):
            out[k] = self.natural_ts(p)
        return out

    def drift_tables(self):
        """(group[N_DRIFT][N_CAC], ngroups[N_DRIFT], bt[N_DRIFT][N_CAC], vol[N_DRIFT][N_CAC], x_drift[N_DRIFT][N_CAC])."""
        m = self.model
        nd = len(m.drift_par_proc)
        grp = np.zeros((max(nd, 1), m.N_CAC), dtype=np.int32)
        ng = np.ones(max(nd, 1), dtype=np.int32)
        bt = [[(0, 0, 0, 0.0, 0.0, 1.0)] * m.N_CAC for _ in range(max(nd, 1))]
        vol = np.zeros((max(nd, 1), m.N_CAC))
        xd = np.zeros((max(nd, 1), m.N_CAC))
        for i, (p, v) in enumerate(zip(m.drift_par_proc, m.vol_par_proc)):
            r = self.routers[p]
            rv = self.routers[v]
            grp[i] = r.map
            ng[i] = r.n_gp
            for g in range(r.n_gp):
                bt[i][g] = r.bt(g)
                # volatility indexed by the drifted parameter's group (drift.c:38-39)
                vol[i, g] = rv.natural(g) if g < rv.n_gp else rv.natural(rv.n_gp - 1)
                xd[i, g] = r.transformed_guess(g)
        return grp, ng, bt, vol, xd

    def x0(self, pop_size_t0):
        """Initial particle: proportions x population size, drift words, zero incidences."""
        m = self.model
        nd = len(m.drift_par_proc)
        S = len(m.par_sv) * m.N_CAC + nd * m.N_CAC + m.N_TS_INC_UNIQUE
        x = np.zeros(S)
        tot = np.zeros(m.N_CAC)
        for i, s in enumerate(m.par_sv):
            prop = np.array(self.natural_cac(s))
            tot += prop
            x[i * m.N_CAC:(i + 1) * m.N_CAC] = prop * np.asarray(pop_size_t0)
        if m.remainder is not None and np.any(tot > 1.0):
            raise ThetaError('sum of the initial conditions without remainder is greater than 1.0')
        if nd:
            _, _, _, _, xd = self.drift_tables()
            off = len(m.par_sv) * m.N_CAC
            for i in range(nd):
                x[off + i * m.N_CAC: off + (i + 1) * m.N_CAC] = xd[i]
        return x
