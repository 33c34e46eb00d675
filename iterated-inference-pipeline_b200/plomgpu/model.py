"""Model description parsing: plom JSON (context / process / link) -> model IR.

This is the builder half of plom's code generator restated for a CUDA
back-end.  The semantics follow the reference:

* state / remainder / parameter bookkeeping and the white-noise, drift and
  observation-variable rules of ``Cmodel.__init__``
  (model_builder/Cmodel.py:31-184), including the resolution of ``N`` and
  of the remainder compartment inside rates (Cmodel.py:150-182) and the
  tokenizer ``change_user_input`` (Cmodel.py:188-209);
* population / time-series bookkeeping of ``Context.__init__``
  (model_builder/Context.py:32-82);
* the time-series sort, ``get_obs2ts`` and the ``.settings.json`` writer of
  ``PlomModelBuilder`` (model_builder/Builder.py:70-113, 118-169, 173-259).

Extension beyond the reference DSL (documented, not expressible there):
``context["coupling"]`` may hold an ``N_CAC x N_CAC`` matrix; rates may then
use the special function ``foi(X)`` = sum_c' W[cac][c'] * X[c'] / Npop[c']
where ``Npop`` is the population size of compartment-age-class c' (the sum
of the state variables when there is no remainder, else the ``N``
covariate).  The reference only declares such a matrix
(model_builder/C/core/build.c:872-874, prediction_util.c:354-364) and never
emits it.
"""

import copy
import datetime

OPS = set(['+', '-', '*', '/', ',', '(', ')'])
SPECIAL_FUNCTIONS = set(['terms_forcing', 'heaviside', 'ramp', 'slowstep',
                         'sin', 'cos', 'correct_rate', 'foi'])
UNIVERSE = 'U'


class PlomModelError(Exception):
    pass


def tokenize(expr):
    """Split an expression on the operators ``+-*/,()`` after removing blanks.

    Same contract as ``Cmodel.change_user_input`` (Cmodel.py:188-209):
    ``tokenize('r0*2*correct_rate(v)') == ['r0','*','2','*','correct_rate','(','v',')']``.
    """
    s = expr.replace(' ', '')
    out, cur = [], ''
    for ch in s:
        if ch in OPS:
            if cur:
                out.append(cur)
                cur = ''
            out.append(ch)
        else:
            cur += ch
    if cur:
        out.append(cur)
    return out


def _has_tag(state, tag):
    t = state.get('tag', [])
    # the reference tests ``'remainder' in x.get('tag', [])`` which accepts a
    # list of tags or a single tag string
    return tag in t


def _days(d):
    return datetime.datetime.strptime(d, "%Y-%m-%d").date()


class PlomModel(object):
    """Parsed model: process + link (+ optional context).

    ``context`` may be a minimal dict (``{'data': {}, 'metadata': [...]}``)
    when only the process/link bookkeeping is needed (as in the reference's
    ``Cmodel`` unit tests).
    """

    def __init__(self, context, process, link):
        self.context = copy.deepcopy(context)
        self.process = copy.deepcopy(process)
        self.link = copy.deepcopy(link)

        # --- states --------------------------------------------------------
        self.remainder = None
        self.par_sv = []
        for x in process['state']:
            if _has_tag(x, 'remainder'):
                self.remainder = x['id']
            else:
                self.par_sv.append(x['id'])

        # --- covariates: N first when present (Cmodel.py:51-53) -------------
        meta = context.get('metadata', [])
        self.par_fixed = [x['id'] for x in meta if x['id'] == 'N']
        self.par_fixed += [x['id'] for x in meta if x['id'] != 'N']
        fixed = set(self.par_fixed)
        self.par_proc = [x['id'] for x in process['parameter'] if x['id'] not in fixed]
        self.par_obs = [x['id'] for x in link['observation'][0]['parameter'] if x['id'] not in fixed]

        # --- reactions and white noises ------------------------------------
        self.proc_model = copy.deepcopy(process['model'])
        self.white_noise = []
        for j, wn in enumerate(process.get('white_noise', [])):
            noise = {'name': 'white_noise__%d' % j, 'sd': wn['sd']}
            self.white_noise.append(noise)
            for r in self.proc_model:
                for nr in wn['reaction']:
                    if self._reaction_matches(r, nr):
                        r['white_noise'] = noise

        # --- observation process and drift ---------------------------------
        self.obs_model = copy.deepcopy(link['observation'][0]['model'])
        self.drift_par_proc = [x['parameter'] for x in process.get('diffusion', [])]
        self.vol_par_proc = [x['volatility'] for x in process.get('diffusion', [])]
        self.drift_par_obs = []
        self.vol_par_obs = []
        self.par_fixed_obs = set()
        for k, v in self.obs_model.items():
            if k not in ('distribution', 'comment'):
                for e in tokenize(v):
                    if e in fixed:
                        self.par_fixed_obs.add(e)
        self.drift_var = ['drift__par_proc__' + x for x in self.drift_par_proc]
        self.drift_var += ['drift__par_obs__' + x for x in self.drift_par_obs]

        # --- observed variables: incidences first (stable) -----------------
        observed = copy.deepcopy(link['observed'])
        observed.sort(key=lambda x: 0 if isinstance(x['definition'][0], dict) else 1)
        rate_of = {}
        for r in self.proc_model:
            rate_of[(r['from'], r['to'])] = r['rate']
        self.obs_var = []
        self.obs_var_def = []
        for x in observed:
            self.obs_var.append(x['id'])
            d = copy.deepcopy(x['definition'])
            for item in d:
                if isinstance(item, dict) and 'rate' not in item:
                    item['rate'] = rate_of[(item['from'], item['to'])]
            self.obs_var_def.append(d)
        for j, wn in enumerate(process.get('white_noise', [])):
            for defs in self.obs_var_def:
                for item in defs:
                    if isinstance(item, dict):
                        for nr in wn['reaction']:
                            if self._reaction_matches(item, nr):
                                item['white_noise'] = {'name': 'white_noise__%d' % j, 'sd': wn['sd']}

        # --- resolve N / remainder (Cmodel.py:150-182) ---------------------
        if self.remainder is None:
            for k in list(self.obs_model.keys()):
                if k != 'distribution':
                    self.obs_model[k] = self._resolve_N(self.obs_model[k])
        for r in self.proc_model:
            r['rate'] = self._resolve_rate(r)
        for defs in self.obs_var_def:
            for item in defs:
                if isinstance(item, dict):
                    item['rate'] = self._resolve_rate(item)

        self.coupling = None
        if 'coupling' in context:
            self.coupling = [list(map(float, row)) for row in context['coupling']]

        if 'population' in context:
            self._init_context(context)

    # ------------------------------------------------------------------
    @staticmethod
    def _reaction_matches(r, nr):
        return (r['from'] == nr['from'] and r['to'] == nr['to'] and
                (('rate' in nr and r['rate'] == nr['rate']) or ('rate' not in nr)))

    def _resolve_N(self, expr):
        tot = '(%s)' % '+'.join(self.par_sv)
        return ''.join(tot if t == 'N' else t for t in tokenize(expr))

    def _resolve_rate(self, r):
        rate = r['rate']
        if self.remainder:
            if r['from'] == self.remainder:
                rate = '(%s)*%s' % (rate, self.remainder)
            rem = '(N-%s)' % '-'.join(self.par_sv)
            return ''.join(rem if t == self.remainder else t for t in tokenize(rate))
        return self._resolve_N(rate)

    # ------------------------------------------------------------------
    def _init_context(self, context):
        """Context bookkeeping + time-series sort (Context.py:32-82, Builder.py:70-113)."""
        self.cac_id = [x['id'] for x in context['population']]
        heads = [x.split('__') for x in self.cac_id]
        cities = [h[0] for h in heads]
        ages = [h[1] for h in heads]
        self.cities_id = [cities[i] for i in sorted(set(cities.index(c) for c in cities))]
        self.ages_id = [ages[i] for i in sorted(set(ages.index(a) for a in ages))]
        self.N_C = len(self.cities_id)
        self.N_AC = len(self.ages_id)
        self.N_CAC = self.N_C * self.N_AC
        # cac index convention of the C side: cac = c*N_AC + ac, and the
        # per-cac covariate / router order is the order of cac_id
        ts_id = [x['id'] for x in context['time_series']]
        self.map_ts_cac = dict((x['id'], list(x['population_id'])) for x in context['time_series'])

        self.map_ts_obs = {}
        for x in self.link['observed']:
            for ts in x['time_series_id']:
                self.map_ts_obs[ts] = x['id']

        data_src = context.get('data', {}).get('source', {})
        dates = []
        rows = []
        if data_src:
            dates = [v[0] for v in data_src[ts_id[0]]['value']]
            for i in range(len(dates)):
                rows.append([data_src[ts]['value'][i][1] for ts in ts_id])

        def parts(ts):
            h = ts.split('__')
            return h[0], h[1], h[2]

        order = sorted(range(len(ts_id)),
                       key=lambda i: (self.obs_var.index(self.map_ts_obs[ts_id[i]]),
                                      parts(ts_id[i])[0], parts(ts_id[i])[1]))
        self.ts_id = [ts_id[i] for i in order]
        self.data = [[r[i] for i in order] for r in rows]
        self.dates = dates
        self.N_TS = len(self.ts_id)
        self._name_ts = [parts(t)[0] for t in self.ts_id]
        self._stream = [parts(t)[1] for t in self.ts_id]
        self._obs_type = [parts(t)[2] for t in self.ts_id]
        inc_names = [self._name_ts[i] for i in range(self.N_TS) if self._obs_type[i] == 'inc']
        self.N_TS_INC = len(inc_names)
        self.N_TS_INC_UNIQUE = len(set(inc_names))
        self.N_DATA = len(self.data)
        t0s = [data_src[t]['t0'] for t in ts_id if t in data_src]
        self.date_0 = _days(t0s[0]) if t0s else None
        self.par_fixed_values = dict((d['id'], copy.deepcopy(d)) for d in context.get('metadata', []))
        self.obs2ts = self._obs2ts()
        self.N_OBS_INC = len([d for d in self.obs_var_def if isinstance(d[0], dict)])
        self.N_OBS_PREV = len(self.obs_var_def) - self.N_OBS_INC
        if self.coupling is not None:
            if len(self.coupling) != self.N_CAC or any(len(r) != self.N_CAC for r in self.coupling):
                raise PlomModelError('coupling matrix must be N_CAC x N_CAC')

    def _obs2ts(self):
        """Per observed variable: unique series, streams and aggregated cac (Builder.py:118-169)."""
        out = []
        for o in self.obs_var:
            idx = [i for i, t in enumerate(self.ts_id) if self.map_ts_obs[t] == o]
            names = [self._name_ts[i] for i in idx]
            uniq = []
            for n in names:
                if n not in uniq:
                    uniq.append(n)
            info = {'n_ts_unique': len(uniq), 'n_stream': [], 'n_cac': [], 'cac': []}
            for u in uniq:
                sel = [idx[k] for k, n in enumerate(names) if n == u]
                streams = set(self._stream[i] for i in sel)
                cacs = self.map_ts_cac[self.ts_id[sel[0]]]
                info['n_stream'].append(len(streams))
                info['n_cac'].append(len(cacs))
                info['cac'].append([(self.cities_id.index(x.split('__')[0]),
                                     self.ages_id.index(x.split('__')[1])) for x in cacs])
            out.append(info)
        off = 0
        for x in out:
            x['offset'] = off
            off += sum(x['n_stream'])
        return out

    # ------------------------------------------------------------------
    @property
    def times(self):
        return [0] + [(_days(d) - self.date_0).days for d in self.dates]

    def settings(self):
        """The ``.settings.json`` document (same keys as Builder.py:173-259)."""
        s = {'POP_SIZE_EQ_SUM_SV': self.remainder is None}
        data = {'obs2ts': self.obs2ts, 'data': self.data}
        pfv = {}
        for k, v in self.par_fixed_values.items():
            order = self.ts_id if k in self.par_fixed_obs else self.cac_id
            vals = []
            for ts in order:
                x, y = [], []
                for d in v['source'][ts]['value']:
                    if d[1] is not None:
                        x.append((_days(d[0]) - self.date_0).days)
                        y.append(d[1])
                obj = {'id': ts, 'x': x, 'y': y, 'size': len(y)}
                if 'unit' in v:
                    obj['unit'] = v['unit']
                if 'type' in v:
                    obj['type'] = v['type']
                vals.append(obj)
            pfv[k] = vals
        data['par_fixed_values'] = pfv
        data['dates'] = self.dates
        data['times'] = self.times
        if self.coupling is not None:
            data['coupling'] = self.coupling
        s['data'] = data
        all_order = self.par_sv + self.par_proc + self.par_obs
        s['drift'] = {'ind_par_Xdrift_applied': [all_order.index(x) for x in self.drift_par_proc + self.drift_par_obs],
                      'ind_volatility_Xdrift': [all_order.index(x) for x in self.vol_par_proc + self.vol_par_obs]}
        s['ind_noise_sd'] = sorted(set(all_order.index(x['sd']) for x in self.white_noise))
        s['remainder'] = self.remainder
        s['date_0'] = str(self.date_0)
        s['cst'] = {'N_C': self.N_C, 'N_AC': self.N_AC,
                    'N_PAR_PROC': len(self.par_proc), 'N_PAR_OBS': len(self.par_obs),
                    'N_PAR_SV': len(self.par_sv), 'N_PAR_FIXED': len(self.par_fixed),
                    'N_TS': self.N_TS, 'N_TS_INC': self.N_TS_INC,
                    'N_TS_INC_UNIQUE': self.N_TS_INC_UNIQUE, 'N_DATA': self.N_DATA,
                    'N_OBS_ALL': len(self.obs_var_def), 'N_OBS_INC': self.N_OBS_INC,
                    'N_OBS_PREV': self.N_OBS_PREV,
                    'N_DRIFT': len(self.drift_par_proc) + len(self.drift_par_obs),
                    'IS_SCHOOL_TERMS': 1 if any('terms_forcing' in r['rate'] for r in self.proc_model) else 0}
        s['orders'] = {'par_sv': self.par_sv, 'par_proc': self.par_proc,
                       'par_fixed': self.par_fixed, 'par_obs': self.par_obs,
                       'ts_id': self.ts_id, 'cac_id': self.cac_id,
                       'drift_var': self.drift_var}
        return s
