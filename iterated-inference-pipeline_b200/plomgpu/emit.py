"""CUDA emitter: model IR -> ``__host__ __device__`` model header.

Restates the equation generation of plom's ``Ccoder`` for a CUDA target:

* rate caching and translation of rate expressions through sympy
  (``make_C_term`` / ``toC`` / ``generator_C``, model_builder/Ccoder.py:34-139);
* the ODE / Euler-Maruyama right-hand sides of the four SDE variants and the
  observed-incidence equations (``step_ode_sde`` incl. ``eq_dem_env``,
  Ccoder.py:366-508);
* prevalence observations (``print_obs_prev``, Ccoder.py:142-152) and the
  observation model (``print_like``, Ccoder.py:526-532);
* the loop structure and clamping of the generated step template
  (model_builder/C/templates/core_template.c:52-102, 215-339).

The emitted header is plain C++ templated on the state precision ``T``; the
same text is compiled into the sm_100a kernels and into the CPU oracle.
Differences from the reference's generated C, each one forced by the target:

* rates of one compartment-age class (cac) are computed and its states
  updated in the same loop iteration, so the state can live in registers or
  shared memory; the reference computes all rates first and writes a second
  buffer ``f`` (core_template.c:258-295).  Both read only the previous
  values of the same cac, so the arithmetic is the same;
* observed incidences are accumulated inside that loop in cac order, then
  added to the incidence word and clamped, as ``X[offset] + sum_inc``
  (core_template.c:305-335);
* noises are requested from a draw source in the reference's order
  (cac-major, then ``dem_sto__*`` then ``white_noise__*``,
  core_template.c:282-283, Ccoder.py:446-476), which is what makes common
  random numbers possible between the GPU and the oracle.
"""

import os
import re

import sympy
from sympy.printing.c import C99CodePrinter

from .model import PlomModel, tokenize, PlomModelError, UNIVERSE

VARIANTS = {  # bit 0: no demographic noise, bit 1: no environmental noise
    'full': 0, 'no_dem_sto': 1, 'no_env_sto': 2, 'no_dem_sto_no_env_sto': 3,
}

_PREFIX = 'plom___'


class _Printer(C99CodePrinter):
    """sympy C printer with a symbol map and literals typed as ``T``."""

    def __init__(self, symmap):
        super().__init__({'strict': False})
        self.symmap = symmap

    def _print_Symbol(self, expr):
        name = expr.name
        if name.startswith(_PREFIX):
            key = name[len(_PREFIX):]
            if key not in self.symmap:
                raise PlomModelError('symbol %r cannot be used here' % key)
            return self.symmap[key]
        raise PlomModelError('unknown symbol %r' % name)

    def _print_Integer(self, expr):
        return 'T(%d)' % int(expr)

    def _print_Float(self, expr):
        return 'T(%s)' % repr(float(expr))

    def _print_Rational(self, expr):
        return '(T(%d)/T(%d))' % (expr.p, expr.q)

    def _print_Pi(self, expr):
        return 'T(3.141592653589793)'

    def _print_Exp1(self, expr):
        return 'T(2.718281828459045)'

    def _print_Pow(self, expr):
        b, e = expr.base, expr.exp
        pb = self.parenthesize(b, sympy.printing.precedence.PRECEDENCE['Pow'])
        if e == -1:
            return '(T(1)/%s)' % pb
        if e == sympy.Rational(1, 2):
            return 'sqrt(%s)' % self._print(b)
        if e == -sympy.Rational(1, 2):
            return '(T(1)/sqrt(%s))' % self._print(b)
        if e == 2:
            return '(%s*%s)' % (pb, pb)
        if e == -2:
            return '(T(1)/(%s*%s))' % (pb, pb)
        return 'pow(%s, %s)' % (self._print(b), self._print(e))

    def _print_Function(self, expr):
        name = expr.func.__name__
        args = ', '.join(self._print(a) for a in expr.args)
        if name in ('heaviside', 'ramp', 'slowstep'):
            return 'plom_%s<T>(%s)' % (name, args)
        if name == 'foi':
            a = expr.args[0]
            if not (isinstance(a, sympy.Symbol) and a.name.startswith(_PREFIX)):
                raise PlomModelError('foi() takes a state variable')
            return 'foi_%s' % a.name[len(_PREFIX):]
        if name == 'terms_forcing':
            raise PlomModelError('terms_forcing (school terms) is not supported by the CUDA back-end')
        return '%s(%s)' % (name, args)

    def _print_sin(self, expr):
        return 'sin(%s)' % self._print(expr.args[0])

    def _print_cos(self, expr):
        return 'cos(%s)' % self._print(expr.args[0])


def _sympify(expr, names, drop_correct_rate):
    toks = tokenize(expr)
    out = []
    i = 0
    while i < len(toks):
        t = toks[i]
        if t == 'correct_rate' and drop_correct_rate:
            i += 1  # "correct_rate(v)" -> "(v)" (Ccoder.toC, Ccoder.py:55-56)
            continue
        out.append(_PREFIX + t if t in names else t)
        i += 1
    s = ''.join(out)
    local = {n: sympy.Function(n) for n in ('heaviside', 'ramp', 'slowstep', 'foi', 'terms_forcing')}
    for n in names:
        local[_PREFIX + n] = sympy.Symbol(_PREFIX + n)
    return sympy.sympify(s, locals=local)


# Calls of the rates that depend on time only (seasonal forcing such as
# cos(2 pi t / 364)) are evaluated once per substep instead of once per cac.
HOIST_TIME_TERMS = os.environ.get('PLOM_HOIST_TIME_TERMS', '1') != '0'
_TIME_FUNCS = ('cos', 'sin', 'tan', 'exp', 'log', 'sqrt', 'pow', 'cosh', 'sinh', 'tanh')


def _time_only(arg):
    names = set(re.findall(r'[A-Za-z_][A-Za-z_0-9]*', arg))
    return names <= {'t', 'T'} and 't' in names


def hoist_time_terms(exprs):
    """(expressions with time-only calls replaced by pre.tt_k, [call text of tt_k])."""
    terms = []
    out = []
    for e in exprs:
        i = 0
        res = ''
        while i < len(e):
            m = re.compile(r'\b(%s)\(' % '|'.join(_TIME_FUNCS)).search(e, i)
            if not m:
                res += e[i:]
                break
            depth, j = 0, m.end() - 1
            while j < len(e):
                if e[j] == '(':
                    depth += 1
                elif e[j] == ')':
                    depth -= 1
                    if depth == 0:
                        break
                j += 1
            call = e[m.start():j + 1]
            arg = e[m.end():j]
            if _time_only(arg):
                if call not in terms:
                    terms.append(call)
                res += e[i:m.start()] + 'pre.tt_%d' % terms.index(call)
                i = j + 1
            else:
                res += e[i:m.end()]
                i = m.end()
        out.append(res)
    return out, terms


class Emitter(object):
    """Builds the model header for one :class:`PlomModel` with context."""

    def __init__(self, model):
        if not hasattr(model, 'cac_id'):
            raise PlomModelError('the emitter needs a model with a context')
        m = self.m = model
        self._check_cac_order()
        self.names = set(m.par_sv + ([m.remainder] if m.remainder else []) + m.par_proc +
                         m.par_obs + m.par_fixed + ['x', 't', 'N'])
        self.cov_obs = [p for p in m.par_fixed if p in m.par_fixed_obs]
        self.cov_cac = [p for p in m.par_fixed if p not in m.par_fixed_obs]
        self.drift = list(m.drift_par_proc)
        self.R = len(m.proc_model)
        self.W = len(m.white_noise)

    def _check_cac_order(self):
        m = self.m
        for c, city in enumerate(m.cities_id):
            for a, age in enumerate(m.ages_id):
                k = c * m.N_AC + a
                if k >= len(m.cac_id) or m.cac_id[k] != '%s__%s' % (city, age):
                    raise PlomModelError('populations must be listed city-major with every age class')

    # ------------------------------------------------------------------ symbols
    def _proc_symmap(self):
        m = self.m
        sm = {}
        for i, s in enumerate(m.par_sv):
            sm[s] = 'xo_%s' % s
        for k, p in enumerate(m.par_proc):
            sm[p] = ('drift_%d' % self.drift.index(p)) if p in self.drift else 'e.par(%d, cac)' % k
        for k, p in enumerate(self.cov_cac):
            sm[p] = 'e.cov(%d, cac)' % k
        sm['t'] = 't'
        return sm

    def _obs_symmap(self):
        m = self.m
        sm = {'x': 'x', 't': 't'}
        for k, p in enumerate(m.par_obs):
            sm[p] = 'e.par_ts(%d, ts)' % k
        for k, p in enumerate(self.cov_obs):
            sm[p] = 'e.cov_ts(%d, ts)' % k
        return sm

    def c_expr(self, expr, symmap, drop_correct_rate=True):
        e = _sympify(expr, self.names, drop_correct_rate)
        return _Printer(symmap).doprint(e)

    # ------------------------------------------------------------------ equations
    def equations(self):
        """Rates, per-state terms and incidence terms (Ccoder.step_ode_sde)."""
        m = self.m
        rates = []
        for r in m.proc_model:
            if r['rate'] not in rates:
                rates.append(r['rate'])
        sm = self._proc_symmap()
        caches = [self.c_expr(r, sm) for r in rates]
        caches, self.time_terms = hoist_time_terms(caches) if HOIST_TIME_TERMS else (caches, [])
        univ = (UNIVERSE, m.remainder)

        def term(r):
            k = rates.index(r['rate'])
            if r['from'] in univ:
                t = 'r%d' % k
            else:
                t = 'r%d*xo_%s' % (k, r['from'])
            wn = r.get('white_noise')
            sd = None
            if wn:
                sd = self._proc_symmap()[wn['sd']] if wn['sd'] in m.par_proc else None
                if sd is None:
                    raise PlomModelError('white-noise intensity must be a process parameter')
            return {'term': t, 'noise': (wn['name'] if wn else None), 'sd': sd,
                    'dem': m.proc_model.index(r)}

        ode = dict((s, []) for s in m.par_sv)
        for r in m.proc_model:
            if r['from'] not in univ:
                d = term(r)
                d['sign'] = '-'
                ode[r['from']].append(d)
        for r in m.proc_model:
            if r['to'] not in univ:
                d = term(r)
                d['sign'] = '+'
                ode[r['to']].append(d)

        inc = []
        for defs in m.obs_var_def:
            if not isinstance(defs[0], dict):
                continue
            eq = []
            for item in defs:
                for r in m.proc_model:
                    if r['from'] == item['from'] and r['to'] == item['to'] and r['rate'] == item['rate']:
                        d = term(r)
                        d['sign'] = '+'
                        eq.append(d)
            inc.append(eq)
        return caches, ode, inc

    @staticmethod
    def _rhs(terms, variant):
        """``(eq)*dt + dem + env`` of one equation for one noise variant (eq_dem_env)."""
        no_dem = variant & 1
        no_env = variant & 2
        eq = ' '.join('%s (%s)' % (d['sign'], d['term']) for d in terms) or '0'
        s = '(%s)*dt' % eq
        if not no_dem:
            for d in terms:
                s += ' %s sqrt(%s)*dem_%d' % (d['sign'], d['term'], d['dem'])
        if not no_env:
            for d in terms:
                if d['noise']:
                    s += ' %s (%s)*%s*%s' % (d['sign'], d['term'], d['sd'], d['noise'].replace('white_noise__', 'wn_'))
        return s

    # ------------------------------------------------------------------ header
    def header(self, name):
        m = self.m
        caches, ode, inc = self.equations()
        L = []
        a = L.append
        nsv = len(m.par_sv)
        nd = len(self.drift)
        a('// Generated by plomgpu.emit for model "%s".  Do not edit.' % name)
        a('#pragma once')
        a('#include "plom_rt.h"')
        a('#include "psr_samplers.h"')
        a('namespace plomgen {')
        self._emit_inc_link_table(a)
        a('struct Model {')
        a('  static constexpr const char* NAME = "%s";' % name)
        a('  static constexpr int N_PAR_SV = %d, N_C = %d, N_AC = %d, N_CAC = %d;' % (nsv, m.N_C, m.N_AC, m.N_CAC))
        a('  static constexpr int N_TS = %d, N_TS_INC_UNIQUE = %d, N_OBS_INC = %d, N_OBS_PREV = %d;' %
          (m.N_TS, m.N_TS_INC_UNIQUE, m.N_OBS_INC, m.N_OBS_PREV))
        a('  static constexpr int N_DRIFT = %d;  // drifted parameters, N_CAC words each' % nd)
        a('  static constexpr int OFF_DRIFT = N_PAR_SV*N_CAC, OFF_INC = OFF_DRIFT + N_DRIFT*N_CAC;')
        a('  static constexpr int S = OFF_INC + N_TS_INC_UNIQUE;  // words per particle')
        a('  static constexpr int N_PAR_PROC = %d, N_PAR_OBS = %d, N_COV_CAC = %d, N_COV_TS = %d;' %
          (len(m.par_proc), len(m.par_obs), len(self.cov_cac), len(self.cov_obs)))
        a('  static constexpr int N_REAC = %d, N_WN = %d;' % (self.R, self.W))
        a('  static constexpr bool COUPLED = %s;' % ('true' if m.coupling is not None else 'false'))
        a('  static constexpr bool POP_SIZE_EQ_SUM_SV = %s;' % ('true' if m.remainder is None else 'false'))
        a('  static constexpr int COV_N = %d;  // index of N among cac covariates, -1 if none' %
          (self.cov_cac.index('N') if 'N' in self.cov_cac else -1))
        a('  // normals drawn per cac and substep for a noise variant (bit0 no dem, bit1 no env)')
        a('  static constexpr PLOM_HD int draws_per_cac(int v) { return ((v & 1) ? 0 : N_REAC) + ((v & 2) ? 0 : N_WN); }')
        # incidence word of each cac: a cac may feed several series
        a('  static constexpr int N_INC_LINKS = %d;' % self._n_inc_links())
        self._emit_inc_tables(a)
        self._emit_step(a, caches, ode, inc)
        self._emit_deriv(a, caches, ode, inc)
        self._emit_step_psr(a, caches)
        self._emit_proj2obs(a)
        self._emit_obs(a)
        a('};')
        a('}  // namespace plomgen')
        return '\n'.join(L) + '\n'

    def _inc_words(self):
        """[(incidence obs index, word index, [cac...])] in word order."""
        m = self.m
        out = []
        w = 0
        for o in range(m.N_OBS_INC):
            info = m.obs2ts[o]
            for u in range(info['n_ts_unique']):
                cacs = [c * m.N_AC + ac for (c, ac) in info['cac'][u]]
                out.append((o, w, cacs))
                w += 1
        return out

    def _n_inc_links(self):
        return sum(len(c) for (_, _, c) in self._inc_words())

    def _inc_link_rows(self):
        """(links per cac, flat [N_CAC * links] table of obs * 1024 + word, -1 after a cac's last)."""
        m = self.m
        words = self._inc_words()
        # per cac, the (obs, word) pairs it feeds, in word order
        per = [[] for _ in range(m.N_CAC)]
        for (o, w, cacs) in words:
            for c in cacs:
                per[c].append((o, w))
        nmax = max([len(p) for p in per] + [1])
        flat = []
        for p in per:
            flat += [o * 1024 + w for (o, w) in p] + [-1] * (nmax - len(p))
        return nmax, flat

    def _emit_inc_link_table(self, a):
        """The links at namespace scope: the step reads them with a run-time cac, and a
        table local to the function would be rebuilt on the stack at every call."""
        _, flat = self._inc_link_rows()
        vals = ','.join('%d' % v for v in flat)
        a('// incidence links of each cac (obs * 1024 + word, -1 after its last), read with a run-time')
        a('// cac: from constant memory on the device')
        a('#if defined(__CUDACC__)')
        a('__constant__ int kIncLinkDev[%d] = {%s};' % (len(flat), vals))
        a('#endif')
        a('static const int kIncLinkHost[%d] = {%s};' % (len(flat), vals))

    def _emit_inc_tables(self, a):
        nmax, _ = self._inc_link_rows()
        a('  static constexpr int INC_PER_CAC = %d;' % nmax)
        a('  PLOM_HD static int inc_link(int cac, int k) {')
        a('#if defined(__CUDA_ARCH__)')
        a('    return kIncLinkDev[cac * INC_PER_CAC + k];')
        a('#else')
        a('    return kIncLinkHost[cac * INC_PER_CAC + k];')
        a('#endif')
        a('  }')

    def _emit_step(self, a, caches, ode, inc):
        m = self.m
        foi_states = sorted(set(self._foi_states()))
        # values computed once per substep from the previous state (coupling)
        a('  template <class T>')
        a('  struct Pre {')
        for s in foi_states:
            a('    T yf_%s[N_CAC];' % s)
        for k in range(len(self.time_terms)):
            a('    T tt_%d;  // %s' % (k, self.time_terms[k]))
        a('    int unused;')
        a('  };')
        # one compartment-age class: rates, noises, equations, incidence
        a('  template <int V, bool DRIFT, class T, class X, class E, class IA>')
        a('  PLOM_HD static void cac_body(X& x, const int cac, const T* nz, const T t, const T dt, const E& e,')
        a('                               IA& inc_acc, const Pre<T>& pre) {')
        a('    (void)t; (void)nz; (void)pre;')
        for i, s in enumerate(m.par_sv):
            a('    const T xo_%s = x[%d*N_CAC+cac];' % (s, i))
        for k, p in enumerate(self.drift):
            pk = m.par_proc.index(p)
            a('    T drift_%d;' % k)
            a('    if (DRIFT) {')
            a('      const int g = e.drift_group(%d, cac);' % k)
            a('      T xw = T(0);')
            a('      if constexpr (X::DYNAMIC) {')
            a('        xw = x[OFF_DRIFT+%d*N_CAC+g];' % k)
            a('      } else {')
            a('        PLOM_UNROLL')
            a('        for (int gg = 0; gg < N_CAC; ++gg) if (gg == g) xw = x[OFF_DRIFT+%d*N_CAC+gg];' % k)
            a('      }')
            a('      drift_%d = e.drift_value(%d, g, xw);' % (k, k))
            a('    } else {')
            a('      drift_%d = e.par(%d, cac);' % (k, pk))
            a('    }')
        for s in foi_states:
            a('    T foi_%s = T(0);' % s)
            if m.N_CAC % 4 == 0:
                a('    PLOM_UNROLL')
                a('    for (int c2 = 0; c2 < N_CAC; c2 += 4) {')
                a('      const plomrt::V4<T> w4 = e.coupling4(cac, c2);')
                a('      foi_%s += w4.a * pre.yf_%s[c2];' % (s, s))
                a('      foi_%s += w4.b * pre.yf_%s[c2 + 1];' % (s, s))
                a('      foi_%s += w4.c * pre.yf_%s[c2 + 2];' % (s, s))
                a('      foi_%s += w4.d * pre.yf_%s[c2 + 3];' % (s, s))
                a('    }')
            else:
                a('    PLOM_UNROLL')
                a('    for (int c2 = 0; c2 < N_CAC; ++c2) foi_%s += e.coupling(cac, c2) * pre.yf_%s[c2];' % (s, s))
        for k, c in enumerate(caches):
            a('    const T r%d = %s;' % (k, c))
        a('    const T sqdt = sqrt(dt);')
        a('    (void)sqdt;')
        a('    int q = 0; (void)q;')
        for i in range(self.R):
            a('    const T dem_%d = (V & 1) ? T(0) : sqdt*nz[q++];' % i)
        for j in range(self.W):
            a('    const T wn_%d = (V & 2) ? T(0) : sqdt*nz[q++];' % j)
        for o, eq in enumerate(inc):
            a('    T incterm_%d;' % o)
            a('    switch (V) {')
            for vname, v in VARIANTS.items():
                a('      case %d: incterm_%d = %s; break;' % (v, o, self._rhs(eq, v)))
            a('    }')
        for i, s in enumerate(m.par_sv):
            a('    T f_%s;' % s)
            a('    switch (V) {')
            for vname, v in VARIANTS.items():
                a('      case %d: f_%s = xo_%s + %s; break;' % (v, s, s, self._rhs(ode[s], v)))
            a('    }')
        if inc:
            a('    PLOM_UNROLL')
            a('    for (int k = 0; k < INC_PER_CAC; ++k) {')
            a('      const int l = inc_link(cac, k);')
            a('      if (l < 0) break;')
            a('      const int o = l >> 10, w = l & 1023;')
            for o in range(len(inc)):
                a('      if (o == %d) inc_acc.add(w, incterm_%d);' % (o, o))
            a('    }')
        for i, s in enumerate(m.par_sv):
            a('    x[%d*N_CAC+cac] = (f_%s < T(0)) ? T(0) : f_%s;' % (i, s, s))
        a('  }')
        # one Euler-Maruyama substep of the whole particle
        a('  // cacs drawn together so that whole draw blocks are used (PER_BLOCK normals per block);')
        a('  // for generators of more than 2 normals per block (FP32) PLOM_MAX_DRAW_GROUP caps the')
        a('  // group, leaving part of the last block of a group unused (SEIR 20x2: 4 cacs = 9 whole')
        a('  // blocks measured 10 % faster than 1 cac = 3 blocks with 3 of their 12 normals unused)')
        a('  // without draws (Euler skeleton) a group of 4 cacs only sets the unrolling of the cac loop')
        a('  static constexpr PLOM_HD int draw_group(int nw, int per_block) {')
        a('    if (nw == 0) return N_CAC >= 4 ? 4 : 1;')
        a('    int g = 1;')
        a('    while (nw > 0 && (g * nw) % per_block != 0 && g < per_block) ++g;')
        a('    g = (nw > 0 && (g * nw) % per_block == 0 && g <= N_CAC) ? g : 1;')
        a('#if defined(PLOM_MAX_DRAW_GROUP)')
        a('    if (per_block > 2 && g > PLOM_MAX_DRAW_GROUP) g = PLOM_MAX_DRAW_GROUP;')
        a('#endif')
        a('    return g;')
        a('  }')
        a('  template <int V, bool DRIFT, class T, class X, class E, class D>')
        a('  PLOM_HD static void step(X& x, const T t, const T dt, const E& e, D& draws) {')
        a('    constexpr int NW = draws_per_cac(V);')
        a('    constexpr int G = draw_group(NW, D::PER_BLOCK);')
        a('    constexpr int NMAIN = N_CAC - (N_CAC % G);')
        a('    typename plomrt::IncAccFor<X, T, N_TS_INC_UNIQUE>::type inc_acc(x);')
        a('    inc_acc.zero();')
        a('    Pre<T> pre;')
        a('    pre.unused = 0;')
        for k, tt in enumerate(self.time_terms):
            a('    pre.tt_%d = %s;' % (k, tt))
        for s in foi_states:
            si = m.par_sv.index(s)
            a('    PLOM_UNROLL')
            a('    for (int c2 = 0; c2 < N_CAC; ++c2) {')
            a('      pre.yf_%s[c2] = x[%d*N_CAC+c2] / %s;' % (s, si, self._npop_expr('c2')))
            a('    }')
        a('    PLOM_PRAGMA_CAC')
        a('    for (int cac0 = 0; cac0 < NMAIN; cac0 += G) {')
        a('      T nz[NW * G > 0 ? NW * G : 1];')
        a('      draws.template normals<NW * G>(cac0, nz);')
        a('      PLOM_PRAGMA_GROUP')
        a('      for (int g = 0; g < G; ++g) cac_body<V, DRIFT, T>(x, cac0 + g, nz + g * NW, t, dt, e, inc_acc, pre);')
        a('    }')
        a('    PLOM_UNROLL')
        a('    for (int cac = NMAIN; cac < N_CAC; ++cac) {')
        a('      T nz[NW > 0 ? NW : 1];')
        a('      draws.template normals<NW>(cac, nz);')
        a('      cac_body<V, DRIFT, T>(x, cac, nz, t, dt, e, inc_acc, pre);')
        a('    }')
        a('    PLOM_UNROLL')
        a('    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) {')
        a('      const T f = x[OFF_INC+w] + inc_acc.get(w);')
        a('      x[OFF_INC+w] = (f < T(0)) ? T(0) : f;')
        a('    }')
        a('    if (DRIFT) {')
        a('      // Brownian walk of the drifted parameters (model_builder/C/core/drift.c:27-41)')
        a('      PLOM_UNROLL')
        a('      for (int i = 0; i < N_DRIFT; ++i) {')
        a('        const int ng = e.drift_ngroups(i);')
        a('        PLOM_UNROLL')
        a('        for (int g = 0; g < N_CAC; ++g) {')
        a('          if (g < ng) x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);')
        a('        }')
        a('      }')
        a('    }')
        a('  }')
        self._emit_step_team(a, foi_states)

    def _emit_step_team(self, a, foi_states):
        """The substep of one particle shared by a team of TM::TP threads.

        Team member `rank` takes the draw groups rank, rank + TP, ... (the same
        Philox blocks as the single-thread step, so the same draws); the
        coupling terms of the substep start are written by the team into the
        particle's shared-memory Pre; incidence partial sums are reduced over the
        team in a fixed order (TM::sum) and applied by rank 0; drift groups are
        split by rank.  Team barriers (TM::sync) separate the reads of the
        substep-start state from its updates.
        """
        m = self.m
        a('  template <int V, bool DRIFT, class T, class X, class E, class D, class TM>')
        a('  PLOM_HD static void step_team(X& x, const T t, const T dt, const E& e, D& draws, const TM& tm, Pre<T>& pre) {')
        a('    constexpr int NW = draws_per_cac(V);')
        a('    constexpr int G = draw_group(NW, D::PER_BLOCK);')
        a('    constexpr int NG = N_CAC / G;')
        a('    constexpr int NMAIN = NG * G;')
        a('    plomrt::RegIncAcc<T, N_TS_INC_UNIQUE> inc_acc;')
        a('    inc_acc.zero();')
        for s_ in foi_states:
            si = m.par_sv.index(s_)
            a('    for (int c2 = tm.rank; c2 < N_CAC; c2 += TM::TP) pre.yf_%s[c2] = x[%d*N_CAC+c2] / %s;'
              % (s_, si, self._npop_expr('c2')))
        if self.time_terms:
            a('    if (tm.rank == 0) {')
            for k, tt in enumerate(self.time_terms):
                a('      pre.tt_%d = %s;' % (k, tt))
            a('    }')
        if foi_states or self.time_terms:
            a('    tm.sync();')
        a('    PLOM_PRAGMA_CAC')
        a('    for (int gi = tm.rank; gi < NG; gi += TM::TP) {')
        a('      const int cac0 = gi * G;')
        a('      T nz[NW * G > 0 ? NW * G : 1];')
        a('      draws.template normals<NW * G>(cac0, nz);')
        a('      PLOM_UNROLL')
        a('      for (int g = 0; g < G; ++g) cac_body<V, DRIFT, T>(x, cac0 + g, nz + g * NW, t, dt, e, inc_acc, pre);')
        a('    }')
        a('    for (int cac = NMAIN + tm.rank; cac < N_CAC; cac += TM::TP) {')
        a('      T nz[NW > 0 ? NW : 1];')
        a('      draws.template normals<NW>(cac, nz);')
        a('      cac_body<V, DRIFT, T>(x, cac, nz, t, dt, e, inc_acc, pre);')
        a('    }')
        a('    PLOM_UNROLL')
        a('    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) inc_acc.v[w] = tm.sum(inc_acc.v[w]);')
        a('    tm.sync();')
        a('    if (tm.rank == 0) {')
        a('      PLOM_UNROLL')
        a('      for (int w = 0; w < N_TS_INC_UNIQUE; ++w) {')
        a('        const T f = x[OFF_INC+w] + inc_acc.v[w];')
        a('        x[OFF_INC+w] = (f < T(0)) ? T(0) : f;')
        a('      }')
        a('    }')
        a('    if (DRIFT) {')
        a('      for (int i = 0; i < N_DRIFT; ++i) {')
        a('        const int ng = e.drift_ngroups(i);')
        a('        for (int g = tm.rank; g < ng; g += TM::TP)')
        a('          x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);')
        a('      }')
        a('    }')
        a('    tm.sync();')
        a('  }')

    def _emit_deriv(self, a, caches, ode, inc):
        """Right-hand side of the deterministic skeleton (step_ode,
        model_builder/C/templates/core_template.c:215-339 with noises_off == 'ode'):
        f = dX/dt for the compartment words, the incidence words, and zero for the
        drift words (drifted parameters take their table values)."""
        m = self.m
        foi_states = sorted(set(self._foi_states()))
        a('  template <class T, class X, class F, class E>')
        a('  PLOM_HD static void deriv(const X& x, F& f, const T t, const E& e) {')
        a('    (void)t;')
        a('    T inc_acc[N_TS_INC_UNIQUE > 0 ? N_TS_INC_UNIQUE : 1];')
        a('    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) inc_acc[w] = T(0);')
        a('    Pre<T> pre;')
        a('    pre.unused = 0;')
        for k, tt in enumerate(self.time_terms):
            a('    pre.tt_%d = %s;' % (k, tt))
        for s_ in foi_states:
            si = m.par_sv.index(s_)
            a('    for (int c2 = 0; c2 < N_CAC; ++c2) pre.yf_%s[c2] = x[%d*N_CAC+c2] / %s;' % (s_, si, self._npop_expr('c2')))
        a('    for (int cac = 0; cac < N_CAC; ++cac) {')
        for i, s_ in enumerate(m.par_sv):
            a('      const T xo_%s = x[%d*N_CAC+cac];' % (s_, i))
        for k, p_ in enumerate(self.drift):
            a('      const T drift_%d = e.par(%d, cac);' % (k, m.par_proc.index(p_)))
        for s_ in foi_states:
            a('      T foi_%s = T(0);' % s_)
            a('      for (int c2 = 0; c2 < N_CAC; ++c2) foi_%s += e.coupling(cac, c2) * pre.yf_%s[c2];' % (s_, s_))
        for k, c in enumerate(caches):
            a('      const T r%d = %s;' % (k, c))
        for o, eq in enumerate(inc):
            rhs = ' '.join('%s (%s)' % (d['sign'], d['term']) for d in eq) or '0'
            a('      const T incterm_%d = %s;' % (o, rhs))
        for i, s_ in enumerate(m.par_sv):
            rhs = ' '.join('%s (%s)' % (d['sign'], d['term']) for d in ode[s_]) or '0'
            a('      f[%d*N_CAC+cac] = %s;' % (i, rhs))
        if inc:
            a('      for (int k = 0; k < INC_PER_CAC; ++k) {')
            a('        const int l = inc_link(cac, k);')
            a('        if (l < 0) break;')
            a('        const int o = l >> 10, w = l & 1023;')
            for o in range(len(inc)):
                a('        if (o == %d) inc_acc[w] += incterm_%d;' % (o, o))
            a('      }')
        a('    }')
        a('    for (int w = OFF_DRIFT; w < OFF_INC; ++w) f[w] = T(0);')
        a('    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) f[OFF_INC+w] = inc_acc[w];')
        a('  }')

    def _emit_step_psr(self, a, caches):
        """Poisson system with stochastic rates (step_psr,
        model_builder/C/templates/core_template.c:105-209; equations of
        Ccoder.step_psr / psr_multinomial / obs_inc_step_psr,
        model_builder/Ccoder.py:155-322).  Per cac: Gamma white noises (rate 1
        mean) unless NOENV; for every compartment with exits a multinomial
        split of its (integer) content into the exits and the stay, with exit
        probabilities (1 - exp(-sum h)) h / sum h, h = rate * dt; Poisson
        arrivals from outside (U, remainder); the new contents; incidence
        words summed from the split counts.  The coupling terms are those of
        the substep start, as in the SDE step."""
        m = self.m
        univ = (UNIVERSE, m.remainder)
        rates = []
        for r in m.proc_model:
            if r['rate'] not in rates:
                rates.append(r['rate'])
        sm = self._proc_symmap()
        foi_states = sorted(set(self._foi_states()))
        noises = []
        for r in m.proc_model:
            wn = r.get('white_noise')
            if wn and wn['name'] not in [n for n, _ in noises]:
                noises.append((wn['name'], sm[wn['sd']]))

        def rate_expr(r):
            k = rates.index(r['rate'])
            e = 'r%d' % k
            wn = r.get('white_noise')
            if wn:
                e = '%s*wn_%d' % (e, [n for n, _ in noises].index(wn['name']))
            return e

        a('  template <bool DRIFT, bool NOENV, class T, class X, class E, class IA>')
        a('  PLOM_HD static void psr_cac(X& x, const int cac, const T t, const T dt, const E& e,')
        a('                              typename plomrt::PsrStream<T>::type& rs, IA& inc_acc, const Pre<T>& pre) {')
        a('    (void)t; (void)pre;')
        a('    const T ddt = dt;')
        for i, s_ in enumerate(m.par_sv):
            a('    const T xo_%s = x[%d*N_CAC+cac];' % (s_, i))
        for k, p_ in enumerate(self.drift):
            pk = m.par_proc.index(p_)
            a('    T drift_%d;' % k)
            a('    if (DRIFT) {')
            a('      const int g = e.drift_group(%d, cac);' % k)
            a('      T xw = T(0);')
            a('      if constexpr (X::DYNAMIC) {')
            a('        xw = x[OFF_DRIFT+%d*N_CAC+g];' % k)
            a('      } else {')
            a('        PLOM_UNROLL')
            a('        for (int gg = 0; gg < N_CAC; ++gg) if (gg == g) xw = x[OFF_DRIFT+%d*N_CAC+gg];' % k)
            a('      }')
            a('      drift_%d = e.drift_value(%d, g, xw);' % (k, k))
            a('    } else {')
            a('      drift_%d = e.par(%d, cac);' % (k, pk))
            a('    }')
        for s_ in foi_states:
            a('    T foi_%s = T(0);' % s_)
            a('    PLOM_UNROLL')
            a('    for (int c2 = 0; c2 < N_CAC; ++c2) foi_%s += e.coupling(cac, c2) * pre.yf_%s[c2];' % (s_, s_))
        # 1: white noises
        for j, (name, sd) in enumerate(noises):
            a('    T wn_%d = T(1);' % j)
            a('    if (!NOENV) {')
            a('      const T sd = (T)(%s);' % sd)
            a('      wn_%d = plomrt::gamma(rs, ddt / (sd * sd), sd * sd) / ddt;' % j)
            a('    }')
        # 2: rates
        for k, c in enumerate(caches):
            a('    const T r%d = %s;' % (k, c))
        # 3: multinomial splits, in compartment order
        for s_ in m.par_sv:
            exits = [r for r in m.proc_model if r['from'] == s_]
            if not exits:
                continue
            K = len(exits) + 1
            a('    T inc_%s[%d];' % (s_, K))
            a('    {')
            for q, r in enumerate(exits):
                a('      const T h%d = %s * ddt;' % (q, rate_expr(r)))
            a('      const T sum = %s;' % ' + '.join('h%d' % q for q in range(len(exits))))
            a('      T p[%d];' % K)
            a('      if (sum > T(0)) {')
            a('        const T ome = T(1) - plomrt::s_exp(-sum);')
            for q in range(len(exits)):
                a('        p[%d] = ome * (h%d / sum);' % (q, q))
            a('        p[%d] = T(1)%s;' % (len(exits), ''.join(' - p[%d]' % q for q in range(len(exits)))))
            a('      } else {')
            for q in range(len(exits)):
                a('        p[%d] = T(0);' % q)
            a('        p[%d] = T(1);' % len(exits))
            a('      }')
            a('      const T xs = xo_%s;' % s_)
            a('      plomrt::multinomial<%d>(rs, xs > T(0) ? floor(xs) : T(0), p, inc_%s);' % (K, s_))
            a('    }')
        # 4: arrivals from outside
        for src in univ:
            if src is None:
                continue
            arr = [r for r in m.proc_model if r['from'] == src]
            if not arr:
                continue
            a('    T inc_%s[%d];' % (self._univ_name(src), len(arr)))
            for q, r in enumerate(arr):
                a('    inc_%s[%d] = plomrt::poisson(rs, %s * ddt);' % (self._univ_name(src), q, rate_expr(r)))
        # 5: new contents
        for i, s_ in enumerate(m.par_sv):
            exits = [r for r in m.proc_model if r['from'] == s_]
            terms = ['inc_%s[%d]' % (s_, len(exits))] if exits else ['xo_%s' % s_]
            for s2 in m.par_sv:
                for q, r in enumerate([r for r in m.proc_model if r['from'] == s2]):
                    if r['to'] == s_:
                        terms.append('inc_%s[%d]' % (s2, q))
            for src in univ:
                if src is None:
                    continue
                for q, r in enumerate([r for r in m.proc_model if r['from'] == src]):
                    if r['to'] == s_:
                        terms.append('inc_%s[%d]' % (self._univ_name(src), q))
            a('    x[%d*N_CAC+cac] = (T)(%s);' % (i, ' + '.join(terms)))
        # 6: incidence of the observed flows
        inc_terms = []
        for defs in m.obs_var_def:
            if not isinstance(defs[0], dict):
                continue
            t_ = []
            for item in defs:
                for r in m.proc_model:
                    if r['from'] == item['from'] and r['to'] == item['to'] and r['rate'] == item['rate']:
                        src = r['from']
                        same = [x for x in m.proc_model if x['from'] == src]
                        name = self._univ_name(src) if src in univ else src
                        t_.append('inc_%s[%d]' % (name, same.index(r)))
            inc_terms.append(' + '.join(t_) or 'T(0)')
        if inc_terms:
            a('    for (int k = 0; k < INC_PER_CAC; ++k) {')
            a('      const int l = inc_link(cac, k);')
            a('      if (l < 0) break;')
            a('      const int o = l >> 10, w = l & 1023;')
            for o, t_ in enumerate(inc_terms):
                a('      if (o == %d) inc_acc.add(w, %s);' % (o, t_))
            a('    }')
        a('  }')
        a('  template <bool DRIFT, bool NOENV, class T, class X, class E, class D>')
        a('  PLOM_HD static void step_psr(X& x, const T t, const T dt, const E& e, const plomrt::PhiloxKey key,')
        a('                               const uint32_t j, const uint32_t n, const uint32_t sub, D& draws) {')
        a('    typename plomrt::IncAccFor<X, T, N_TS_INC_UNIQUE>::type inc_acc(x);')
        a('    inc_acc.zero();')
        a('    Pre<T> pre;')
        a('    pre.unused = 0;')
        for k, tt in enumerate(self.time_terms):
            a('    pre.tt_%d = %s;' % (k, tt))
        for s_ in foi_states:
            si = m.par_sv.index(s_)
            a('    PLOM_UNROLL')
            a('    for (int c2 = 0; c2 < N_CAC; ++c2) pre.yf_%s[c2] = x[%d*N_CAC+c2] / %s;' % (s_, si, self._npop_expr('c2')))
        a('    for (int cac = 0; cac < N_CAC; ++cac) {')
        a('      typename plomrt::PsrStream<T>::type rs;')
        a('      rs.init(key, j, n, sub * (uint32_t)(N_CAC + 1) + (uint32_t)cac);')
        a('      psr_cac<DRIFT, NOENV, T>(x, cac, t, dt, e, rs, inc_acc, pre);')
        a('    }')
        a('    PLOM_UNROLL')
        a('    for (int w = 0; w < N_TS_INC_UNIQUE; ++w) x[OFF_INC+w] = x[OFF_INC+w] + inc_acc.get(w);')
        a('    if (DRIFT) {')
        a('      // Brownian walk of the drifted parameters (model_builder/C/core/drift.c:27-41)')
        a('      for (int i = 0; i < N_DRIFT; ++i) {')
        a('        const int ng = e.drift_ngroups(i);')
        a('        for (int g = 0; g < ng; ++g)')
        a('          x[OFF_DRIFT+i*N_CAC+g] += e.drift_vol(i, g)*sqrt(dt)*draws.drift_normal(i, g);')
        a('      }')
        a('    }')
        a('  }')

    @staticmethod
    def _univ_name(src):
        return 'U' if src == UNIVERSE else 'rem_' + src

    def _foi_states(self):
        out = []
        for r in self.m.proc_model:
            toks = tokenize(r['rate'])
            for i, t in enumerate(toks):
                if t == 'foi':
                    out.append(toks[i + 2])
        if out and self.m.coupling is None:
            raise PlomModelError('foi() needs a coupling matrix in the context')
        return out

    def _npop_expr(self, c):
        m = self.m
        if m.remainder is None:
            return '(' + '+'.join('x[%d*N_CAC+%s]' % (i, c) for i in range(len(m.par_sv))) + ')'
        return 'e.cov(COV_N, %s)' % c

    def _emit_proj2obs(self, a):
        """obs[N_TS] from a particle (core_template.c:52-102)."""
        m = self.m
        a('  template <class T, class X>')
        a('  PLOM_HD static void proj2obs(const X& x, double* obs) {')
        ind = 0
        w = 0
        for o in range(m.N_OBS_INC):
            info = m.obs2ts[o]
            for u in range(info['n_ts_unique']):
                for s in range(info['n_stream'][u]):
                    a('    obs[%d] = (double)x[OFF_INC+%d];' % (ind, w))
                    ind += 1
                w += 1
        for po in range(m.N_OBS_PREV):
            o = m.N_OBS_INC + po
            info = m.obs2ts[o]
            defs = m.obs_var_def[o]
            for u in range(info['n_ts_unique']):
                terms = []
                for (c, ac) in info['cac'][u]:
                    cac = c * m.N_AC + ac
                    for s in defs:
                        if s == m.remainder or s not in m.par_sv:
                            raise PlomModelError('prevalence of the remainder is not supported')
                        terms.append('(double)x[%d*N_CAC+%d]' % (m.par_sv.index(s), cac))
                a('    { double sum_prev = 0.0;')
                for t in terms:
                    a('      sum_prev += %s;' % t)
                for s in range(info['n_stream'][u]):
                    a('      obs[%d] = sum_prev;' % ind)
                    ind += 1
                a('    }')
        a('  }')

    def _emit_obs(self, a):
        m = self.m
        om = m.obs_model
        if om.get('distribution', 'discretized_normal') != 'discretized_normal':
            raise PlomModelError('only the discretized normal observation model is supported')
        sm = self._obs_symmap()
        mean = self.c_expr(om['mean'], sm, drop_correct_rate=False)
        var = self.c_expr(om['var'], sm, drop_correct_rate=False)
        a('  // observation model, evaluated in double (Ccoder.print_like)')
        a('  template <class E>')
        a('  PLOM_HD static double obs_mean(const double x, const int ts, const double t, const E& e) {')
        a('    typedef double T; (void)x; (void)ts; (void)t; (void)e;')
        a('    return %s;' % mean)
        a('  }')
        a('  template <class E>')
        a('  PLOM_HD static double obs_var(const double x, const int ts, const double t, const E& e) {')
        a('    typedef double T; (void)x; (void)ts; (void)t; (void)e;')
        a('    return %s;' % var)
        a('  }')


def emit_header(context, process, link, name):
    return Emitter(PlomModel(context, process, link)).header(name)
