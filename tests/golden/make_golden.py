"""Generates the golden fixtures of tests/golden/ from the reference's own code.

Run in a container that holds the reference checkout:

    python tests/golden/make_golden.py /path/to/reference

The reference's model builder (model_builder/Cmodel.py, Ccoder.py,
Context.py, Builder.py) is Python 2 with a Django dependency; it is loaded
here with a minimal source shim (print statements, ``iteritems``, list-valued
``map``/``zip``, non-strict ``sympy.ccode``, stub Django modules) and run on:

* the in-memory models of the reference's own unit tests (model_builder/test_Cmodel.py:7-70);
* the example models ``noise`` and ``drift`` (model_builder/example/);
* the ``sir`` workload and ``seir_local`` (the SEIR workload with the
  force of infection restricted to the own population, the part of the
  coupled model the reference language can express).

Recorded per model: the parsed model (``Cmodel``), the settings document
(``PlomModelBuilder.make_settings_json``), the generated equations
(``Ccoder.step_ode_sde``, ``print_like``, ``print_obs_prev``, and the
Poisson-system code of ``step_psr``, ``psr_multinomial`` and
``obs_inc_step_psr``) and, for seeded
random inputs, the numbers those generated C expressions produce for one
Euler-Maruyama step of every noise variant and for the observation model.
The C expressions are evaluated in IEEE double through a mechanical
translation to Python (same operator order; ``gsl_cdf_gaussian_P`` as
0.5*erfc(-z/sqrt(2))).  The fixtures hold only numbers and strings produced
by the reference's code, never its source.
"""

import copy
import json
import math
import os
import re
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, 'iterated-inference-pipeline_b200'))


def _stub_django():
    for name in ('django', 'django.conf', 'django.template', 'django.template.loader'):
        sys.modules[name] = types.ModuleType(name)
    sys.modules['django.conf'].settings = types.SimpleNamespace(configured=True)
    sys.modules['django.template'].Context = dict
    sys.modules['django.template.loader'].get_template = lambda *a, **k: None


def load_reference(ref_root):
    """Imports Cmodel, Ccoder, Context and Builder from the reference under the shim."""
    import sympy
    mb = os.path.join(ref_root, 'model_builder')
    _stub_django()
    mods = {}

    def load(name):
        src = open(os.path.join(mb, name + '.py')).read()
        src = re.sub(r"^(\s*)print (.*)$", r"\1print(\2)", src, flags=re.M)
        src = src.replace('.iteritems()', '.items()')
        src = re.sub(r'(?<![\w.])map\(', 'list_map(', src)
        src = re.sub(r'(?<![\w.])zip\(', 'list_zip(', src)
        mod = types.ModuleType(name)
        mod.__dict__['__file__'] = os.path.join(mb, name + '.py')
        mod.__dict__['list_map'] = lambda *a: list(map(*a))
        mod.__dict__['list_zip'] = lambda *a: list(zip(*a))
        sys.modules[name] = mod
        exec(compile(src, os.path.join(mb, name + '.py'), 'exec'), mod.__dict__)
        if 'ccode' in mod.__dict__:
            mod.__dict__['ccode'] = lambda e, **k: '\n'.join(
                l for l in sympy.ccode(e, strict=False, **k).splitlines() if not l.startswith('/*'))
        mods[name] = mod
        return mod

    load('Cmodel')
    load('Ccoder')
    load('Context')
    load('Builder')
    return mods


# ------------------------------------------------------------------ C -> Python
def c_to_py(expr):
    e = expr
    e = re.sub(r'X\[ORDER_(\w+)\*N_CAC\+cac\]', r"X['\1']", e)
    e = re.sub(r'_r\[cac\]\[(\d+)\]', r'R[\1]', e)
    e = re.sub(r'_sf\[cac\]\[(\d+)\]', r'SF[\1]', e)
    e = re.sub(r'par\[ORDER_(\w+)\]\[routers\[ORDER_\w+\]->map\[(cac|ts)\]\]', r"P['\1']", e)
    e = re.sub(r'gsl_spline_eval\(p_calc->spline\[ORDER_(\w+)\]\[(cac|ts)\],t,p_calc->acc\[ORDER_\w+\]\[(cac|ts)\]\)',
               r"COV['\1']", e)
    e = re.sub(r'drifted\[ORDER_drift__par_proc__(\w+)\]\[cac\]', r"DRIFT['\1']", e)
    e = re.sub(r'(dem_sto__\d+|white_noise__\d+)\[cac\]', r"NZ['\1']", e)
    e = e.replace('M_PI', 'math.pi')
    e = re.sub(r'(?<![\w.])sqrt\(', 'math.sqrt(', e)
    e = re.sub(r'(?<![\w.])pow\(', 'math.pow(', e)
    e = re.sub(r'(?<![\w.])sin\(', 'math.sin(', e)
    e = re.sub(r'(?<![\w.])cos\(', 'math.cos(', e)
    e = re.sub(r'(\d)\.(?!\d)', r'\1.0', e)
    return e


def phi(z):
    return 0.5 * math.erfc(-z * 0.70710678118654752440)


def ref_like(y, mu, var, like_min):
    sd = math.sqrt(var)
    if y > 0.0:
        like = phi((y + 0.5 - mu) / sd) - phi((y - 0.5 - mu) / sd)
    else:
        like = phi((y + 0.5 - mu) / sd)
    if math.isinf(like) or math.isnan(like) or like < 0.0:
        return like_min
    return like_min if like <= like_min else like


# ------------------------------------------------------------------ fixtures
def ir_of(m):
    return {'par_sv': m.par_sv, 'remainder': m.remainder, 'par_proc': m.par_proc, 'par_obs': m.par_obs,
            'par_fixed': m.par_fixed, 'par_fixed_obs': sorted(m.par_fixed_obs),
            'drift_par_proc': m.drift_par_proc, 'vol_par_proc': m.vol_par_proc,
            'proc_model': m.proc_model, 'obs_var': m.obs_var, 'obs_var_def': m.obs_var_def,
            'white_noise': m.white_noise}


def step_cases(ref, ctx, proc, link, n_cases, rng):
    """Golden one-step results of the reference's generated equations."""
    from plomgpu.model import PlomModel
    mine = PlomModel(ctx, proc, link)
    sode = ref.step_ode_sde()
    caches = [c_to_py(c) for c in sode['caches']]
    sfs = [c_to_py(c) for c in sode['sf']]
    like = ref.print_like()
    mean_py, var_py = c_to_py(like['mean']), c_to_py(like['var'])
    prev_py = [c_to_py(p) for p in ref.print_obs_prev()]
    N_CAC = mine.N_CAC
    par_sv = ref.par_sv
    cov_cac = [p for p in ref.par_fixed if p not in ref.par_fixed_obs]
    noises_all = ['dem_sto__%d' % i for i in range(len(ref.proc_model))] + [w['name'] for w in ref.white_noise]
    cases = []
    for _ in range(n_cases):
        dt = float(rng.choice([1.0, 0.5, 0.25]))
        t = float(rng.uniform(0.0, 400.0))
        X = dict((s, [float(rng.uniform(1.0, 5e4)) for _ in range(N_CAC)]) for s in par_sv)
        P = dict((p, [float(rng.uniform(0.05, 2.0)) for _ in range(N_CAC)]) for p in ref.par_proc)
        COV = dict((p, [float(rng.uniform(0.5, 1.5)) * (2e5 if p == 'N' else 1e-3) for _ in range(N_CAC)])
                   for p in cov_cac)
        DRIFT = dict((p, [float(rng.uniform(0.5, 2.0)) for _ in range(N_CAC)]) for p in ref.drift_par_proc)
        Z = [[float(rng.standard_normal()) for _ in noises_all] for _ in range(N_CAC)]
        inc0 = [float(rng.uniform(0.0, 100.0)) for _ in range(mine.N_TS_INC_UNIQUE)]
        out = {}
        for variant, func in sode['func'].items():
            if variant == 'ode':
                continue
            newX = dict((s, [0.0] * N_CAC) for s in par_sv)
            terms = []  # per cac, per incidence obs
            for cac in range(N_CAC):
                env = {'math': math, 'dt': dt, 't': t,
                       'X': dict((s, X[s][cac]) for s in par_sv),
                       'P': dict((p, P[p][cac]) for p in P),
                       'COV': dict((p, COV[p][cac]) for p in COV),
                       'DRIFT': dict((p, DRIFT[p][cac]) for p in DRIFT)}
                env['SF'] = [eval(c, env) for c in sfs]
                env['R'] = [eval(c, env) for c in caches]
                env['NZ'] = dict((nm, math.sqrt(dt) * Z[cac][k]) for k, nm in enumerate(noises_all))
                for eq in func['proc']['system']:
                    s = par_sv[eq['index']]
                    f = eval('X[%r] + %s' % (s, c_to_py(eq['eq'])), env)
                    newX[s][cac] = 0.0 if f < 0.0 else f
                terms.append(dict((o['index'], eval(c_to_py(o['eq']), env)) for o in func['obs']))
            inc = []
            w = 0
            for o in range(mine.N_OBS_INC):
                info = mine.obs2ts[o]
                for u in range(info['n_ts_unique']):
                    s = 0.0
                    for (c, a) in info['cac'][u]:
                        s += terms[c * mine.N_AC + a][o]
                    f = inc0[w] + s
                    inc.append(0.0 if f < 0.0 else f)
                    w += 1
            out[variant] = {'X': newX, 'inc': inc}
        # observation model at a few points
        obs_cases = []
        ts = int(rng.integers(0, mine.N_TS))
        par_obs = dict((p, float(rng.uniform(0.05, 0.95))) for p in ref.par_obs)
        cov_obs = dict((p, float(rng.uniform(0.5, 1.0))) for p in ref.par_fixed_obs)
        for _k in range(4):
            x = float(rng.uniform(0.0, 300.0))
            y = float(rng.integers(0, 300))
            env = {'math': math, 'x': x, 't': t, 'P': par_obs, 'COV': cov_obs}
            mu = eval(mean_py, env)
            var = eval(var_py, env)
            obs_cases.append({'x': x, 'y': y, 'mu': mu, 'var': var, 'like': ref_like(y, mu, var, 1e-17)})
        prev = []
        for pexpr in prev_py:
            prev.append([eval(pexpr, {'math': math, 'X': dict((s, X[s][c]) for s in par_sv)}) for c in range(N_CAC)])
        cases.append({'dt': dt, 't': t, 'X': X, 'P': P, 'COV': COV, 'DRIFT': DRIFT, 'Z': Z, 'inc0': inc0,
                      'out': out, 'obs_ts': ts, 'par_obs': par_obs, 'cov_obs': cov_obs, 'obs': obs_cases,
                      'prev': prev})
    return {'caches': sode['caches'], 'sf': sode['sf'], 'func': sode['func'], 'like': like, 'obs_prev': ref.print_obs_prev(),
            'noises': noises_all, 'cases': cases}


def seir_local():
    from plomgpu import workloads
    ctx, proc, link, theta = workloads.seir20x2(n_obs=10, n_pop=3)
    proc = copy.deepcopy(proc)
    for r in proc['model']:
        r['rate'] = r['rate'].replace('foi(I)', 'I/N')
    ctx = dict(ctx)
    ctx.pop('coupling', None)
    return ctx, proc, link, theta


def main(ref_root):
    import numpy as np
    mods = load_reference(ref_root)
    Cmodel, Ccoder, Builder = mods['Cmodel'].Cmodel, mods['Ccoder'].Ccoder, mods['Builder'].PlomModelBuilder
    rng = np.random.Generator(np.random.Philox(20240601))
    from plomgpu import workloads

    fixtures = {}
    # unit-test models of model_builder/test_Cmodel.py (rebuilt from its setUp)
    src = open(os.path.join(ref_root, 'model_builder', 'test_Cmodel.py')).read()
    ns = {}
    setup = src[src.index('        m = {'):src.index('        self.m = Cmodel')]
    setup = '\n'.join(l[8:] for l in setup.splitlines())
    exec(setup, {'copy': copy}, ns)
    unit = {}
    for key in ('m', 'm2', 'm3'):
        cm = Cmodel(ns['c'], ns[key], ns['l'])
        unit[key] = {'process': ns[key], 'context': ns['c'], 'link': ns['l'], 'ir': ir_of(cm)}
    fixtures['cmodel_unit'] = unit

    models = {}
    ex = os.path.join(ref_root, 'model_builder', 'example')
    for name in ('noise', 'drift'):
        models[name] = [json.load(open(os.path.join(ex, name, f)))
                        for f in ('context.json', 'process.json', 'link.json', 'theta.json')]
    models['sir'] = workloads.sir(n_obs=6)
    models['seir_local'] = seir_local()

    out_models = {}
    for name, (c, p, l, th) in models.items():
        ref = Ccoder(c, p, l)
        b = Builder('/tmp/plom_golden_%s' % name, c, p, l)
        settings = json.loads(b.make_settings_json())
        entry = {'context': c, 'process': p, 'link': l, 'theta': th, 'ir': ir_of(ref), 'settings': settings,
                 'ts_id': b.ts_id, 'cac_id': b.cac_id}
        entry.update(step_cases(ref, c, p, l, 6, rng))
        # Poisson-system-with-stochastic-rates code generation (Ccoder.step_psr,
        # psr_multinomial, obs_inc_step_psr)
        psr = ref.step_psr()
        entry['psr'] = {'caches': list(psr['caches']), 'code': psr['code'], 'poisson': list(psr['poisson']),
                        'update': psr['update'], 'multinomial': ref.psr_multinomial(),
                        'obs_inc': ref.obs_inc_step_psr()}
        out_models[name] = entry
    fixtures['models'] = out_models
    path = os.path.join(HERE, 'reference_codegen.json')
    with open(path, 'w') as f:
        json.dump(fixtures, f, indent=0, sort_keys=True)
    print(path, os.path.getsize(path))


if __name__ == '__main__':
    # the reference iterates over sets when it orders its rate caches: fix the
    # string hash so that the fixture is reproducible
    if os.environ.get('PYTHONHASHSEED') != '0':
        os.execve(sys.executable, [sys.executable] + sys.argv, dict(os.environ, PYTHONHASHSEED='0'))
    if len(sys.argv) != 2:
        sys.exit('usage: python tests/golden/make_golden.py /path/to/reference')
    main(sys.argv[1])
