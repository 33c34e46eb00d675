"""The builder and the emitted model checked against the reference's own code
generator (golden fixtures made by tests/golden/make_golden.py from
model_builder/Cmodel.py, Ccoder.py and Builder.py)."""

import json
import math

import numpy as np
import pytest

from plomgpu.model import PlomModel, tokenize
from plomgpu import native

import models

G = models.golden()
MODELS = sorted(G['models'])


def _ir(m):
    return {'par_sv': m.par_sv, 'remainder': m.remainder, 'par_proc': m.par_proc, 'par_obs': m.par_obs,
            'par_fixed': m.par_fixed, 'par_fixed_obs': sorted(m.par_fixed_obs),
            'drift_par_proc': m.drift_par_proc, 'vol_par_proc': m.vol_par_proc,
            'proc_model': m.proc_model, 'obs_var': m.obs_var, 'obs_var_def': m.obs_var_def,
            'white_noise': m.white_noise}


def _norm(x):
    return json.loads(json.dumps(x))


def test_tokenizer_matches_reference_unit_test():
    # model_builder/test_Cmodel.py:73-75
    assert tokenize('r0*2*correct_rate(v)') == ['r0', '*', '2', '*', 'correct_rate', '(', 'v', ')']


@pytest.mark.parametrize('key', ['m', 'm2', 'm3'])
def test_ir_matches_reference_unit_models(key):
    u = G['cmodel_unit'][key]
    m = PlomModel(u['context'], u['process'], u['link'])
    assert _norm(_ir(m)) == _norm(u['ir'])


@pytest.mark.parametrize('name', MODELS)
def test_ir_matches_reference(name):
    g = G['models'][name]
    m = PlomModel(g['context'], g['process'], g['link'])
    assert _norm(_ir(m)) == _norm(g['ir'])


@pytest.mark.parametrize('name', MODELS)
def test_settings_match_reference(name):
    g = G['models'][name]
    m = PlomModel(g['context'], g['process'], g['link'])
    mine = _norm(m.settings())
    ref = g['settings']
    assert mine['orders'] == ref['orders']
    assert mine['cst'] == ref['cst']
    assert mine['data']['obs2ts'] == ref['data']['obs2ts']
    assert mine['data']['times'] == ref['data']['times']
    assert mine['data']['data'] == ref['data']['data']
    assert mine['data']['par_fixed_values'] == ref['data']['par_fixed_values']
    assert mine['drift'] == ref['drift']
    assert sorted(mine['ind_noise_sd']) == sorted(ref['ind_noise_sd'])
    assert mine['remainder'] == ref['remainder']
    assert mine['POP_SIZE_EQ_SUM_SV'] == ref['POP_SIZE_EQ_SUM_SV']


class _StepProblem(object):
    """A one-substep descriptor holding the golden inputs of one case."""

    def __init__(self, m, case, info):
        self.J, self.n_obs = 1, 1
        self.n_sub = np.array([1], dtype=np.int32)
        self.t_sub = np.array([case['t']])
        self.t_obs = np.array([case['t']])
        self.dt = case['dt']
        self.data = np.full((1, m.N_TS), np.nan)
        P = dict(case['P'])
        for p, v in case['DRIFT'].items():
            P[p] = v  # the reference's drifted value of this step
        self.par_cac = np.array([P[p] for p in m.par_proc]).reshape(len(m.par_proc), m.N_CAC)
        self.par_ts = np.zeros((max(len(m.par_obs), 1), m.N_TS))
        for k, p in enumerate(m.par_obs):
            self.par_ts[k, :] = case['par_obs'][p]
        cov_cac = [p for p in m.par_fixed if p not in m.par_fixed_obs]
        cov_ts = [p for p in m.par_fixed if p in m.par_fixed_obs]
        self.cov_cac = np.array([case['COV'][p] for p in cov_cac]).reshape(1, len(cov_cac), m.N_CAC)
        self.cov_ts = np.zeros((1, max(len(cov_ts), 1), m.N_TS))
        for k, p in enumerate(cov_ts):
            self.cov_ts[0, k, :] = case['cov_obs'][p]
        self.coupling = None
        nd = max(len(m.drift_par_proc), 1)
        self.drift_group = np.zeros((nd, m.N_CAC), dtype=np.int32)
        self.drift_ngroups = np.ones(nd, dtype=np.int32)
        self.drift_bt = [[(0, 0, 0, 0.0, 0.0, 1.0)] * m.N_CAC for _ in range(nd)]
        self.drift_vol = np.zeros((nd, m.N_CAC))
        self.x0 = np.zeros(info.n_state)
        self.noises_off, self.filter, self.like_min, self.seed, self.precision = 0, 1, 1e-17, 0, 64


VARIANT_BITS = {'full': 0, 'no_dem_sto': 1, 'no_env_sto': 2, 'no_dem_sto_no_env_sto': 3}


@pytest.mark.parametrize('name', MODELS)
def test_emitted_step_matches_reference_equations(name):
    """One Euler-Maruyama step of every noise variant equals the reference's generated C."""
    g = G['models'][name]
    m = PlomModel(g['context'], g['process'], g['link'])
    orc = models.build_oracle(name)
    info = orc.info
    R, W = len(m.proc_model), len(m.white_noise)
    nsv = len(m.par_sv)
    worst = 0.0
    for case in g['cases']:
        sp = _StepProblem(m, case, info)
        for variant, expect in case['out'].items():
            bits = VARIANT_BITS[variant]
            x = np.zeros(info.n_state)
            for i, s in enumerate(m.par_sv):
                x[i * m.N_CAC:(i + 1) * m.N_CAC] = case['X'][s]
            x[info.off_inc:info.off_inc + m.N_TS_INC_UNIQUE] = case['inc0']
            Z = np.array(case['Z'])
            sel = {0: slice(0, R + W), 1: slice(R, R + W), 2: slice(0, R), 3: slice(0, 0)}[bits]
            normals = np.concatenate([Z[c, sel] for c in range(m.N_CAC)] + [np.zeros(max(1, m.N_CAC))])
            sp.noises_off = bits | 4  # drifted values come from the parameter table here
            y = orc.step(sp, x, case['t'], 0, normals, noises_off=bits | 4)
            for i, s in enumerate(m.par_sv):
                got = y[i * m.N_CAC:(i + 1) * m.N_CAC]
                ref = np.array(expect['X'][s])
                np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-9)
                worst = max(worst, float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))))
            np.testing.assert_allclose(y[info.off_inc:info.off_inc + m.N_TS_INC_UNIQUE], expect['inc'],
                                       rtol=1e-12, atol=1e-9)
    assert worst < 1e-12


@pytest.mark.parametrize('name', MODELS)
def test_observation_model_matches_reference(name):
    """Mean, variance and clamped discretised-normal likelihood (core_template.c:342-393)."""
    g = G['models'][name]
    m = PlomModel(g['context'], g['process'], g['link'])
    orc = models.build_oracle(name)
    info = orc.info
    for case in g['cases']:
        sp = _StepProblem(m, case, info)
        ts = case['obs_ts']
        for oc in case['obs']:
            mu, var = orc.obs_moments(sp, oc['x'], ts, case['t'])
            assert mu == pytest.approx(oc['mu'], rel=1e-14, abs=1e-300)
            assert var == pytest.approx(oc['var'], rel=1e-13, abs=1e-300)
            like = orc.like(oc['y'], mu, var, 1e-17)
            assert like == pytest.approx(oc['like'], rel=1e-9, abs=1e-17)


@pytest.mark.parametrize('name', ['noise'])
def test_prevalence_observation_matches_reference(name):
    """proj2obs prevalence series = sum over the series' populations of the generated expression."""
    g = G['models'][name]
    m = PlomModel(g['context'], g['process'], g['link'])
    orc = models.build_oracle(name)
    info = orc.info
    o_prev = m.N_OBS_INC
    for case in g['cases']:
        x = np.zeros(info.n_state)
        for i, s in enumerate(m.par_sv):
            x[i * m.N_CAC:(i + 1) * m.N_CAC] = case['X'][s]
        obs = orc.proj2obs(x)
        k = sum(sum(m.obs2ts[o]['n_stream']) for o in range(o_prev))
        info_o = m.obs2ts[o_prev]
        for u in range(info_o['n_ts_unique']):
            cacs = [c * m.N_AC + a for (c, a) in info_o['cac'][u]]
            expect = sum(case['prev'][0][c] for c in cacs)
            for _s in range(info_o['n_stream'][u]):
                assert obs[k] == pytest.approx(expect, rel=1e-15)
                k += 1
