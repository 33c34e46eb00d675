"""CPU tests: the C ABI library loads and exports its header, the host-side
parameter / time / covariate logic, and known answers of the oracle."""

import ctypes
import math
import os
import re

import numpy as np
import pytest

import models
from plomgpu import native, problem, theta, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, 'include', 'plomgpu.h')).read()
    return sorted(set(re.findall(r'\b(plomgpu_\w+)\s*\(', text)))


def test_header_symbols_are_bound():
    assert header_symbols() == sorted(native.API_SYMBOLS)


def test_failure_boundary_is_exact():
    """The filters fail a particle when loglik <= b, b the largest double with
    exp(b) <= LIKE_MIN^N_TS (host code of the library, no GPU): on both sides
    of b the host's exp decides as weight() does (smc.c:44), including
    thresholds that underflow to zero and the all-survive edge."""
    import math
    models.build_gpu('sir')
    lib = native.load(models.lib_name('sir'))
    for like_min, n_ts in ((1e-17, 1), (1e-17, 2), (1e-17, 20), (1e-300, 3), (0.5, 1), (1e-5, 7)):
        thresh = like_min ** n_ts
        b = lib.plomgpu_debug_fail_boundary(thresh)
        assert math.isfinite(b)
        assert math.exp(b) <= thresh
        assert math.exp(math.nextafter(b, math.inf)) > thresh
    assert lib.plomgpu_debug_fail_boundary(0.0) < -700.0
    assert lib.plomgpu_debug_fail_boundary(math.inf) == math.inf


@pytest.mark.parametrize('name', ['sir', 'seir3'])
def test_library_loads_and_exports_every_symbol(name):
    path = models.build_gpu(name)
    lib = ctypes.CDLL(path)
    for sym in header_symbols():
        assert hasattr(lib, sym), sym
    eng = native.Engine(models.lib_name(name))
    m = models.plom_model(name)
    info = eng.info
    assert info.n_cac == m.N_CAC and info.n_ts == m.N_TS and info.n_par_sv == len(m.par_sv)
    assert info.n_state == len(m.par_sv) * m.N_CAC + len(m.drift_par_proc) * m.N_CAC + m.N_TS_INC_UNIQUE
    assert eng.draws_per_substep(0) == m.N_CAC * (len(m.proc_model) + len(m.white_noise))
    assert eng.draws_per_substep(3) == 0


def test_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip('a GPU is present')
    except ImportError:
        pass
    eng = models.engine('sir')
    p = models.make_problem('sir', J=16, dt=1.0)
    with pytest.raises(native.PlomGpuError) as e:
        eng.smc(p)
    assert e.value.code in (2, 5)


def test_bad_descriptor_is_rejected():
    eng = models.engine('sir')
    p = models.make_problem('sir', J=16, dt=1.0)
    p.J = 0
    with pytest.raises(native.PlomGpuError) as e:
        eng.smc(p)
    assert e.value.code == 1


# ------------------------------------------------------------------ host logic
def test_units_and_transforms():
    # rate_as_duration 5 days in data unit days -> 1/(1e-5 + 5) (transform.c:462-481)
    r = theta.Router('v', {'unit': 'D', 'type': 'rate_as_duration', 'transformation': 'log',
                           'group': {'all': {'min': {'value': 5}, 'max': {'value': 5}, 'guess': {'value': 5}}}},
                     {'group': [{'id': 'all', 'population_id': ['a']}]}, ['a'], 'population_id')
    assert r.natural(0) == pytest.approx(1.0 / (1e-5 + 5.0), rel=1e-15)
    # a rate per year in day units
    assert theta.get_multiplier('D', {'unit': 'Y'}) == pytest.approx(1.0 / 365.0)
    # logit round trip and its clamps
    for x in (1e-20, 0.3, 0.999999999999):
        z = theta.f_forward('logit', x, 0, 0)
        back = theta.back_transform(z, (2, 0, 0, 0.0, 0.0, 1.0))
        assert back == pytest.approx(min(max(x, theta.ZERO_LOG), theta.ONE_LOGIT), rel=1e-9)
    # logit_ab stays in [a, b]
    for z in (-50.0, -1.0, 0.0, 2.0, 50.0):
        v = theta.back_transform(z, (3, 0, 0, 2.0, 7.0, 1.0))
        assert 2.0 <= v <= 7.0


def test_dt_rounding_and_substeps():
    assert problem.round_dt(0.3) == 1.0 / 3.0
    assert problem.round_dt(1.0) == 1.0
    # replaying ``while (t < t1) t += dt`` (prediction_util.c:275-287): 0.1 accumulates
    # rounding and gives one extra step over 7 days
    assert len(problem.substep_times(0, 7, 1.0)) == 7
    n = len(problem.substep_times(0, 7, 0.1))
    t, k = 0.0, 0
    while t < 7:
        t += 0.1
        k += 1
    assert n == k


def test_natural_cubic_spline_matches_definition():
    x = [0.0, 7.0, 14.0, 21.0, 35.0, 50.0]
    y = [1.0, 3.0, 2.0, 5.0, 4.0, 4.5]
    sp = problem.Spline(x, y)
    for xi, yi in zip(x, y):
        assert sp(xi) == pytest.approx(yi, abs=1e-12)
    # second derivative vanishes at the ends and is continuous inside
    h = 1e-4
    d2 = lambda t: (sp(t + h) - 2 * sp(t) + sp(t - h)) / h ** 2
    assert abs(d2(0.0 + 2 * h)) < 1e-3 and abs(d2(50.0 - 2 * h)) < 1e-3
    assert d2(7.0 - 1e-3) == pytest.approx(d2(7.0 + 1e-3), abs=5e-3)
    lin = problem.Spline([0.0, 10.0], [1.0, 3.0])
    assert lin(5.0) == pytest.approx(2.0)
    assert problem.Spline([0.0], [4.0])(123.0) == 4.0


def test_initial_conditions_and_tables():
    p = models.make_problem('sir', J=8, dt=1.0)
    assert p.x0[:3] == pytest.approx([4e5, 100.0, 599900.0])
    assert p.x0[3] == 0.0
    m = p.model
    assert p.par_cac.shape == (len(m.par_proc), m.N_CAC)
    assert p.cov_cac.shape[0] == int(p.n_sub.sum())


# ------------------------------------------------------------------ oracle known answers
def test_systematic_sampling_known_answer():
    orc = models.build_oracle('sir')
    likes = [0.1, 0.2, 0.3, 0.4]
    w, sel, ll, ess, fail = orc.weight_and_resample(likes, U=0.5 / 4)
    # points 0.125, 0.375, 0.625, 0.875 against cumulative 0.1, 0.3, 0.6, 1.0
    assert list(sel) == [1, 2, 3, 3]
    assert ll == pytest.approx(math.log(1.0 / 4))
    assert ess == pytest.approx(1.0 / (0.01 + 0.04 + 0.09 + 0.16))
    assert fail == 0
    assert w == pytest.approx([0.1, 0.2, 0.3, 0.4])


def test_weight_failure_rule_known_answer():
    orc = models.build_oracle('sir')   # one series: failure iff like <= LIKE_MIN
    likes = [1e-17, 1e-17, 1e-17]
    w, sel, ll, ess, fail = orc.weight_and_resample(likes, U=0.1)
    assert fail == 1 and list(sel) == [0, 1, 2] and ess == 0.0
    assert ll == pytest.approx(math.log(1e-17))
    likes = [1e-17, 2e-17, 0.0]
    w, sel, ll, ess, fail = orc.weight_and_resample(likes, U=0.1)
    assert fail == 0 and list(sel) == [1, 1, 1]


@pytest.mark.parametrize('J', [1, 7, 1000, 12345, 1 << 17])
def test_systematic_closed_form_matches_sequential_additions(J):
    orc = models.build_oracle('sir')
    rng = np.random.default_rng(J)
    inc = 1.0 / J
    for U in [0.0, 5e-324, inc * 1e-9, np.nextafter(inc, 0.0)] + list(rng.uniform(0, inc, 20)):
        np.testing.assert_array_equal(orc.systematic_points(U, J, table=True), orc.systematic_points(U, J))


def test_oracle_threads_do_not_change_results():
    orc = models.build_oracle('seir3')
    p = models.make_problem('seir3', J=300, dt=1.0, precision=64, seed=9)
    a = orc.smc(p, n_threads=1, ancestors=True)
    b = orc.smc(p, n_threads=4, ancestors=True)
    assert a.loglik == b.loglik
    np.testing.assert_array_equal(a.ancestors, b.ancestors)


def test_oracle_crn_is_deterministic_and_sensitive():
    orc = models.build_oracle('sir_short')
    p = models.make_problem('sir_short', J=200, dt=1.0, precision=64)
    D = orc.draws_per_substep(0)
    rng = np.random.default_rng(1)
    z = rng.standard_normal(p.J * int(p.n_sub.sum()) * D)
    u = rng.uniform(size=p.n_obs)
    a = orc.smc(p, crn_normals=z, crn_uniforms=u)
    b = orc.smc(p, crn_normals=z, crn_uniforms=u)
    assert a.loglik == b.loglik
    z2 = z.copy()
    z2[0] += 1.0
    assert orc.smc(p, crn_normals=z2, crn_uniforms=u).loglik != a.loglik


# ------------------------------------------------------------------ filtered summaries (oracle)
def test_ci95_known_answer():
    """get_CI95 (model_builder/C/core/hat.c:28-57): the value at which the sorted running weight reaches the level."""
    orc = models.build_oracle('sir')
    v = [3.0, 1.0, 2.0, 4.0]
    w = [0.1, 0.02, 0.5, 0.38]
    # sorted 1 (0.02), 2 (0.52), 3 (0.62), 4 (1.0)
    assert orc.ci95(v, w) == (2.0, 4.0)
    # equal weights: 40 values, the running sum of 1/40 reaches 0.025 at the first value
    vals = np.arange(40.0)[::-1].copy()
    lo, hi = orc.ci95(vals)
    assert lo == 0.0
    # 0.975 * 40 = 39 terms of 1/40 summed in sequence
    cum, k = 0.0, 0
    while cum < 0.975:
        cum += 1.0 / 40
        k += 1
    assert hi == float(k - 1)


def test_oracle_summaries_are_consistent():
    """Summaries of the oracle's filter: ordered intervals, a constant start, the remainder identity."""
    orc = models.build_oracle('sir')
    p = models.make_problem('sir', J=300, dt=1.0, precision=64, seed=3)
    out = orc.smc(p, hat=True)
    h = out.hat
    assert h.shape == (p.n_obs + 1, orc.n_hat, 3)
    assert np.all(h[:, :, 0] <= h[:, :, 2])
    # time 0: every particle starts from the same state
    np.testing.assert_allclose(h[0, :, 0], h[0, :, 2])
    assert np.all(np.isfinite(out.pred_res[:, :, 0]))  # res is 0/0 = nan once the epidemic is over, as in the reference
    # a model with a remainder: its rows are N(t) minus the summed states
    orc = models.build_oracle('noise')
    p = models.make_problem('noise', J=200, dt=1.0, precision=64, seed=3)
    h = orc.smc(p, hat=True).hat
    info = orc.info
    nc, nsv = info.n_cac, info.n_par_sv * info.n_cac
    states = h[:, :nsv, 1].reshape(len(h), info.n_par_sv, nc).sum(axis=1)
    np.testing.assert_allclose(h[:, nsv:nsv + nc, 1], p.pop_size - states, rtol=1e-9)


def test_mif_components_per_group():
    """A parameter fitted per group gives one component per group; its slot is -2 and the
    per-population / per-series table names the component of every member."""
    from plomgpu import mif
    from plomgpu.native import MifDescHolder
    p = models.make_problem('noise', J=10, dt=1.0, precision=64)
    comp = mif.components(p, names=['r0', 'v', 'phi'])
    names = [(c['name'], c['g']) for c in comp]
    assert names == [('r0', 0), ('r0', 1), ('v', 0), ('phi', 0), ('phi', 1)]
    m = p.model
    h = MifDescHolder(1, [(c['kind'], c['index'], c['bt'], True, c['members']) for c in comp],
                      len(m.par_proc), len(m.par_obs), m.N_CAC, m.N_TS)
    r0, v, phi = m.par_proc.index('r0'), m.par_proc.index('v'), m.par_obs.index('phi')
    assert h.proc_slot[r0] == -2 and h.proc_slot[v] == 2
    assert list(h.proc_cac[r0]) == [0, 1]
    assert h.obs_slot[phi] == -2 and list(h.obs_ts[phi]) == [3, 4, 3, 3]
    orc = models.build_oracle('noise')
    import numpy as np
    th = np.array([[c['theta0'] for c in comp]])
    Q, T = len(comp), p.n_obs
    ll, nf, bart, vt = orc.mif_iteration(p, h, th, np.full(Q, 0.05), np.full((T, Q), 0.01), np.zeros((T, Q)), 3)
    assert np.isfinite(ll).all()


def test_single_precision_log_density_matches_double():
    """The FP32 particle states' discretised-normal log-density: narrow intervals (sd >= 20) by the midpoint
    expansion, wide ones by tail-aware erfc; counts and means up to 1e7.  Against tail-accurate values (the
    double version, a difference of two CDFs like the reference's, loses the upper tail to cancellation below
    about 1e-12) and against the double version where that one is accurate."""
    from scipy import stats
    orc = models.build_oracle('sir')
    like_min = 1e-17
    y, mu, var = [], [], []
    for yy in [0.0, 1.0, 3.0, 17.0, 250.0, 4.0e3, 1.0e5, 2.5e6, 1.0e7]:
        for sd in [0.3, 0.7, 1.0, 2.5, 7.0, 19.9, 20.0, 20.1, 55.0, 300.0, 4.0e3, 1.5e5]:
            for k in np.linspace(-9.0, 9.0, 37):
                m = yy + k * sd
                if m < 0.0:
                    continue
                y.append(yy)
                mu.append(m)
                var.append(sd * sd)
    y, mu, var = np.array(y), np.array(mu), np.array(var)
    o64, o32, f64, f32 = orc.log_like_terms(y, mu, var, like_min)
    sd = np.sqrt(var)
    lo, hi = (y - 0.5 - mu) / sd, (y + 0.5 - mu) / sd
    truth = np.where(y > 0, np.where(lo >= 0, stats.norm.sf(lo) - stats.norm.sf(hi),
                                     stats.norm.cdf(hi) - stats.norm.cdf(lo)), stats.norm.cdf(hi))
    ok = truth > 10 * like_min
    assert ok.sum() > 2500
    assert np.all(f32[ok] == 0)
    assert np.abs(o32[ok] - np.log(truth[ok])).max() < 5e-5
    accurate = ok & (o64 > math.log(1e-12))
    assert accurate.sum() > 2000
    assert np.abs(o32[accurate] - o64[accurate]).max() < 5e-5
    # below the floor both clamp to it
    under = truth < 0.1 * like_min
    assert np.all(f32[under] == 1) and np.all(o32[under] == math.log(like_min))


def test_oracle_interval_from_cloud_equals_interval_in_filter():
    """One interval run alone from the resampled particles of the interval
    before (x0_particles) equals the same interval inside the whole filter,
    with the same CRN draws: the basis of the conditional precision-error
    measurement."""
    orc = models.build_oracle('seir3')
    p = models.make_problem('seir3', J=200, dt=1.0, precision=64, seed=3, nb_obs=6)
    D = orc.draws_per_substep(0)
    rng = np.random.Generator(np.random.Philox(78))
    z = rng.standard_normal(p.J * int(p.n_sub.sum()) * D)
    u = rng.uniform(size=p.n_obs)
    full = orc.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True)
    off_inc = orc.info.off_inc
    for n in (1, 3, 5):
        cloud = full.x_pred[n - 1][:off_inc, full.ancestors[n - 1]]
        sub0 = int(p.n_sub[:n].sum())
        zn = z[p.J * sub0 * D:p.J * (sub0 + int(p.n_sub[n])) * D]
        o = orc.smc(p.interval_problem(n, cloud), crn_normals=zn, crn_uniforms=u[n:n + 1], ancestors=True)
        assert o.llike_n[0] == full.llike_n[n]
        np.testing.assert_array_equal(o.ancestors[0], full.ancestors[n])
    # the replicated cloud is the plain initial particle
    rep = np.repeat(p.x0[:off_inc, None], p.J, axis=1)
    q = p.interval_problem(0, rep)
    zn = z[:p.J * int(p.n_sub[0]) * D]
    a = orc.smc(q, crn_normals=zn, crn_uniforms=u[:1])
    assert a.llike_n[0] == full.llike_n[0]


def test_interval_problem_rejects_bad_cloud():
    p = models.make_problem('sir', J=16, dt=1.0, nb_obs=4)
    q = p.interval_problem(2, np.zeros((2, 16)))
    with pytest.raises(ValueError):
        native.DescHolder(q)
    with pytest.raises(ValueError):
        p.interval_problem(4)
