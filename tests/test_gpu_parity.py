"""GPU engine (through the C ABI) against the FP64 CPU oracle.

* CRN mode: both sides consume the same injected normals and resampling
  uniforms; FP64 state.  Trajectories within 1e-6 relative (observed ~1e-13),
  ancestors bit-exact, log-likelihood within 1e-9 relative.
* Deterministic Euler skeleton (no noise) in FP64: within 1e-10 relative.
* Philox mode in FP64: the same counter-based streams on both sides.
* FP32 production mode: the log-likelihood estimator over replicates has the
  oracle's mean and variance within Monte Carlo error.
"""

import numpy as np
import pytest

import models

pytestmark = pytest.mark.gpu

CRN_CASES = [('sir', 1000, 1.0, 0), ('sir_short', 777, 0.5, 0), ('noise', 300, 1.0, 0), ('drift', 257, 1.0, 0),
             ('seir3', 500, 1.0, 0), ('sir', 400, 1.0, 1), ('sir', 400, 1.0, 2), ('noise', 200, 1.0, 3),
             ('drift', 128, 1.0, 4)]


def crn_draws(problem, D, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    total = problem.J * int(np.sum(problem.n_sub)) * D
    return rng.standard_normal(total), rng.uniform(0.0, 1.0, size=problem.n_obs)


@pytest.mark.parametrize('name,J,dt,noises_off', CRN_CASES)
def test_crn_parity(name, J, dt, noises_off):
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=J, dt=dt, noises_off=noises_off, precision=64, seed=11)
    D = eng.draws_per_substep(noises_off)
    assert D == orc.draws_per_substep(noises_off)
    z, u = crn_draws(p, D, 1234 + J)
    g = eng.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True, x_final=True)
    o = orc.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True, x_final=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    np.testing.assert_allclose(g.x_pred, o.x_pred, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(g.x_final, o.x_final, rtol=1e-6, atol=1e-9)
    assert g.n_all_fail == o.n_all_fail
    np.testing.assert_allclose(g.llike_n[:p.n_obs], o.llike_n[:p.n_obs], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(g.ess_n[:p.n_obs], o.ess_n[:p.n_obs], rtol=1e-8, atol=1e-8)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)


@pytest.mark.parametrize('name', ['sir', 'seir3'])
def test_skeleton_1e10(name):
    """Deterministic Euler skeleton (sde --no_dem_sto --no_white_noise), FP64."""
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=64, dt=1.0, noises_off=3, precision=64, filter=False)
    g = eng.smc(p, x_pred=True)
    o = orc.smc(p, x_pred=True)
    np.testing.assert_allclose(g.x_pred, o.x_pred, rtol=1e-10, atol=1e-10)
    # every particle follows the same deterministic path
    assert np.all(g.x_pred == g.x_pred[:, :, :1])


@pytest.mark.parametrize('name,J', [('sir', 2000), ('seir3', 300), ('drift', 500)])
def test_philox_fp64_parity(name, J):
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=J, dt=1.0, precision=64, seed=99)
    g = eng.smc(p, ancestors=True)
    o = orc.smc(p, ancestors=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)


def test_fp32_loglik_statistics_match_oracle():
    """200 replicates: mean and variance of the FP32 estimator vs the FP64 oracle."""
    from plomgpu.native import Plan
    eng = models.engine('sir')
    orc = models.build_oracle('sir')
    R = 200
    p32 = models.make_problem('sir', J=1000, dt=1.0, precision=32, seed=0)
    plan = Plan(eng, p32)
    g = []
    for r in range(R):
        plan.update(seed=1000 + r)
        plan.launch()
        g.append(plan.results().loglik)
    plan.close()
    o = []
    for r in range(R):
        p64 = models.make_problem('sir', J=1000, dt=1.0, precision=64, seed=50000 + r)
        o.append(orc.smc(p64).loglik)
    g, o = np.array(g), np.array(o)
    se = np.sqrt(g.var(ddof=1) / R + o.var(ddof=1) / R)
    assert abs(g.mean() - o.mean()) < 4.0 * se + 0.05
    ratio = g.var(ddof=1) / o.var(ddof=1)
    assert 0.6 < ratio < 1.6


def test_fp32_vs_fp64_same_draws_close():
    """The FP32 path stays within 0.5 nats of the FP64 path of the same model and data."""
    eng = models.engine('sir')
    lls = []
    for prec in (32, 64):
        vals = []
        for s in range(20):
            p = models.make_problem('sir', J=4000, dt=1.0, precision=prec, seed=7000 + s)
            vals.append(eng.smc(p).loglik)
        lls.append(np.mean(vals))
    assert abs(lls[0] - lls[1]) < 0.5


@pytest.mark.parametrize('J', [1, 2, 3, 1000, 4096, 65537, 200000])
def test_systematic_points_exact(J):
    """Device closed form of ``ran += 1/J`` equals the sequential double additions."""
    eng = models.engine('sir')
    orc = models.build_oracle('sir')
    rng = np.random.default_rng(J)
    inc = 1.0 / J
    for U in [0.0, 5e-324, inc * 1e-12, inc * 0.5, np.nextafter(inc, 0.0), float(rng.uniform(0, inc))]:
        np.testing.assert_array_equal(eng.systematic_points(U, J), orc.systematic_points(U, J))


def test_all_fail_rule():
    """Data far above the model: every particle fails (smc.c:55-69)."""
    eng = models.engine('sir_short')
    orc = models.build_oracle('sir_short')
    p = models.make_problem('sir_short', J=500, dt=1.0, precision=64, seed=3)
    p.data[3:6, :] = 1e9
    g = eng.smc(p, ancestors=True)
    o = orc.smc(p, ancestors=True)
    assert o.n_all_fail >= 3
    assert g.n_all_fail == o.n_all_fail
    for n in range(3, 6):
        np.testing.assert_array_equal(g.ancestors[n], np.arange(p.J))
        assert g.llike_n[n] == pytest.approx(np.log(1e-17) * 1, rel=1e-12)
        assert g.ess_n[n] == 0.0
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)


def test_missing_rows_and_no_filter():
    eng = models.engine('sir_short')
    orc = models.build_oracle('sir_short')
    p = models.make_problem('sir_short', J=300, dt=1.0, precision=64, seed=4)
    p.data[[0, 5, 6, 11], :] = np.nan
    g = eng.smc(p, ancestors=True)
    o = orc.smc(p, ancestors=True)
    for n in (0, 5, 6, 11):
        np.testing.assert_array_equal(g.ancestors[n], np.arange(p.J))
        assert g.llike_n[n] == 0.0
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)
    q = models.make_problem('sir_short', J=300, dt=1.0, precision=32, seed=4, filter=False)
    assert eng.smc(q).loglik == 0.0


def test_large_population_properties():
    """Size-independent checks at J = 2^20: sorted in-range ancestors, finite likelihood,
    offspring counts within one of J * normalised weight."""
    eng = models.engine('sir')
    p = models.make_problem('sir', J=1 << 20, dt=1.0, precision=32, seed=5, nb_obs=8)
    g = eng.smc(p, ancestors=True)
    assert np.isfinite(g.loglik)
    a = g.ancestors.astype(np.int64)
    assert a.min() >= 0 and a.max() < p.J
    assert np.all(np.diff(a, axis=1) >= 0)
    ess = g.ess_n[:p.n_obs]
    assert np.all((ess > 0) & (ess <= p.J * (1 + 1e-9)))


def test_plan_reuse_matches_one_shot():
    from plomgpu.native import Plan
    eng = models.engine('seir3')
    p = models.make_problem('seir3', J=2048, dt=1.0, precision=32, seed=21)
    one = eng.smc(p).loglik
    plan = Plan(eng, p)
    vals = []
    for _ in range(3):
        plan.update(seed=21)
        plan.launch()
        vals.append(plan.results().loglik)
    plan.close()
    assert vals == [one, one, one]


def test_fp32_precision_bias_with_common_draws():
    """FP32 state vs the FP64 oracle on the same injected draws.  A single path
    comparison diverges once an ancestor flips at the last bits of a weight, so
    the precision error is assessed as the bias over replicates: the signed mean
    difference stays well inside 0.5 nats, as does the median absolute one."""
    eng = models.engine('sir')
    orc = models.build_oracle('sir')
    diffs = []
    for s in range(24):
        p32 = models.make_problem('sir', J=1000, dt=1.0, precision=32, seed=s)
        D = eng.draws_per_substep(0)
        z, u = crn_draws(p32, D, 500 + s)
        g = eng.smc(p32, crn_normals=z, crn_uniforms=u)
        o = orc.smc(models.make_problem('sir', J=1000, dt=1.0, precision=64, seed=s), crn_normals=z, crn_uniforms=u)
        diffs.append(g.loglik - o.loglik)
    diffs = np.array(diffs)
    assert abs(diffs.mean()) < 0.25
    assert np.median(np.abs(diffs)) < 0.5


@pytest.mark.parametrize('noises_off', [0, 3])
def test_crn_parity_shared_memory_state(noises_off):
    """seir20x2 (180 state words per particle, held in shared memory) against the oracle with
    common draws, FP64: trajectories, ancestors, log-likelihood."""
    eng = models.engine('seir20x2')
    orc = models.build_oracle('seir20x2')
    p = models.make_problem('seir20x2', J=300, dt=1.0, noises_off=noises_off, precision=64, seed=11, nb_obs=30)
    D = eng.draws_per_substep(noises_off)
    z, u = crn_draws(p, D, 77)
    g = eng.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True)
    o = orc.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    np.testing.assert_allclose(g.x_pred, o.x_pred, rtol=1e-6, atol=1e-9)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)


def test_concentrated_weights_shared_memory_state_match_oracle():
    """seir20x2 at J = 4000 (tiles of 128 particles): the weights of its 20 series concentrate on a
    few particles, so single tiles take more than 8 tiles' worth of systematic points and are
    finished by the second resampling launch; ancestors still equal the oracle's (FP64 Philox)."""
    eng = models.engine('seir20x2')
    orc = models.build_oracle('seir20x2')
    p = models.make_problem('seir20x2', J=4000, dt=1.0, precision=64, seed=9, nb_obs=12)
    g = eng.smc(p, ancestors=True)
    o = orc.smc(p, ancestors=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)
    per_tile = [np.bincount(a // 128, minlength=4000 // 128 + 1).max() for a in g.ancestors]
    assert max(per_tile) > 8 * 128


def test_philox_fp64_shared_memory_state_matches_oracle():
    """The shared-memory-state kernel consumes the same Philox blocks as the oracle (FP64)."""
    eng = models.engine('seir20x2')
    orc = models.build_oracle('seir20x2')
    p = models.make_problem('seir20x2', J=200, dt=1.0, precision=64, seed=5, nb_obs=20)
    g = eng.smc(p, ancestors=True)
    o = orc.smc(p, ancestors=True)
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)
