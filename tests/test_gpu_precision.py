"""Log-likelihood error of the FP32 production filter against FP64.

The production filter keeps particle states, rates, noises, observation
densities and log-weights in FP32 and the log-likelihood accumulation, the
log-sum-exp normalisation and the cumulative weights in FP64
(weight(), model_builder/C/core/smc.c:27-83, is the rule both follow).  The
error of that split is measured with paired draws: an FP32 filter consumes
the normals and resampling uniforms of the FP64 filter of the same seed
(rounded to FP32), so the difference of the two log-likelihoods is due to
precision alone.  The FP64 filter itself equals the FP64 oracle (CRN and
Philox parity tests).

* paired FP64 = Philox FP64: the paired draws are the FP64 filter's draws;
* one interval from a given particle cloud equals the same interval inside
  the whole filter (the conditional measurement below rests on it);
* conditional per-interval error on the SEIR 20x2 model (the model of the
  J = 1e5, T = 520 benchmark): the same FP64 particle cloud advanced over
  one interval in FP32 and in FP64, at every interval of an FP64 filter path
  (plomgpu.precision);
* whole filters: paired FP32 - FP64 log-likelihood over seeds on the SIR
  model of the batched workload (on SEIR 20x2 whole filters diverge: the
  estimator's own spread, see plomgpu.precision).
"""

import copy
import math

import numpy as np
import pytest

import models
from plomgpu import precision

pytestmark = pytest.mark.gpu


def _with(prob, **kw):
    p = copy.copy(prob)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize('name,J', [('sir', 1000), ('seir3', 500), ('drift', 300)])
def test_paired_fp64_equals_philox_fp64(name, J):
    eng = models.engine(name)
    p = models.make_problem(name, J=J, dt=1.0, precision=64, seed=21)
    a = eng.smc(p, ancestors=True)
    b = eng.smc(_with(p, paired_draws=True), ancestors=True)
    np.testing.assert_array_equal(a.ancestors, b.ancestors)
    np.testing.assert_allclose(b.llike_n[:p.n_obs], a.llike_n[:p.n_obs], rtol=1e-12, atol=1e-12)
    assert b.loglik == pytest.approx(a.loglik, rel=1e-12)


def test_interval_from_cloud_equals_interval_in_filter():
    """Interval n run alone from the resampled particles after interval n - 1
    (plomgpu_smc_desc.x0_particles) gives the whole filter's llike_n[n] and
    ancestors, on the GPU and on the oracle (CRN draws, FP64)."""
    eng = models.engine('seir3')
    orc = models.build_oracle('seir3')
    p = models.make_problem('seir3', J=300, dt=1.0, precision=64, seed=3, nb_obs=8)
    D = eng.draws_per_substep(0)
    rng = np.random.Generator(np.random.Philox(77))
    z = rng.standard_normal(p.J * int(p.n_sub.sum()) * D)
    u = rng.uniform(size=p.n_obs)
    full = eng.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True)
    off_inc = orc.info.off_inc
    for n in (1, 4, 7):
        cloud = full.x_pred[n - 1][:off_inc, full.ancestors[n - 1]]
        sub0 = int(p.n_sub[:n].sum())
        zn = z[p.J * sub0 * D:p.J * (sub0 + int(p.n_sub[n])) * D]
        q = p.interval_problem(n, cloud)
        g = eng.smc(q, crn_normals=zn, crn_uniforms=u[n:n + 1], ancestors=True)
        o = orc.smc(q, crn_normals=zn, crn_uniforms=u[n:n + 1], ancestors=True)
        assert g.llike_n[0] == pytest.approx(full.llike_n[n], rel=1e-12, abs=1e-12)
        np.testing.assert_array_equal(g.ancestors[0], full.ancestors[n])
        assert o.llike_n[0] == pytest.approx(full.llike_n[n], rel=1e-9)
        np.testing.assert_array_equal(o.ancestors[0], full.ancestors[n])


def test_conditional_interval_error_seir20x2():
    """Per-interval precision error on the benchmark's model (SEIR 20x2, J = 20000), every interval
    of a 60-interval FP64 filter path: bias and standard error below 0.005 nats per interval, and
    the whole-filter bias they imply within the 0.5-nat budget."""
    eng = models.engine('seir20x2')
    p = models.make_problem('seir20x2', J=20000, dt=1.0, precision=32, seed=1, nb_obs=60)
    n, d = precision.conditional_interval_errors(eng, p, stride=1, seed=100)
    st = precision.summary(p, n, d)
    assert st['per_interval_se'] < 0.005, st
    assert abs(st['per_interval_mean']) < 0.005, st
    assert abs(st['implied_filter_bias']) < 0.5, st


def test_paired_filter_error_sir():
    """The SIR model of the batched workload (J = 1000, T = 52) over 64 seeds:
    bias within 0.5 nats."""
    eng = models.engine('sir')
    p = models.make_problem('sir', J=1000, dt=1.0, precision=32, seed=1)
    d = precision.paired_filter_errors(eng, p, range(64))
    se = d.std(ddof=1) / math.sqrt(len(d))
    assert abs(d.mean()) < 0.5, (d.mean(), se)
    assert se < 0.5, (d.mean(), se)
