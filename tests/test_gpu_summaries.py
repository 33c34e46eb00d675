"""Filtered summaries and prediction residuals on the GPU against the oracle's
restatement of compute_hat / get_CI95 (model_builder/C/core/hat.c:28-260) and
print_prediction_residuals (model_builder/C/core/print.c:632-711).

CRN mode, FP64 state: both sides see the same particles (to ~1e-13) and the
same ancestors, so the means agree to 1e-9 relative and the quantiles pick
the same particle.  Quantiles under equal weights use the reference's exact
ranks (its running sum of 1/J replayed on the host).
"""

import numpy as np
import pytest

import models
from test_gpu_parity import crn_draws

pytestmark = pytest.mark.gpu

CASES = [('sir', 1000, 1.0, 0, True), ('sir', 1000, 1.0, 0, False), ('noise', 300, 1.0, 0, True),
         ('drift', 257, 1.0, 0, True), ('seir3', 500, 1.0, 0, True), ('sir', 40, 1.0, 3, True)]


def _run(name, J, dt, noises_off, filt):
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=J, dt=dt, noises_off=noises_off, precision=64, seed=11, filter=filt)
    D = eng.draws_per_substep(noises_off)
    z, u = crn_draws(p, D, 4321 + J)
    g = eng.smc(p, crn_normals=z, crn_uniforms=u, hat=True, ancestors=True)
    o = orc.smc(p, crn_normals=z, crn_uniforms=u, hat=True, ancestors=True)
    return eng, p, g, o


@pytest.mark.parametrize('name,J,dt,noises_off,filt', CASES)
def test_summaries_match_oracle(name, J, dt, noises_off, filt):
    eng, p, g, o = _run(name, J, dt, noises_off, filt)
    assert eng.info.n_hat == g.hat.shape[1]
    np.testing.assert_array_equal(g.ancestors, o.ancestors)
    np.testing.assert_allclose(g.hat[:, :, 1], o.hat[:, :, 1], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(g.hat[:, :, 0], o.hat[:, :, 0], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(g.hat[:, :, 2], o.hat[:, :, 2], rtol=1e-9, atol=1e-9)
    weighted = np.zeros(p.n_obs, bool)
    if filt:
        weighted = ~np.all(np.isnan(p.data), axis=1)
    rows = np.nonzero(weighted)[0]
    gp, op = g.pred_res[rows], o.pred_res[rows]
    np.testing.assert_allclose(gp[:, :, 0], op[:, :, 0], rtol=1e-9, atol=1e-9)
    fin = np.isfinite(op[:, :, 1])
    np.testing.assert_array_equal(np.isfinite(gp[:, :, 1]), fin)
    np.testing.assert_allclose(gp[:, :, 1][fin], op[:, :, 1][fin], rtol=1e-7, atol=1e-9)


@pytest.mark.parametrize('name', ['sir', 'noise'])
def test_summaries_large_J_properties(name):
    """J = 2^18, FP32 production mode: intervals ordered, the time-0 row constant,
    the remainder rows (where the model has one) equal to N(t) minus the summed states."""
    eng = models.engine(name)
    p = models.make_problem(name, J=1 << 18, dt=1.0, precision=32, seed=5)
    g = eng.smc(p, hat=True)
    h = g.hat
    assert np.all(np.isfinite(h))
    assert np.all(h[:, :, 0] <= h[:, :, 2])
    np.testing.assert_allclose(h[0, :, 0], h[0, :, 2])
    info = eng.info
    if not info.pop_size_eq_sum_sv:
        nc, nsv = info.n_cac, info.n_par_sv * info.n_cac
        states = h[:, :nsv, 1].reshape(len(h), info.n_par_sv, nc).sum(axis=1)
        np.testing.assert_allclose(h[:, nsv:nsv + nc, 1], p.pop_size - states, rtol=1e-5,
                                   atol=1e-6 * p.pop_size.max())
    # the log-likelihood is unchanged by asking for summaries (same draws)
    assert eng.smc(p).loglik == g.loglik


def test_summaries_need_pop_size():
    """A model with a remainder needs N(t) for its summaries: a clear error, not a guess."""
    from plomgpu.native import PlomGpuError
    eng = models.engine('noise')
    p = models.make_problem('noise', J=100, dt=1.0, precision=64)
    p.pop_size = None
    with pytest.raises(PlomGpuError):
        eng.smc(p, hat=True)
