"""The "ode" implementation: the deterministic skeleton integrated by the
embedded RKF45 pair with step control (plomrt::rkf45_interval, shared by the
GPU engine and the oracle).

CPU: the emitted right-hand side (deriv) against the emitted Euler step
(cac_body with noise off) through a converged fine-step Euler skeleton, and
the step control honouring its tolerance.  GPU: engine against oracle on the
same tolerances (FP64), and FP32.
"""

import numpy as np
import pytest

import models


def _problem(name, **kw):
    return models.make_problem(name, J=1, dt=1.0, precision=64, seed=1, **kw)


@pytest.mark.parametrize('name', ['sir', 'seir3', 'noise'])
def test_ode_skeleton_converges_to_fine_euler(name):
    orc = models.build_oracle(name)
    tight = _problem(name, nb_obs=8, ode=True, eps_abs=1e-10, eps_rel=1e-10)
    a = orc.smc(tight, x_pred=True)
    fine = models.make_problem(name, J=1, dt=1.0 / 2048, precision=64, seed=1, nb_obs=8, noises_off=3)
    b = orc.smc(fine, x_pred=True)
    # Euler is first order: error ~ dt * |x''| / 2 per unit time
    np.testing.assert_allclose(a.x_pred, b.x_pred, rtol=2e-3, atol=1e-6 * np.abs(b.x_pred).max())
    assert a.loglik == pytest.approx(b.loglik, rel=2e-3, abs=1e-2)


@pytest.mark.parametrize('eps', [1e-3, 1e-6])
def test_ode_step_control_meets_tolerance(eps):
    orc = models.build_oracle('sir')
    ref = orc.smc(_problem('sir', nb_obs=20, ode=True, eps_abs=1e-12, eps_rel=1e-12), x_pred=True)
    got = orc.smc(_problem('sir', nb_obs=20, ode=True, eps_abs=eps, eps_rel=eps), x_pred=True)
    err = np.abs(got.x_pred - ref.x_pred) / (eps + eps * np.abs(ref.x_pred))
    # global error over 20 intervals of accumulated local errors held below the tolerance
    assert err.max() < 50.0
    assert err.max() > 0.0 or eps < 1e-5


def test_ode_is_deterministic_and_ignores_noise_flags():
    orc = models.build_oracle('sir')
    p = models.make_problem('sir', J=5, dt=1.0, precision=64, seed=1, nb_obs=10, ode=True)
    a = orc.smc(p, x_pred=True)
    assert p.noises_off == 7
    assert np.all(a.x_pred == a.x_pred[:, :, :1])


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['sir', 'seir3', 'seir20x2'])
def test_ode_gpu_matches_oracle(name):
    eng = models.engine(name)
    orc = models.build_oracle(name)
    p = models.make_problem(name, J=3, dt=1.0, precision=64, seed=1, nb_obs=25, ode=True)
    g = eng.smc(p, x_pred=True)
    o = orc.smc(p, x_pred=True)
    np.testing.assert_allclose(g.x_pred, o.x_pred, rtol=1e-9, atol=1e-9)
    assert g.loglik == pytest.approx(o.loglik, rel=1e-9)
    p32 = models.make_problem(name, J=3, dt=1.0, precision=32, seed=1, nb_obs=25, ode=True)
    g32 = eng.smc(p32)
    assert g32.loglik == pytest.approx(o.loglik, rel=1e-3)
