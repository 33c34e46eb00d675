"""plomgpu_resample_noalloc: the resampling step for callers that cannot
allocate device memory (a plug-in whose host runtime owns the GPU memory
through its own caching allocator, or a latency-bounded serving loop where
cudaMalloc would synchronise the device).

The entry point is checked against the regular entry point plomgpu_smc_run:
one observation interval is filtered with common random numbers, the
log-weights of its propagated particles are recomputed with the oracle, and
the no-allocation call on those log-weights must give the same ancestors
(bit-exact), log mean weight (1e-9) and ESS (1e-8), on two calls in a row
and on a second, different problem (the fixed scratch keeps the previous
call's contents).  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

import models
from plomgpu import native

pytestmark = pytest.mark.gpu


def _reference_interval(J, seed):
    eng = models.engine('sir_short')
    orc = models.build_oracle('sir_short')
    p = models.make_problem('sir_short', J=J, dt=1.0, precision=64, seed=seed, nb_obs=1)
    D = eng.draws_per_substep(0)
    rng = np.random.Generator(np.random.Philox(seed))
    z = rng.standard_normal(p.J * int(p.n_sub.sum()) * D)
    u = rng.uniform(0.0, 1.0, size=p.n_obs)
    g = eng.smc(p, crn_normals=z, crn_uniforms=u, ancestors=True, x_pred=True)
    x = g.x_pred[0]
    lw = np.array([orc.obs_loglik(p, x[:, j], 0) for j in range(J)])
    return eng, g, lw, float(u[0])


def _noalloc(eng, lw, u, like_min=1e-17, precision=64):
    import torch
    J = len(lw)
    d_lw = torch.tensor(lw, dtype=torch.float64 if precision == 64 else torch.float32, device='cuda')
    d_anc = torch.full((J,), -1, dtype=torch.int32, device='cuda')
    d_out = torch.full((4,), -7.0, dtype=torch.float64, device='cuda')
    stream = torch.cuda.current_stream()
    rc = eng.lib.plomgpu_resample_noalloc(ctypes.c_void_p(d_lw.data_ptr()), precision, J, like_min, u,
                                          ctypes.c_void_p(d_anc.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                          ctypes.c_void_p(stream.cuda_stream))
    native.check(eng.lib, rc)
    torch.cuda.synchronize()
    return d_anc.cpu().numpy().astype(np.uint32), d_out.cpu().numpy()


def _check(g, anc, out):
    np.testing.assert_array_equal(anc, g.ancestors[0])
    assert out[0] == pytest.approx(g.llike_n[0], rel=1e-9)
    assert out[1] == pytest.approx(g.ess_n[0], rel=1e-8)
    assert out[2] == 0.0
    assert out[3] == 0.0


def test_noalloc_matches_smc_run_twice_in_a_row():
    eng, g, lw, u = _reference_interval(3000, seed=41)
    anc1, out1 = _noalloc(eng, lw, u)
    _check(g, anc1, out1)
    anc2, out2 = _noalloc(eng, lw, u)
    _check(g, anc2, out2)
    np.testing.assert_array_equal(anc1, anc2)
    assert np.array_equal(out1, out2)
    # a different problem size right after: nothing of the previous call leaks
    eng, g, lw, u = _reference_interval(4097, seed=42)
    anc3, out3 = _noalloc(eng, lw, u)
    _check(g, anc3, out3)


def test_noalloc_single_precision_log_weights():
    """FP32 log-weights (the production precision): the weights are read as
    float and reduced in double, so the ancestors equal those of the same
    values widened to double, and the oracle's weight() + systematic_sampling()
    on their linear likelihoods; two calls in a row agree."""
    eng, g, lw, u = _reference_interval(5000, seed=43)
    lw32 = lw.astype(np.float32)
    wide = lw32.astype(np.float64)
    anc32, out32 = _noalloc(eng, lw32, u, precision=32)
    anc64, out64 = _noalloc(eng, wide, u, precision=64)
    np.testing.assert_array_equal(anc32, anc64)
    assert np.array_equal(out32, out64)
    orc = models.build_oracle('sir_short')
    J = len(lw)
    _, sel, ll, ess, fail = orc.weight_and_resample(np.exp(wide), (1.0 / J) * u)
    assert not fail
    np.testing.assert_array_equal(anc32, sel)
    assert out32[0] == pytest.approx(ll, rel=1e-9)
    assert out32[1] == pytest.approx(ess, rel=1e-8)
    assert out32[2] == 0.0 and out32[3] == 0.0
    anc32b, out32b = _noalloc(eng, lw32, u, precision=32)
    np.testing.assert_array_equal(anc32, anc32b)
    assert np.array_equal(out32, out32b)


@pytest.mark.parametrize('precision', [64, 32])
def test_noalloc_concentrated_weights(precision):
    """Weights concentrated on a few particles: the tiles holding them take far
    more than 8 tiles' worth of systematic points, which the second resampling
    launch spreads over all blocks.  Ancestors equal the oracle's weight() +
    systematic_sampling() bit for bit, with failing particles mixed in, and
    every particle failing gives identity ancestors."""
    eng = models.engine('sir_short')
    orc = models.build_oracle('sir_short')
    rng = np.random.default_rng(7)
    J = 200000
    lw = -30.0 + rng.standard_normal(J)          # survive, but carry no points
    lw[rng.integers(0, J, 5000)] = -1000.0       # fail: exp(l) <= LIKE_MIN^N_TS
    lw[51200:51500] = rng.uniform(-1.0, 0.0, 300)          # tile 50: most of the mass
    lw[153700:153710] = rng.uniform(-2.0, -1.0, 10)        # tile 150: some of it
    lw[2000:3000] = rng.uniform(-9.0, -8.0, 1000)          # tiles 1-2: a few points
    if precision == 32:
        lw = lw.astype(np.float32)
    wide = lw.astype(np.float64)
    for u in (0.25, 0.8125):
        anc, out = _noalloc(eng, lw, u, precision=precision)
        _, sel, ll, ess, fail = orc.weight_and_resample(np.exp(wide), (1.0 / J) * u)
        assert not fail
        np.testing.assert_array_equal(anc, sel)
        assert out[0] == pytest.approx(ll, rel=1e-9)
        assert out[1] == pytest.approx(ess, rel=1e-8)
        assert out[2] == 0.0 and out[3] == 0.0
        counts = np.bincount(anc // 1024, minlength=J // 1024 + 1)
        assert counts[50] > 8 * 1024 and counts[150] > 0
    dead = np.full(J, -1000.0, dtype=lw.dtype)
    anc, out = _noalloc(eng, dead, 0.5, precision=precision)
    np.testing.assert_array_equal(anc, np.arange(J, dtype=np.uint32))
    assert out[2] == 1.0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    eng = models.engine('sir_short')
    J = (1 << 18) + 1
    d = torch.zeros(4, dtype=torch.float64, device='cuda')
    rc = eng.lib.plomgpu_resample_noalloc(ctypes.c_void_p(d.data_ptr()), 64, J, 1e-17, 0.5,
                                          ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), None)
    assert rc == 1
    assert b'no-allocation limit' in eng.lib.plomgpu_last_error()
