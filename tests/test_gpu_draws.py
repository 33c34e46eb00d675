"""Distribution tests of the random draws as the GPU computes them.

The model libraries are built with the special-function-unit forms of the
single-precision elementary functions (log, exp, sin, cos, pow) and with
hardware-rate division and square roots, so the FP32 production draws run
other arithmetic than the host build of the same headers that
``test_psr.py`` checks.  Here the device's own draws (test hook
plomgpu_debug_draws, compiled into the same library as the filters) go
through the same checks, with the parameter grid of ``test_psr.py``:

* the Box-Muller normals of the sde step (model_builder/C/templates/
  core_template.c:283 draws one gsl_ran_ugaussian per noise term): moments,
  Kolmogorov-Smirnov, tail frequencies beyond 3, 4 and 4.5 sd, independence of
  the normals of one Philox block and of neighbouring streams;
* the psr samplers (core_template.c:105-209, prediction_util.c:327-345):
  binomial and Poisson moments and chi-square, Gamma Kolmogorov-Smirnov;
* the normals of the psr uniform stream (Gamma white noise).
"""

import math

import numpy as np
import pytest
from scipy import stats

import models

pytestmark = pytest.mark.gpu

STREAMS, PER_STREAM = 1024, 128  # 131072 draws per sampler case


@pytest.fixture(scope='module')
def eng():
    return models.engine('sir')


@pytest.mark.parametrize('precision', [32, 64])
def test_sde_normals(eng, precision):
    n_streams, per = 8192, 512  # 4.2 M normals
    z = eng.draws('normal', seed=7 + precision, streams=n_streams, per_stream=per, precision=precision)
    n = len(z)
    assert np.all(np.isfinite(z))
    assert abs(z.mean()) < 5.0 / math.sqrt(n)
    assert abs(z.var() - 1.0) < 5.0 * math.sqrt(2.0 / n)
    assert abs(stats.skew(z)) < 5.0 * math.sqrt(6.0 / n)
    assert abs(stats.kurtosis(z)) < 5.0 * math.sqrt(24.0 / n)
    assert stats.kstest(z, 'norm').pvalue > 1e-4
    # tails: the frequency of |z| > k against 2 (1 - Phi(k)), within 5 Poisson sd
    a = np.abs(z)
    for k in (3.0, 4.0, 4.5):
        expect = n * 2.0 * stats.norm.sf(k)
        got = int(np.count_nonzero(a > k))
        assert abs(got - expect) < 5.0 * math.sqrt(expect) + 1, (k, got, expect)
    # independence: the normals of one Philox block (positions within a
    # block of 4 in FP32, 2 in FP64) and the same draw of neighbouring streams
    per_block = 4 if precision == 32 else 2
    blocks = z.reshape(-1, per_block)
    lim = 5.0 / math.sqrt(blocks.shape[0])
    for i in range(per_block):
        for j in range(i + 1, per_block):
            assert abs(np.corrcoef(blocks[:, i], blocks[:, j])[0, 1]) < lim
            assert abs(np.corrcoef(blocks[:, i] ** 2, blocks[:, j] ** 2)[0, 1]) < lim
    by_stream = z.reshape(n_streams, per)
    r = np.corrcoef(by_stream[:-1].ravel(), by_stream[1:].ravel())[0, 1]
    assert abs(r) < 5.0 / math.sqrt(by_stream[1:].size)


@pytest.mark.parametrize('precision', [32, 64])
def test_psr_stream_normals(eng, precision):
    z = eng.draws('psr_normal', seed=5, streams=STREAMS, per_stream=PER_STREAM, precision=precision)
    n = len(z)
    assert abs(z.mean()) < 5.0 / math.sqrt(n)
    assert abs(z.var() - 1.0) < 5.0 * math.sqrt(2.0 / n)
    assert stats.kstest(z, 'norm').pvalue > 1e-4


def _chi2_pvalue(x, pmf, support):
    obs = np.bincount(x.astype(int), minlength=len(support))[:len(support)]
    exp = pmf(support) * len(x)
    keep = exp > 5
    chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
    return stats.chi2.sf(chi, keep.sum() - 1)


@pytest.mark.parametrize('precision', [32, 64])
@pytest.mark.parametrize('n,p', [(7, 0.3), (40, 0.2), (100, 0.3), (1000, 0.035), (1000, 0.05), (100000, 0.3),
                                 (2_000_000, 0.9), (50, 0.97), (80, 0.5),
                                 (10_000_000, 1e-6), (10_000_000, 2e-6), (8_000_000, 1e-3)])
def test_binomial_sampler_device(eng, n, p, precision):
    x = eng.draws('binomial', n, p, seed=n + precision, streams=STREAMS, per_stream=PER_STREAM, precision=precision)
    assert np.all(x == np.floor(x)) and x.min() >= 0 and x.max() <= n
    mu, var = n * p, n * p * (1 - p)
    assert abs(x.mean() - mu) < 5 * math.sqrt(var / len(x))
    assert abs(x.var() / var - 1.0) < 0.04
    if n <= 1000:
        assert _chi2_pvalue(x, lambda k: stats.binom.pmf(k, n, p), np.arange(n + 1)) > 1e-4


@pytest.mark.parametrize('precision', [32, 64])
@pytest.mark.parametrize('mu', [0.3, 4.0, 9.99, 10.0, 37.5, 39.9, 40.0, 55.0, 2e4, 3e6])
def test_poisson_sampler_device(eng, mu, precision):
    x = eng.draws('poisson', mu, seed=int(mu * 100) + 1 + precision, streams=STREAMS, per_stream=PER_STREAM,
                  precision=precision)
    assert np.all(x == np.floor(x)) and x.min() >= 0
    assert abs(x.mean() - mu) < 5 * math.sqrt(mu / len(x))
    assert abs(x.var() / mu - 1.0) < 0.04
    if mu < 100:
        assert _chi2_pvalue(x, lambda k: stats.poisson.pmf(k, mu), np.arange(int(mu * 4 + 20))) > 1e-4


@pytest.mark.parametrize('precision', [32, 64])
@pytest.mark.parametrize('a,theta', [(0.3, 2.0), (1.0, 1.0), (100.0, 0.01), (7.0, 3.0)])
def test_gamma_sampler_device(eng, a, theta, precision):
    x = eng.draws('gamma', a, theta, seed=int(a * 10) + 3 + precision, streams=STREAMS, per_stream=PER_STREAM,
                  precision=precision)
    assert x.min() > 0
    assert stats.kstest(x, stats.gamma(a, scale=theta).cdf).pvalue > 1e-4
    assert abs(x.mean() / (a * theta) - 1.0) < 5 * math.sqrt(1.0 / (a * len(x)))
