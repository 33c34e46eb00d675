"""Batched persistent filters against single filters and the oracle."""

import numpy as np
import pytest

import models
from plomgpu import workloads
from plomgpu.native import Batch

pytestmark = pytest.mark.gpu


def small_batch(n=24, seed=8):
    return workloads.sir_batch(n_sets=n, seed=seed, J_range=(1, 3000), T_range=(5, 40))


def test_batch_fp64_matches_oracle_per_filter():
    eng = models.engine('sir')
    orc = models.build_oracle('sir')
    bp = small_batch()
    b = Batch(eng, bp, precision=64)
    b.launch()
    ll, nf, ess = b.results()
    b.close()
    for i in range(len(bp.J)):
        o = orc.smc(bp.single(i, precision=64))
        assert ll[i] == pytest.approx(o.loglik, rel=1e-9, abs=1e-9), i
        assert nf[i] == o.n_all_fail


@pytest.mark.parametrize('ppt', [1, 2])
@pytest.mark.parametrize('bt', [128, 256, 512])
def test_batch_fp32_matches_single_filter_path(bt, ppt):
    eng = models.engine('sir')
    bp = small_batch(n=16, seed=9)
    b = Batch(eng, bp, precision=32, block_threads=bt, particles_per_thread=ppt)
    assert b.config[:2] == (bt, ppt)
    b.launch()
    ll, _, _ = b.results()
    b.launch()
    ll2, _, _ = b.results()
    b.close()
    np.testing.assert_array_equal(ll, ll2)  # replay is deterministic
    for i in range(len(bp.J)):
        single = eng.smc(bp.single(i, precision=32)).loglik
        assert ll[i] == pytest.approx(single, rel=1e-9, abs=1e-9), i


def test_batch_autotune_picks_a_candidate_and_handles_uneven_sizes():
    eng = models.engine('sir')
    bp = workloads.sir_batch(n_sets=300, seed=10, J_range=(256, 4096), T_range=(52, 104))
    b = Batch(eng, bp, precision=32)
    bt, ppt, grid = b.config
    assert bt in (128, 256, 512) and ppt in (1, 2) and grid >= 148
    b.launch()
    ll, nf, ess = b.results()
    b.close()
    assert np.all(np.isfinite(ll))
    assert np.all(ess > 0)
