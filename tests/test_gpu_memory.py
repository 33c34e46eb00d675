"""Plan buffers come from the library's stream-ordered memory pool: one-shot
filters in a row reuse it (same results), plans of other sizes and plans that
live side by side get their own memory, and plomgpu_release_memory hands the
unused memory back to the driver."""

import numpy as np
import pytest

import models
from plomgpu.native import Plan

pytestmark = pytest.mark.gpu


def test_one_shot_filters_reuse_the_pool():
    import torch
    eng = models.engine('seir3')
    p = models.make_problem('seir3', J=4000, dt=1.0, precision=32, seed=5)
    a = eng.smc(p, ancestors=True)
    b = eng.smc(p, ancestors=True)            # the buffers of the first call
    np.testing.assert_array_equal(a.ancestors, b.ancestors)
    assert a.loglik == b.loglik
    q = models.make_problem('seir3', J=1500, dt=1.0, precision=32, seed=5)
    c = eng.smc(q)                            # another size in between
    d = eng.smc(p)
    assert d.loglik == a.loglik
    assert np.isfinite(c.loglik)
    # two plans alive at once do not share buffers
    pa, pb = Plan(eng, p), Plan(eng, q)
    pa.launch()
    pb.launch()
    ra, rb = pa.results(), pb.results()
    pa.close()
    pb.close()
    assert ra.loglik == a.loglik and rb.loglik == c.loglik
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    eng.release_memory()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free0
