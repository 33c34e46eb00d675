"""Likelihood server: results equal alone and in the mix, equal to the
single-filter path, admission bounded by the memory budget."""

import numpy as np
import pytest

import models
from plomgpu.native import Server

pytestmark = pytest.mark.gpu


def _thetas(p, n, rng):
    out = []
    for _ in range(n):
        pc = p.par_cac * np.exp(0.05 * rng.standard_normal(p.par_cac.shape))
        out.append(pc)
    return out


@pytest.mark.parametrize('name,J,n_mix,precision', [('sir_short', 700, 120, 32), ('sir_short', 300, 40, 64),
                                                    ('seir3', 1500, 12, 32)])
def test_result_same_alone_and_in_the_mix(name, J, n_mix, precision):
    eng = models.engine(name)
    p = models.make_problem(name, J=J, dt=1.0, precision=precision, seed=1)
    rng = np.random.default_rng(3)
    pcs = _thetas(p, n_mix, rng)
    sv = Server(eng, p, max_J=4 * J, precision=precision)
    alone = sv.wait(sv.submit(J, par_cac=pcs[0], seed=77))[0]
    tickets = []
    for i, pc in enumerate(pcs):
        Ji = J if i == 0 else int(rng.integers(J // 2, 4 * J))
        tickets.append(sv.submit(Ji, par_cac=pc, seed=77 if i == 0 else 1000 + i))
    mixed = [sv.wait(t) for t in tickets]
    st = sv.stats()
    sv.close()
    assert mixed[0][0] == alone  # bit-identical: the request's result does not depend on the mix
    assert st['completed'] == n_mix + 1 and st['pending'] == 0 and st['in_flight'] == 0
    # and equal to the plain single-filter path with the same parameters and seed
    q = models.make_problem(name, J=J, dt=1.0, precision=precision, seed=77)
    q.par_cac = pcs[0]
    assert eng.smc(q).loglik == pytest.approx(alone, rel=1e-9)


def test_admission_respects_memory_budget():
    eng = models.engine('sir_short')
    p = models.make_problem('sir_short', J=2000, dt=1.0, precision=32, seed=1)
    one = 2000 * (2 * 4 * 4 + 4 + 8 + 4) + 4096
    sv = Server(eng, p, max_J=2000, memory_budget=3.5 * one, precision=32)
    ts = [sv.submit(2000, seed=i) for i in range(30)]
    res = [sv.wait(t) for t in ts]
    st = sv.stats()
    sv.close()
    assert all(np.isfinite(r[0]) for r in res)
    assert st['peak_bytes'] <= 3.5 * one
    assert st['peak_in_flight'] <= 3


@pytest.mark.parametrize('precision', [32, 64])
def test_tiled_loop_same_alone_in_the_mix_and_plain(precision):
    """Models whose particle does not fit registers (SEIR 20x2, 180 words) run on the tiled device
    loop: tiles of many requests share the SMs; a request's result is bit-identical alone and in
    the mix, and equal to the plain filter with the same parameters and seed (same tiles, same
    reduction order)."""
    eng = models.engine('seir20x2')
    p = models.make_problem('seir20x2', J=1000, dt=1.0, precision=precision, seed=1, nb_obs=30)
    rng = np.random.default_rng(5)
    pcs = _thetas(p, 9, rng)
    sv = Server(eng, p, max_J=3000, precision=precision)
    alone = sv.wait(sv.submit(1000, par_cac=pcs[0], seed=5))[0]
    Js = [1000] + [int(rng.integers(300, 3000)) for _ in pcs[1:]]
    ts = [sv.submit(Js[i], par_cac=pc, seed=5 if i == 0 else 100 + i) for i, pc in enumerate(pcs)]
    mixed = [sv.wait(t) for t in ts]
    st = sv.stats()
    sv.close()
    assert st['persistent_loop'] == 1
    assert mixed[0][0] == alone
    assert st['completed'] == 10 and st['pending'] == 0 and st['in_flight'] == 0
    q = models.make_problem('seir20x2', J=1000, dt=1.0, precision=precision, seed=5, nb_obs=30)
    q.par_cac = pcs[0]
    assert eng.smc(q).loglik == alone
    # other requests of the mix equal their own plain filters too
    for i in (3, 7):
        qi = models.make_problem('seir20x2', J=Js[i], dt=1.0, precision=precision, seed=100 + i, nb_obs=30)
        qi.par_cac = pcs[i]
        assert eng.smc(qi).loglik == mixed[i][0]


def test_plan_pool_same_alone_and_in_the_mix():
    """Models whose particle does not fit registers can also be served by concurrent plans."""
    eng = models.engine('seir20x2')
    p = models.make_problem('seir20x2', J=1024, dt=1.0, precision=32, seed=1, nb_obs=40)
    sv = Server(eng, p, max_J=2048, plan_pool=4, precision=32, use_plan_pool=True)
    alone = sv.wait(sv.submit(1024, seed=5))[0]
    ts = [sv.submit(1024 if i % 2 == 0 else 2048, seed=5 if i == 0 else 100 + i) for i in range(10)]
    mixed = [sv.wait(t) for t in ts]
    st = sv.stats()
    sv.close()
    assert st['persistent_loop'] == 0
    assert mixed[0][0] == alone
    assert st['completed'] == 11
