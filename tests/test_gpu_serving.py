"""Serving form on the GPU: continuous batching of forecast requests.

* a request's result is bitwise identical alone and in a mix of overlapping
  requests of other grids, member counts and lengths, and equals the plain
  drop-in form's result for the same state (FP64 arithmetic in both);
* admission never lets the arena exceed the HBM budget, and requests that do
  not fit wait until earlier ones finish;
* cancellation retires a request without results.
"""
import numpy as np
import pytest

from conftest import generated_input, rel_err
from swe_b200 import capi, gen, swe_input

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models():
    return {lv: swe_input.to_model(generated_input(lv)[1]) for lv in (3, 4)}


def _states(m, members, seed):
    return np.stack([gen.perturb_h(m.H_init, seed + b) for b in range(members)])


def test_alone_equals_mixed_equals_plain(models):
    m3, m4 = models[3], models[4]
    A = _states(m4, 3, 10)
    srv = capi.Server(2 << 30)
    try:
        g4 = srv.add_grid(m4)
        g3 = srv.add_grid(m3)
        ra = srv.submit(g4, A, 30)
        srv.wait([ra])
        alone = srv.fetch(ra)
        # the same request in a mix: others before, with and after it
        others = [srv.submit(g3, _states(m3, 2, 20), 50), srv.submit(g4, _states(m4, 1, 30), 10)]
        rb = srv.submit(g4, A, 30)
        others += [srv.submit(g3, _states(m3, 5, 40), 25), srv.submit(g4, _states(m4, 32, 50), 5)]
        srv.wait(others + [rb])
        mixed = srv.fetch(rb)
        for r in others:
            srv.fetch(r)
        st = srv.stats()
    finally:
        srv.stop()
    assert np.array_equal(alone, mixed)
    assert st["completed"] >= 6
    plain = capi.Plain()
    plain.init_model(m4, "fp64")
    for b in range(3):
        plain.set_state(A[b])
        plain.step(30)
        assert rel_err(alone[b], plain.get_state()).max() <= 1e-12
    plain.finalize()


def test_budget_admission(models):
    m4 = models[4]
    per_request = 4 * 8 * m4.N * 4 * 4          # 8 members: H, Ka, Kb, D
    budget = int(per_request * 2.5)
    srv = capi.Server(budget)
    try:
        g = srv.add_grid(m4)
        rids = [srv.submit(g, _states(m4, 8, 100 + 10 * i), 20) for i in range(6)]
        res = srv.wait(rids)
        st = srv.stats()
        outs = [srv.fetch(r) for r in rids]
    finally:
        srv.stop()
    assert all(v[0] == 1 for v in res.values())
    assert st["peak_bytes"] <= budget
    assert st["peak_bytes"] >= per_request
    assert all(np.isfinite(o).all() for o in outs)
    # at most two requests fit at a time, so later ones waited for admission
    admit = sorted(v[1] for v in res.values())
    assert admit[-1] > admit[0]


def test_cancel(models):
    m4 = models[4]
    srv = capi.Server(1 << 30)
    try:
        g = srv.add_grid(m4)
        r1 = srv.submit(g, _states(m4, 4, 7), 400)
        srv.cancel(r1)
        res = srv.wait([r1])
    finally:
        srv.stop()
    assert res[r1][0] == 2


def test_rejects_oversized_request(models):
    m4 = models[4]
    srv = capi.Server(1 << 20)
    try:
        g = srv.add_grid(m4)
        with pytest.raises(capi.SweError) as e:
            srv.submit(g, _states(m4, 4, 1), 5)
        assert e.value.status == 4
    finally:
        srv.stop()
