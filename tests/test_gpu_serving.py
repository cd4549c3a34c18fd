"""Serving form on the GPU: continuous batching of forecast requests.

* a request's result is bitwise identical alone and in a mix of overlapping
  requests of other grids, member counts and lengths, and equals the plain
  drop-in form's result for the same state (FP64 arithmetic in both);
* admission never lets the arena exceed the HBM budget, and requests that do
  not fit wait until earlier ones finish;
* cancellation retires a request without results;
* every served member equals the FP64 oracle's run of the same state and step
  count (rk4_rbffd_swe.c:30-72) within 1e-12 relative per field;
* a dependency wait that runs out (a work item withheld by the test hook) fails
  the request with SWE_ERR_TIMEOUT, and the server then completes a clean request;
* on the N=40962 grid in the device level order (20 node chunks per member, work
  items of two members), concurrent requests of 1 to 7 members match the oracle.
"""
import numpy as np
import pytest

import oracle
from conftest import generated_input, rel_err
from swe_b200 import capi, gen, layout, swe_input

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


def test_served_members_match_oracle(models):
    """Requests of two grids, several member counts and lengths, overlapping on the
    device; every member of every result against the oracle's own RK4 run."""
    m3, m4 = models[3], models[4]
    plan = [(m4, 3, 40, 11), (m3, 2, 60, 21), (m4, 1, 15, 31), (m3, 5, 25, 41), (m4, 4, 30, 51)]
    srv = capi.Server(2 << 30)
    try:
        gids = {id(m4): srv.add_grid(m4), id(m3): srv.add_grid(m3)}
        states = [_states(m, mb, seed) for m, mb, st, seed in plan]
        rids = [srv.submit(gids[id(m)], H0, st) for (m, mb, st, seed), H0 in zip(plan, states)]
        srv.wait(rids)
        outs = [srv.fetch(r) for r in rids]
    finally:
        srv.stop()
    ports = {id(m4): oracle.Port(m4, "fp64"), id(m3): oracle.Port(m3, "fp64")}
    for (m, mb, st, seed), H0, out in zip(plan, states, outs):
        for b in range(mb):
            want = ports[id(m)].run(H0[b], st)
            assert rel_err(out[b], want).max() <= 1e-12, (m.N, mb, st, b)


def test_dependency_timeout_fails_request_then_server_recovers(models):
    """The test hook withholds one work item of stage 5 (step 1, stage 1); the items
    of stage 6 wait for it until the 0.2 s limit runs out.  The request fails with
    SWE_ERR_TIMEOUT, the server counts the failure, and a clean request submitted
    afterwards completes and matches the oracle."""
    m3 = models[3]
    srv = capi.Server(1 << 30)
    try:
        g = srv.add_grid(m3)
        srv.set_dep_limit(0.2)
        srv.test_withhold(-1, 5)            # armed for the next submission
        bad = srv.submit(g, _states(m3, 1, 3), 6)
        with pytest.raises(capi.SweError, match="dependency wait") as e:
            srv.wait([bad], timeout=60.0)
        assert e.value.status == 6
        assert srv.stats()["dependency_failures"] == 1
        H0 = _states(m3, 2, 9)
        good = srv.submit(g, H0, 12)
        res = srv.wait([good], timeout=60.0)
        assert res[good][0] == 1
        out = srv.fetch(good)
    finally:
        srv.stop()
    port = oracle.Port(m3, "fp64")
    for b in range(2):
        assert rel_err(out[b], port.run(H0[b], 12)).max() <= 1e-12


def test_n40962_device_order_requests_match_oracle():
    """Several requests on the N=40962 grid registered in the device level order (the
    serving bench's setup): member counts 1, 2, 5 and 7 (odd counts end in a one-member
    block), different lengths, all in flight together; every member against the
    oracle's own RK4 run (1e-12 relative per field)."""
    _, d = generated_input(6)
    m = swe_input.to_model(d)
    m = layout.reorder(m, layout.rcm_mapping(m, device=True))
    plan = [(1, 30, 3), (2, 20, 13), (5, 12, 23), (7, 25, 33)]
    srv = capi.Server(4 << 30)
    try:
        g = srv.add_grid(m)
        states = [_states(m, mb, seed) for mb, st, seed in plan]
        rids = [srv.submit(g, H0, st) for (mb, st, seed), H0 in zip(plan, states)]
        srv.wait(rids)
        outs = [srv.fetch(r) for r in rids]
    finally:
        srv.stop()
    port = oracle.Port(m, "fp64")
    for (mb, st, seed), H0, out in zip(plan, states, outs):
        for b in range(mb):
            assert rel_err(out[b], port.run(H0[b], st)).max() <= 1e-12, (mb, st, b)
