"""Grid-sharded stepping (swe_b200/shard.py) on the host: world_size-2 and -3 gloo
ranks, each stepping its patch with the oracle as engine and exchanging halo rows
between substeps by point-to-point sends, reproduce the full-grid oracle run bit for
bit.  The plan itself is checked on its own: every stencil row of a rank's compute
rows lies in its patch, and what one rank sends is what its peer receives.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import generated_input
from swe_b200 import layout, shard, swe_input

STEPS = 6


def _model():
    _, d = generated_input(3)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=1)
    return m


def test_plan_covers_every_stencil_and_matches_peers():
    m = _model()
    for nranks in (1, 2, 3, 5):
        plans = shard.plan(m.idx, nranks)
        assert plans[0].c0 == 0 and plans[-1].c1 == m.N
        for p in plans:
            need = np.unique(m.idx[p.c0:p.c1])
            assert need.min() >= p.p0 and need.max() < p.p1
            halo = need[(need < p.c0) | (need >= p.c1)]
            got = np.sort(np.concatenate(list(p.recv.values()) or [np.zeros(0, int)]))
            assert np.array_equal(got, halo)
            for q, rows in p.send.items():
                assert np.array_equal(rows, plans[q].recv[p.rank])
                assert ((rows >= p.c0) & (rows < p.c1)).all()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    res = {}
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from shard_oracle import OracleEngine

        m = _model()
        p = shard.plan(m.idx, world)[rank]
        eng = OracleEngine(m, p)
        eng.set_patch_state(m.H_init[p.p0:p.p1])
        stepper = shard.HaloStepper(p, eng, device="cpu")
        stepper.step(STEPS)
        H = eng.patch_state()[p.c0 - p.p0:p.c1 - p.p0]
        res["H"] = H
        res["range"] = (p.c0, p.c1)
        res["exchanges"] = stepper.exchanges
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        res["error"] = repr(e)
    out[rank] = res


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_oracle_run_equals_full_grid(world):
    import oracle

    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for pr in procs:
            pr.start()
        for pr in procs:
            pr.join(180)
            assert pr.exitcode == 0
        res = dict(out)
    m = _model()
    full = oracle.Port(m, "fp64").run(m.H_init, STEPS)
    H = np.zeros_like(full)
    for r in range(world):
        assert "error" not in res[r], res[r]
        c0, c1 = res[r]["range"]
        H[c0:c1] = res[r]["H"]
        assert res[r]["exchanges"] == 4 * STEPS
    assert np.array_equal(H, full)
