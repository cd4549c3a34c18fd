"""The N>1 path of bench.py on CPU: two gloo ranks stand in for two GPUs.

bench.py runs one independent replica per GPU (the path shards by replica only;
no collective touches the data).  What crosses ranks is the timing: every rank's
elapsed time is reduced with MAX, so the job's time is the slowest replica's,
and the whole-job rate counts all ranks' units over that time.  The reference
arm prints from rank 0 only; the other ranks leave without work.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    res = {}
    try:
        bench.init_replicas("gloo", timeout_s=30.0)
        res["info"] = bench.world_info()
        bench.sync_ranks()
        res["tmax"] = bench.max_over_ranks(1.0 + rank)             # rank 1 is the slow one
        res["rate"] = bench.job_rate(100.0, 1.0 + rank)            # 100 units per rank
        if rank != 0:
            # the reference arm does no work on ranks other than 0
            res["ref"] = bench.run_reference(None, 6, "fp64", "plain_fp64_n40962", "")
        bench.sync_ranks()
        bench.finish_replicas()
    except Exception as e:                                            # reported to the parent
        res["error"] = repr(e)
    out.put((rank, res))


def test_two_gloo_ranks_reduce_time_and_rate():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    for rank, res in results.items():
        assert "error" not in res, res
        assert res["info"] == (rank, rank, world)
        assert res["tmax"] == 2.0                      # max over ranks, the same on every rank
        assert res["rate"] == pytest.approx(100.0 * world / 2.0)
    assert results[1]["ref"] is None


def test_single_process_is_its_own_job(monkeypatch):
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    assert bench.world_info() == (0, 0, 1)
    bench.init_replicas("gloo")                        # no process group for one process
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(10.0, 2.0) == 5.0


def test_plain_kernel_names_match_selection_codes():
    """bench.py --plain-kernel names map to the swe_cuda_select_kernel codes that the
    wrapper's lane_shape() gives for the same node-per-lane shape."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "rbf-fd-swe_b200"))
    import bench
    from swe_b200 import capi

    for lanes in (1, 2, 4):
        for wide, ctas in (("", 4), ("w", 5), ("d", 3)):
            for pf in (False, True):
                name = f"lane{lanes}{wide}{'pf' if pf else ''}"
                assert bench.PLAIN_KERNELS[name] == capi.Plain.lane_shape(lanes, ctas, pf), name
    codes = [v for v in bench.PLAIN_KERNELS.values() if v is not None]
    assert len(codes) == len(set(codes)) and max(codes) == 23 and min(codes) == 1


def test_reference_arm_line_on_rank0(capsys, monkeypatch):
    """bench.py --impl reference on rank 0: one JSON line with the contract's keys, the
    reference's own CPU code timed on the host cores, and vs_baseline against the
    reference's recorded rate for this workload."""
    import json
    import types

    sys.path.insert(0, ROOT)
    import bench
    import oracle

    if not oracle.reference_available("fp64", "cfdl"):
        pytest.skip("the reference was not built here")
    monkeypatch.setenv("RANK", "0")
    args = types.SimpleNamespace(gpus=1, steps=1, warmup=1)
    desc = bench.WORKLOADS["plain_fp64_n40962"][2]
    bench.run_reference(args, 6, "fp64", "plain_fp64_n40962", desc)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    # both arms read one input file and print one config dict
    _, d, sha = bench.workload_input(6)
    assert line["config"] == bench.plain_config("plain_fp64_n40962", desc, d, sha)
    cpu = line["cpu_baseline"]
    assert cpu["cores"] == cpu["cpu"]["threads_used"] >= 1 and cpu["one_thread_value"] > 0
    assert cpu["cpu"]["affinity_cpus"] >= cpu["cores"] or os.environ.get("OMP_NUM_THREADS")
    for key in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert abs(line["vs_baseline"] - line["value"] / bench.RECORDED_RATE["plain_fp64_n40962"][0]) < 1e-12
