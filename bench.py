"""Benchmark of the RK4 + RBF-FD hot path on B200.

Default workload: the plain GPU drop-in on the N=40962 (level-6) icosahedral
grid in FP64, CFDL layout, RCM order, dt = 225 s -- the configuration the
reference's "plain GPU drop-in vs reference OpenMP" comparison is quoted on.
A step is one full RK4 step (4 fused stage kernels) of one state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` = node-stage updates/s (4 * N * steps / s)
with the state resident in HBM, timed with CUDA events around each step on the
library's stream, L2 flushed between timed steps (a 256 MB write, then a 256 MB
read so that the write's dirty lines are written back before the step: each
step starts from a cold, clean L2); `e2e` = the
same metric through the C ABI with host buffers (pinned H2D of the state,
one RK4 step, D2H of the state every step); `roofline` = the fused stage
kernel's algorithmic bytes (1396 B per FP64 node-stage, 760 B FP32; 62 B less when
the node-per-lane kernel reads the stencil rows as 16-bit offsets) over its
average duration in the timed region (a timed step is the four stage kernels and
nothing else, so step time / 4) against the measured HBM copy bandwidth.  Multi-GPU runs
are independent replicas (the path does not shard across GPUs here): every
rank steps its own state, time is the max over ranks, value is the sum.

The default run also carries the targets quoted for the larger workloads, in
`targets`: the plain FP64 form at N=163842 and N=655362 (data far beyond L2, so
their roofline is an HBM roofline) and the 64-member batched form at N=163842 in
3xTF32 and in split FP16 (member-steps/s, the ratio to the plain FP64 form on the
same grid, and the h error of all 64 members after 1000 steps against the plain
FP64 GPU run).
The default workload's own data (57 MB of algorithmic bytes per stage) fits the
126 MB L2, so its roofline is labelled L2-resident.

--impl reference times the reference's own CPU code (oracle/_ref, built from
the reference's sources; the oracle port if that is absent) on the host cores
with OpenMP, on the same workload.  Both arms read one input file: the
workload's grid is generated once (seeded, CPU generator) into the reference's
binary format and reused by the other arm; its SHA-256 prefix is in `config`.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rbf-fd-swe_b200"))

WORKLOADS = {
    # name: (level, precision, description)
    "plain_fp64_n40962": (6, "fp64", "plain FP64, N=40962 (level 6), CFDL, RCM, dt=225 s"),
    "plain_fp64_n163842": (7, "fp64", "plain FP64, N=163842 (level 7), CFDL, RCM, dt=120 s"),
    "plain_fp64_n655362": (8, "fp64", "plain FP64, N=655362 (level 8), CFDL, RCM, dt=60 s"),
    "plain_fp32_n655362": (8, "fp32", "plain FP32, N=655362 (level 8), CFDL, RCM, dt=60 s"),
    "ens_tf32_n163842_b64": (7, "tf32x3", "batched ensemble, N=163842 (level 7), 64 members, 3xTF32 on tcgen05, dt=120 s"),
    "ens_tf32_n40962_b64": (6, "tf32x3", "batched ensemble, N=40962 (level 6), 64 members, 3xTF32 on tcgen05, dt=225 s"),
    "ens_bf16_n163842_b64": (7, "bf16x3", "batched ensemble, N=163842 (level 7), 64 members, split BF16 on tcgen05, "
                                          "dt=120 s"),
    "ens_fp16_n163842_b64": (7, "fp16x3", "batched ensemble, N=163842 (level 7), 64 members, split FP16 with "
                                          "power-of-two scales on tcgen05, dt=120 s"),
    "serve_mix": (0, "serve", "serving: Poisson arrivals over N in {2562, 10242, 40962, 163842}, 1-32 members, "
                              "10-500 steps, 80 GB budget, FP64"),
}
# The reference's own recorded rate for a workload's metric and configuration, where one
# exists: Eval_Rhs at N=40962 in the CFDL layout took 1.267690e-3 s per RK4 step (4
# eval_RHS calls) with its OpenACC build on a V100 (run/psg/output/output_cfdl.txt:41;
# precision not recorded) = 4 * 40962 / 1.267690e-3 node-stage updates/s.
RECORDED_RATE = {"plain_fp64_n40962": (4 * 40962 / 1.267690e-3,
                                       "reference run log run/psg/output/output_cfdl.txt:41 "
                                       "(Eval_Rhs, N=40962, CFDL, OpenACC on V100)")}


def vs_recorded(workload: str, value: float):
    """(value / the reference's recorded rate, its source), or (None, None)."""
    rec = RECORDED_RATE.get(workload)
    return (value / rec[0], rec[1]) if rec else (None, None)


ALG_BYTES = {"fp64": 1396, "fp32": 760}      # per node-stage (FP64: 4*31*8+31*4+17*8+4*8+14*8)


def plain_alg_bytes(prec: str, kinfo: dict) -> int:
    """Bytes per node-stage of the representation the stage kernel reads: the
    node-per-lane kernel reads the 31 stencil rows as 16-bit offsets (2 B, not 4)
    when every offset fits."""
    narrow = kinfo["in_use"] == "lane" and kinfo.get("index_offsets_16bit", False)
    return ALG_BYTES[prec] - (31 * 2 if narrow else 0)
# batched form, per node-stage: shared 4*31*4 (weights) + 31*4 (idx) + 17*4 (pointwise)
# plus per member 4*4 (K read once) + 14*4 (RK combine) + 4 (FP64 h registers)
ENS_SHARED_BYTES = 4 * 31 * 4 + 31 * 4 + 17 * 4
ENS_MEMBER_BYTES = 4 * 4 + 14 * 4 + 4
# --plain-kernel choices -> swe_cuda_select_kernel codes (laneN: N lanes per node at 4 CTAs per
# SM; "w": 5 CTAs per SM; "d": 3 CTAs per SM; "pf": with the L2 prefetch)
PLAIN_KERNELS = {"auto": None, "register": 1, "pipelined64": 2, "pipelined32": 3, "pipelined16": 4,
                 "lane1": 6, "lane2": 7, "lane4": 8, "lane1w": 9, "lane2w": 10, "lane4w": 11,
                 "lane1pf": 12, "lane2pf": 13, "lane4pf": 14, "lane1wpf": 15, "lane2wpf": 16, "lane4wpf": 17,
                 "lane1d": 18, "lane2d": 19, "lane4d": 20, "lane1dpf": 21, "lane2dpf": 22, "lane4dpf": 23}
L2_FLUSH_BYTES = 256 << 20
L2_NOTE = "flushed between timed steps: 256 MB write, then 256 MB read (cold, clean L2 at each step)"
L2_NOTE_BOTH = ("GPU arm: L2 flushed between timed steps (256 MB write, then 256 MB read: cold, clean L2 at "
                "each step); CPU arm: no flush")
# DRAM bytes (read + write) per launch of the dominant kernel, from ncu captures of the same
# command (dram__bytes_read.sum + dram__bytes_write.sum, averaged over the captured launches);
# the profile summaries under profiles/ give the commands.
TRAFFIC_BYTES = {
    # DRAM read + write bytes per stage launch, mean over 8 launches of the timed
    # steps (ncu --cache-control none inside the bench's own flushed loop, so
    # stage 0 of each step starts cold and stages 1-3 see what L2 kept; plain
    # kernels reading the stencil rows as 16-bit offsets)
    "plain_fp64_n40962": 45.27e6,       # swe::stage_lane_kernel<double, *, 2, 5, true>
    "plain_fp64_n163842": 181.62e6,     # swe::stage_lane_kernel<double, *, 1, 3, true>
    "plain_fp64_n655362": 887.10e6,     # swe::stage_lane_kernel<double, *, 1, 4, true>
    "plain_fp32_n655362": 452.35e6,     # swe::stage_lane_kernel<float, *, 1, 5, true>
    # swe::ens_stage_kernel<32, 64, stage, 3xTF32>, 12 launches (cold); 707 MB of it is
    # the streamed A-operand image (16 KB per 16-row chunk, 43128 chunks)
    "ens_tf32_n163842_b64": 1668.31e6,
    # swe::ens_stage_kernel<32, 64, stage, BF16>, 12 launches (cold); 353 MB of it is the
    # streamed A-operand image (8 KB per 16-row chunk)
    "ens_bf16_n163842_b64": 1294.82e6,
    # swe::ens_stage_kernel<32, 64, stage, FP16>, 12 launches (cold); 353 MB of it is the
    # streamed A-operand image (8 KB per 16-row chunk)
    "ens_fp16_n163842_b64": 1297.55e6,
}


class L2Flush:
    """Run between timed steps, untimed: a 256 MB write evicts every line of the
    126 MB L2, and a 256 MB read then replaces the write's dirty lines, so their
    write-back is not charged to the next step.  The step starts from an L2 that
    holds none of its data."""

    def __init__(self, device):
        import torch

        self.torch = torch
        self.wr = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
        self.rd = torch.zeros(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
        self.out = torch.empty((), dtype=torch.float32, device=device)

    def __call__(self):
        self.wr.zero_()
        self.torch.sum(self.rd, dim=0, out=self.out)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---- replicas (one process per GPU, no data-path collective) --------------------------------

def world_info():
    """(rank, local_rank, world_size) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def init_replicas(backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Process group for the timing reductions only; a short timeout ends a rank that waits
    for a peer which died, instead of hanging."""
    import datetime

    import torch.distributed as dist
    if world_info()[2] > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def sync_ranks() -> None:
    """Barrier across replicas (no-op for one process)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(x: float, device="cpu") -> float:
    """The job's time is the slowest replica's: max over ranks of a per-rank time."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, t_per_rank: float, device="cpu") -> float:
    """Whole-job throughput of N replicas: all ranks' units over the slowest rank's time."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    return units_per_rank * world / max_over_ranks(t_per_rank, device)


def finish_replicas() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


SPEC_HBM_GBS = 8000.0   # the B200 HBM3e specification figure the hot path's targets are stated against


def measured_peak_bf16_tflops():
    """Dense BF16 GEMM throughput (cuBLAS, burst) of this pool's B200s, or the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def ensemble_tensor_roofline(cfg: dict, members: int, precision: str, t_stage: float) -> dict:
    """Tensor-core side of the batched kernel: the MMA work one stage issues (every 16-row
    chunk: M = 4 x tile nodes, N = 4 x members over the member blocks, K = 16, three
    products) over the stage time, against the dense peak of the MMA kind (TF32 runs at half
    the BF16 rate, FP16 at the BF16 rate)."""
    flops = cfg["chunks"] * 16 * (4 * cfg["tile_nodes"]) * (4 * members) * 2 * 3
    bf16, src = measured_peak_bf16_tflops()
    peak = bf16 / 2 if precision == "tf32x3" else bf16
    achieved = flops / t_stage / 1e12
    return {"mma_flops_per_launch": flops, "achieved": round(achieved, 1), "peak": round(peak, 1),
            "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
            "peak_source": f"{src} BF16 GEMM" + (" / 2 for TF32" if precision == "tf32x3" else "")}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def _rows(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        return rows

    def count(self) -> int:
        return len(self._rows())

    def wait_for(self, n: int, timeout: float, keep_busy=None) -> None:
        """Until n samples exist (or timeout), calling keep_busy() meanwhile."""
        t0 = time.time()
        while self.proc and self.count() < n and time.time() - t0 < timeout:
            if keep_busy:
                keep_busy()
            else:
                time.sleep(0.05)

    def summary(self, first: int = 0):
        rows = self._rows()[first:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def build_workload(level: int, prec: str, device: str):
    from swe_b200 import gen, layout, swe_input

    t0 = time.time()
    d = gen.generate(level, seed=1, device=device)
    m = swe_input.to_model(d)
    pm, mapping = layout.prepare(m, use_rcm=True, simd_length=32)
    log(f"[bench] generated level {level} (N={d.N}) in {time.time() - t0:.1f}s")
    return d, m, pm


def workload_input(level: int):
    """(path, SweInput, sha256 prefix) of the workload's input file, which both arms read.
    The first arm to run generates it (seeded, CPU generator) in the reference's binary
    format; later runs on the same host read it back."""
    from swe_b200 import gen, swe_input

    ddir = os.environ.get("SWE_BENCH_DATA") or os.path.join(tempfile.gettempdir(), "swe_b200_bench")
    os.makedirs(ddir, exist_ok=True)
    path = os.path.join(ddir, f"icos{10 * 4 ** level + 2}_seed1.bin")
    t0 = time.time()
    try:
        d = swe_input.read_input(path)
        how = "read"
    except (OSError, ValueError):
        d = gen.generate(level, seed=1, device="cpu")
        swe_input.write_input(path, d)
        how = "generated"
    h = hashlib.sha256()
    with open(path, "rb") as fh:
        for block in iter(lambda: fh.read(1 << 24), b""):
            h.update(block)
    log(f"[bench] input {path} {how} in {time.time() - t0:.1f}s")
    return path, d, h.hexdigest()[:16]


def plain_config(wl: str, desc: str, d, sha: str) -> dict:
    """The workload's config, the same dict in both arms."""
    return {"workload": wl, "description": desc, "nodes": d.N, "nnbr": d.Nnbr, "dt": d.dt, "layout": "CFDL",
            "rcm": True, "input": f"icos{d.N}_seed1.bin sha256:{sha}", "l2": L2_NOTE_BOTH}


def cpu_baseline_sample(path: str, d, prec: str, target_s: float = 12.0):
    """The reference's own CPU code (oracle/_ref) on a bounded number of steps, on every
    CPU this process may use (affinity set and cgroup quota), and on one thread beside
    it.  Each sample runs in a process of its own (oracle/cpu_baseline.py) that holds
    no GPU context or PyTorch thread pool, so the OpenMP team has the host cores to
    itself.  Rates are whole RK_substep loops (RHS and combine), 4 N steps / seconds;
    the reference's own Eval_Rhs timer (profiling.c:118-126) gives eval_rhs_value."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    cpu = oracle.usable_cpus()
    threads = int(os.environ.get("OMP_NUM_THREADS", cpu["threads"]))
    script = os.path.join(ROOT, "oracle", "cpu_baseline.py")

    def sample(nthreads: int, budget: float) -> dict:
        env = dict(os.environ, OMP_NUM_THREADS=str(nthreads), OMP_SCHEDULE="static")
        env.setdefault("OMP_PROC_BIND", "close")
        out = subprocess.run([sys.executable, script, path, prec, str(budget)], env=env, capture_output=True,
                             text=True, timeout=max(120.0, 20 * budget))
        if out.returncode != 0:
            raise RuntimeError(f"cpu_baseline.py failed: {out.stderr[-300:]}")
        return json.loads(out.stdout.strip().splitlines()[-1])

    full = sample(threads, target_s)
    one = sample(1, target_s / 3)
    rate = 4.0 * d.N * full["steps"] / full["seconds"]
    one_rate = 4.0 * d.N * one["steps"] / one["seconds"]
    what = "the reference's RK_substep (CFDL, RCM)" if full["kind"] == "reference" else "the oracle's C restatement"
    return {"value": rate, "unit": "node-stage updates/s", "cores": threads, "kind": full["kind"],
            "sample": f"{full['steps']} RK4 steps of {what}, OpenMP on {threads} threads, on N={d.N}, in a process "
                      f"of its own (one-thread figure: {one['steps']} steps)",
            "seconds": round(full["seconds"], 3),
            "eval_rhs_value": (4.0 * d.N * full["steps"] / full["eval_rhs_seconds"]) if full["eval_rhs_seconds"]
            else None,
            "one_thread_value": one_rate, "speedup_vs_one_thread": rate / one_rate,
            "cpu": {"model": cpu["model"], "threads_used": threads, "affinity_cpus": cpu["affinity"],
                    "cgroup_quota_cpus": cpu["cgroup_quota_cpus"], "os_cpu_count": cpu["cpu_count"],
                    "omp": {"OMP_NUM_THREADS": str(threads), "OMP_PROC_BIND": os.environ.get("OMP_PROC_BIND", "close"),
                            "OMP_SCHEDULE": "static"}}}


def run_reference(args, level, prec, wl, desc):
    """--impl reference: the reference's own CPU implementation, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    path, d, sha = workload_input(level)
    base = cpu_baseline_sample(path, d, prec, target_s=max(5.0, 0.6 * args.steps))
    line = {
        "metric": "node-stage updates/s (RK4 + RBF-FD stage, plain form)",
        "value": base["value"], "unit": "node-stage updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * 4.0 * d.N / base["value"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": vs_recorded(wl, base["value"])[0], "vs_baseline_source": vs_recorded(wl, base["value"])[1],
        "dtype": "f64" if prec == "fp64" else "f32", "data": "synthetic",
        "config": plain_config(wl, desc, d, sha),
        "parallelism": f"OpenMP x{base['cores']} on the host (rank 0 only)",
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "node-stage updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed_steps(step, stream, steps: int, flush) -> list:
    """Seconds of each of `steps` calls of step(), CUDA events on the library's stream,
    L2 flushed (untimed) before each."""
    import torch

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sync_ranks()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for s in range(steps):
            flush()
            starts[s].record(stream)
            step()
            stops[s].record(stream)
    torch.cuda.synchronize()
    sync_ranks()
    return [a.elapsed_time(b) * 1e-3 for a, b in zip(starts, stops)]


def sample_clocks(local: int, run, keep_busy):
    """run() inside an nvidia-smi sampler; keep_busy() repeats untimed work until 3 samples
    cover the region.  Returns (run's result, clock summary)."""
    with ClockSampler(local) as clocks:
        clocks.wait_for(1, 5.0)
        first = clocks.count()
        out = run()
        clocks.wait_for(first + 3, 5.0, keep_busy=keep_busy)
    return out, clocks.summary(first)


def plain_target(wl: str, local: int, steps: int, warmup: int, flush, world: int) -> dict:
    """One plain workload, timed like the headline line (per-step events, L2 flushed between
    steps); an HBM roofline where the data is far beyond L2."""
    import torch

    from swe_b200 import capi

    level, prec, desc = WORKLOADS[wl]
    d, m, pm = build_workload(level, prec, device=f"cuda:{local}")
    N = d.N
    plain = capi.Plain()
    plain.init_model(pm, prec)
    plain.set_state(pm.H_init.astype(np.float64 if prec == "fp64" else np.float32))
    for _ in range(warmup):
        plain.step(1)
    plain.sync()
    stream = torch.cuda.ExternalStream(plain.stream())

    def busy():
        for _ in range(20):
            plain.step(1)
        plain.sync()
    t, clocks = sample_clocks(local, lambda: timed_steps(lambda: plain.step(1), stream, steps, flush), busy)
    t_total = max_over_ranks(sum(t), f"cuda:{local}")
    t_kernel = t_total / (4 * steps)
    peak, peak_kind = measured_peak_hbm()
    kinfo = plain.kernel_info()
    alg = plain_alg_bytes(prec, kinfo)
    achieved = alg * N / t_kernel / 1e9
    plain.finalize()
    return {"workload": wl, "description": desc, "value": 4.0 * N * steps * world / t_total,
            "unit": "node-stage updates/s", "member_steps_per_s": steps * world / t_total,
            "steps": steps, "ms_per_step": 1e3 * t_total / steps, "dtype": "f64" if prec == "fp64" else "f32",
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "frac_of_spec_8tbs": round(achieved / SPEC_HBM_GBS, 4),
                         "traffic": TRAFFIC_BYTES.get(wl),
                         "peak_source": peak_kind, "kernel": "swe::stage_lane_kernel" if kinfo["in_use"] == "lane"
                         else kinfo["in_use"], "kernel_us": round(t_kernel * 1e6, 2),
                         "alg_bytes_per_node_stage": alg, "kernel_choice": kinfo},
            "clocks": clocks}


def ensemble_target(wl: str, local: int, steps: int, warmup: int, flush, world: int, err_steps: int = 1000,
                    err_members: int = 64, members: int = 64, plain_rate: float | None = None,
                    with_e2e: bool = False) -> dict:
    """member-steps/s of the batched form (3xTF32 or split BF16), its ratio to the plain FP64
    form on the same grid (timed the same way: per-step events, L2 flushed between steps),
    and the per-field error of `err_members` members after `err_steps` steps against the
    plain FP64 GPU run of the same member (u, v, w on the velocity scale, h on max|h|)."""
    import torch

    from swe_b200 import capi, gen

    level, precision, desc = WORKLOADS[wl]
    d, m, pm = build_workload(level, "fp64", device=f"cuda:{local}")
    N = d.N
    H0 = np.stack([gen.perturb_h(m.H_init, 1000 + b) for b in range(members)])
    ens = capi.Ensemble()
    ens.init(m, members)
    ens.set_precision(precision)
    ens.set_state(H0)
    tune_ms = ens.tune().tolist()
    cfg = ens.config()
    ens.set_state(H0)
    for _ in range(warmup):
        ens.step(1)
    ens.sync()
    stream = torch.cuda.ExternalStream(ens.stream())
    counted = {}

    def timed():
        # launches of the timed steps only (the clock sampler's keep-busy steps come after)
        launches0 = capi.kernel_launches()
        out = timed_steps(lambda: ens.step(1), stream, steps, flush)
        counted["launches"] = capi.kernel_launches() - launches0
        return out

    def busy():
        for _ in range(5):
            ens.step(1)
        ens.sync()
    t, clocks = sample_clocks(local, timed, busy)
    launches = counted["launches"]
    t_total = max_over_ranks(sum(t), f"cuda:{local}")
    member_steps = members * steps * world / t_total
    t_stage = t_total / (4 * steps)
    ens_bytes = ENS_SHARED_BYTES + members * ENS_MEMBER_BYTES
    peak, peak_kind = measured_peak_hbm()
    achieved = ens_bytes * N / t_stage / 1e9

    e2e = None
    if with_e2e:
        # through the C ABI with pinned host buffers: host state in, one step, host state out
        H_pin = torch.from_numpy(np.ascontiguousarray(H0, dtype=np.float64).reshape(-1)).pin_memory()
        H_back = torch.empty_like(H_pin).pin_memory()
        e2e_steps = max(3, steps // 4)
        ens.set_state_ptr(H_pin.data_ptr())
        ens.step(1)
        ens.get_state_ptr(H_back.data_ptr())
        sync_ranks()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ens.set_state_ptr(H_pin.data_ptr())
            ens.step(1)
            ens.get_state_ptr(H_back.data_ptr())       # synchronises
        t_e2e = max_over_ranks(time.perf_counter() - t0, f"cuda:{local}")
        nbytes = H_pin.numel() * H_pin.element_size()
        e2e = {"value": members * e2e_steps * world / t_e2e, "unit": "member-steps/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}

    plain = capi.Plain()
    if plain_rate is None:
        # plain FP64 on the same grid (RCM order, the drop-in's own order): member-steps/s =
        # steps/s of one state
        plain.init_model(pm, "fp64")
        plain.set_state(pm.H_init)
        for _ in range(3):
            plain.step(1)
        plain.sync()
        pt = timed_steps(lambda: plain.step(1), torch.cuda.ExternalStream(plain.stream()), steps, flush)
        plain_rate = steps / max_over_ranks(sum(pt), f"cuda:{local}")

    # error after err_steps steps against the plain FP64 GPU run of the same members
    # (natural node order, as the batched form exchanges states)
    plain.init_model(m, "fp64")
    err_idx = list(range(0, members, max(1, members // err_members)))[:err_members]
    ens.set_state(H0)
    ens.step(err_steps)
    Hens = ens.get_state()
    errs = []
    for b in err_idx:
        plain.set_state(H0[b])
        plain.step(err_steps)
        Hp = plain.get_state().reshape(-1, 4)
        vel = np.abs(Hp[:, :3]).max()
        scale = np.array([vel, vel, vel, np.abs(Hp[:, 3]).max()])
        errs.append(np.abs(Hens[b] - Hp).max(0) / scale)
    errs = np.array(errs)
    plain.finalize()
    ens.finalize()
    return {"workload": wl, "description": desc, "value": member_steps, "unit": "member-steps/s",
            "steps": steps, "ms_per_step": 1e3 * t_total / steps,
            "dtype": f"{precision} (fp32 state, fp64 h accumulation)", "members": members,
            "kernel_variant": cfg,
            "tune_ms_per_step": {f"tile{t}_mpc{mp}": (v if v > 0 else None)
                                 for (t, mp), v in zip(capi.Ensemble.TUNE_VARIANTS, tune_ms)},
            "plain_fp64_member_steps_per_s": plain_rate, "ratio_vs_plain_fp64": member_steps / plain_rate,
            "h_err_vs_fp64": {"steps": err_steps, "members": len(err_idx),
                              "reference": "plain FP64 GPU run of the same member (itself within 1e-12 of the "
                                           "oracle in the GPU tests)",
                              "max_norm_rel_per_field_max": errs.max(0).tolist(),
                              "h_max": float(errs[:, 3].max()), "h_median": float(np.median(errs[:, 3])),
                              "h_worst_member": int(err_idx[int(errs[:, 3].argmax())])},
            "e2e": e2e, "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "frac_of_spec_8tbs": round(achieved / SPEC_HBM_GBS, 4),
                         "traffic": TRAFFIC_BYTES.get(wl),
                         "peak_source": peak_kind, "kernel": "swe::ens_stage_kernel",
                         "kernel_us": round(t_stage * 1e6, 2), "alg_bytes_per_node_stage": ens_bytes,
                         "tensor": ensemble_tensor_roofline(cfg, members, precision, t_stage)},
            "clocks": clocks, "state_finite": bool(np.isfinite(Hens).all())}


def run_ensemble(args, desc):
    """--workload ens_*: the batched form as the line's own metric."""
    import torch

    rank, local, world = world_info()
    torch.cuda.set_device(local)
    init_replicas()
    from swe_b200 import capi
    capi.check("swe_cuda_select_device", capi.load().swe_cuda_select_device(local))
    flush = L2Flush(f"cuda:{local}")
    r = ensemble_target(args.workload, local, args.steps, args.warmup, flush, world, err_steps=args.err_steps,
                        err_members=args.err_members, with_e2e=True)
    if rank == 0:
        line = {
            "metric": "member-steps/s (batched ensemble, "
                      f"{'3xTF32' if 'tf32' in args.workload else 'split FP16' if 'fp16' in args.workload else 'split BF16'} "
                      "tcgen05) and ratio to plain FP64",
            "value": r["value"], "unit": "member-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": r["dtype"],
            "data": "synthetic (seeded icosahedral grid, PHS RBF-FD weights, TC5 ICs, per-member 1e-3 h noise)",
            "config": {"workload": args.workload, "description": desc, "members": r["members"],
                       "kernel_variant": r["kernel_variant"], "l2": L2_NOTE},
            "parallelism": f"replicas x{world}",
            **{k: r[k] for k in ("plain_fp64_member_steps_per_s", "ratio_vs_plain_fp64", "h_err_vs_fp64", "e2e",
                                 "gpu_launches", "roofline", "clocks", "state_finite", "tune_ms_per_step")},
        }
        print(json.dumps(line), flush=True)
    finish_replicas()


def run_serving(args, desc):
    """Seeded Poisson stream of forecast requests through the serving form."""
    from swe_b200 import capi, gen, layout, swe_input

    rank, local, world = world_info()
    import torch
    torch.cuda.set_device(local)
    init_replicas()
    rng = np.random.default_rng(args.seed)
    levels = [4, 5, 6, 7]
    models = {}
    t0 = time.time()
    order_s = {}
    for lv in levels:
        d = gen.generate(lv, seed=1, device=f"cuda:{local}")
        m = swe_input.to_model(d)
        if args.serve_order == "device":
            # registered in the device's breadth-first level order (bandwidth-reducing, like
            # the reference's RCM), which keeps each work item's gathers local
            t1 = time.time()
            m = layout.reorder(m, layout.rcm_mapping(m, device=True))
            order_s[lv] = time.time() - t1
        models[lv] = m
    log(f"[bench] serving grids generated in {time.time() - t0:.1f}s (ordering {order_s})")
    srv = capi.Server(args.budget_gb * 1e9, max_requests=512)
    capi.check("swe_cuda_select_device", srv.lib.swe_cuda_select_device(local))
    gids = {lv: srv.add_grid(models[lv]) for lv in levels}
    nreq = args.requests
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, nreq))
    reqs = []
    for k in range(nreq):
        lv = levels[rng.integers(len(levels))]
        members = int(rng.integers(1, 33))
        steps = int(rng.integers(10, 501))
        seed = int(rng.integers(1 << 30))
        reqs.append((lv, members, steps, seed))
    # initial states drawn as in the single-state case, per-request seeds
    states = [np.stack([gen.perturb_h(models[lv].H_init, seed + b) for b in range(mb)])
              for lv, mb, st, seed in reqs]
    launches0 = capi.kernel_launches()
    ids = []
    start = time.perf_counter()
    for k, (lv, mb, st, seed) in enumerate(reqs):
        delay = arrivals[k] - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(gids[lv], states[k], st))
    res = srv.wait(ids, timeout=600.0)
    wall = time.perf_counter() - start
    stats = srv.stats()
    outs = [srv.fetch(r) for r in ids]
    srv.stop()
    lat = np.array([res[r][2] for r in ids])
    wait_admit = np.array([res[r][1] for r in ids])
    member_steps = sum(mb * st for lv, mb, st, seed in reqs)
    wall = max_over_ranks(wall, f"cuda:{local}")      # each replica serves its own stream
    node_stages = sum(4.0 * models[lv].N * mb * st for lv, mb, st, seed in reqs)
    if rank == 0:
        line = {
            "metric": "serving: aggregate member-steps/s with p50/p99 request latency",
            "value": member_steps * world / wall, "unit": "member-steps/s", "n_gpus": world, "steps": None,
            "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic seeded request stream",
            "config": {"workload": args.workload, "description": desc, "requests": nreq,
                       "arrival_rate_per_s": args.rate, "seed": args.seed, "budget_bytes": args.budget_gb * 1e9,
                       "grid_order": args.serve_order},
            "grid_order_seconds": order_s,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "admission_wait_s": {"p50": float(np.percentile(wait_admit, 50)),
                                 "p99": float(np.percentile(wait_admit, 99))},
            "node_stage_updates_per_s": node_stages * world / wall,
            "wall_s": wall, "server": stats,
            "gpu_launches": int(capi.kernel_launches() - launches0),
            "state_finite": bool(all(np.isfinite(o).all() for o in outs)),
        }
        print(json.dumps(line), flush=True)
    finish_replicas()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain_fp64_n40962", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-targets", action="store_true",
                    help="skip the nested lines of the larger workloads in the default run")
    ap.add_argument("--target-steps", type=int, default=10, help="timed steps of each nested line")
    ap.add_argument("--err-steps", type=int, default=1000)
    ap.add_argument("--err-members", type=int, default=64)
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--budget-gb", type=float, default=80.0)
    ap.add_argument("--serve-order", default="device", choices=["device", "natural"],
                    help="node order the serving grids are registered in")
    ap.add_argument("--plain-kernel", default="auto", choices=sorted(PLAIN_KERNELS),
                    help="plain stage kernel: auto = the one swe_cuda_init timed fastest; the others pin a kernel "
                         "and shape (for profiling runs, where the init-time timing is not representative)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    level, prec, desc = WORKLOADS[args.workload]
    if args.impl == "reference":
        rlevel = level if level else 6
        rprec = "fp64" if prec in ("tf32x3", "bf16x3", "fp16x3", "serve") else prec
        return run_reference(args, rlevel, rprec, args.workload, desc)
    if prec in ("tf32x3", "bf16x3", "fp16x3"):
        return run_ensemble(args, desc)
    if prec == "serve":
        return run_serving(args, desc)

    import torch

    from swe_b200 import capi, layout, swe_input

    rank, local, world = world_info()
    torch.cuda.set_device(local)
    init_replicas()

    if level <= 6:
        # the input file the reference arm reads too
        path, d, sha = workload_input(level)
        m = swe_input.to_model(d)
        pm, _ = layout.prepare(m, use_rcm=True, simd_length=32)
    else:
        path, sha = None, None
        d, m, pm = build_workload(level, prec, device=f"cuda:{local}")
    N = d.N
    dt_np = np.float64 if prec == "fp64" else np.float32
    plain = capi.Plain()
    capi.check("swe_cuda_select_device", plain.lib.swe_cuda_select_device(local))
    plain.init_model(pm, prec)
    if args.plain_kernel != "auto":
        plain.select_kernel(PLAIN_KERNELS[args.plain_kernel])
    stream = torch.cuda.ExternalStream(plain.stream())
    flush = L2Flush(f"cuda:{local}")

    plain.set_state(pm.H_init.astype(dt_np))
    for _ in range(args.warmup):
        plain.step(1)
    plain.sync()

    # ---- device-resident timed region -------------------------------------------------
    launches0 = capi.kernel_launches()
    with ClockSampler(local) as clocks:
        clocks.wait_for(1, 5.0)
        first_sample = clocks.count()
        torch.cuda.profiler.start()                 # a profiler run with --profile-from-start off sees this loop only
        t_steps = timed_steps(lambda: plain.step(1), stream, args.steps, flush)
        torch.cuda.profiler.stop()
        launches = capi.kernel_launches() - launches0
        t_total = float(sum(t_steps))

        # ---- per-stage kernel durations (same stream, events), right after the timed
        # steps and at the same clocks -------------------------------------------------------
        plain.set_timing(True)
        with torch.cuda.stream(stream):
            for s in range(max(3, args.steps // 4)):
                flush()
                for st in range(4):
                    plain.rk_substep(st)
        k_time, k_launches, _ = plain.timings()
        plain.set_timing(False)

        # The timed region is far shorter than nvidia-smi's 200 ms period: keep
        # the same step loop running (untimed) until 3 samples cover it.
        def busy():
            for _ in range(200):
                plain.step(1)
            plain.sync()
        clocks.wait_for(first_sample + 3, 5.0, keep_busy=busy)
    t_total = max_over_ranks(t_total, f"cuda:{local}")
    value = 4.0 * N * args.steps * world / t_total

    # ---- end to end through the C ABI with pinned host buffers --------------------------
    H_host = torch.from_numpy(np.ascontiguousarray(pm.H_init, dtype=dt_np).reshape(-1)).pin_memory()
    H_out = torch.empty_like(H_host).pin_memory()
    nbytes = H_host.numel() * H_host.element_size()
    e2e_steps = max(3, args.steps // 2)
    for _ in range(2):
        plain.set_state_ptr(H_host.data_ptr())
        plain.step(1)
        plain.get_state_ptr(H_out.data_ptr())
    sync_ranks()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plain.set_state_ptr(H_host.data_ptr())
        plain.step(1)
        plain.get_state_ptr(H_out.data_ptr())     # synchronises
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(t_e2e, f"cuda:{local}")
    e2e = 4.0 * N * e2e_steps * world / t_e2e
    finite = bool(np.isfinite(H_out.numpy()).all())

    # ---- roofline of the fused stage kernel ------------------------------------------
    peak, peak_kind = measured_peak_hbm()
    # a timed step is the four stage kernels and nothing else: their average
    # duration in the timed region is step time / 4 (stages overlap by
    # programmatic dependent launch, which per-launch events would break up)
    t_kernel = t_total / (4 * args.steps)
    t_isolated = k_time / max(k_launches, 1)
    kinfo = plain.kernel_info()
    alg = plain_alg_bytes(prec, kinfo)
    achieved = alg * N / t_kernel / 1e9
    alg_per_launch = alg * N
    traffic = TRAFFIC_BYTES.get(args.workload)
    # data that fits the 126 MB L2 (with the flush's lines and headroom) is served from L2
    # for most of each step: its roofline is not an HBM roofline
    l2_resident = alg_per_launch < 100e6
    roofline = {"bound": "l2-resident" if l2_resident else "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "frac_of_spec_8tbs": round(achieved / SPEC_HBM_GBS, 4),
                "traffic": traffic, "peak_source": peak_kind,
                "kernel": {"pipelined": "swe::stage_tma_kernel", "register": "swe::stage_kernel",
                           "lane": "swe::stage_lane_kernel"}[kinfo["in_use"]],
                "kernel_us": round(t_kernel * 1e6, 2), "kernel_us_isolated": round(t_isolated * 1e6, 2),
                "alg_bytes_per_node_stage": alg, "alg_bytes_per_launch": alg_per_launch,
                "kernel_choice": kinfo}
    if l2_resident:
        roofline["note"] = (f"{alg_per_launch / 1e6:.1f} MB of algorithmic bytes per launch fit the 126 MB L2: "
                            "'achieved' counts them over the stage time and 'frac' divides that by the measured "
                            "HBM copy peak, an effective-bandwidth figure, not an HBM fraction; the HBM rooflines "
                            "are the targets' lines (N=163842 and N=655362)")
        if traffic:
            roofline["dram_achieved"] = round(traffic / t_kernel / 1e9, 1)
            roofline["dram_frac"] = round(traffic / t_kernel / 1e9 / peak, 4)
    plain.finalize()

    targets = None
    if args.workload == "plain_fp64_n40962" and not args.no_targets:
        targets = {}
        for wl in ("plain_fp64_n163842", "plain_fp64_n655362", "plain_fp32_n655362"):
            targets[wl] = plain_target(wl, local, args.target_steps, args.warmup, flush, world)
        for wl in ("ens_tf32_n163842_b64", "ens_fp16_n163842_b64"):
            targets[wl] = ensemble_target(
                wl, local, args.target_steps, args.warmup, flush, world,
                err_steps=args.err_steps, err_members=args.err_members,
                plain_rate=targets["plain_fp64_n163842"]["member_steps_per_s"] / world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if path is None:
                path, d, _ = workload_input(level)
            cpu = cpu_baseline_sample(path, d, prec)
        except Exception as e:            # reported, not fatal
            cpu = {"value": None, "unit": "node-stage updates/s", "error": str(e)[:200]}

    if rank == 0:
        config = plain_config(args.workload, desc, d, sha) if sha else \
            {"workload": args.workload, "description": desc, "nodes": N, "nnbr": d.Nnbr, "dt": d.dt,
             "layout": "CFDL", "rcm": True, "input": "generated on the GPU (seed 1)", "l2": L2_NOTE}
        line = {
            "metric": "node-stage updates/s (RK4 + RBF-FD stage, plain form)",
            "value": value, "unit": "node-stage updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": vs_recorded(args.workload, value)[0],
            "vs_baseline_source": vs_recorded(args.workload, value)[1],
            "dtype": "f64" if prec == "fp64" else "f32",
            "data": "synthetic (seeded icosahedral grid, PHS RBF-FD weights, TC5 Gaussian-mountain ICs)",
            "config": config,
            "parallelism": f"replicas x{world}",
            "e2e": {"value": e2e, "unit": "node-stage updates/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(first_sample),
            "state_finite": finite,
        }
        if targets is not None:
            line["targets"] = targets
        print(json.dumps(line), flush=True)
    finish_replicas()


if __name__ == "__main__":
    main()
