"""Test infrastructure (oracle): time the reference's own CPU code on one input file.

    python oracle/cpu_baseline.py <input.bin> <fp64|fp32> <seconds>

Run as a fresh process by bench.py's CPU-baseline leg and its reference arm, with
OMP_NUM_THREADS / OMP_PROC_BIND / OMP_SCHEDULE set by the caller.  A process of its
own keeps the timed OpenMP team alone on the host cores: in a process that also
holds a GPU context and PyTorch's own thread pool, the reference's static schedule
waited at every barrier for descheduled threads (2.6e6 node-stage/s on 16 threads
there, against 9.6e7 alone on the same host).

Prints one JSON object: steps, loop seconds, the reference's own Eval_Rhs seconds
(profiling.c:118-126), and which code ran ("reference": oracle/_ref, the reference's
sources compiled here; "port": the oracle's C restatement, where the reference was
not built).
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import oracle  # noqa: E402


def main() -> None:
    path, prec, budget = sys.argv[1], sys.argv[2], float(sys.argv[3])
    if oracle.reference_available(prec, "cfdl"):
        ref = oracle.Ref(path, prec, "cfdl", use_rcm=1)
        H0 = ref.H_init()

        def run(k):
            _, t, t_rhs = ref.run(H0, k)
            return t, t_rhs
        kind = "reference"
    else:
        sys.path.insert(0, os.path.join(os.path.dirname(HERE), "rbf-fd-swe_b200"))
        from swe_b200 import swe_input

        m = swe_input.load_model(path)
        port = oracle.Port(m, prec)

        def run(k):
            t0 = time.perf_counter()
            port.run(m.H_init, k)
            return time.perf_counter() - t0, None
        kind = "port"
    run(1)                                        # warm-up (page faults, thread team)
    t1, _ = run(1)                                # sizes the sample
    steps = max(1, min(500, int(budget / max(t1, 1e-5))))
    t, t_rhs = run(steps)
    print(json.dumps({"steps": steps, "seconds": t, "eval_rhs_seconds": t_rhs, "kind": kind}))


if __name__ == "__main__":
    main()
