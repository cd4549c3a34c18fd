"""Host-side pieces of bench.py's JSON line that need no GPU: the tensor-core roofline
of the batched stage and the HBM fractions."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_tensor_roofline_counts_every_chunk_product():
    # 43128 chunks of 16 rows, M = 4 x 32 (operators x tile nodes), N = 4 x 64 member-fields,
    # three products of 2 flops per multiply-add
    cfg = {"chunks": 43128, "tile_nodes": 32}
    r = bench.ensemble_tensor_roofline(cfg, 64, "tf32x3", 334e-6)
    assert r["mma_flops_per_launch"] == 43128 * 16 * 128 * 256 * 2 * 3
    bf16, _ = bench.measured_peak_bf16_tflops()
    assert r["peak"] == round(bf16 / 2, 1)                      # TF32 at half the BF16 rate
    assert abs(r["achieved"] - r["mma_flops_per_launch"] / 334e-6 / 1e12) < 0.05
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    rb = bench.ensemble_tensor_roofline(cfg, 64, "bf16x3", 334e-6)
    assert rb["peak"] == round(bf16, 1)
    # split FP16 runs kind::f16 at the 16-bit rate, like split BF16
    assert bench.ensemble_tensor_roofline(cfg, 64, "fp16x3", 334e-6)["peak"] == round(bf16, 1)
    # 16-node tiles: M = 64
    r16 = bench.ensemble_tensor_roofline({"chunks": 1000, "tile_nodes": 16}, 32, "tf32x3", 1e-3)
    assert r16["mma_flops_per_launch"] == 1000 * 16 * 64 * 128 * 2 * 3


def test_spec_fraction_uses_8_tbs():
    assert bench.SPEC_HBM_GBS == 8000.0


def test_plain_bytes_follow_the_index_width():
    lane16 = {"in_use": "lane", "index_offsets_16bit": True}
    lane32 = {"in_use": "lane", "index_offsets_16bit": False}
    assert bench.plain_alg_bytes("fp64", lane16) == 4 * 31 * 8 + 31 * 2 + 17 * 8 + 4 * 8 + 14 * 8
    assert bench.plain_alg_bytes("fp64", lane32) == 1396
    assert bench.plain_alg_bytes("fp32", lane16) == 760 - 62
    # the other kernels read 32-bit indices whatever the lane kernel would read
    assert bench.plain_alg_bytes("fp64", {"in_use": "pipelined", "index_offsets_16bit": True}) == 1396


def test_fp16_ensemble_workload_is_registered():
    level, prec, desc = bench.WORKLOADS["ens_fp16_n163842_b64"]
    assert (level, prec) == (7, "fp16x3") and "FP16" in desc
    assert bench.TRAFFIC_BYTES["ens_fp16_n163842_b64"] > 0
