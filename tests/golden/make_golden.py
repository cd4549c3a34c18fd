"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root after `make -C oracle` has built the reference
libraries (oracle/_ref, which needs the reference sources):

    python tests/golden/make_golden.py

Outputs
  icos162_seed7.bin   a level-2 (N=162) synthetic input in the reference's binary
                      format (swe_b200.gen, seed 7; H_100 = the reference's own
                      100-step FP64 result)
  icos162_ref.npz     outputs of the reference's own eval_RHS_swe and RK_substep
                      (swe_code/main/rk4_rbffd_swe.c, built from source, CFDL
                      layout, no RCM) on that input:
                        F0      eval_RHS_swe(H_init)                 FP64 [192, 4]
                        K1      H_init + seeded perturbation          FP64
                        F1      eval_RHS_swe(K1)                      FP64
                        H10     10 RK4 steps from H_init              FP64
                        F0_32   eval_RHS_swe(H_init) of the FP32 build
                        H10_32  10 RK4 steps of the FP32 build
                        mapping the reference's RCM permutation (rcm.c:9-62)
                        H10_rcm 10 RK4 steps with RCM on (reference order)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rbf-fd-swe_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from swe_b200 import gen, swe_input  # noqa: E402


def main():
    d = gen.generate(2, seed=7)
    path = os.path.join(HERE, "icos162_seed7.bin")
    swe_input.write_input(path, d)
    ref = oracle.Ref(path, "fp64", "cfdl", use_rcm=0)
    H, _, _ = ref.run(ref.H_init(), 100)
    d.H_100[:] = H.reshape(-1, 4)[: d.N]
    swe_input.write_input(path, d)

    ref = oracle.Ref(path, "fp64", "cfdl", use_rcm=0)
    H0 = ref.H_init()
    rng = np.random.default_rng(11)
    K1 = H0 * (1.0 + 1e-3 * rng.standard_normal(H0.shape))
    out = {
        "F0": ref.eval_rhs(H0).reshape(-1, 4),
        "K1": K1.reshape(-1, 4),
        "F1": ref.eval_rhs(K1).reshape(-1, 4),
        "H10": ref.run(H0, 10)[0].reshape(-1, 4),
    }
    assert ref.verify(ref.run(H0, 100)[0])[0] == 0
    r32 = oracle.Ref(path, "fp32", "cfdl", use_rcm=0)
    out["F0_32"] = r32.eval_rhs(r32.H_init()).reshape(-1, 4)
    out["H10_32"] = r32.run(r32.H_init(), 10)[0].reshape(-1, 4)
    rr = oracle.Ref(path, "fp64", "cfdl", use_rcm=1)
    out["mapping"] = rr.mapping()
    out["H10_rcm"] = rr.run(rr.H_init(), 10)[0].reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "icos162_ref.npz"), **out)
    print("wrote", path, "and icos162_ref.npz")


if __name__ == "__main__":
    main()
