"""swe_cuda_step_noalloc: RK4 steps for callers that cannot allocate device memory.

Callers whose device memory belongs to an outer framework's pool, or whose
loops may not pay an allocation's implicit device synchronisation, own every
buffer themselves and pass device pointers; the entry point keeps its K/D
registers in a static device array instead of calling cudaMalloc.  This test
owns its buffers through torch (the test is the caller), runs the entry point
twice in a row through the C ABI, and compares each result with the
allocating entry point (swe_cuda_init + swe_cuda_step) at the tolerance the
other plain-form tests use, in FP64 and FP32, on a small grid and on one that
fills most of the static array.  It lives in its own file so that it is collected
last.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, scaled_err
from swe_b200 import capi, swe_input

pytestmark = pytest.mark.gpu

NSTEPS = 20
# FP64: the other plain-form tests' 1e-12 relative bar.  FP32: both paths round every
# operation to FP32 in different summation orders (this path sums slots in the 8-lane
# tree, the allocating one in the kernel its init timing picked), so they are held to
# each other within 1e-4 of each field's scale after 20 steps (u, v, w on the velocity
# scale max|(u, v, w)|, h on max|h|) and to the reference's FP32 verify tolerance,
# 4e-2 absolute (swe_config.h:80).
REL_BAR = {"fp64": 1e-12, "fp32": 1e-4}


def _bind():
    lib = capi.load()
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.swe_cuda_step_noalloc.argtypes = [i, i, i, d, d] + [vp] * 15 + [i, vp]
    lib.swe_cuda_step_noalloc.restype = i
    return lib


def _model(which):
    if which == "n162":
        return swe_input.load_model(os.path.join(GOLDEN, "icos162_seed7.bin"))
    # N=40962 (level 6): 94% of the FP64 node limit, so K, K and D fill most of the array
    from swe_b200 import gen
    return swe_input.to_model(gen.generate(6, seed=1, device="cuda"))


def _reference_steps(m, prec):
    plain = capi.Plain()
    plain.init_model(m, prec)
    plain.set_state(m.H_init.astype(np.float64 if prec == "fp64" else np.float32))
    plain.step(NSTEPS)
    H = plain.get_state().reshape(-1, 4)
    plain.finalize()
    return H


@pytest.mark.parametrize("which", ["n162", "n40962"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_noalloc_matches_allocating_entry_point_twice(prec, which):
    import torch

    lib = _bind()
    m = _model(which)
    fsize = 8 if prec == "fp64" else 4
    assert m.N <= capi.NOALLOC_SCRATCH_BYTES // (12 * fsize)
    dt = np.float64 if prec == "fp64" else np.float32
    want = _reference_steps(m, prec)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(m, k), dtype=dt)).to(dev) for k in
         ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")}
    t["idx"] = torch.from_numpy(np.ascontiguousarray(m.idx, dtype=np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        H = torch.from_numpy(np.ascontiguousarray(m.H_init, dtype=dt)).to(dev)
        st = lib.swe_cuda_step_noalloc(
            fsize, m.N, m.Nnbr, float(m.gh0), float(m.dt), t["idx"].data_ptr(),
            *[t[k].data_ptr() for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm",
                                        "p_u", "p_v", "p_w", "gradghm")],
            H.data_ptr(), NSTEPS, stream.cuda_stream)
        assert st == 0, lib.swe_cuda_last_error()
        # nsteps = 0 waits for the stream and reports any out-of-range stencil index
        # the kernels met: none here
        st = lib.swe_cuda_step_noalloc(
            fsize, m.N, m.Nnbr, float(m.gh0), float(m.dt), t["idx"].data_ptr(),
            *[t[k].data_ptr() for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm",
                                        "p_u", "p_v", "p_w", "gradghm")],
            H.data_ptr(), 0, stream.cuda_stream)
        assert st == 0, lib.swe_cuda_last_error()
        got = H.cpu().numpy().reshape(-1, 4)
        assert np.isfinite(got).all(), f"call {call}"
        err = scaled_err(got, want)
        print(f"{prec} {which} call {call}: rel err per field {err}")
        assert err.max() <= REL_BAR[prec], f"call {call}"
        if prec == "fp32":
            assert np.abs(got.astype(np.float64) - want).max() <= 4e-2


def test_noalloc_rejects_sizes_beyond_its_static_scratch():
    lib = _bind()
    limit = capi.NOALLOC_SCRATCH_BYTES // (12 * 8)
    dummy = ctypes.c_void_p(16)          # never dereferenced: the size check comes first
    st = lib.swe_cuda_step_noalloc(8, limit + 1, 31, 0.0, 1.0, *([dummy] * 15), 1, None)
    assert st == 1
    assert b"static scratch" in lib.swe_cuda_last_error()
