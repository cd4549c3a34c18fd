"""swe_cuda_step_noalloc: RK4 steps for callers that cannot allocate device memory.

Callers whose device memory belongs to an outer framework's pool, or whose
loops may not pay an allocation's implicit device synchronisation, own every
buffer themselves and pass device pointers; the entry point keeps its K/D
registers in a static device array instead of calling cudaMalloc.  This test
owns its buffers through torch (the test is the caller), runs the entry point
twice in a row through the C ABI, and compares each result with the
allocating entry point (swe_cuda_init + swe_cuda_step) at the tolerance the
other plain-form tests use.  It lives in its own file so that it is collected
last.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
from swe_b200 import capi, swe_input

pytestmark = pytest.mark.gpu

NSTEPS = 20


def _bind():
    lib = capi.load()
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.swe_cuda_step_noalloc.argtypes = [i, i, i, d, d] + [vp] * 15 + [i, vp]
    lib.swe_cuda_step_noalloc.restype = i
    return lib


def _model():
    return swe_input.load_model(os.path.join(GOLDEN, "icos162_seed7.bin"))


def _reference_steps(m):
    plain = capi.Plain()
    plain.init_model(m, "fp64")
    plain.set_state(m.H_init)
    plain.step(NSTEPS)
    H = plain.get_state().reshape(-1, 4)
    plain.finalize()
    return H


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    lib = _bind()
    m = _model()
    want = _reference_steps(m)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(m, k))).to(dev) for k in
         ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")}
    t["idx"] = torch.from_numpy(np.ascontiguousarray(m.idx, dtype=np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        H = torch.from_numpy(np.ascontiguousarray(m.H_init)).to(dev)
        st = lib.swe_cuda_step_noalloc(
            8, m.N, m.Nnbr, float(m.gh0), float(m.dt), t["idx"].data_ptr(),
            *[t[k].data_ptr() for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm",
                                        "p_u", "p_v", "p_w", "gradghm")],
            H.data_ptr(), NSTEPS, stream.cuda_stream)
        assert st == 0, lib.swe_cuda_last_error()
        torch.cuda.synchronize(dev)
        got = H.cpu().numpy()
        assert np.isfinite(got).all(), f"call {call}"
        assert rel_err(got, want).max() <= 1e-12, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_static_scratch():
    lib = _bind()
    limit = (4 << 20) // (12 * 8)
    dummy = ctypes.c_void_p(16)          # never dereferenced: the size check comes first
    st = lib.swe_cuda_step_noalloc(8, limit + 1, 31, 0.0, 1.0, *([dummy] * 15), 1, None)
    assert st == 1
    assert b"static scratch" in lib.swe_cuda_last_error()
