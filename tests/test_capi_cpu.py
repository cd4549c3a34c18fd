"""The C-ABI library loads and exports what include/swe_b200.h declares.

No compute calls: only entry points whose argument checks fail before any
CUDA call are exercised, so this runs without a GPU.
"""
import ctypes

import numpy as np
import pytest

from swe_b200 import capi


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = capi.declared_symbols()
    assert "swe_cuda_init" in names and "swe_cuda_eval_rhs" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_calls_before_init_report_state_error():
    lib = capi.load()
    assert lib.swe_cuda_step(1) == 2               # SWE_ERR_STATE
    assert lib.swe_cuda_rk_substep(0) == 2
    assert b"swe_cuda_init" in lib.swe_cuda_last_error()


def test_init_argument_checks_fail_before_device_work():
    lib = capi.load()
    z = np.zeros(64)
    i = np.zeros(64, dtype=np.int32)
    ptrs = [z.ctypes.data] * 9 + [i.ctypes.data] + [z.ctypes.data] * 4
    # fsize 3 is neither FP32 nor FP64
    assert lib.swe_cuda_init(3, 1, 1, 2, 2, 0, 1, 1, 0.0, 1.0, *ptrs) == 1
    # stencils wider than 32 slots are rejected
    assert lib.swe_cuda_init(8, 1, 1, 2, 2, 0, 33, 33, 0.0, 1.0, *ptrs) == 1
    assert b"nnbr" in lib.swe_cuda_last_error()
    # patch smaller than the compute range
    assert lib.swe_cuda_init(8, 1, 1, 4, 2, 0, 1, 1, 0.0, 1.0, *ptrs) == 1
    # null array
    assert lib.swe_cuda_init(8, 1, 1, 2, 2, 0, 1, 1, 0.0, 1.0, *([None] + ptrs[1:])) == 1
