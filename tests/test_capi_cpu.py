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


def test_header_compiles_as_c_and_links(tmp_path):
    """The reference's host is C99: include/swe_b200.h must compile as C with warnings
    as errors, and a C program must link against the library and call it (a call that
    fails before any device work, so no GPU is needed)."""
    import os
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(capi.LIB_PATH)
    src = tmp_path / "use_swe.c"
    src.write_text(
        '#include <stdio.h>\n'
        '#include "swe_b200.h"\n'
        'int main(void) {\n'
        '    int st = swe_cuda_step(1);          /* before swe_cuda_init: a state error */\n'
        '    const char* msg = swe_cuda_last_error();\n'
        '    printf("%d %s\\n", st, msg);\n'
        '    return (st == SWE_ERR_STATE && swe_b200_kernel_launches() >= 0) ? 0 : 1;\n'
        '}\n')
    exe = tmp_path / "use_swe"
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(root, "include"),
                    str(src), "-L", libdir, "-lswe_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("2 ") and "swe_cuda_init" in out.stdout


def test_noalloc_argument_checks_fail_before_device_work():
    """swe_cuda_step_noalloc checks its arguments before any CUDA call: a bad fsize,
    stencil width, step count, node count or null pointer is rejected with
    SWE_ERR_ARG.  The dummy pointers are never dereferenced."""
    lib = capi.load()
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.swe_cuda_step_noalloc.argtypes = [i, i, i, d, d] + [vp] * 15 + [i, vp]
    dummy = [ctypes.c_void_p(16)] * 15
    limit = capi.NOALLOC_SCRATCH_BYTES // (12 * 8)
    assert lib.swe_cuda_step_noalloc(3, 100, 31, 0.0, 1.0, *dummy, 1, None) == 1
    assert lib.swe_cuda_step_noalloc(8, 100, 33, 0.0, 1.0, *dummy, 1, None) == 1
    assert b"nnbr" in lib.swe_cuda_last_error()
    assert lib.swe_cuda_step_noalloc(8, 100, 31, 0.0, 1.0, *dummy, -1, None) == 1
    assert lib.swe_cuda_step_noalloc(8, 0, 31, 0.0, 1.0, *dummy, 1, None) == 1
    assert lib.swe_cuda_step_noalloc(8, limit + 1, 31, 0.0, 1.0, *dummy, 1, None) == 1
    assert b"static scratch" in lib.swe_cuda_last_error()
    assert lib.swe_cuda_step_noalloc(4, 2 * limit + 2, 31, 0.0, 1.0, *dummy, 1, None) == 1
    assert lib.swe_cuda_step_noalloc(8, 100, 31, 0.0, 1.0, *([None] + dummy[1:]), 1, None) == 1
    assert b"null" in lib.swe_cuda_last_error()


def test_device_order_argument_checks_fail_before_device_work():
    lib = capi.load()
    lib.swe_dev_rcm_mapping.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    idx = np.zeros((4, 3), dtype=np.int32)
    out = np.zeros(4, dtype=np.int32)
    assert lib.swe_dev_rcm_mapping(0, 3, idx.ctypes.data, out.ctypes.data) == 1
    assert lib.swe_dev_rcm_mapping(4, 1, idx.ctypes.data, out.ctypes.data) == 1
    assert lib.swe_dev_rcm_mapping(4, 3, None, out.ctypes.data) == 1
    idx[2, 1] = 9
    assert lib.swe_dev_rcm_mapping(4, 3, idx.ctypes.data, out.ctypes.data) == 5      # SWE_ERR_INDEX
    assert b"outside" in lib.swe_cuda_last_error()
