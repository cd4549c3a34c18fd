"""The reference's own main program, built with a SWE_USE_CUDA switch beside its
SWE_USE_OCL one (oracle/patch_main.py, `make -C oracle host`), on its shipped
N=2562 input: 100 RK4 steps per attempt and the reference's own verify_output
against H_100 (main.c:439-477, FP64 tolerance 1e-9).

* CPU: SWE_USE_CUDA=0 is the reference's unchanged CPU path through the same
  executable.
* GPU: SWE_USE_CUDA=1 steps through libswe_b200.so (swe_cuda_init_psmd,
  swe_cuda_set_state, swe_cuda_rk_substep, swe_cuda_get_state) and the
  reference's host code verifies the result.
"""
import os
import subprocess

import pytest

import oracle

EXE = os.path.join(oracle.REF_DIR, "swe_host_cuda_fp64_cfdl.exe")


def _run(use_cuda: int, attempts: int):
    if not os.path.exists(EXE) or not os.path.exists(oracle.SHIPPED_INPUT):
        pytest.skip("the reference host was not built (make -C oracle host)")
    env = dict(os.environ, SWE_INPUT_FILE=oracle.SHIPPED_INPUT, SWE_USE_NETCDF="0", SWE_NUM_COMPUTE_UNITS="1",
               SWE_NSTEPS="100", SWE_NATTEMPTS=str(attempts), SWE_USE_RCM="1", SWE_USE_OCL="0",
               SWE_USE_CUDA=str(use_cuda), OMP_NUM_THREADS="4")
    return subprocess.run([EXE], env=env, capture_output=True, text=True, timeout=600)


def test_reference_host_cpu_path_verifies():
    out = _run(0, 1)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert out.stdout.count("VERIFICATION SUCCEEDED") == 1


@pytest.mark.gpu
def test_reference_host_drives_the_library_and_verifies():
    out = _run(1, 2)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert out.stdout.count("VERIFICATION SUCCEEDED") == 2, out.stdout[-2000:]
    assert "VERIFICATION FAILED" not in out.stdout
