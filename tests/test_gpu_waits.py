"""The bounded-wait path of the pipelined kernels, exercised without a fault:
a wait that nothing completes gives up after its limit, the kernel returns,
the host reads SWE_ERR_TIMEOUT and the same context keeps working."""
import ctypes

import numpy as np
import pytest

from conftest import generated_input
from swe_b200 import capi, swe_input

pytestmark = pytest.mark.gpu


def test_wait_that_never_completes_times_out_and_context_survives():
    lib = capi.load()
    waited = ctypes.c_double(0.0)
    st = lib.swe_selftest_wait_timeout(0.05, ctypes.byref(waited))
    assert st == 6, (st, lib.swe_cuda_last_error())         # SWE_ERR_TIMEOUT
    assert 0.05 <= waited.value < 1.0, waited.value
    # the context is intact: a normal run afterwards
    _, d = generated_input(4)
    m = swe_input.to_model(d)
    p = capi.Plain()
    p.init_model(m, "fp64")
    p.set_state(m.H_init)
    p.step(3)
    assert np.isfinite(p.get_state()).all()
    p.finalize()


def test_selftest_rejects_unbounded_limits():
    lib = capi.load()
    assert lib.swe_selftest_wait_timeout(0.0, None) == 1      # SWE_ERR_ARG
    assert lib.swe_selftest_wait_timeout(5.0, None) == 1
