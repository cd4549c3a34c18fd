"""Node ordering on the device (swe_dev_rcm_mapping), against its plain-Python
statement (tests/levelset_order.py) and the reference's RCM bandwidth.

* the device order is exactly the breadth-first level order stated in Python
  (keys are unique, so there is one answer), on generated grids up to N=40962;
* its bandwidth (rcm.c:68-96's max and mean of max - min stencil index) is no
  larger than 1.05x the reference's RCM order's, at every size up to N=655362;
* a patch ordered by it steps like the oracle (the order changes the node
  numbering only).
"""
import time

import numpy as np
import pytest

import oracle
from conftest import generated_input, rel_err
from levelset_order import levelset_mapping
from swe_b200 import capi, layout, swe_input

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [3, 4, 6])
def test_device_order_equals_statement(level):
    _, d = generated_input(level)
    m = swe_input.to_model(d)
    got = layout.rcm_mapping(m, device=True)
    assert np.array_equal(np.sort(got), np.arange(m.N))
    assert np.array_equal(got, levelset_mapping(m.idx))


@pytest.mark.parametrize("level", [4, 6, 8])
def test_device_order_bandwidth_vs_reference_rcm(level):
    _, d = generated_input(level, device="cuda" if level >= 7 else "cpu")
    m = swe_input.to_model(d)
    t0 = time.perf_counter()
    dev = layout.rcm_mapping(m, device=True)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref = layout.rcm_mapping(m)
    t_host = time.perf_counter() - t0
    bw_dev = layout.bandwidth(layout.reorder(m, dev).idx)
    bw_ref = layout.bandwidth(layout.reorder(m, ref).idx)
    print(f"N={m.N}: device order bandwidth {bw_dev} in {t_dev:.3f} s, reference RCM {bw_ref} in {t_host:.3f} s")
    assert bw_dev[0] <= 1.05 * bw_ref[0] and bw_dev[1] <= 1.05 * bw_ref[1]


def test_patch_in_device_order_steps_like_oracle():
    _, d = generated_input(4, fill_fc=True)
    m, mapping = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32, device_order=True)
    plain = capi.Plain()
    try:
        plain.init_model(m, "fp64")
        plain.set_state(m.H_init)
        plain.step(20)
        H = plain.get_state().reshape(-1, 4)
    finally:
        plain.finalize()
    assert rel_err(H, oracle.Port(m, "fp64").run(m.H_init, 20)).max() <= 1e-12
