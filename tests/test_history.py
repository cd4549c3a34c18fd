"""History files (swe_hist_open): the format on CPU, and the writer on the GPU.

The reference declares a history output (USE_HIST, runtime_params.c:24-27) but
writes nothing, so the bar is internal consistency: every record equals, bit for
bit, what swe_cuda_get_state returns after that many RK4 steps.
"""
import numpy as np
import pytest

from conftest import generated_input
from swe_b200 import capi, history, layout, swe_input


def test_format_round_trip(tmp_path):
    states = np.random.default_rng(3).standard_normal((3, 40))
    p = tmp_path / "h.bin"
    history.write_history(p, interval=5, dt=900.0, steps=[5, 10, 15], states=states, layout=1, simd=32)
    h = history.read_history(p)
    assert (h.value_bytes, h.interval, h.dt, h.layout, h.simd) == (8, 5, 900.0, 1, 32)
    assert h.steps.tolist() == [5, 10, 15] and h.times.tolist() == [4500.0, 9000.0, 13500.0]
    assert np.array_equal(h.states, states)
    (tmp_path / "bad.bin").write_bytes(b"NOTAHIST" + bytes(56))
    with pytest.raises(ValueError):
        history.read_history(tmp_path / "bad.bin")
    (tmp_path / "cut.bin").write_bytes(p.read_bytes()[:-3])
    with pytest.raises(ValueError):
        history.read_history(tmp_path / "cut.bin")


@pytest.fixture(scope="module")
def plain():
    pl = capi.Plain()
    yield pl
    pl.finalize()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_records_equal_states_bitwise(plain, tmp_path, prec):
    _, d = generated_input(4)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    plain.init_model(m, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    H0 = m.H_init.astype(dt)
    # the states after 2, 4, 6 and 8 steps, one run each
    want = {}
    for k in (2, 4, 6, 8):
        plain.set_state(H0)
        plain.step(k)
        want[k] = plain.get_state().copy()
    path = tmp_path / f"hist_{prec}.bin"
    plain.set_state(H0)
    plain.hist_open(str(path), 2)
    plain.step(7)                        # records at steps 2, 4, 6
    for s in range(4):                   # step 8 by substeps: a record when substep 3 completes it
        plain.rk_substep(s)
    final = plain.get_state().copy()
    st = plain.hist_stats()
    plain.hist_close()
    assert st["open"] and st["steps"] == 8
    h = history.read_history(path)
    assert h.value_bytes == np.dtype(dt).itemsize and h.interval == 2
    assert h.steps.tolist() == [2, 4, 6, 8]
    assert np.allclose(h.times, h.steps * m.dt)
    for i, k in enumerate(h.steps):
        assert np.array_equal(h.states[i].reshape(want[k].shape), want[k]), k
    assert np.array_equal(h.states[-1].reshape(final.shape), final)
    assert plain.hist_stats()["open"] is False


@pytest.mark.gpu
def test_many_records_keep_order_under_back_pressure(plain, tmp_path):
    """interval 1 over 40 steps: more snapshots than copy slots, all written in order."""
    _, d = generated_input(4)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    plain.init_model(m, "fp64")
    plain.set_state(m.H_init)
    path = tmp_path / "many.bin"
    plain.hist_open(str(path), 1)
    plain.step(40)
    final = plain.get_state().copy()
    plain.hist_close()
    h = history.read_history(path)
    assert h.steps.tolist() == list(range(1, 41))
    assert np.array_equal(h.states[-1].reshape(final.shape), final)


@pytest.mark.gpu
def test_rejects_bad_interval(plain, tmp_path):
    _, d = generated_input(4)
    plain.init_model(swe_input.to_model(d), "fp64")
    with pytest.raises(capi.SweError):
        plain.hist_open(str(tmp_path / "x.bin"), 0)
