"""The split-FP16 ensemble's state-field scales (ens::fp16_field_scale), compiled for the
host from the kernel's own header: each field's largest |value| lands at 2^11..2^12, the
three velocity components share one scale, a zero field gets 1, and every scale is an
exact power of two whose inverse multiplies back to 1; exponents are clamped to
+-60."""
import math
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("fp16") / "fp16_scale_check")
    subprocess.run([NVCC, "-std=c++17", "-o", exe, os.path.join(HERE, "fp16_scale_check.cu")], check=True,
                   capture_output=True)
    return exe


def scales(exe, maxima):
    out = subprocess.run([exe] + [repr(float(m)) for m in maxima], check=True, capture_output=True, text=True)
    return [tuple(float.fromhex(x) for x in line.split()) for line in out.stdout.strip().splitlines()]


@pytest.mark.parametrize("maxima", [(20.0, 20.0, 0.0, 9511.9), (2.5e-3, 7.0, 1e-9, 1.0), (0.0, 0.0, 0.0, 3.0e4),
                                    (1e-30, 0.0, 0.0, 0.125)])
def test_field_scales(checker, maxima):
    s = scales(checker, maxima)
    vmax = max(maxima[:3])
    for f, (sc, inv) in enumerate(s):
        m = vmax if f < 3 else maxima[3]
        assert sc * inv == 1.0
        assert math.frexp(sc)[0] == 0.5           # a power of two
        if m == 0.0:
            assert sc == 1.0
        else:
            e = min(60, max(-60, 12 - math.frexp(m)[1]))
            assert sc == 2.0 ** e, (f, m, sc)
            if abs(e) < 60:
                assert 2.0 ** 11 <= m * sc < 2.0 ** 12, (f, m, sc)
    assert s[0] == s[1] == s[2]                    # u, v, w share one scale
