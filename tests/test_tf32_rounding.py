"""The operand converters round to TF32 with integer operations
(csrc/tcgen05.cuh:tf32_rna): (bits + 0x1000) & 0xffffe000.  This checks that
formula, on the CPU, against an exact restatement of round-to-nearest with ties
away from zero at 11 significant bits, over random and edge-case finite floats."""
from fractions import Fraction

import numpy as np


def _formula(x: np.ndarray) -> np.ndarray:
    b = x.astype(np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def _exact_rna_tf32(v: float) -> float:
    """Nearest TF32 value (ties away from zero), by exact arithmetic: 11 significant
    bits for normal values; below 2**-126 TF32, like FP32, keeps the fixed quantum of
    its smallest exponent (2**-136)."""
    if v == 0.0:
        return v
    _, e = np.frexp(np.float64(v))                 # |v| = m * 2**e, 0.5 <= m < 1
    quantum = Fraction(2) ** (max(int(e), -125) - 11)
    q = abs(Fraction(float(v))) / quantum
    n = int(q)
    if q - n >= Fraction(1, 2):
        n += 1
    r = n * quantum
    return float(np.float32(float(r) if v > 0 else -float(r)))


def test_tf32_rounding_formula_matches_exact_rounding():
    rng = np.random.default_rng(7)
    vals = np.concatenate([
        rng.standard_normal(20000).astype(np.float32) * np.float32(6000.0),
        rng.standard_normal(20000).astype(np.float32) * np.float32(1e-4),
        (rng.integers(0, 2**31 - 2**24, 20000, dtype=np.uint32)).view(np.float32),   # any finite bit pattern
    ])
    vals = vals[np.isfinite(vals) & (np.abs(vals) < np.float32(3e38))]
    # exact ties and the carry into the exponent
    ties = np.array([1 + 2**-11, 1 + 3 * 2**-11, 2 - 2**-11, -(1 + 2**-11), 0.5 - 2**-13, 0.0, -0.0],
                    dtype=np.float32)
    vals = np.concatenate([vals, ties])
    got = _formula(vals)
    want = np.array([_exact_rna_tf32(float(v)) for v in vals], dtype=np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the remainder x - hi is exact in FP32 and at most half a TF32 ulp
    x64, hi64 = vals.astype(np.float64), got.astype(np.float64)
    lo = (vals - got).astype(np.float64)
    assert np.array_equal(lo, x64 - hi64)
    normal = np.abs(x64) >= 2.0**-126
    assert np.all(np.abs(lo[normal]) <= np.abs(x64[normal]) * 2.0**-11 * (1 + 2.0**-10))
