"""Reader (and, for tests and tools, writer) of the history files that
swe_hist_open produces: snapshots of the plain form's state every few RK4 steps.

Layout (little endian):
    header, 64 bytes: b"SWEHIST1", int32 value bytes (4 or 8), int32 interval,
        int64 values per record, float64 dt, int32 layout flags (bit 0 CFDL,
        bit 1 SFDL), int32 SIMD length, 24 zero bytes;
    record: int64 step, float64 time (= step * dt), then the values -- the
        state in the caller's layout, exactly what swe_cuda_get_state returns.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

MAGIC = b"SWEHIST1"
HEADER = np.dtype([("magic", "S8"), ("value_bytes", "<i4"), ("interval", "<i4"), ("nvalues", "<i8"),
                   ("dt", "<f8"), ("layout", "<i4"), ("simd", "<i4"), ("pad", "V24")])
assert HEADER.itemsize == 64


@dataclass
class History:
    value_bytes: int
    interval: int
    dt: float
    layout: int
    simd: int
    steps: np.ndarray          # [records] int64
    times: np.ndarray          # [records] float64
    states: np.ndarray         # [records, values] float32 or float64


def _record_dtype(value_bytes: int, nvalues: int) -> np.dtype:
    return np.dtype([("step", "<i8"), ("time", "<f8"), ("values", "<f%d" % value_bytes, (nvalues,))])


def read_history(path: str | os.PathLike) -> History:
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < HEADER.itemsize:
        raise ValueError(f"{path}: shorter than the 64-byte header")
    h = raw[:HEADER.itemsize].view(HEADER)[0]
    if bytes(h["magic"]) != MAGIC:
        raise ValueError(f"{path}: not a history file (magic {bytes(h['magic'])!r})")
    vb, nv = int(h["value_bytes"]), int(h["nvalues"])
    if vb not in (4, 8) or nv <= 0:
        raise ValueError(f"{path}: bad header (value bytes {vb}, values {nv})")
    rec = _record_dtype(vb, nv)
    body = raw[HEADER.itemsize:]
    if body.size % rec.itemsize:
        raise ValueError(f"{path}: {body.size} bytes of records is not a whole number of {rec.itemsize}-byte records")
    r = body.view(rec)
    return History(vb, int(h["interval"]), float(h["dt"]), int(h["layout"]), int(h["simd"]),
                   r["step"].copy(), r["time"].copy(), r["values"].copy())


def write_history(path: str | os.PathLike, interval: int, dt: float, steps, states, layout: int = 0,
                  simd: int = 1) -> None:
    """The same format from numpy (test fixtures, converting other runs)."""
    states = np.asarray(states)
    vb = states.dtype.itemsize
    if states.ndim != 2 or vb not in (4, 8):
        raise ValueError("states must be [records, values] float32 or float64")
    h = np.zeros(1, HEADER)
    h["magic"], h["value_bytes"], h["interval"], h["nvalues"] = MAGIC, vb, interval, states.shape[1]
    h["dt"], h["layout"], h["simd"] = dt, layout, simd
    r = np.zeros(states.shape[0], _record_dtype(vb, states.shape[1]))
    r["step"] = np.asarray(steps, dtype=np.int64)
    r["time"] = r["step"] * dt
    r["values"] = states
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(r.tobytes())
