"""Reader and writer for the mini-app's binary input format.

The format is the one ``swe_code/io/input.c:189-414`` reads and
``swe_code/io/nc2bin.c:32-80`` writes (all little-endian)::

    int32 N, int32 Nnbr
    f64 a, gh0, dt, gamma
    f64 x[N], y[N], z[N], f[N], ghm[N]
    f64 p_u[N][3], p_v[N][3], p_w[N][3], gradghm[N][3]
    f64 Dx[N][Nnbr], Dy[N][Nnbr], Dz[N][Nnbr], L[N][Nnbr]   (unit sphere, unscaled)
    int32 idx[N][Nnbr]                                        (1-based)
    f64 H_init[N][4], H_100[N][4]                             (u, v, w, h per node)

``load_model`` applies what ``get_GSMD_bin`` applies after reading
(input.c:314-328): Dx, Dy, Dz divided by ``a`` and L multiplied by ``gamma``,
both in FP64 (the input precision), and idx shifted to 0-based.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class SweInput:
    """Raw contents of one input file (no scaling applied)."""

    N: int
    Nnbr: int
    a: float
    gh0: float
    dt: float
    gamma: float
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    f: np.ndarray
    ghm: np.ndarray
    p_u: np.ndarray        # [N, 3]
    p_v: np.ndarray
    p_w: np.ndarray
    gradghm: np.ndarray
    Dx: np.ndarray         # [N, Nnbr] unit-sphere weights
    Dy: np.ndarray
    Dz: np.ndarray
    L: np.ndarray          # unscaled hyperviscosity weights
    idx1: np.ndarray       # [N, Nnbr] int32, 1-based
    H_init: np.ndarray     # [N, 4]
    H_100: np.ndarray      # [N, 4]


@dataclasses.dataclass
class SweModel:
    """Model-ready static data in canonical order (the reader's scaling applied).

    Arrays are FP64 node-major; idx is 0-based int32 [N, Nnbr].
    """

    N: int
    Nnbr: int
    gh0: float
    dt: float
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    f: np.ndarray
    ghm: np.ndarray
    p_u: np.ndarray
    p_v: np.ndarray
    p_w: np.ndarray
    gradghm: np.ndarray
    idx: np.ndarray
    Dx: np.ndarray
    Dy: np.ndarray
    Dz: np.ndarray
    L: np.ndarray
    H_init: np.ndarray
    H_100: np.ndarray


def file_size(N: int, Nnbr: int) -> int:
    """Byte size of a file with N nodes and Nnbr-point stencils (input.c:358, :399)."""
    return 4 * (2 + N * Nnbr) + 8 * (4 + 5 * N + 4 * N * 3 + 4 * N * Nnbr + 2 * N * 4)


def read_input(path: str) -> SweInput:
    """Parse one binary input file; raises ValueError on a truncated or inconsistent file."""
    size = os.path.getsize(path)
    with open(path, "rb") as fh:
        head = fh.read(8)
        if len(head) != 8:
            raise ValueError(f"{path}: truncated header")
        N, Nnbr = (int(v) for v in np.frombuffer(head, dtype="<i4"))
        if N <= 0 or Nnbr <= 0 or Nnbr > N:
            raise ValueError(f"{path}: bad header N={N} Nnbr={Nnbr}")
        if size != file_size(N, Nnbr):
            raise ValueError(f"{path}: size {size} != expected {file_size(N, Nnbr)} for N={N}, Nnbr={Nnbr}")

        def f64(count):
            return np.frombuffer(fh.read(8 * count), dtype="<f8").copy()

        a, gh0, dt, gamma = f64(4)
        x, y, z, f, ghm = (f64(N) for _ in range(5))
        p_u, p_v, p_w, gradghm = (f64(3 * N).reshape(N, 3) for _ in range(4))
        Dx, Dy, Dz, L = (f64(N * Nnbr).reshape(N, Nnbr) for _ in range(4))
        idx1 = np.frombuffer(fh.read(4 * N * Nnbr), dtype="<i4").reshape(N, Nnbr).copy()
        H_init = f64(4 * N).reshape(N, 4)
        H_100 = f64(4 * N).reshape(N, 4)
    return SweInput(N, Nnbr, float(a), float(gh0), float(dt), float(gamma), x, y, z, f, ghm,
                    p_u, p_v, p_w, gradghm, Dx, Dy, Dz, L, idx1, H_init, H_100)


def write_input(path: str, d: SweInput) -> None:
    """Write ``d`` in the reference's binary layout (nc2bin.c:32-80 order)."""
    N, Nnbr = d.N, d.Nnbr
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(np.asarray([N, Nnbr], dtype="<i4").tobytes())
        fh.write(np.asarray([d.a, d.gh0, d.dt, d.gamma], dtype="<f8").tobytes())
        for arr in (d.x, d.y, d.z, d.f, d.ghm):
            fh.write(np.ascontiguousarray(arr, dtype="<f8").reshape(N).tobytes())
        for arr in (d.p_u, d.p_v, d.p_w, d.gradghm):
            fh.write(np.ascontiguousarray(arr, dtype="<f8").reshape(N, 3).tobytes())
        for arr in (d.Dx, d.Dy, d.Dz, d.L):
            fh.write(np.ascontiguousarray(arr, dtype="<f8").reshape(N, Nnbr).tobytes())
        fh.write(np.ascontiguousarray(d.idx1, dtype="<i4").reshape(N, Nnbr).tobytes())
        fh.write(np.ascontiguousarray(d.H_init, dtype="<f8").reshape(N, 4).tobytes())
        fh.write(np.ascontiguousarray(d.H_100, dtype="<f8").reshape(N, 4).tobytes())
    os.replace(tmp, path)


def to_model(d: SweInput) -> SweModel:
    """Apply get_GSMD_bin's post-read scaling (input.c:314-328)."""
    if d.idx1.min() < 1 or d.idx1.max() > d.N:
        raise ValueError("stencil index out of range [1, N]")
    return SweModel(
        N=d.N, Nnbr=d.Nnbr, gh0=d.gh0, dt=d.dt,
        x=d.x, y=d.y, z=d.z, f=d.f, ghm=d.ghm,
        p_u=d.p_u, p_v=d.p_v, p_w=d.p_w, gradghm=d.gradghm,
        idx=(d.idx1 - 1).astype(np.int32),
        Dx=d.Dx / d.a, Dy=d.Dy / d.a, Dz=d.Dz / d.a, L=d.L * d.gamma,
        H_init=d.H_init, H_100=d.H_100,
    )


def load_model(path: str) -> SweModel:
    return to_model(read_input(path))
