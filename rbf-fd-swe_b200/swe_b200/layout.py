"""Host-side preparation of a patch, mirroring the reference's host code.

* ``rcm_mapping``   the reference's RCM permutation (rcm/rcm.c:9-62), computed by
                    the library's host restatement swe_host_rcm_mapping
* ``reorder``       reorder_GSMD_struct (rcm/reorder_nodes.c:46-87): permute rows
                    and renumber stencil indices
* ``pad``           pad_GSMD_data (layout/layout.c:10-45): round the node count up
                    to a multiple of the tile width by replicating the last node
                    (matrix_transformations.c:9-32)

All functions take and return swe_input.SweModel objects (canonical node-major
arrays), so the result can go straight to capi.Plain.init_model.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import capi
from .swe_input import SweModel

_ROW_FIELDS = ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "Dx", "Dy", "Dz", "L",
               "H_init", "H_100")


def rcm_mapping(model: SweModel, device: bool = False) -> np.ndarray:
    """mapping[new] = old.  device=False: identical to the reference's rcm_mapping (the
    library's host restatement).  device=True: the breadth-first level order built on
    the GPU (swe_dev_rcm_mapping), of the same bandwidth but not the same permutation."""
    lib = capi.load()
    fn = lib.swe_dev_rcm_mapping if device else lib.swe_host_rcm_mapping
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    idx = np.ascontiguousarray(model.idx, dtype=np.int32)
    out = np.empty(model.N, dtype=np.int32)
    name = "swe_dev_rcm_mapping" if device else "swe_host_rcm_mapping"
    capi.check(name, fn(model.N, model.Nnbr, idx.ctypes.data, out.ctypes.data))
    return out


def bandwidth(idx: np.ndarray) -> tuple[int, float]:
    """(max, mean) over nodes of max - min stencil index, as the reference's
    print_max_bandwidth (rcm/rcm.c:68-96) reports it for a reordered idx."""
    idx = np.asarray(idx)
    bw = idx.max(1) - idx.min(1)
    return int(bw.max()), float(bw.mean())


def reorder(model: SweModel, mapping: np.ndarray) -> SweModel:
    """Rows new <- old = mapping[new]; idx renumbered through the inverse map."""
    inv = np.empty_like(mapping)
    inv[mapping] = np.arange(len(mapping), dtype=mapping.dtype)
    kw = {f: np.ascontiguousarray(getattr(model, f)[mapping]) for f in _ROW_FIELDS}
    kw["idx"] = np.ascontiguousarray(inv[model.idx[mapping]]).astype(np.int32)
    return dataclasses.replace(model, **kw)


def pad(model: SweModel, simd_length: int) -> SweModel:
    """Replicate the last node until N is a multiple of simd_length (layout.c:10-45)."""
    N = model.N
    Np = ((N - 1) // simd_length + 1) * simd_length
    if Np == N:
        return model
    rows = np.concatenate([np.arange(N), np.full(Np - N, N - 1)])
    kw = {f: np.ascontiguousarray(getattr(model, f)[rows]) for f in _ROW_FIELDS}
    kw["idx"] = np.ascontiguousarray(model.idx[rows])
    return dataclasses.replace(model, N=Np, **kw)


def prepare(model: SweModel, use_rcm: bool = True, simd_length: int = 32,
            device_order: bool = False) -> tuple[SweModel, np.ndarray]:
    """The reference's host pipeline for one serial patch (main.c:107-140): optional
    RCM, then padding.  Returns (patch model, mapping[new] = old over real nodes).
    device_order=True orders by the GPU's breadth-first level order instead of the
    reference's exact RCM permutation."""
    mapping = rcm_mapping(model, device_order) if use_rcm else np.arange(model.N, dtype=np.int32)
    m = reorder(model, mapping) if use_rcm else model
    return pad(m, simd_length), mapping
