"""Grid-sharded stepping across ranks (one process per GPU).

The reference splits a grid into MPI patches (swe_code/mpi/init_patches.c:21-92):
each rank owns a contiguous range of compute rows in RCM order and holds, around
them, the rows its stencils read; after every stage it refreshes those halo rows
from their owners (exchange_SVM_halos, swe_code/mpi/halos.c:11-35, called after
eval_K and update_H, rk4_rbffd_swe.c:86-158).  Here:

* ``plan``         the split: balanced contiguous compute ranges, each rank's patch
                   [p0, p1) (the compute range widened to every row its stencils
                   read), and per peer the rows it sends and receives;
* ``patch_arrays`` the patch's static arrays in the library's canonical layout
                   (compute rows, stencil indices patch-local);
* ``HaloStepper``  RK4 steps of one rank: a substep on the rank's engine, then the
                   exchange of the halo rows of the buffer the next substep reads,
                   by ``torch.distributed`` point-to-point operations (NCCL between
                   GPUs, gloo on the host) with no collective in the data path.

The engine is the library (``PlainEngine``: swe_cuda_rk_substep and the halo
pack/unpack entry points, device buffers handed to NCCL) or, for host-only tests, any
object with the same four methods.  Nothing reads another GPU's memory: rows cross
between ranks only through the communication library's send/recv.
"""
from __future__ import annotations

import dataclasses

import numpy as np

_STATIC = ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "Dx", "Dy", "Dz", "L")


@dataclasses.dataclass
class ShardPlan:
    rank: int
    nranks: int
    n: int
    c0: int                       # compute rows [c0, c1), global (RCM order)
    c1: int
    p0: int                       # patch rows [p0, p1), global; patch row = global - p0
    p1: int
    send: dict                    # peer -> global rows (sorted) this rank's compute rows send
    recv: dict                    # peer -> global halo rows (sorted) this rank receives

    @property
    def peers(self) -> list:
        return sorted(set(self.send) | set(self.recv))

    def send_rows_local(self) -> np.ndarray:
        """Patch-local send rows, peers in ascending order (the send buffer's layout)."""
        return np.concatenate([self.send[q] for q in sorted(self.send)] or [np.zeros(0, np.int32)]).astype(
            np.int32) - self.p0

    def recv_rows_local(self) -> np.ndarray:
        return np.concatenate([self.recv[q] for q in sorted(self.recv)] or [np.zeros(0, np.int32)]).astype(
            np.int32) - self.p0


def plan(idx: np.ndarray, nranks: int) -> list[ShardPlan]:
    """Split N rows (stencil indices idx [N][n], global, 0-based) into nranks
    contiguous compute ranges of near-equal size, as the reference's patch setup
    does for a serial RCM order; every rank's patch is the smallest contiguous range
    holding its compute rows and every row they read."""
    idx = np.asarray(idx)
    n = len(idx)
    if not 1 <= nranks <= n:
        raise ValueError(f"cannot split {n} rows over {nranks} ranks")
    bounds = np.array([n * r // nranks for r in range(nranks + 1)])
    plans = []
    for r in range(nranks):
        c0, c1 = int(bounds[r]), int(bounds[r + 1])
        need = np.unique(idx[c0:c1])
        halo = need[(need < c0) | (need >= c1)]
        owner = np.searchsorted(bounds, halo, side="right") - 1
        recv = {int(q): halo[owner == q].astype(np.int32) for q in np.unique(owner)}
        p0 = int(min(c0, need.min()))
        p1 = int(max(c1, need.max() + 1))
        plans.append(ShardPlan(r, nranks, n, c0, c1, p0, p1, {}, recv))
    for r in range(nranks):
        for q, rows in plans[r].recv.items():
            plans[q].send[r] = rows
    return plans


def patch_arrays(model, p: ShardPlan, dtype=np.float64) -> dict:
    """Static arrays of rank p's patch for capi.Plain.init: compute rows only, stencil
    indices made patch-local (global - p0)."""
    rows = slice(p.c0, p.c1)
    out = {k: np.ascontiguousarray(getattr(model, k)[rows], dtype=dtype) for k in _STATIC}
    out["idx"] = np.ascontiguousarray(np.asarray(model.idx)[rows] - p.p0, dtype=np.int32)
    return out


class PlainEngine:
    """The library as one rank's engine: its patch initialised with halo rows."""

    def __init__(self, model, p: ShardPlan, prec: str = "fp64"):
        from . import capi

        self.p = p
        self.dtype = np.float64 if prec == "fp64" else np.float32
        self.plain = capi.Plain()
        arrays = patch_arrays(model, p, self.dtype)
        self.plain.init(np.dtype(self.dtype).itemsize, capi.SWE_LAYOUT_CFDL, 1, p.c1 - p.c0, p.p1 - p.p0,
                        p.c0 - p.p0, model.Nnbr, model.Nnbr, model.gh0, model.dt, arrays)
        self.plain.halo_setup(p.send_rows_local(), p.recv_rows_local())

    def set_patch_state(self, H_patch: np.ndarray) -> None:
        self.plain.set_state(np.ascontiguousarray(H_patch, dtype=self.dtype))

    def patch_state(self) -> np.ndarray:
        return self.plain.get_state().reshape(-1, 4)

    def substep(self, s: int) -> None:
        self.plain.rk_substep(s)

    def pack(self, sub: int, buf) -> None:
        self.plain.halo_pack(sub, buf.data_ptr())
        self.plain.sync()

    def unpack(self, sub: int, buf) -> None:
        self.plain.halo_unpack(sub, buf.data_ptr())

    def finalize(self) -> None:
        self.plain.finalize()


class HaloStepper:
    """RK4 steps of this rank's patch with halo exchanges between substeps.

    ``engine`` has substep(s), pack(sub, tensor), unpack(sub, tensor) and the state
    accessors; ``device`` is where the exchange buffers live ("cuda:k" for NCCL,
    "cpu" for gloo).  Every rank must call step() the same number of times: each
    exchange is one batch of point-to-point sends and receives with the rank's
    neighbours."""

    def __init__(self, p: ShardPlan, engine, device: str = "cpu", dtype=None):
        import torch

        self.p, self.engine = p, engine
        tdt = torch.float64 if (dtype or np.float64) == np.float64 else torch.float32
        self.send_n = {q: len(v) for q, v in sorted(p.send.items())}
        self.recv_n = {q: len(v) for q, v in sorted(p.recv.items())}
        self.send_buf = torch.zeros((max(sum(self.send_n.values()), 1), 4), dtype=tdt, device=device)
        self.recv_buf = torch.zeros((max(sum(self.recv_n.values()), 1), 4), dtype=tdt, device=device)
        self.exchanges = 0

    @staticmethod
    def _segments(counts: dict):
        off = 0
        for q, c in counts.items():
            yield q, off, c
            off += c

    def exchange(self, sub: int) -> None:
        import torch.distributed as dist

        self.engine.pack(sub, self.send_buf)
        ops = [dist.P2POp(dist.isend, self.send_buf[o:o + c], q) for q, o, c in self._segments(self.send_n) if c]
        ops += [dist.P2POp(dist.irecv, self.recv_buf[o:o + c], q) for q, o, c in self._segments(self.recv_n) if c]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self.recv_buf.is_cuda:
            import torch
            torch.cuda.synchronize(self.recv_buf.device)
        self.engine.unpack(sub, self.recv_buf)
        self.exchanges += 1

    def step(self, nsteps: int) -> None:
        for _ in range(nsteps):
            for s in range(4):
                self.engine.substep(s)
                self.exchange((s + 1) % 4)
