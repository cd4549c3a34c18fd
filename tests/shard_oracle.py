"""Test infrastructure: the oracle as one rank's stepping engine for
swe_b200.shard.HaloStepper (host-only runs of the sharded path).

The rank's patch rows [p0, p1) become an oracle grid of p1 - p0 rows: compute rows
keep their stencils (made patch-local), halo rows get a stencil of their own row
with zero weights (their results are never used: the exchange overwrites them
before any compute row reads them).  Each compute row's arithmetic is then the
full grid's, so a sharded oracle run equals the full-grid oracle run bit for bit.
"""
import dataclasses

import numpy as np

import oracle


class OracleEngine:
    def __init__(self, model, p):
        self.p = p
        rows = np.arange(p.p0, p.p1)
        m = len(rows)
        kw = {k: np.ascontiguousarray(getattr(model, k)[rows]) for k in
              ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "H_init", "H_100")}
        idx = np.repeat(np.arange(m, dtype=np.int32)[:, None], model.Nnbr, axis=1)
        comp = slice(p.c0 - p.p0, p.c1 - p.p0)
        idx[comp] = np.asarray(model.idx)[p.c0:p.c1] - p.p0
        for k in ("Dx", "Dy", "Dz", "L"):
            w = np.zeros((m, model.Nnbr))
            w[comp] = getattr(model, k)[p.c0:p.c1]
            kw[k] = w
        self.model = dataclasses.replace(model, N=m, idx=idx, **kw)
        self.port = oracle.Port(self.model, "fp64")
        self.send_local = p.send_rows_local()
        self.recv_local = p.recv_rows_local()
        self.H = np.zeros((m, 4))
        self.K = np.zeros((m, 4))
        self.F = np.zeros((m, 4))
        self.D = np.zeros((m, 4))

    def set_patch_state(self, H_patch):
        self.H[:] = H_patch
        self.K[:] = H_patch

    def patch_state(self):
        return self.H.copy()

    def substep(self, s):
        self.port.rk_substep(self.H, self.K, self.F, self.D, s)

    def _buf(self, sub):
        return self.H if sub == 0 else self.K

    def pack(self, sub, buf):
        import torch
        n = len(self.send_local)
        if n:
            buf[:n] = torch.from_numpy(self._buf(sub)[self.send_local])

    def unpack(self, sub, buf):
        n = len(self.recv_local)
        if n:
            self._buf(sub)[self.recv_local] = buf[:n].numpy()
