"""The library's side of grid-sharded stepping, on one GPU: a rank's patch with halo
rows steps by swe_cuda_rk_substep, and its halo rows are refreshed between substeps
by swe_cuda_halo_unpack.  The peer is played by the full-grid oracle run in lockstep
(no second GPU, and no two ranks' kernels on one GPU): after each substep the halo
rows of the buffer the next substep reads come from the oracle's state at the same
point.  After 10 steps the patch's compute rows equal the oracle's full-grid run
within 1e-12, and what swe_cuda_halo_pack hands out for the peers matches the
oracle's rows too.  The host-side plan and the point-to-point exchange are covered
by tests/test_shard.py on gloo ranks.
"""
import numpy as np
import pytest

import oracle
from conftest import generated_input, rel_err
from swe_b200 import capi, layout, shard, swe_input

pytestmark = pytest.mark.gpu

STEPS = 10


@pytest.mark.parametrize("rank", [0, 1, 2])
def test_patch_with_halo_rows_steps_like_full_grid(rank):
    import torch

    _, d = generated_input(4)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=1)
    p = shard.plan(m.idx, 3)[rank]
    assert p.recv and p.send                     # a middle or end rank with peers
    eng = shard.PlainEngine(m, p, "fp64")
    try:
        eng.set_patch_state(m.H_init[p.p0:p.p1])
        with pytest.raises(capi.SweError, match="halo"):
            eng.plain.step(1)                    # whole-step graphs do not exchange halos
        port = oracle.Port(m, "fp64")
        Hf, Kf = m.H_init.copy(), m.H_init.copy()
        Ff, Df = np.zeros_like(Hf), np.zeros_like(Hf)
        recv_g = np.concatenate([p.recv[q] for q in sorted(p.recv)])
        send_g = np.concatenate([p.send[q] for q in sorted(p.send)])
        recv = torch.zeros((len(recv_g), 4), dtype=torch.float64, device="cuda")
        send = torch.zeros((len(send_g), 4), dtype=torch.float64, device="cuda")
        worst_send = 0.0
        for _ in range(STEPS):
            for s in range(4):
                eng.substep(s)
                port.rk_substep(Hf, Kf, Ff, Df, s)
                sub = (s + 1) % 4
                src = Hf if sub == 0 else Kf
                eng.pack(sub, send)
                worst_send = max(worst_send, rel_err(send.cpu().numpy(), src[send_g]).max())
                recv.copy_(torch.from_numpy(np.ascontiguousarray(src[recv_g])))
                eng.unpack(sub, recv)
        H = eng.patch_state()[p.c0 - p.p0:p.c1 - p.p0]
    finally:
        eng.finalize()
    err = rel_err(H, Hf[p.c0:p.c1])
    print(f"rank {rank} of 3: compute rows {p.c0}..{p.c1}, patch {p.p0}..{p.p1}, "
          f"{len(send_g)} rows sent / {len(recv_g)} received per exchange; rel err {err}, send {worst_send:.2e}")
    assert err.max() <= 1e-12 and worst_send <= 1e-12


def test_halo_setup_rejects_rows_outside_their_range():
    _, d = generated_input(3)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=1)
    p = shard.plan(m.idx, 2)[0]
    eng = shard.PlainEngine(m, p, "fp64")
    try:
        comp = p.c0 - p.p0
        with pytest.raises(capi.SweError) as e:      # a halo row listed as a send row
            eng.plain.halo_setup(np.array([p.c1 - p.p0], dtype=np.int32), np.zeros(0, dtype=np.int32))
        assert e.value.status == 5
        with pytest.raises(capi.SweError) as e:      # a compute row listed as a receive row
            eng.plain.halo_setup(np.zeros(0, dtype=np.int32), np.array([comp], dtype=np.int32))
        assert e.value.status == 5
    finally:
        eng.finalize()
