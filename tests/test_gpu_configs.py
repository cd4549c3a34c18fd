"""Parity at the sizes and lengths of the configured workloads, on the GPU.

The other GPU test files check every kernel and layout on small grids (N=162 to
N=40962, up to 100 steps).  This file runs the configured workloads themselves:

* N=40962 (level 6), FP64, dt=225 s, 1000 RK4 steps, in each of the reference's
  four layouts, with and without RCM ordering: the library initialised from the
  reference's own PSMD_struct (oracle.Ref), eval_rhs against the reference's own
  eval_RHS_swe, and the 1000-step state against the oracle's 1000-step run.
* N=655362 (level 8), FP64 and FP32, dt=60 s: eval_rhs against the oracle and the
  configured 200 RK4 steps against the oracle's run.
* N=163842 (level 7), 64 members, 3xTF32 batched form, 1000 steps at dt=120 s:
  h error of every member against the plain FP64 GPU run of that member, with
  that plain run itself checked against the oracle over the same 1000 steps.
* N=40962, 32 members (32 per CTA), both precisions, 200 steps: every member
  against its plain FP64 GPU run.

Bars and why:
* FP64 states after 1000 steps, 1e-12 relative per field.  Two FP64 summation
  orders of the same formula stay close here: the reference's OpenMP-SIMD build
  and the oracle's sequential loops differ by 4.5e-15 after 1000 steps at
  N=40962 (measured), so 1e-12 leaves more than two decades for the GPU's own
  order while still catching any wrong term (a missing or misplaced term moves
  the state by >1e-6 within a few steps).
* FP64 eval_rhs, 1e-12 relative (the drop-in contract), and FP32 eval_rhs within
  the FP32 bound of the condition-normalised error (conftest.cond_err).
* FP32 200-step states: within 4x the error the oracle's own FP32 restatement
  makes against the FP64 oracle (two FP32 orders of one formula), and within the
  reference's FP32 verify tolerance, 4e-2 absolute (swe_config.h:80).
* Batched h after 1000 steps: 1e-6 of max|h| for every member (the stated target
  for the batched form); the plain FP64 run it is measured against is itself
  within 1e-12 of the oracle.

Grids of level >= 7 are generated by the library's GPU generator; the oracle and
the library then read the same arrays.
"""
import numpy as np
import pytest

import oracle
from conftest import abs_rhs, cond_err, generated_input, rel_err, scaled_err
from swe_b200 import capi, gen, layout, swe_input

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain():
    p = capi.Plain()
    yield p
    p.finalize()


def _perturbed(H, seed=5, eps=1e-3):
    rng = np.random.default_rng(seed)
    return H * (1.0 + eps * rng.standard_normal(H.shape))


@pytest.mark.parametrize("rcm", [1, 0])
def test_n40962_1000_steps_every_reference_layout(plain, rcm):
    path, d = generated_input(6)
    m = swe_input.to_model(d)
    assert m.N == 40962 and d.dt == 225.0
    H_port = None
    ran = 0
    for lay in oracle.LAYOUTS:
        if not oracle.reference_available("fp64", lay):
            continue
        ref = oracle.Ref(path, "fp64", lay, use_rcm=rcm)
        if H_port is None:
            pm = layout.reorder(m, ref.mapping())
            H0 = ref.state_to_canonical(ref.H_init())[: m.N]
            assert np.array_equal(H0, pm.H_init)
            H_port = oracle.Port(pm, "fp64").run(H0, 1000)
        plain.init_psmd(ref.psmd_ptr(), 8, ref.layout_flags, ref.simd_length)
        K = _perturbed(ref.H_init())
        F = ref.state_to_canonical(plain.eval_rhs(K))[: m.N]
        F_ref = ref.state_to_canonical(ref.eval_rhs(K))[: m.N]
        assert rel_err(F, F_ref).max() <= 1e-12, lay
        plain.set_state(ref.H_init())
        plain.step(1000)
        H = ref.state_to_canonical(plain.get_state())[: m.N]
        err = rel_err(H, H_port)
        print(f"N=40962 rcm={rcm} {lay}: 1000-step rel err per field {err}")
        assert np.isfinite(H).all() and err.max() <= 1e-12, lay
        ran += 1
    if not ran:
        pytest.skip("reference not built")


@pytest.fixture(scope="module")
def model_l8():
    _, d = generated_input(8, device="cuda")
    assert d.N == 655362
    # RCM order, padded to a multiple of 32 nodes by replicating the last one (layout.c)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    return m


def test_n655362_fp64_eval_rhs_and_200_steps(plain, model_l8):
    m = model_l8
    plain.init_model(m, "fp64")
    port = oracle.Port(m, "fp64")
    K = _perturbed(m.H_init)
    F = plain.eval_rhs(K)
    F_ref = port.eval_rhs(K)
    assert rel_err(F, F_ref).max() <= 1e-12
    assert cond_err(F, F_ref, m, K) <= 4e-16
    assert m.dt == 60.0
    plain.set_state(m.H_init)
    plain.step(200)
    H = plain.get_state().reshape(-1, 4)
    err = rel_err(H, port.run(m.H_init, 200))
    print(f"N=655362 FP64 200-step rel err per field {err}")
    assert err.max() <= 1e-12


def test_n655362_fp32_eval_rhs_and_200_steps(plain, model_l8):
    m = model_l8
    plain.init_model(m, "fp32")
    K = _perturbed(m.H_init).astype(np.float32)
    F = plain.eval_rhs(K)
    port64 = oracle.Port(m, "fp64")
    scale = abs_rhs(m, K).max(0)
    F64 = port64.eval_rhs(K.astype(np.float64))
    assert (np.abs(F.reshape(-1, 4) - F64).max(0) / scale).max() <= 4e-6
    plain.set_state(m.H_init.astype(np.float32))
    plain.step(200)
    H = plain.get_state().reshape(-1, 4).astype(np.float64)
    H64 = port64.run(m.H_init, 200)
    H32 = oracle.Port(m, "fp32").run(m.H_init.astype(np.float32), 200)
    err, err32 = scaled_err(H, H64), scaled_err(H32, H64)
    print(f"N=655362 FP32 200-step error per field {err}, FP32 oracle's {err32}")
    assert err.max() <= 4 * err32.max()
    assert np.abs(H - H64).max() <= 4e-2


def test_n163842_b64_1000_steps_h_error_every_member(plain):
    """The batched form's §8 configuration in both precisions that meet its h bar (3xTF32
    and split FP16): 64 members at N=163842, 1000 steps at dt=120 s, every member against
    its plain FP64 GPU run (itself checked against the oracle for member 0)."""
    _, d = generated_input(7, device="cuda")
    m = swe_input.to_model(d)
    assert m.N == 163842 and d.dt == 120.0
    members, steps = 64, 1000
    H0 = np.stack([gen.perturb_h(m.H_init, 1000 + b) for b in range(members)])
    # the plain FP64 run the batched form is measured against, itself checked
    # against the oracle (natural node order, as the batched form exchanges states)
    plain.init_model(m, "fp64")
    plain.set_state(H0[0])
    plain.step(steps)
    err = rel_err(plain.get_state(), oracle.Port(m, "fp64").run(H0[0], steps))
    print(f"N=163842 plain FP64 {steps} steps vs oracle: rel err per field {err}")
    assert err.max() <= 1e-12, err
    Hs = {}
    for precision in ("tf32x3", "fp16x3"):
        ens = capi.Ensemble()
        try:
            ens.init(m, members)
            ens.set_precision(precision)
            ens.tune()
            ens.set_state(H0)
            ens.step(steps)
            Hs[precision] = ens.get_state()
        finally:
            ens.finalize()
    errs = {p: np.empty((members, 4)) for p in Hs}
    for b in range(members):
        plain.set_state(H0[b])
        plain.step(steps)
        ref = plain.get_state()
        for p, H in Hs.items():
            errs[p][b] = scaled_err(H[b], ref)
    for p, e in errs.items():
        worst = int(e[:, 3].argmax())
        print(f"N=163842 B=64 {p} {steps} steps: per-field max over members {e.max(0)}, "
              f"h worst member {worst}, h median {np.median(e[:, 3]):.3e}")
        assert np.isfinite(Hs[p]).all()
        assert e[:, 3].max() <= 1e-6, (p, worst, e[worst])


@pytest.mark.parametrize("precision", ["tf32x3", "bf16x3", "fp16x3"])
def test_n40962_b32_200_steps_every_member(plain, precision):
    """A 32-member ensemble (32 members per CTA: the (32, 32) and (16, 32) tile shapes the
    tuner chooses between) on the N=40962 grid, 200 steps at dt=225 s, every member
    against its plain FP64 GPU run.  3xTF32 is held to the batched form's h bar, 1e-6 of
    max|h|, and so is split FP16; split BF16 (2^-17 operand splits) to 1e-5."""
    _, d = generated_input(6)
    m = swe_input.to_model(d)
    members, steps = 32, 200
    H0 = np.stack([gen.perturb_h(m.H_init, 500 + b) for b in range(members)])
    ens = capi.Ensemble()
    try:
        ens.init(m, members)
        ens.set_precision(precision)
        ens.tune()
        cfg = ens.config()
        ens.set_state(H0)
        ens.step(steps)
        H = ens.get_state()
    finally:
        ens.finalize()
    assert cfg["members_per_cta"] == 32
    plain.init_model(m, "fp64")
    errs = np.empty((members, 4))
    for b in range(members):
        plain.set_state(H0[b])
        plain.step(steps)
        errs[b] = scaled_err(H[b], plain.get_state())
    print(f"N=40962 B=32 {precision} {cfg} {steps} steps: per-field max over members {errs.max(0)}")
    assert np.isfinite(H).all()
    assert errs[:, 3].max() <= (1e-5 if precision == "bf16x3" else 1e-6)
