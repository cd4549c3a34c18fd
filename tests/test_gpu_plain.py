"""Plain form on the GPU, called through the C ABI (capi -> libswe_b200.so).

Parity bars:
* FP64 eval_rhs: <= 1e-12 per-field max-norm relative error against the oracle
  and against the reference's own eval_RHS_swe on the generated (noised)
  inputs, plus a condition-normalised bound (conftest.cond_err) that also holds
  on the balanced shipped input;
* 100 RK4 steps on an input whose H_100 came from the reference: the
  reference's own verify_output criterion, |H - H_100| <= 1e-9 (FP64) and
  <= 4e-2 (FP32) absolute (swe_config.h:80, :88);
* the stage-by-stage API and the graph-captured step are bit-identical, and
  reruns are bit-identical;
* the pipelined and register kernels agree bit for bit; the node-per-lane
  kernel (another slot order) meets the same oracle bars.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, abs_rhs, cond_err, generated_input, rel_err
from swe_b200 import capi, layout, swe_input

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain():
    p = capi.Plain()
    yield p
    p.finalize()


@pytest.fixture(scope="module")
def grid_l6():
    return generated_input(6)


def _perturbed(H, seed=5, eps=1e-3):
    rng = np.random.default_rng(seed)
    return H * (1.0 + eps * rng.standard_normal(H.shape))


@pytest.mark.parametrize("level", [4, 6])
def test_eval_rhs_fp64_matches_oracle(plain, level):
    _, d = generated_input(level, fill_fc=(level == 4))
    m = swe_input.to_model(d)
    plain.init_model(m, "fp64")
    port = oracle.Port(m, "fp64")
    for K in (m.H_init, _perturbed(m.H_init)):
        F = plain.eval_rhs(K)
        F_ref = port.eval_rhs(K)
        assert rel_err(F, F_ref).max() <= 1e-12
        assert cond_err(F, F_ref, m, K) <= 4e-16


@pytest.mark.parametrize("lay", oracle.LAYOUTS)
@pytest.mark.parametrize("rcm", [0, 1])
def test_drop_in_all_reference_layouts(plain, lay, rcm, grid_l4):
    """The reference builds LPSMD in its own layout (and RCM order); the library
    takes the PSMD_struct as is and must agree with the reference's eval_RHS_swe."""
    if not oracle.reference_available("fp64", lay):
        pytest.skip("reference not built")
    path, d = grid_l4
    ref = oracle.Ref(path, "fp64", lay, use_rcm=rcm)
    plain.init_psmd(ref.psmd_ptr(), 8, ref.layout_flags, ref.simd_length)
    for K in (ref.H_init(), _perturbed(ref.H_init())):
        F = ref.state_to_canonical(plain.eval_rhs(K))
        F_ref = ref.state_to_canonical(ref.eval_rhs(K))
        assert rel_err(F, F_ref).max() <= 1e-12


@pytest.mark.parametrize("lay", oracle.LAYOUTS)
@pytest.mark.parametrize("rcm", [0, 1])
def test_drop_in_all_reference_layouts_fp32(plain, lay, rcm, grid_l4):
    """The same through the reference's FP32 builds: F within the FP32 bound of the
    condition-normalised error (two FP32 summation orders of the same formula)."""
    if not oracle.reference_available("fp32", lay):
        pytest.skip("reference not built")
    path, d = grid_l4
    ref = oracle.Ref(path, "fp32", lay, use_rcm=rcm)
    plain.init_psmd(ref.psmd_ptr(), 4, ref.layout_flags, ref.simd_length)
    m = layout.reorder(swe_input.to_model(d), ref.mapping())
    for K in (ref.H_init(), _perturbed(ref.H_init()).astype(np.float32)):
        F = ref.state_to_canonical(plain.eval_rhs(K))[: m.N]
        F_ref = ref.state_to_canonical(ref.eval_rhs(K))[: m.N]
        Kc = ref.state_to_canonical(K)[: m.N]
        assert cond_err(F, F_ref, m, Kc) <= 4e-6


@pytest.mark.parametrize("lay", ["cfdl", "default"])
def test_shipped_input_100_steps_verify(plain, shipped_input, lay):
    """The reference's own end-to-end check on its shipped input, through its PSMD."""
    if not oracle.reference_available("fp64", lay):
        pytest.skip("reference not built")
    ref = oracle.Ref(shipped_input, "fp64", lay, use_rcm=1)
    plain.init_psmd(ref.psmd_ptr(), 8, ref.layout_flags, ref.simd_length)
    K = ref.H_init()
    m = swe_input.load_model(shipped_input)
    F = ref.state_to_canonical(plain.eval_rhs(K))[: m.N]
    F_ref = ref.state_to_canonical(ref.eval_rhs(K))[: m.N]
    perm = ref.mapping()
    assert cond_err(F, F_ref, layout.reorder(m, perm), K=ref.state_to_canonical(K)[: m.N]) <= 4e-16
    plain.set_state(ref.H_init())
    plain.step(100)
    count, max_err = ref.verify(plain.get_state())
    assert count == 0, max_err


def test_generated_input_100_steps_vs_oracle_H100(plain, grid_l4):
    path, d = grid_l4
    m, mapping = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    plain.init_model(m, "fp64")
    plain.set_state(m.H_init)
    plain.step(100)
    H = plain.get_state().reshape(-1, 4)
    assert np.abs(H - m.H_100).max() <= 1e-9


def test_substeps_equal_graph_steps_and_rerun_bitwise(plain, grid_l4):
    _, d = grid_l4
    m = swe_input.to_model(d)
    plain.init_model(m, "fp64")
    plain.set_state(m.H_init)
    for _ in range(5):
        for s in range(4):
            plain.rk_substep(s)
    a = plain.get_state()
    plain.set_state(m.H_init)
    plain.step(5)
    b = plain.get_state()
    plain.set_state(m.H_init)
    plain.step(5)
    c = plain.get_state()
    assert np.array_equal(a, b) and np.array_equal(b, c)


def test_fp32_form(plain, grid_l4):
    _, d = grid_l4
    m = swe_input.to_model(d)
    plain.init_model(m, "fp32")
    K = _perturbed(m.H_init).astype(np.float32)
    F = plain.eval_rhs(K)
    assert cond_err(F, oracle.Port(m, "fp32").eval_rhs(K), m, K) <= 4e-6
    assert cond_err(F, oracle.Port(m, "fp64").eval_rhs(K.astype(np.float64)), m, K) <= 4e-6
    plain.set_state(m.H_init.astype(np.float32))
    plain.step(100)
    H = plain.get_state().reshape(-1, 4)
    assert np.abs(H - m.H_100).max() <= 4e-2          # the reference's FP32 TOLERANCE


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_patch_with_halo_rows(plain, grid_l4, prec):
    """A patch as the reference's MPI decomposition builds one (init_patches.c): the
    compute rows start at compute_pid_s inside a longer gather patch, and stencil
    indices refer to patch rows, some of them halo rows.  eval_rhs of the compute
    rows matches the oracle's rows of the whole grid, for every kernel and shape."""
    _, d = grid_l4
    m = swe_input.to_model(d)
    pid0, nc = 100, 1000                              # compute rows [100, 1100) of 2562
    dt = np.float64 if prec == "fp64" else np.float32
    rows = slice(pid0, pid0 + nc)
    arrays = {k: np.ascontiguousarray(getattr(m, k)[rows], dtype=dt)
              for k in ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "Dx", "Dy", "Dz", "L")}
    arrays["idx"] = np.ascontiguousarray(m.idx[rows], dtype=np.int32)
    assert (arrays["idx"] < pid0).any() and (arrays["idx"] >= pid0 + nc).any()   # halo rows on both sides
    plain.init(np.dtype(dt).itemsize, capi.SWE_LAYOUT_CFDL, 1, nc, m.N, pid0, m.Nnbr, m.Nnbr, m.gh0, m.dt, arrays)
    K = _perturbed(m.H_init).astype(dt)
    want64 = oracle.Port(m, "fp64").eval_rhs(K.astype(np.float64)).reshape(-1, 4)[rows]
    for which in (1, 3, 4, 6, 7, 8, 15, 18, 19):
        plain.select_kernel(which)
        F = plain.eval_rhs(K).reshape(-1, 4)
        assert F.shape == (nc, 4)
        if prec == "fp64":
            assert rel_err(F, want64).max() <= 1e-12, which
        else:
            scale = abs_rhs(m, K)[rows].max(0)             # term scale of these rows
            assert (np.abs(F - want64).max(0) / scale).max() <= 4e-6, which


def test_padded_weight_columns_are_never_read(plain):
    """Non-CFDL callers pass [N][32] rows whose column 31 the reference fills by
    replication (matrix_transformations.c:20-21); garbage there must not matter."""
    m = swe_input.load_model(os.path.join(GOLDEN, "icos162_seed7.bin"))
    m = layout.pad(m, 32)
    arrays = {}
    for k in ("Dx", "Dy", "Dz", "L"):
        a = np.zeros((m.N, 32))
        a[:, :31] = getattr(m, k)
        a[:, 31] = 1e300
        arrays[k] = a
    idx = np.full((m.N, 32), 10 ** 8, dtype=np.int32)
    idx[:, :31] = m.idx
    arrays["idx"] = idx
    for k in ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm"):
        arrays[k] = np.ascontiguousarray(getattr(m, k))
    plain.init(8, capi.SWE_LAYOUT_CFDL, 32, m.N, m.N, 0, 31, 32, m.gh0, m.dt, arrays)
    F = plain.eval_rhs(m.H_init)
    assert np.isfinite(F).all()
    assert rel_err(F, oracle.Port(m, "fp64").eval_rhs(m.H_init)).max() <= 1e-12


def test_out_of_range_index_is_rejected(plain):
    """The static data is packed on the device; the first out-of-range stencil index
    in row-major order is reported with its (node, slot), and the library stays usable."""
    m = swe_input.load_model(os.path.join(GOLDEN, "icos162_seed7.bin"))
    good = m.idx.copy()
    m.idx[7, 3] = m.N + 5
    m.idx[9, 0] = -1
    with pytest.raises(capi.SweError, match=r"idx\[node 7\]\[nbr 3\] = %d outside the patch" % (m.N + 5)) as e:
        plain.init_model(m, "fp64")
    assert e.value.status == 5
    m.idx[:] = good
    plain.init_model(m, "fp64")
    assert rel_err(plain.eval_rhs(m.H_init), oracle.Port(m, "fp64").eval_rhs(m.H_init)).max() <= 1e-12


def test_invariants_watchdog_reports_non_finite_state(plain, grid_l4):
    """A NaN in the state (here one node's h in the initial state) makes the FP64
    conservation sums non-finite; swe_cuda_invariants reports SWE_ERR_NONFINITE and
    the library stays usable."""
    _, d = grid_l4
    m = swe_input.to_model(d)
    plain.init_model(m, "fp64")
    H = m.H_init.copy().reshape(-1, 4)
    H[17, 3] = np.nan
    plain.set_state(H)
    plain.step(2)
    with pytest.raises(capi.SweError, match="NaN or Inf") as e:
        plain.invariants()
    assert e.value.status == 7
    plain.set_state(m.H_init)
    plain.step(2)
    assert np.isfinite(plain.invariants()).all()


def test_invariants_match_oracle(plain, grid_l4):
    _, d = grid_l4
    m = swe_input.to_model(d)
    plain.init_model(m, "fp64")
    plain.set_state(m.H_init)
    plain.step(3)
    H = plain.get_state()
    got = plain.invariants()
    want = oracle.Port(m, "fp64").invariants(H)[0]
    assert np.allclose(got, want, rtol=1e-13)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pipelined_and_register_kernels_agree_bitwise(plain, prec):
    """The bulk-copy pipelined kernel and the register-streaming kernel do the
    same arithmetic in the same order."""
    _, d = generated_input(6)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    plain.init_model(m, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    K = _perturbed(m.H_init).astype(dt)
    results = {}
    # 2 / 3 / 4: pipelined kernel with 64- / 32- / 16-node tiles (1 / 2 / 4 CTAs per SM); 1: register
    for which, kind, tile in ((2, "pipelined", 64), (3, "pipelined", 32), (4, "pipelined", 16), (1, "register", None)):
        plain.select_kernel(which)
        info = plain.kernel_info()
        assert info["in_use"] == kind
        if tile:
            assert info["pipelined_tile"] == tile
        F = plain.eval_rhs(K)
        plain.set_state(m.H_init.astype(dt))
        plain.step(7)
        results[which] = (F, plain.get_state())
    F0, H0 = results[1]
    for which in (2, 3, 4):
        assert np.array_equal(results[which][0], F0) and np.array_equal(results[which][1], H0), which
    if prec == "fp64":
        assert rel_err(F0, oracle.Port(m, "fp64").eval_rhs(K)).max() <= 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_lane_kernel_16bit_offsets_equal_32bit_indices(plain, prec):
    """The node-per-lane kernel reads the stencil rows as 16-bit offsets from each node's
    own row when every offset fits (the RCM order keeps them within about 1500 rows at
    N=40962). Both widths name the same rows, so eval_rhs and 7 RK4 steps agree bit for
    bit with every lanes-per-node shape. In the generator's own order the offsets reach
    38432 rows: the library falls back to 32-bit indices and refuses 16."""
    _, d = generated_input(6)
    m0 = swe_input.to_model(d)
    m, _ = layout.prepare(m0, use_rcm=True, simd_length=32)
    assert np.abs(m.idx.reshape(m.N, -1) - np.arange(m.N)[:, None]).max() <= 32767
    plain.init_model(m, prec)
    assert plain.kernel_info()["index_offsets_16bit"]
    dt = np.float64 if prec == "fp64" else np.float32
    K = _perturbed(m.H_init).astype(dt)
    for lpn in (1, 2, 4):
        plain.select_kernel(capi.Plain.lane_shape(lpn))
        res = {}
        for bits in (16, 32):
            plain.set_index_width(bits)
            assert plain.kernel_info()["index_offsets_16bit"] == (bits == 16)
            F = plain.eval_rhs(K)
            plain.set_state(m.H_init.astype(dt))
            plain.step(7)
            res[bits] = (F, plain.get_state())
        assert np.array_equal(res[16][0], res[32][0]), lpn
        assert np.array_equal(res[16][1], res[32][1]), lpn
    plain.set_index_width(16)
    m_raw, _ = layout.prepare(m0, use_rcm=False, simd_length=32)
    assert np.abs(m_raw.idx.reshape(m_raw.N, -1) - np.arange(m_raw.N)[:, None]).max() > 32767
    plain.init_model(m_raw, prec)
    plain.select_kernel(capi.Plain.lane_shape(1))
    assert not plain.kernel_info()["index_offsets_16bit"]
    with pytest.raises(capi.SweError) as e:
        plain.set_index_width(16)
    assert capi.STATUS[e.value.status] == "SWE_ERR_ARG"
    plain.set_index_width(32)
    F = plain.eval_rhs(m_raw.H_init.astype(dt))
    if prec == "fp64":
        assert rel_err(F, oracle.Port(m_raw, "fp64").eval_rhs(m_raw.H_init)).max() <= 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_lane_kernel_matches_oracle(plain, prec):
    """The node-per-lane kernel sums each node's slots serially per lane (1, 2 or 4
    lanes per node) instead of in the 8-lane tree, so it is held to the oracle's bars
    rather than to the other kernels' bits: eval_rhs within 1e-12 relative and a few
    ulps of the condition scale (FP64), FP32 within the FP32 condition bound, and
    7 RK4 steps within 1e-12 of the register kernel (FP64)."""
    _, d = generated_input(6)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    plain.init_model(m, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    K = _perturbed(m.H_init).astype(dt)
    F64 = oracle.Port(m, "fp64").eval_rhs(K.astype(np.float64))
    plain.select_kernel(1)
    plain.set_state(m.H_init.astype(dt))
    plain.step(7)
    H_reg = plain.get_state().reshape(-1, 4)
    F_first = {}
    for pf in (False, True):
        for ctas in (4, 5, 3):
            for lpn in (1, 2, 4):
                plain.select_kernel(capi.Plain.lane_shape(lpn, ctas, pf))
                info = plain.kernel_info()
                assert info["in_use"] == "lane" and info["lanes_per_node"] == lpn
                assert info["l2_prefetch"] == pf and info["ctas_per_sm"] == ctas
                F = plain.eval_rhs(K)
                # neither the prefetch nor the register bound moves any arithmetic
                if lpn in F_first:
                    assert np.array_equal(F, F_first[lpn]), (lpn, ctas, pf)
                    continue
                F_first[lpn] = F
                if prec == "fp64":
                    assert rel_err(F, F64).max() <= 1e-12, lpn
                    assert cond_err(F, F64, m, K) <= 4e-16, lpn
                else:
                    assert cond_err(F, F64, m, K) <= 4e-6, lpn
                plain.set_state(m.H_init.astype(dt))
                plain.step(7)
                H = plain.get_state().reshape(-1, 4)
                assert np.isfinite(H).all()
                if prec == "fp64":
                    assert rel_err(H, H_reg).max() <= 1e-12, lpn


def test_select_kernel_rejects_unknown_choice(plain, grid_l4):
    _, d = grid_l4
    plain.init_model(swe_input.to_model(d), "fp64")
    for bad in (-1, 24):
        with pytest.raises(capi.SweError):
            plain.select_kernel(bad)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_short_stencils_match_oracle(plain, prec):
    """20-point stencils (the reference takes any Nnbr up to the padded width): slots
    20..31 carry no weight in either kernel, and the results still match the oracle."""
    _, d = generated_input(4, nnbr=20)
    m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
    assert m.Nnbr == 20
    plain.init_model(m, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    K = _perturbed(m.H_init).astype(dt)
    port = oracle.Port(m, prec)
    # register, pipelined 64 / 32 / 16, node-per-lane shapes (18-20: 3 CTAs per SM, whose
    # gather rows are read before the dependent-launch wait, and a lane's last slot skipped
    # as padding)
    for which in (1, 2, 3, 4, 6, 7, 8, 10, 16, 18, 19, 20):
        plain.select_kernel(which)
        F = plain.eval_rhs(K)
        want = port.eval_rhs(K)
        if prec == "fp64":
            assert rel_err(F, want).max() <= 1e-12, which
        else:
            assert cond_err(F, oracle.Port(m, "fp64").eval_rhs(K.astype(np.float64)), m, K) <= 4e-6, which
    plain.set_state(m.H_init.astype(dt))
    plain.step(10)
    H = plain.get_state()
    if prec == "fp64":
        assert np.abs(H - port.run(m.H_init, 10).reshape(H.shape)).max() <= 1e-9
