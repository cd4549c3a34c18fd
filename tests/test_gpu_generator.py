"""GPU input generator (swe_gen_stencils, swe_gen_weights) against the host generator.

The reference has no generator (it reads a shipped file), so the checks are:
* stencils: the same neighbour set and the same sorted distances as scipy's
  cKDTree on every node, self first (distance ties may be ordered differently);
* weights: the same local solves as the torch path (FP64, partial pivoting in a
  different elimination order) within a tolerance set by the systems'
  conditioning, and the property every operator here has exactly: it
  annihilates constants (derivatives and Delta^4 of a constant are zero), to
  rounding of the solve;
* an input generated on the GPU gives, after 200 RK4 steps, the state that the
  host-weighted input on the same stencils gives.
"""
import numpy as np
import pytest

from swe_b200 import capi, gen, layout, swe_input

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [3, 5])
def test_stencils_match_kdtree(level):
    X = gen.icosahedral_nodes(level)
    got = gen.stencils_gpu(X)
    want = gen.stencils(X)
    assert got.shape == want.shape
    assert np.array_equal(got[:, 0], np.arange(len(X)))
    d_got = np.linalg.norm(X[got] - X[:, None, :], axis=2)
    d_want = np.linalg.norm(X[want] - X[:, None, :], axis=2)
    assert np.all(np.diff(d_got, axis=1) >= -1e-15)            # ascending distance (ties: last-bit rounding)
    np.testing.assert_allclose(d_got, d_want, rtol=0, atol=1e-15)
    # neighbour sets agree except where a distance tie straddles the k-th place
    differ = np.array([set(a) != set(b) for a, b in zip(got, want)])
    if differ.any():
        kth = d_want[differ, -1]
        nxt = np.array([np.sort(np.linalg.norm(X - X[i], axis=1))[want.shape[1]] for i in np.where(differ)[0]])
        assert np.allclose(kth, nxt, rtol=0, atol=1e-15), "sets differ without a tie at the k-th distance"


@pytest.mark.parametrize("level", [3, 4])
def test_weights_match_host_solve(level):
    X = gen.icosahedral_nodes(level)
    idx = gen.stencils(X)
    got = gen.rbffd_weights_gpu(X, idx)
    want = gen.rbffd_weights(X, idx, device="cpu")
    for name, g, w in zip(("Dx", "Dy", "Dz", "L"), got, want):
        # (rows can be all zero -- Dz at the poles -- so the scale is the operator's largest weight)
        rel = np.abs(g - w).max() / np.abs(w).max()
        # constants are annihilated: sum_j w_j = 0 to rounding of the local solve
        ann = (np.abs(g.sum(1)) / np.maximum(np.abs(g).sum(1), np.abs(g).max())).max()
        print(f"level {level} {name}: max |gpu - host| / max|w| = {rel:.2e}, annihilation {ann:.2e}")
        assert rel <= 1e-8, (name, rel)
        assert ann <= 1e-10, (name, ann)


def test_gpu_generated_input_steps_like_host_generated():
    """200 steps from the GPU-generated input agree with 200 steps from the host-weighted
    input on the same stencils (the stencil search itself is checked above)."""
    d_gpu = gen.generate(5, seed=3, device="cuda")
    d_host = gen.generate(5, seed=3, device="cpu", idx=d_gpu.idx1.astype(np.int64) - 1)
    runs = []
    for d in (d_gpu, d_host):
        m, _ = layout.prepare(swe_input.to_model(d), use_rcm=True, simd_length=32)
        p = capi.Plain()
        p.init_model(m, "fp64")
        p.set_state(m.H_init)
        p.step(200)
        runs.append(p.get_state().reshape(-1, 4))
        p.finalize()
    g, h = runs
    assert np.isfinite(g).all()
    scale = np.abs(h).max(0)
    scale[:3] = np.abs(h[:, :3]).max()
    rel = (np.abs(g - h).max(0) / scale).max()
    print(f"200 steps, GPU- vs host-weighted input: {rel:.2e}")
    assert rel <= 1e-8, rel
