"""Shared test setup: import paths, the `gpu` marker and cached synthetic grids."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("rbf-fd-swe_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# The oracle's OpenMP loops get the CPUs this process may use (affinity and cgroup
# quota), set before any oracle library loads.
import oracle as _oracle  # noqa: E402

os.environ.setdefault("OMP_NUM_THREADS", str(_oracle.usable_cpus()["threads"]))
os.environ.setdefault("OMP_SCHEDULE", "static")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


_grid_cache = {}


def generated_input(level: int, seed: int = 1, fill_fc: bool = False, nnbr: int = 31, device: str = "cpu"):
    """(path, SweInput) of a generated grid, written once per session under a temp dir.
    device="cuda" makes the stencils and weights with the library's GPU generator (the
    large grids); the oracle and the library then read the same arrays either way."""
    import tempfile

    from swe_b200 import gen, swe_input

    key = (level, seed, fill_fc, nnbr, device)
    if key in _grid_cache:
        return _grid_cache[key]
    d = gen.generate(level, seed=seed, nnbr=nnbr, device=device)
    if fill_fc:
        import oracle

        m = swe_input.to_model(d)
        d.H_100[:] = oracle.Port(m, "fp64").run(m.H_init, 100)
    tmpdir = tempfile.mkdtemp(prefix="swe_b200_test_")
    path = os.path.join(tmpdir, f"icos{d.N}_seed{seed}.bin")
    swe_input.write_input(path, d)
    _grid_cache[key] = (path, d)
    return path, d


@pytest.fixture(scope="session")
def grid_l3():
    return generated_input(3)


@pytest.fixture(scope="session")
def grid_l4():
    return generated_input(4, fill_fc=True)


@pytest.fixture(scope="session")
def shipped_input():
    import oracle

    if not os.path.exists(oracle.SHIPPED_INPUT):
        pytest.skip("the reference's shipped input was not staged (oracle/_ref absent)")
    return oracle.SHIPPED_INPUT


def rel_err(a, b):
    """Per-field max-norm relative error of [.., 4] arrays."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 4)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 4)
    return np.abs(a - b).max(axis=0) / np.maximum(np.abs(b).max(axis=0), 1e-300)


def scaled_err(a, b):
    """Per-field max-norm error of [.., 4] states, u, v, w over the velocity scale
    max|(u, v, w)| of b (w starts at zero in the test cases) and h over max|h|."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 4)
    b = np.asarray(b, dtype=np.float64).reshape(-1, 4)
    vel = max(np.abs(b[:, :3]).max(), 1e-300)
    scale = np.array([vel, vel, vel, max(np.abs(b[:, 3]).max(), 1e-300)])
    return np.abs(a - b).max(axis=0) / scale


def abs_rhs(model, K, chunk: int = 65536):
    """eval_RHS_swe (rk4_rbffd_swe.c:285-353) evaluated on absolute values with every
    subtraction turned into an addition: the running-error scale of each F entry."""
    Kf = np.abs(np.asarray(K, dtype=np.float64).reshape(-1, 4))
    dX = [np.empty((model.N, 4)) for _ in range(3)]
    LX = np.empty((model.N, 4))
    for r0 in range(0, model.N, chunk):                           # [chunk, n, 4] gathers
        rows = slice(r0, min(model.N, r0 + chunk))
        G = Kf[model.idx[rows]]
        for D, out in zip((model.Dx, model.Dy, model.Dz, model.L), dX + [LX]):
            out[rows] = (np.abs(D[rows])[:, :, None] * G).sum(1)
    u, v, w, h = Kf[:, 0], Kf[:, 1], Kf[:, 2], Kf[:, 3]
    f, x, y, z = np.abs(model.f), np.abs(model.x), np.abs(model.y), np.abs(model.z)
    adv = [u * dX[0][:, c] + v * dX[1][:, c] + w * dX[2][:, c] for c in range(3)]
    cor = [f * (y * w + z * v), f * (z * u + x * w), f * (x * v + y * u)]
    rhs = [adv[c] + cor[c] + dX[c][:, 3] for c in range(3)]
    out = np.empty((model.N, 4))
    for r, P in enumerate((model.p_u, model.p_v, model.p_w)):
        Pa = np.abs(P)
        out[:, r] = Pa[:, 0] * rhs[0] + Pa[:, 1] * rhs[1] + Pa[:, 2] * rhs[2] + LX[:, r]
    gg = np.abs(model.gradghm)
    out[:, 3] = (u * (dX[0][:, 3] + gg[:, 0]) + v * (dX[1][:, 3] + gg[:, 1]) + w * (dX[2][:, 3] + gg[:, 2]) +
                 (h + abs(model.gh0) + np.abs(model.ghm)) * (dX[0][:, 0] + dX[1][:, 1] + dX[2][:, 2]) + LX[:, 3])
    return out


def cond_err(F, F_ref, model, K):
    """max |F - F_ref| / max |F|_abs per field, maximised over fields, where |F|_abs is
    abs_rhs(): the error relative to the size of the terms F is summed from.  Any
    FP64 evaluation order of the reference's formula stays within a few ulps of 1
    on this scale, whatever the cancellation."""
    F = np.asarray(F, dtype=np.float64).reshape(-1, 4)[: model.N]
    F_ref = np.asarray(F_ref, dtype=np.float64).reshape(-1, 4)[: model.N]
    scale = abs_rhs(model, K).max(0)
    return float((np.abs(F - F_ref).max(0) / np.maximum(scale, 1e-300)).max())
