"""Binary input format and the synthetic generator (host logic, no GPU)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN
from swe_b200 import gen, swe_input


def test_roundtrip(tmp_path):
    d = swe_input.read_input(os.path.join(GOLDEN, "icos162_seed7.bin"))
    p = tmp_path / "x.bin"
    swe_input.write_input(str(p), d)
    e = swe_input.read_input(str(p))
    for k, v in d.__dict__.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, getattr(e, k)), k
        else:
            assert v == getattr(e, k), k
    assert os.path.getsize(p) == swe_input.file_size(d.N, d.Nnbr)


def test_truncated_and_bad_files_raise(tmp_path):
    src = open(os.path.join(GOLDEN, "icos162_seed7.bin"), "rb").read()
    p = tmp_path / "t.bin"
    p.write_bytes(src[:-8])
    with pytest.raises(ValueError):
        swe_input.read_input(str(p))
    bad = bytearray(src)
    bad[0:4] = np.int32(161).tobytes()      # wrong N for the size
    p.write_bytes(bytes(bad))
    with pytest.raises(ValueError):
        swe_input.read_input(str(p))
    d = swe_input.read_input(os.path.join(GOLDEN, "icos162_seed7.bin"))
    d.idx1[3, 4] = d.N + 1                   # out-of-range stencil index
    with pytest.raises(ValueError):
        swe_input.to_model(d)


def test_reader_scaling_matches_reference_convention():
    d = swe_input.read_input(os.path.join(GOLDEN, "icos162_seed7.bin"))
    m = swe_input.to_model(d)
    assert np.array_equal(m.Dx, d.Dx / d.a)          # input.c:314-319
    assert np.array_equal(m.L, d.L * d.gamma)
    assert np.array_equal(m.idx, d.idx1 - 1)          # input.c:326-328


@pytest.mark.parametrize("level", [0, 1, 2, 3])
def test_icosahedral_counts_and_unit_norm(level):
    X = gen.icosahedral_nodes(level)
    assert len(X) == 10 * 4 ** level + 2
    assert np.allclose(np.linalg.norm(X, axis=1), 1.0, atol=1e-15)
    assert len(np.unique(np.round(X, 12), axis=0)) == len(X)


def test_generator_operators(grid_l3):
    _, d = grid_l3
    N, n = d.N, d.Nnbr
    X = np.c_[d.x, d.y, d.z]
    idx = d.idx1 - 1
    assert n == 31 and np.array_equal(idx[:, 0], np.arange(N))
    M = lambda W: sp.csr_matrix((W.ravel(), (np.repeat(np.arange(N), n), idx.ravel())), shape=(N, N))
    # projected gradient of z on the unit sphere is e_z - z x
    for k, D in enumerate((d.Dx, d.Dy, d.Dz)):
        exact = np.eye(3)[2][k] - d.z * X[:, k]
        assert np.abs(M(D) @ d.z - exact).max() < 1e-4
        assert np.abs(D.sum(1)).max() < 1e-8 * np.abs(D).max()      # constants annihilated
    assert np.abs(d.L.sum(1)).max() < 1e-8 * np.abs(d.L).max()
    # P = I - x x^T rows
    assert np.allclose(d.p_u, np.eye(3)[0] - X * d.x[:, None])
    # gradghm follows the shipped file's convention (Dx/a) . ghm
    gx = (M(d.Dx) @ d.ghm) / d.a
    assert np.abs(d.gradghm[:, 0] - gx).max() <= 1e-12 * np.abs(gx).max()
    assert d.gamma == -gen.GAMMA_COEF * float(N) ** -4


def test_generator_is_seeded():
    a, _ = gen.tc5_state(gen.icosahedral_nodes(2), seed=3)
    b, _ = gen.tc5_state(gen.icosahedral_nodes(2), seed=3)
    c, _ = gen.tc5_state(gen.icosahedral_nodes(2), seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
