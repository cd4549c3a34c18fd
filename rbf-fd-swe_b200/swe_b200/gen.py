"""Synthetic input generator: icosahedral nodes, RBF-FD weights, TC5-style ICs.

The reference ships one input (N=2562) and not the tool that made it, so the
larger grids are generated here and written in the reference's binary format
(swe_code/io/input.c:189-414).  Everything is FP64 and seeded.

Grid
    Recursive bisection of the icosahedron (the same 12 base vertices, in the
    same order, as the shipped N=2562 file), N = 10*4^level + 2.  Nodes are
    kept in creation order (base vertices, then each level's edge midpoints).

Stencils
    The n=31 nearest nodes by chordal distance (self first), 1-based in the file.

Weights (local solves, one per node, FP64)
    Projected Cartesian derivatives P*d/dx, P*d/dy, P*d/dz (P = I - x x^T):
    polyharmonic spline phi(r) = r^7 on the chordal distance plus the 15
    polynomials of degree <= 4 in the node's tangent-plane coordinates
    (xi, eta).  Degree-4 polynomials in x, y, z restricted to the sphere span
    25 functions, too many for a 31-point stencil to stay well-posed, so the
    tangent-plane basis of the same degree is used instead.
    Hyperviscosity Delta^4: phi(r) = r^9 on tangent-plane distances with
    Delta^4 r^9 = 9^2 7^2 5^2 3^2 r (the flat 2-D formula; r^7 would make
    Delta^4 phi singular at the stencil centre), with the same polynomials,
    which Delta^4 annihilates.
    Weights are for the unit sphere; the reader divides Dx, Dy, Dz by a and
    multiplies L by gamma = -GAMMA_COEF * N^-4.

State (Williamson TC5 with a Gaussian mountain)
    u = u0 (-y, x, 0) (solid-body zonal flow, u0 = 20 m/s);
    h = -(a Omega u0 + u0^2/2) z^2 (geopotential anomaly; total = h + gh0);
    gh0 = g * 5960; ghm = g * 2000 * exp(-(d/R)^2), d the great-circle distance
    to (lon 3pi/2, lat pi/6), R = pi/9; f = 2 Omega z; gradghm = (Dx,Dy,Dz)/a . ghm
    (the shipped file's convention).  h gets multiplicative noise 1e-3 * N(0,1)
    from numpy.random.default_rng(seed).
"""
from __future__ import annotations

import math

import numpy as np

from .swe_input import SweInput

A_EARTH = 6.37122e6
OMEGA = 7.292e-5
G = 9.80616
H0 = 5960.0
U0 = 20.0
MOUNTAIN_H = 2000.0
MOUNTAIN_LON = 1.5 * math.pi
MOUNTAIN_LAT = math.pi / 6.0
MOUNTAIN_R = math.pi / 9.0
NNBR = 31
NOISE = 1e-3
# gamma = -GAMMA_COEF * N^-4.  With these weights dt*|gamma*lambda_max(L)| is about
# 2.6 * dt/900 s at every N (inside RK4's real-axis bound 2.78 up to dt = 900 s), and the
# configured runs (N=2562/100 steps, 10242/1000, 40962/1000 at LEVEL_DT) stay bounded.
GAMMA_COEF = 2.5e-3

# (level, dt) of the configured grids: dt keeps the gravity-wave CFL near 0.55 from
# level 4 up; coarser grids stay at 900 s, the hyperviscosity bound above.
LEVEL_DT = {2: 900.0, 3: 900.0, 4: 900.0, 5: 450.0, 6: 225.0, 7: 120.0, 8: 60.0}


def icosahedral_nodes(level: int) -> np.ndarray:
    """Unit vectors of the level-`level` bisected icosahedron, [10*4^level + 2, 3]."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = np.array([[0, t, 1], [0, -t, 1], [0, t, -1], [0, -t, -1],
                  [1, 0, t], [-1, 0, t], [1, 0, -t], [-1, 0, -t],
                  [t, 1, 0], [-t, 1, 0], [t, -1, 0], [-t, -1, 0]], dtype=np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    # the 20 faces: vertex triples at mutual (edge) distance
    d = np.linalg.norm(V[:, None, :] - V[None, :, :], axis=2)
    edge = np.isclose(d, d[d > 1e-9].min())
    F = np.array([(i, j, k) for i in range(12) for j in range(i + 1, 12) for k in range(j + 1, 12)
                  if edge[i, j] and edge[j, k] and edge[i, k]], dtype=np.int64)
    for _ in range(level):
        nF, nV = len(F), len(V)
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * nV + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        mid = V[uniq // nV] + V[uniq % nV]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        ids = nV + np.arange(len(uniq))
        m01, m12, m20 = ids[inv[:nF]], ids[inv[nF:2 * nF]], ids[inv[2 * nF:]]
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        F = np.concatenate([np.stack([a, m01, m20], 1), np.stack([m01, b, m12], 1),
                            np.stack([m20, m12, c], 1), np.stack([m01, m12, m20], 1)])
        V = np.concatenate([V, mid])
    return V


def _on_cuda(device) -> bool:
    return str(device).startswith("cuda")


def stencils_gpu(X: np.ndarray, nnbr: int = NNBR, device: str = "cuda") -> np.ndarray:
    """The same stencils from the library's GPU kernel (swe_gen_stencils): k nearest by
    chordal distance, self first, ties by node index."""
    import torch

    from . import capi
    lib = capi.load()
    Xt = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(device)
    out = torch.empty((len(X), nnbr), dtype=torch.int32, device=device)
    with torch.cuda.device(Xt.device):
        capi.check("swe_gen_stencils", lib.swe_gen_stencils(len(X), nnbr, Xt.data_ptr(), out.data_ptr()))
    return out.cpu().numpy()


def rbffd_weights_gpu(X: np.ndarray, idx: np.ndarray, device: str = "cuda"):
    """The same unit-sphere weights from the library's GPU kernel (swe_gen_weights)."""
    import torch

    from . import capi
    lib = capi.load()
    N, n = idx.shape
    Xt = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(device)
    It = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).to(device)
    D = torch.empty((4, N, n), dtype=torch.float64, device=device)
    with torch.cuda.device(Xt.device):
        capi.check("swe_gen_weights", lib.swe_gen_weights(N, n, Xt.data_ptr(), It.data_ptr(), D.data_ptr()))
    D = D.cpu().numpy()
    return D[0], D[1], D[2], D[3]


def stencils(X: np.ndarray, nnbr: int = NNBR) -> np.ndarray:
    """0-based [N, nnbr] nearest-neighbour stencils, self first."""
    from scipy.spatial import cKDTree

    _, idx = cKDTree(X).query(X, k=nnbr)
    idx = idx.astype(np.int32)
    self_ = np.arange(len(X), dtype=np.int32)
    if not np.array_equal(idx[:, 0], self_):
        raise RuntimeError("nearest-neighbour query did not return self first")
    return idx


def _poly(xi, eta, deg: int = 4):
    """Monomials xi^a eta^b, a+b <= deg, ordered by total degree: [..., 15]."""
    import torch

    cols = [xi ** (t - b) * eta ** b for t in range(deg + 1) for b in range(t + 1)]
    return torch.stack(cols, dim=-1)


def rbffd_weights(X: np.ndarray, idx: np.ndarray, chunk: int = 32768, device: str = "cpu"):
    """Unit-sphere weights (Dx, Dy, Dz, L), each [N, n] FP64, for stencils idx.

    One augmented (n + 15) x (n + 15) FP64 solve per node and operator, batched
    with torch on ``device`` ("cpu" or a CUDA device for the large grids).
    """
    import torch

    dev = torch.device(device)
    N, n = idx.shape
    out = np.empty((4, N, n))
    npoly = 15
    c_lap4 = float((9 * 7 * 5 * 3) ** 2)
    Xt = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(dev)
    It = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int64)).to(dev)
    for s in range(0, N, chunk):
        e = min(N, s + chunk)
        B = e - s
        c = Xt[s:e]                                   # [B,3] centres
        S = Xt[It[s:e]]                               # [B,n,3] stencil nodes
        ax = torch.zeros_like(c)
        polar = c[:, 2].abs() >= 0.9
        ax[~polar, 2] = 1.0
        ax[polar, 0] = 1.0
        e1 = torch.linalg.cross(c, ax)
        e1 = e1 / e1.norm(dim=1, keepdim=True)
        e2 = torch.linalg.cross(c, e1)
        dv = S - c[:, None, :]
        rho = dv.norm(dim=2).amax(dim=1)              # stencil radius (chordal)
        xi = torch.einsum("bjk,bk->bj", dv, e1) / rho[:, None]
        eta = torch.einsum("bjk,bk->bj", dv, e2) / rho[:, None]
        P = _poly(xi, eta)                            # [B,n,15]
        Pt = P.transpose(1, 2)
        Z = torch.zeros(B, npoly, npoly, dtype=P.dtype, device=dev)
        # projected gradient: phi = r^7 on chordal distance (scaled by rho)
        r = torch.cdist(S, S) / rho[:, None, None]
        A = torch.cat([torch.cat([r ** 7, P], 2), torch.cat([Pt, Z], 2)], 1)
        rc = dv.norm(dim=2) / rho[:, None]                             # |c - x_j| / rho
        cdot = torch.einsum("bk,bjk->bj", c, S)                        # c . x_j
        proj = c[:, None, :] * cdot[:, :, None] - S                    # c_k (c.x_j) - x_jk
        rhs_phi = 7.0 * (rc ** 5)[:, :, None] * proj / (rho ** 2)[:, None, None]
        rhs_p = torch.zeros(B, npoly, 3, dtype=P.dtype, device=dev)
        rhs_p[:, 1, :] = e1 / rho[:, None]
        rhs_p[:, 2, :] = e2 / rho[:, None]
        w = torch.linalg.solve(A, torch.cat([rhs_phi, rhs_p], 1))[:, :n, :]
        # hyperviscosity: phi = r^9 on tangent-plane distance, Delta^4 r^9 = c_lap4 r
        T = torch.stack([xi, eta], 2)
        r2 = torch.cdist(T, T)
        A2 = torch.cat([torch.cat([r2 ** 9, P], 2), torch.cat([Pt, Z], 2)], 1)
        rhs2 = torch.zeros(B, n + npoly, 1, dtype=P.dtype, device=dev)
        rhs2[:, :n, 0] = c_lap4 * T.norm(dim=2) / (rho ** 8)[:, None]
        wl = torch.linalg.solve(A2, rhs2)[:, :n, 0]
        out[0, s:e] = w[:, :, 0].cpu().numpy()
        out[1, s:e] = w[:, :, 1].cpu().numpy()
        out[2, s:e] = w[:, :, 2].cpu().numpy()
        out[3, s:e] = wl.cpu().numpy()
    return out[0], out[1], out[2], out[3]


def tc5_state(X: np.ndarray, seed: int, noise: float = NOISE) -> tuple[np.ndarray, np.ndarray]:
    """(H [N,4], ghm [N]) for the Gaussian-mountain TC5 variant."""
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    H = np.empty((len(X), 4))
    H[:, 0] = -U0 * y
    H[:, 1] = U0 * x
    H[:, 2] = 0.0
    h = -(A_EARTH * OMEGA * U0 + 0.5 * U0 * U0) * z * z
    rng = np.random.default_rng(seed)
    H[:, 3] = h * (1.0 + noise * rng.standard_normal(len(X)))
    lat = np.arcsin(np.clip(z, -1.0, 1.0))
    lon = np.arctan2(y, x)
    cosd = (math.sin(MOUNTAIN_LAT) * np.sin(lat) +
            math.cos(MOUNTAIN_LAT) * np.cos(lat) * np.cos(lon - MOUNTAIN_LON))
    d = np.arccos(np.clip(cosd, -1.0, 1.0))
    ghm = G * MOUNTAIN_H * np.exp(-(d / MOUNTAIN_R) ** 2)
    return H, ghm


def perturb_h(H: np.ndarray, seed: int, noise: float = NOISE) -> np.ndarray:
    """A copy of H with independent multiplicative 1e-3 noise on h (ensemble members)."""
    out = np.array(H, copy=True)
    rng = np.random.default_rng(seed)
    out[:, 3] = out[:, 3] * (1.0 + noise * rng.standard_normal(len(H)))
    return out


def generate(level: int, seed: int = 0, dt: float | None = None, device: str = "cpu",
             gamma_coef: float = GAMMA_COEF, native: bool | None = None,
             idx: np.ndarray | None = None, nnbr: int = NNBR) -> SweInput:
    """A complete input.  H_100 is left zero: the generator has no reference run to
    take it from (the tests fill it with the oracle's 100-step state where they need it).

    On a CUDA device the stencils and weights come from the library's GPU kernels
    (native, the default there); on the CPU from scipy and torch.  `idx` (0-based
    [N, nnbr], self first) fixes the stencils instead: nodes at an exact distance tie
    for the last stencil place may be chosen differently by the two searches."""
    X = icosahedral_nodes(level)
    N = len(X)
    if native is None:
        native = _on_cuda(device)
    if idx is None:
        idx = stencils_gpu(X, nnbr, device=device) if native else stencils(X, nnbr)
    if native:
        Dx, Dy, Dz, L = rbffd_weights_gpu(X, idx, device=device)
    else:
        Dx, Dy, Dz, L = rbffd_weights(X, idx, device=device)
    H, ghm = tc5_state(X, seed)
    gradghm = np.stack([np.einsum("ij,ij->i", D, ghm[idx]) / A_EARTH for D in (Dx, Dy, Dz)], 1)
    eye = np.eye(3)
    Pm = eye[None, :, :] - X[:, :, None] * X[:, None, :]      # [N,3,3], rows are p_u, p_v, p_w
    return SweInput(
        N=N, Nnbr=idx.shape[1], a=A_EARTH, gh0=G * H0,
        dt=float(dt if dt is not None else LEVEL_DT.get(level, 900.0 if level < 4 else 900.0 / 2 ** (level - 4))),
        gamma=-gamma_coef * float(N) ** -4,
        x=X[:, 0].copy(), y=X[:, 1].copy(), z=X[:, 2].copy(), f=2.0 * OMEGA * X[:, 2], ghm=ghm,
        p_u=Pm[:, 0, :].copy(), p_v=Pm[:, 1, :].copy(), p_w=Pm[:, 2, :].copy(), gradghm=gradghm,
        Dx=Dx, Dy=Dy, Dz=Dz, L=L, idx1=(idx + 1).astype(np.int32),
        H_init=H, H_100=np.zeros_like(H),
    )


def level_of(N: int) -> int:
    lv = round(math.log((N - 2) / 10.0, 4))
    if 10 * 4 ** lv + 2 != N:
        raise ValueError(f"N={N} is not an icosahedral node count")
    return lv
