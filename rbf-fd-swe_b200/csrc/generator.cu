// Offline input generator on the GPU: nearest-neighbour stencils and RBF-FD
// weights (swe_gen_* entry points of include/swe_b200.h).
//
// The reference ships one input file and not the tool that made it
// (io/input.c:189-414 reads the binary format).  swe_b200/gen.py builds inputs
// for the larger grids; these kernels are its native GPU path.
//
// Stencils: the k nearest nodes of every node by chordal distance, self first,
// then by increasing distance, ties by node index.  Nodes are counting-sorted
// into a uniform grid of cubic cells covering [-1, 1]^3 with an edge h chosen
// from the expected k-nearest radius; a query scans the cells within `ring`
// cells of its own and keeps the k best candidates.  Every node inside the
// scanned block lies within ring * h of the query, so when the k-th distance
// found is at most ring * h the answer is exact; otherwise the query is
// repeated with a wider ring.
//
// Weights, per node c with stencil x_1..x_n (n <= 32), in FP64:
//   tangent frame e1 = c x a / |c x a| (a = z, or x near the poles), e2 = c x e1;
//   rho = max_j |x_j - c|; (xi_j, eta_j) = ((x_j - c).e1, (x_j - c).e2) / rho;
//   P = the 15 monomials xi^(t-b) eta^b, t <= 4, ordered by t then b.
//   Projected gradient: [[r_ij^7, P], [P^T, 0]] w = [[7 rc_j^5 (c (c.x_j) - x_j) / rho^2],
//     [0, e1/rho, e2/rho, 0...]] with r_ij = |x_i - x_j| / rho, rc_j = |x_j - c| / rho
//     (three right-hand sides: x, y, z).
//   Hyperviscosity Delta^4: [[s_ij^9, P], [P^T, 0]] w = [[9^2 7^2 5^2 3^2 s_j / rho^8], [0]]
//     with s the tangent-plane distances (s_j = |(xi_j, eta_j)|).
// Each system (n + 15 unknowns) is solved by Gaussian elimination with partial
// pivoting, one warp per node, the augmented matrix in shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace swe {
namespace gen {

constexpr int kMaxK = 32;          // stencil size limit
constexpr int kNPoly = 15;         // degree-4 polynomials in two variables
constexpr int kMaxSys = kMaxK + kNPoly;
constexpr int kRhs = 3;
constexpr int kLd = kMaxSys + kRhs + 1;   // row stride of the augmented matrix (odd: fewer bank conflicts)
constexpr int kWarpsPerCta = 4;

// ---- kNN ---------------------------------------------------------------------------------

struct Grid {
    int G;          // cells per dimension
    double h;       // cell edge
};

__device__ __forceinline__ int cell_coord(double v, const Grid& g) {
    int c = (int)floor((v + 1.0) / g.h);
    return min(max(c, 0), g.G - 1);
}

__global__ void cell_of_kernel(const double* __restrict__ X, int n, Grid g, int* __restrict__ cell,
                               int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = cell_coord(X[3 * i], g), cy = cell_coord(X[3 * i + 1], g), cz = cell_coord(X[3 * i + 2], g);
    const int c = (cz * g.G + cy) * g.G + cx;
    cell[i] = c;
    atomicAdd(count + c, 1);
}

__global__ void scatter_kernel(const int* __restrict__ cell, int n, int* __restrict__ cursor, int* __restrict__ sorted) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sorted[atomicAdd(cursor + cell[i], 1)] = i;
}

// One thread per query: the k best (d2, index) pairs over the cells within `ring`.
// found[i] = 1 when the answer is exact (k-th distance within the scanned radius).
__global__ void knn_kernel(const double* __restrict__ X, int n, Grid g, const int* __restrict__ start,
                           const int* __restrict__ sorted, int k, int ring, const int* __restrict__ todo,
                           int ntodo, int* __restrict__ idx, int* __restrict__ found) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ntodo) return;
    const int i = todo ? todo[q] : q;
    const double px = X[3 * i], py = X[3 * i + 1], pz = X[3 * i + 2];
    double bd[kMaxK];
    int bi[kMaxK];
    int m = 0;
    const int cx = cell_coord(px, g), cy = cell_coord(py, g), cz = cell_coord(pz, g);
    for (int z = max(cz - ring, 0); z <= min(cz + ring, g.G - 1); ++z)
        for (int y = max(cy - ring, 0); y <= min(cy + ring, g.G - 1); ++y) {
            const int row = (z * g.G + y) * g.G;
            const int c0 = row + max(cx - ring, 0), c1 = row + min(cx + ring, g.G - 1);
            for (int s = start[c0]; s < start[c1 + 1]; ++s) {
                const int j = sorted[s];
                const double dx = X[3 * j] - px, dy = X[3 * j + 1] - py, dz = X[3 * j + 2] - pz;
                const double d = dx * dx + dy * dy + dz * dz;
                if (m == k && (d > bd[k - 1] || (d == bd[k - 1] && j > bi[k - 1]))) continue;
                // insert, keeping (d, j) ascending
                int p = m < k ? m++ : k - 1;
                while (p > 0 && (bd[p - 1] > d || (bd[p - 1] == d && bi[p - 1] > j))) {
                    bd[p] = bd[p - 1];
                    bi[p] = bi[p - 1];
                    --p;
                }
                bd[p] = d;
                bi[p] = j;
            }
        }
    const double reach = ring * g.h;
    const bool ok = m == k && bd[k - 1] <= reach * reach;
    found[i] = ok ? 1 : 0;
    if (ok)
        for (int t = 0; t < k; ++t) idx[(long)i * k + t] = bi[t];
}

// ---- weights -------------------------------------------------------------------------------

__device__ __forceinline__ double ipow(double x, int e) {
    double r = 1.0;
    for (int t = 0; t < e; ++t) r *= x;
    return r;
}

// Solve the (ns x ns) system in M (row stride kLd, right-hand sides in columns ns..ns+nr-1)
// by Gaussian elimination with partial pivoting, one warp; solutions overwrite the
// right-hand-side columns.  Returns false for a singular pivot.
__device__ bool warp_solve(double* M, int ns, int nr) {
    const int lane = threadIdx.x & 31;
    const int nc = ns + nr;
    for (int p = 0; p < ns; ++p) {
        // pivot: largest |M[r][p]|, r >= p (ties: smallest r)
        double best = -1.0;
        int br = p;
        for (int r = p + lane; r < ns; r += 32) {
            const double v = fabs(M[r * kLd + p]);
            if (v > best) { best = v; br = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > best || (ov == best && orr < br)) { best = ov; br = orr; }
        }
        if (!(best > 0.0)) return false;
        if (br != p)
            for (int c = p + lane; c < nc; c += 32) {
                const double t = M[p * kLd + c];
                M[p * kLd + c] = M[br * kLd + c];
                M[br * kLd + c] = t;
            }
        __syncwarp();
        const double piv = M[p * kLd + p];
        // eliminate below the pivot: each lane owns rows
        for (int r = p + 1 + lane; r < ns; r += 32) {
            const double f = M[r * kLd + p] / piv;
            if (f != 0.0)
                for (int c = p + 1; c < nc; ++c) M[r * kLd + c] -= f * M[p * kLd + c];
            M[r * kLd + p] = 0.0;
        }
        __syncwarp();
    }
    // back substitution: one right-hand side per lane
    for (int q = lane; q < nr; q += 32) {
        const int c = ns + q;
        for (int r = ns - 1; r >= 0; --r) {
            double s = M[r * kLd + c];
            for (int t = r + 1; t < ns; ++t) s -= M[r * kLd + t] * M[t * kLd + c];
            M[r * kLd + c] = s / M[r * kLd + r];
        }
    }
    __syncwarp();
    return true;
}

__device__ __forceinline__ void poly15(double xi, double eta, double* out) {
    int col = 0;
    for (int t = 0; t <= 4; ++t)
        for (int b = 0; b <= t; ++b) out[col++] = ipow(xi, t - b) * ipow(eta, b);
}

// D: [4][n][k] (Dx, Dy, Dz, L) unit-sphere weights.
__global__ void __launch_bounds__(32 * kWarpsPerCta) weights_kernel(const double* __restrict__ X, const int* __restrict__ idx,
                                                                   int n, int k, double* __restrict__ D,
                                                                   int* __restrict__ status) {
    extern __shared__ double sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int node = blockIdx.x * kWarpsPerCta + warp;
    if (node >= n) return;
    double* M = sm + (size_t)warp * (kMaxSys * kLd + 6 * kMaxK);
    double* sx = M + kMaxSys * kLd;                   // stencil node coordinates
    double* sy = sx + kMaxK;
    double* sz = sy + kMaxK;
    double* sxi = sz + kMaxK;                          // tangent-plane coordinates
    double* seta = sxi + kMaxK;
    double* src = seta + kMaxK;                        // |x_j - c| / rho
    const int ns = k + kNPoly;
    const double c0 = X[3 * node], c1 = X[3 * node + 1], c2 = X[3 * node + 2];
    // tangent frame
    double ax0 = 0.0, ax1 = 0.0, ax2 = 1.0;
    if (fabs(c2) >= 0.9) { ax0 = 1.0; ax2 = 0.0; }
    double e10 = c1 * ax2 - c2 * ax1, e11 = c2 * ax0 - c0 * ax2, e12 = c0 * ax1 - c1 * ax0;
    const double en = sqrt(e10 * e10 + e11 * e11 + e12 * e12);
    e10 /= en; e11 /= en; e12 /= en;
    const double e20 = c1 * e12 - c2 * e11, e21 = c2 * e10 - c0 * e12, e22 = c0 * e11 - c1 * e10;
    // stencil coordinates, radius
    double dmax = 0.0;
    for (int j = lane; j < k; j += 32) {
        const int s = idx[(long)node * k + j];
        sx[j] = X[3 * s]; sy[j] = X[3 * s + 1]; sz[j] = X[3 * s + 2];
        const double d0 = sx[j] - c0, d1 = sy[j] - c1, d2 = sz[j] - c2;
        dmax = fmax(dmax, sqrt(d0 * d0 + d1 * d1 + d2 * d2));
    }
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    const double rho = dmax;
    for (int j = lane; j < k; j += 32) {
        const double d0 = sx[j] - c0, d1 = sy[j] - c1, d2 = sz[j] - c2;
        sxi[j] = (d0 * e10 + d1 * e11 + d2 * e12) / rho;
        seta[j] = (d0 * e20 + d1 * e21 + d2 * e22) / rho;
        src[j] = sqrt(d0 * d0 + d1 * d1 + d2 * d2) / rho;
    }
    __syncwarp();
    bool ok = true;
    for (int sys = 0; sys < 2; ++sys) {
        const int nr = sys == 0 ? 3 : 1;
        // RBF block and polynomial blocks
        for (int e = lane; e < k * k; e += 32) {
            const int i = e / k, j = e % k;
            double r;
            if (sys == 0) {
                const double d0 = sx[i] - sx[j], d1 = sy[i] - sy[j], d2 = sz[i] - sz[j];
                r = ipow(sqrt(d0 * d0 + d1 * d1 + d2 * d2) / rho, 7);
            } else {
                const double a = sxi[i] - sxi[j], b = seta[i] - seta[j];
                r = ipow(sqrt(a * a + b * b), 9);
            }
            M[i * kLd + j] = r;
        }
        for (int j = lane; j < k; j += 32) {
            double pv[kNPoly];
            poly15(sxi[j], seta[j], pv);
            for (int q = 0; q < kNPoly; ++q) {
                M[j * kLd + k + q] = pv[q];
                M[(k + q) * kLd + j] = pv[q];
            }
            // right-hand sides of the RBF rows
            if (sys == 0) {
                const double cdot = c0 * sx[j] + c1 * sy[j] + c2 * sz[j];
                const double f = 7.0 * ipow(src[j], 5) / (rho * rho);
                M[j * kLd + ns + 0] = f * (c0 * cdot - sx[j]);
                M[j * kLd + ns + 1] = f * (c1 * cdot - sy[j]);
                M[j * kLd + ns + 2] = f * (c2 * cdot - sz[j]);
            } else {
                const double cl = (double)(9 * 7 * 5 * 3) * (double)(9 * 7 * 5 * 3);
                M[j * kLd + ns] = cl * sqrt(sxi[j] * sxi[j] + seta[j] * seta[j]) / ipow(rho, 8);
            }
        }
        for (int e = lane; e < kNPoly * kNPoly; e += 32) M[(k + e / kNPoly) * kLd + k + e % kNPoly] = 0.0;
        for (int e = lane; e < kNPoly * nr; e += 32) {
            const int q = e / nr, c = e % nr;
            double v = 0.0;
            if (sys == 0 && q == 1) v = (c == 0 ? e10 : c == 1 ? e11 : e12) / rho;
            if (sys == 0 && q == 2) v = (c == 0 ? e20 : c == 1 ? e21 : e22) / rho;
            M[(k + q) * kLd + ns + c] = v;
        }
        __syncwarp();
        ok = warp_solve(M, ns, nr) && ok;
        for (int j = lane; j < k; j += 32) {
            if (sys == 0) {
                for (int c = 0; c < 3; ++c) D[((long)c * n + node) * k + j] = M[j * kLd + ns + c];
            } else {
                D[((long)3 * n + node) * k + j] = M[j * kLd + ns];
            }
        }
        __syncwarp();
    }
    if (!ok && lane == 0) atomicExch(status, 1);
}

}  // namespace gen
}  // namespace swe

using namespace swe;
using namespace swe::gen;

extern "C" {

int swe_gen_stencils(int n, int k, const double* X, int* idx) {
    if (n <= 0 || k <= 0 || k > kMaxK || k > n || !X || !idx) {
        set_error("swe_gen_stencils: need n > 0, 1 <= k <= min(n, %d), device X and idx", kMaxK);
        return SWE_ERR_ARG;
    }
    // cell edge from the expected k-nearest radius of n quasi-uniform points on the unit sphere
    Grid g;
    // (at most 256^3 cells: beyond ~3M nodes cells hold more nodes, the answer stays exact)
    g.h = std::max(1.2 * std::sqrt(4.0 * k / n), 2.0 / 256.0);
    g.G = std::max(1, std::min(256, (int)std::ceil(2.0 / g.h)));
    g.h = 2.0 / g.G;
    const long cells = (long)g.G * g.G * g.G;
    int *cell = nullptr, *count = nullptr, *start = nullptr, *sorted = nullptr, *found = nullptr, *todo = nullptr;
    int st = SWE_OK;
    auto cleanup = [&] {
        for (int* p : {cell, count, start, sorted, found, todo}) if (p) cudaFree(p);
    };
#define GEN_TRY(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            set_error("%s: %s", #call, cudaGetErrorString(e_));                        \
            cleanup();                                                                 \
            return SWE_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)
    GEN_TRY(cudaMalloc(&cell, n * sizeof(int)));
    GEN_TRY(cudaMalloc(&count, cells * sizeof(int)));
    GEN_TRY(cudaMalloc(&start, (cells + 1) * sizeof(int)));
    GEN_TRY(cudaMalloc(&sorted, n * sizeof(int)));
    GEN_TRY(cudaMalloc(&found, n * sizeof(int)));
    GEN_TRY(cudaMemset(count, 0, cells * sizeof(int)));
    const int T = 256;
    cell_of_kernel<<<ceil_div(n, T), T>>>(X, n, g, cell, count);
    count_launch();
    GEN_TRY(cudaGetLastError());
    // exclusive scan of the cell counts on the host (at most 256^3 cells)
    {
        std::vector<int> h(cells);
        GEN_TRY(cudaMemcpy(h.data(), count, cells * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> s(cells + 1, 0);
        for (long c = 0; c < cells; ++c) s[c + 1] = s[c] + h[c];
        GEN_TRY(cudaMemcpy(start, s.data(), (cells + 1) * sizeof(int), cudaMemcpyHostToDevice));
        GEN_TRY(cudaMemcpy(count, s.data(), cells * sizeof(int), cudaMemcpyHostToDevice));   // scatter cursors
    }
    scatter_kernel<<<ceil_div(n, T), T>>>(cell, n, count, sorted);
    count_launch();
    GEN_TRY(cudaGetLastError());
    // within a cell the scatter order is arbitrary; the query's (distance, index)
    // ordering makes the result independent of it
    knn_kernel<<<ceil_div(n, 128), 128>>>(X, n, g, start, sorted, k, 1, nullptr, n, idx, found);
    count_launch();
    GEN_TRY(cudaGetLastError());
    std::vector<int> f(n);
    GEN_TRY(cudaMemcpy(f.data(), found, n * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> miss;
    for (int i = 0; i < n; ++i) if (!f[i]) miss.push_back(i);
    for (int ring = 2; !miss.empty(); ++ring) {
        if (ring > g.G) {
            set_error("swe_gen_stencils: %zu nodes found fewer than %d neighbours", miss.size(), k);
            cleanup();
            return SWE_ERR_ARG;
        }
        if (!todo) GEN_TRY(cudaMalloc(&todo, n * sizeof(int)));
        GEN_TRY(cudaMemcpy(todo, miss.data(), miss.size() * sizeof(int), cudaMemcpyHostToDevice));
        knn_kernel<<<ceil_div((long)miss.size(), 128), 128>>>(X, n, g, start, sorted, k, ring, todo, (int)miss.size(),
                                                              idx, found);
        count_launch();
        GEN_TRY(cudaGetLastError());
        GEN_TRY(cudaMemcpy(f.data(), found, n * sizeof(int), cudaMemcpyDeviceToHost));
        std::vector<int> next;
        for (int i : miss) if (!f[i]) next.push_back(i);
        miss.swap(next);
    }
    GEN_TRY(cudaDeviceSynchronize());
#undef GEN_TRY
    cleanup();
    return st;
}

int swe_gen_weights(int n, int k, const double* X, const int* idx, double* D) {
    if (n <= 0 || k <= 0 || k > kMaxK || !X || !idx || !D) {
        set_error("swe_gen_weights: need n > 0, 1 <= k <= %d and device X, idx, D", kMaxK);
        return SWE_ERR_ARG;
    }
    int* status = nullptr;
    SWE_CUDA_TRY(cudaMalloc(&status, sizeof(int)));
    SWE_CUDA_TRY(cudaMemset(status, 0, sizeof(int)));
    const size_t smem = (size_t)kWarpsPerCta * (kMaxSys * kLd + 6 * kMaxK) * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(weights_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        weights_kernel<<<ceil_div(n, kWarpsPerCta), 32 * kWarpsPerCta, smem>>>(X, idx, n, k, D, status);
        count_launch();
        e = cudaGetLastError();
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(status);
    if (e != cudaSuccess) {
        set_error("swe_gen_weights: %s", cudaGetErrorString(e));
        return SWE_ERR_CUDA;
    }
    if (h) {
        set_error("swe_gen_weights: a local system was singular (coincident stencil nodes?)");
        return SWE_ERR_ARG;
    }
    return SWE_OK;
}

}  // extern "C"
