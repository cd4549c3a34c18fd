// Device-side layout transforms of the static data (init of the plain form and
// grid registration of the serving form).
//
// The caller's arrays arrive in the reference's layouts: DM arrays (Dx, Dy, Dz, L,
// idx) of compute_size x padded_Nnbr values indexed by DM_LIN_ID, VECT arrays
// (p_u, p_v, p_w, gradghm) of compute_size x 3 values indexed by VECT_LIN_ID, and
// per-node arrays (x, y, z, f, ghm) -- swe_config.h:31-36.  They are copied to the
// device once and rearranged there by two kernels into every layout the stage
// kernels read:
//   * W / idx:   the 8-lanes-per-node layout (stage_kernel.cuh, stage_tma.cuh),
//   * Wl / idxl: the tile-transposed node-per-lane layout (stage_lane.cuh), and
//     idxs, the same indices as 16-bit offsets from each node's own row,
//   * PT:        the pointwise records [node][kPointStride].
// Slots j >= nnbr get zero weights and gather the node's own row; nodes past n in
// the last 32-node tile of Wl / idxl get zero weights and gather row pid0.  An
// index outside [0, rows) is reported as the first offending (node, slot) in
// row-major order.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <vector>

#include "common.cuh"
#include "stage_kernel.cuh"
#include "stage_lane.cuh"

namespace swe {

template <typename T>
struct PackedStatic {
    T* W = nullptr;       // 8-lanes-per-node weights
    int* idx = nullptr;   // 8-lanes-per-node indices
    T* Wl = nullptr;      // tile-transposed weights
    int* idxl = nullptr;  // tile-transposed indices
    short* idxs = nullptr;  // the same as 16-bit offsets from the node's own row
    bool idxs_ok = false;   // every offset fits 16 bits
    T* PT = nullptr;      // pointwise records
    void release() {
        for (void* p : {(void*)W, (void*)idx, (void*)Wl, (void*)idxl, (void*)idxs, (void*)PT}) if (p) cudaFree(p);
        W = nullptr; idx = nullptr; Wl = nullptr; idxl = nullptr; idxs = nullptr; PT = nullptr;
        idxs_ok = false;
    }
};

// One thread per (node i, slot j), i < npad (n rounded up to whole 32-node tiles).
template <typename T>
__global__ void pack_stencils_kernel(const T* __restrict__ Dx, const T* __restrict__ Dy, const T* __restrict__ Dz,
                                     const T* __restrict__ L, const int* __restrict__ idx_raw, CallerLayout cl,
                                     int n, long npad, int nnbr, int rows, int pid0, T* __restrict__ W,
                                     int* __restrict__ idxp, T* __restrict__ Wl, int* __restrict__ idxl,
                                     short* __restrict__ idxs, int* __restrict__ wide,
                                     unsigned long long* __restrict__ bad) {
    constexpr int U = Quad<T>::kUnits;
    constexpr int per_unit = 16 / (int)sizeof(T);
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kSlots) return;
    const long i = t / kSlots;
    const int j = (int)(t % kSlots);
    T w[4] = {T(0), T(0), T(0), T(0)};
    int p = i < n ? (int)i + pid0 : pid0;
    if (i < n && j < nnbr) {
        const long dm = cl.dm(i, j);
        w[0] = Dx[dm]; w[1] = Dy[dm]; w[2] = Dz[dm]; w[3] = L[dm];
        const int q = idx_raw[dm];
        if (q < 0 || q >= rows) atomicMin(bad, ((unsigned long long)i << 32) | (unsigned)j);
        else p = q;
    }
    if (i < n) {
        const int m = j / 8, k = j % 8;
#pragma unroll
        for (int op = 0; op < 4; ++op) {
            const long unit = ((i * kSlotChunks + m) * U + op / per_unit) * 8 + k;
            W[unit * per_unit + op % per_unit] = w[op];
        }
        idxp[(i * 8 + k) * 4 + m] = p;
    }
    const long b = i / kLaneTile, tt = i % kLaneTile;
#pragma unroll
    for (int op = 0; op < 4; ++op) {
        const long unit = ((b * kSlots + j) * U + op / per_unit) * kLaneTile + tt;
        Wl[unit * per_unit + op % per_unit] = w[op];
    }
    idxl[(b * kSlots + j) * kLaneTile + tt] = p;
    // 16-bit offset from the node's own row (past n: from row n - 1 + pid0, offset 0)
    const int off = i < n ? p - ((int)i + pid0) : 0;
    if (off < -32768 || off > 32767) atomicOr(wide, 1);
    idxs[(b * kSlots + j) * kLaneTile + tt] = (short)off;
}

// One thread per node.
template <typename T>
__global__ void pack_points_kernel(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                                   const T* __restrict__ f, const T* __restrict__ ghm, const T* __restrict__ pu,
                                   const T* __restrict__ pv, const T* __restrict__ pw, const T* __restrict__ gg,
                                   CallerLayout cl, int n, T* __restrict__ PT) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T r[kPointStride];
#pragma unroll
    for (int k = 0; k < kPointStride; ++k) r[k] = T(0);
    r[PT_X] = x[i]; r[PT_Y] = y[i]; r[PT_Z] = z[i]; r[PT_F] = f[i]; r[PT_GHM] = ghm[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const long v = cl.vect(i, c);
        r[PT_PU + c] = pu[v]; r[PT_PV + c] = pv[v]; r[PT_PW + c] = pw[v]; r[PT_GG + c] = gg[v];
    }
#pragma unroll
    for (int k = 0; k < kPointStride; ++k) PT[i * kPointStride + k] = r[k];
}

namespace pack_detail {
// stream-ordered staging buffer: allocating and freeing it never waits for work
// on other streams (a persistent serving kernel may be running)
template <typename A>
inline cudaError_t upload(A** dst, const A* src, size_t count, cudaStream_t st, std::vector<void*>& owned) {
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(dst), count * sizeof(A), st);
    if (e != cudaSuccess) return e;
    owned.push_back(*dst);
    return cudaMemcpyAsync(*dst, src, count * sizeof(A), cudaMemcpyHostToDevice, st);
}
}  // namespace pack_detail

// Uploads the caller's static arrays (n nodes of a patch with `rows` gather rows,
// compute rows starting at pid0) and packs them on the device into `out` (which
// the caller releases).  Everything runs on a private non-blocking stream, so the
// call waits only for its own work.  Returns SWE_OK, SWE_ERR_INDEX (the message
// names the first out-of-range index) or SWE_ERR_CUDA / SWE_ERR_NOMEM.
template <typename T>
int pack_static_device(const CallerLayout& cl, int n, int rows, int pid0, int nnbr, const T* Dx, const T* Dy,
                       const T* Dz, const T* L, const int* idx, const T* x, const T* y, const T* z, const T* f,
                       const T* ghm, const T* pu, const T* pv, const T* pw, const T* gg, PackedStatic<T>& out) {
    const size_t ndm = (size_t)n * cl.pnbr, nv = (size_t)n * 3;
    const long npad = ((long)n + kLaneTile - 1) / kLaneTile * kLaneTile;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_error("static data packing: %s", cudaGetErrorString(e));
        return SWE_ERR_CUDA;
    }
    std::vector<void*> owned;
    auto drop_staging = [&]() {
        for (void* p : owned) cudaFreeAsync(p, st);
        owned.clear();
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    };
    auto fail = [&](cudaError_t err) {
        drop_staging();
        out.release();
        set_error("static data packing: %s", cudaGetErrorString(err));
        return err == cudaErrorMemoryAllocation ? SWE_ERR_NOMEM : SWE_ERR_CUDA;
    };
    T *tDx, *tDy, *tDz, *tL, *tx, *ty, *tz, *tf, *tghm, *tpu, *tpv, *tpw, *tgg;
    int* tidx;
    unsigned long long* bad = nullptr;
    using pack_detail::upload;
    if ((e = upload(&tDx, Dx, ndm, st, owned)) || (e = upload(&tDy, Dy, ndm, st, owned)) ||
        (e = upload(&tDz, Dz, ndm, st, owned)) || (e = upload(&tL, L, ndm, st, owned)) ||
        (e = upload(&tidx, idx, ndm, st, owned)) || (e = upload(&tx, x, (size_t)n, st, owned)) ||
        (e = upload(&ty, y, (size_t)n, st, owned)) || (e = upload(&tz, z, (size_t)n, st, owned)) ||
        (e = upload(&tf, f, (size_t)n, st, owned)) || (e = upload(&tghm, ghm, (size_t)n, st, owned)) ||
        (e = upload(&tpu, pu, nv, st, owned)) || (e = upload(&tpv, pv, nv, st, owned)) ||
        (e = upload(&tpw, pw, nv, st, owned)) || (e = upload(&tgg, gg, nv, st, owned)))
        return fail(e);
    constexpr int U = Quad<T>::kUnits;
    constexpr int per_unit = 16 / (int)sizeof(T);
    if ((e = cudaMalloc(&out.W, (size_t)n * kSlotChunks * U * 8 * per_unit * sizeof(T))) ||
        (e = cudaMalloc(&out.idx, (size_t)n * kSlots * sizeof(int))) ||
        (e = cudaMalloc(&out.Wl, (size_t)npad * kSlots * U * per_unit * sizeof(T))) ||
        (e = cudaMalloc(&out.idxl, (size_t)npad * kSlots * sizeof(int))) ||
        (e = cudaMalloc(&out.idxs, (size_t)npad * kSlots * sizeof(short))) ||
        (e = cudaMalloc(&out.PT, (size_t)n * kPointStride * sizeof(T))))
        return fail(e);
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&bad), sizeof(*bad), st))) return fail(e);
    owned.push_back(bad);
    if ((e = cudaMemsetAsync(bad, 0xff, sizeof(*bad), st))) return fail(e);
    int* wide = nullptr;
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&wide), sizeof(int), st))) return fail(e);
    owned.push_back(wide);
    if ((e = cudaMemsetAsync(wide, 0, sizeof(int), st))) return fail(e);
    const long threads = npad * kSlots;
    pack_stencils_kernel<T><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
        tDx, tDy, tDz, tL, tidx, cl, n, npad, nnbr, rows, pid0, out.W, out.idx, out.Wl, out.idxl, out.idxs, wide,
        bad);
    pack_points_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(tx, ty, tz, tf, tghm, tpu, tpv, tpw, tgg, cl,
                                                                      n, out.PT);
    count_launch(2);
    unsigned long long hb = ULLONG_MAX;
    int hw = 1;
    if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(&hw, wide, sizeof(hw), cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
        return fail(e);
    out.idxs_ok = hw == 0;
    drop_staging();
    if (hb != ULLONG_MAX) {
        const long i = (long)(hb >> 32);
        const int j = (int)(hb & 0xffffffffu);
        set_error("idx[node %ld][nbr %d] = %d outside the patch [0, %d)", i, j, idx[cl.dm(i, j)], rows);
        out.release();
        return SWE_ERR_INDEX;
    }
    return SWE_OK;
}

}  // namespace swe
