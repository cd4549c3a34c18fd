// RK4 steps with no device allocation: swe_cuda_step_noalloc.
//
// Some callers cannot call cudaMalloc: hosts whose device memory is owned by
// an outer framework's pool, and latency-critical loops where an allocation's
// implicit device synchronisation is not allowed.  They hand over every input
// and output as device pointers they already own; the only other memory this
// path needs -- the RK4 registers K (two ping-pong copies) and D -- lives in
// the file-scope array below, of SWE_NOALLOC_SCRATCH_BYTES.
//
// The array occupies that much memory on every GPU that loads this library,
// for the life of the process.  All calls share it: two calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it and give wrong results; serialise them.  Nothing in it has to start at
// zero: within one call every K and D value is written by a stage before any
// stage reads it, so the previous call's contents are never seen.
//
// The kernels are the fused stage kernel's math (stage_kernel.cuh) reading the
// caller's row-major arrays directly instead of the packed device layout that
// swe_cuda_init builds, so no packing buffer is needed either.
//
// The other entry points check every stencil index while packing it; here the
// indices are read straight from the caller's device array, so the kernel
// checks them as it gathers.  An index outside 0..n-1 is never dereferenced:
// the gather reads the node's own row instead (so that call's results are
// wrong), and the first such (node, slot, value) is kept in g_noalloc_bad.  A
// call with nsteps = 0 waits for `stream`, reports a kept record as
// SWE_ERR_INDEX and clears it.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "stage_kernel.cuh"

namespace swe {
namespace {

constexpr size_t kNoallocScratchBytes = (size_t)4 << 20;
static_assert(kNoallocScratchBytes == SWE_NOALLOC_SCRATCH_BYTES, "header and file disagree");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// First out-of-range stencil index met by a kernel: {seen, node, slot, value}.
// Zero at load; cleared by the nsteps = 0 call that reports it.
static __device__ int g_noalloc_bad[4];

__device__ __forceinline__ int checked_neighbour(int v, int n, long node, int slot) {
    if ((unsigned)v < (unsigned)n) return v;
    if (atomicCAS(&g_noalloc_bad[0], 0, 1) == 0) {
        g_noalloc_bad[1] = (int)node;
        g_noalloc_bad[2] = slot;
        g_noalloc_bad[3] = v;
    }
    return (int)node;
}

// Device addresses of the scratch array, one per device, filled by the first
// call on that device (cudaGetSymbolAddress with that device current).  In
// host code the array's name is only a stand-in, so kernels get these.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

template <typename T>
struct RowMajorArgs {
    int n, nnbr;
    const int* idx;                // [n][nnbr], 0-based
    const T *Dx, *Dy, *Dz, *L;     // [n][nnbr]
    const T *x, *y, *z, *f, *ghm;  // [n]
    const T *pu, *pv, *pw, *gg;    // [n][3]
    const T* Kin;                  // gather source [n][4]
    T* H;                          // [n][4] RK base state (the caller's buffer, in/out)
    T* D;                          // [n][4] scratch
    T* Kout;                       // [n][4] scratch
    T gh0;
    T c;                           // dt/2, dt/2, dt for stages 0-2
    double dt6;                    // dt/6
};

template <typename T, int MODE>
__global__ void __launch_bounds__(kStageThreads) rowmajor_stage_kernel(const RowMajorArgs<T> a) {
    __shared__ __align__(16) T red[kStageWarps][4][16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 3, k = lane & 7;
    const long warps_total = (long)gridDim.x * kStageWarps;
    for (long base = ((long)blockIdx.x * kStageWarps + warp) * 4; base < a.n; base += warps_total * 4) {
        const long i = base + g;
        const bool valid = i < a.n;
        const long ii = valid ? i : (long)a.n - 1;
        T acc[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[t] = T(0);
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m) {
            const int j = 8 * m + k;           // same slot-to-lane split as stage_kernel
            if (j < a.nnbr) {
                const long e = ii * a.nnbr + j;
                const T w[4] = {__ldg(a.Dx + e), __ldg(a.Dy + e), __ldg(a.Dz + e), __ldg(a.L + e)};
                T kv[4];
                Quad<T>::load_row(a.Kin + 4L * checked_neighbour(__ldg(a.idx + e), a.n, ii, j), kv);
#pragma unroll
                for (int op = 0; op < 4; ++op)
#pragma unroll
                    for (int fld = 0; fld < 4; ++fld) acc[op * 4 + fld] += w[op] * kv[fld];
            }
        }
        T r0, r1;
        reduce_scatter8(acc, k, r0, r1);
        red[warp][g][2 * k] = r0;
        red[warp][g][2 * k + 1] = r1;
        __syncwarp();
        if (k == 0 && valid) {
            T s[16], pt[kPointStride], q[4], F[4];
#pragma unroll
            for (int t = 0; t < 16; ++t) s[t] = red[warp][g][t];
            pt[PT_X] = a.x[i]; pt[PT_Y] = a.y[i]; pt[PT_Z] = a.z[i]; pt[PT_F] = a.f[i]; pt[PT_GHM] = a.ghm[i];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                pt[PT_PU + c] = a.pu[3 * i + c]; pt[PT_PV + c] = a.pv[3 * i + c];
                pt[PT_PW + c] = a.pw[3 * i + c]; pt[PT_GG + c] = a.gg[3 * i + c];
            }
            Quad<T>::load_row(a.Kin + 4 * i, q);
            pointwise_rhs(s, q, pt, a.gh0, F);
            if (MODE == kStage0) {
                T kn[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) kn[t] = Quad<T>::axpy(q[t], a.c, F[t]);
                Quad<T>::store_row(a.D + 4 * i, F);
                Quad<T>::store_row(a.Kout + 4 * i, kn);
            } else if (MODE == kStage1 || MODE == kStage2) {
                T h[4], d[4], kn[4];
                Quad<T>::load_row_rw(a.H + 4 * i, h);
                Quad<T>::load_row_rw(a.D + 4 * i, d);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    d[t] = Quad<T>::axpy(d[t], T(2), F[t]);
                    kn[t] = Quad<T>::axpy(h[t], a.c, F[t]);
                }
                Quad<T>::store_row(a.D + 4 * i, d);
                Quad<T>::store_row(a.Kout + 4 * i, kn);
            } else {
                T h[4], d[4];
                Quad<T>::load_row_rw(a.H + 4 * i, h);
                Quad<T>::load_row_rw(a.D + 4 * i, d);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    d[t] = Quad<T>::axpy(d[t], T(1), F[t]);
                    h[t] = Quad<T>::update_h(h[t], a.dt6, d[t]);
                }
                Quad<T>::store_row(a.H + 4 * i, h);
            }
        }
        __syncwarp();
    }
}

// First call on the current device: look up the scratch array's address.
int scratch_for_current_device(void** out) {
    int dev = 0;
    SWE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("swe_cuda_step_noalloc: device %d beyond the %d supported", dev, kMaxDevices);
        return SWE_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        SWE_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SWE_OK;
}

// nsteps = 0: wait for the caller's stream, then report (and clear) the first
// out-of-range stencil index any earlier call met.
int report_bad_index(cudaStream_t stream) {
    SWE_CUDA_TRY(cudaStreamSynchronize(stream));
    int bad[4] = {0, 0, 0, 0};
    SWE_CUDA_TRY(cudaMemcpyFromSymbol(bad, g_noalloc_bad, sizeof(bad)));
    if (!bad[0]) return SWE_OK;
    const int zero[4] = {0, 0, 0, 0};
    SWE_CUDA_TRY(cudaMemcpyToSymbol(g_noalloc_bad, zero, sizeof(zero)));
    set_error("swe_cuda_step_noalloc: an earlier call met idx[node %d][nbr %d] = %d outside 0..n-1; it read the "
              "node's own row there, so its results are wrong", bad[1], bad[2], bad[3]);
    return SWE_ERR_INDEX;
}

template <typename T>
int run_noalloc(int n, int nnbr, double gh0, double dt, const int* idx, const void* Dx, const void* Dy,
                const void* Dz, const void* L, const void* x, const void* y, const void* z, const void* f,
                const void* ghm, const void* pu, const void* pv, const void* pw, const void* gg, void* H,
                int nsteps, cudaStream_t stream) {
    void* scratch = nullptr;
    SWE_TRY(scratch_for_current_device(&scratch));
    T* Ka = reinterpret_cast<T*>(scratch);
    T* Kb = Ka + 4L * n;
    T* D = Kb + 4L * n;
    RowMajorArgs<T> a{};
    a.n = n;
    a.nnbr = nnbr;
    a.idx = idx;
    a.Dx = (const T*)Dx; a.Dy = (const T*)Dy; a.Dz = (const T*)Dz; a.L = (const T*)L;
    a.x = (const T*)x; a.y = (const T*)y; a.z = (const T*)z; a.f = (const T*)f; a.ghm = (const T*)ghm;
    a.pu = (const T*)pu; a.pv = (const T*)pv; a.pw = (const T*)pw; a.gg = (const T*)gg;
    a.H = (T*)H;
    a.D = D;
    a.gh0 = (T)gh0;
    const T dtT = (T)dt;
    a.dt6 = (double)dtT / 6.0;
    const int grid = ceil_div(n, 4 * kStageWarps);
    for (int s = 0; s < nsteps; ++s) {
        a.Kin = a.H; a.Kout = Ka; a.c = (T)(dtT / 2.0);
        rowmajor_stage_kernel<T, kStage0><<<grid, kStageThreads, 0, stream>>>(a);
        a.Kin = Ka; a.Kout = Kb;
        rowmajor_stage_kernel<T, kStage1><<<grid, kStageThreads, 0, stream>>>(a);
        a.Kin = Kb; a.Kout = Ka; a.c = dtT;
        rowmajor_stage_kernel<T, kStage2><<<grid, kStageThreads, 0, stream>>>(a);
        a.Kin = Ka; a.Kout = nullptr;
        rowmajor_stage_kernel<T, kStage3><<<grid, kStageThreads, 0, stream>>>(a);
        count_launch(4);
        SWE_CUDA_TRY(cudaGetLastError());
    }
    return SWE_OK;
}

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" int swe_cuda_step_noalloc(int fsize, int n, int nnbr, double gh0, double dt, const int* idx,
                                     const void* Dx, const void* Dy, const void* Dz, const void* L,
                                     const void* x, const void* y, const void* z, const void* f,
                                     const void* ghm, const void* p_u, const void* p_v, const void* p_w,
                                     const void* gradghm, void* H, int nsteps, void* stream) {
    if (fsize != 8 && fsize != 4) { set_error("swe_cuda_step_noalloc: fsize must be 8 or 4, got %d", fsize); return SWE_ERR_ARG; }
    if (nnbr <= 0 || nnbr > kSlots) { set_error("swe_cuda_step_noalloc: nnbr %d not in 1..%d", nnbr, kSlots); return SWE_ERR_ARG; }
    if (nsteps < 0) { set_error("swe_cuda_step_noalloc: nsteps < 0"); return SWE_ERR_ARG; }
    const long max_nodes = (long)(kNoallocScratchBytes / (12L * fsize));
    if (n <= 0 || n > max_nodes) {
        set_error("swe_cuda_step_noalloc: n = %d nodes outside 1..%ld, the most the %zu-byte static scratch "
                  "holds at fsize %d (3 x n x 4 values)", n, max_nodes, kNoallocScratchBytes, fsize);
        return SWE_ERR_ARG;
    }
    if (!idx || !Dx || !Dy || !Dz || !L || !x || !y || !z || !f || !ghm || !p_u || !p_v || !p_w || !gradghm || !H) {
        set_error("swe_cuda_step_noalloc: null device pointer");
        return SWE_ERR_ARG;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (nsteps == 0) return report_bad_index(s);
    return fsize == 8 ? run_noalloc<double>(n, nnbr, gh0, dt, idx, Dx, Dy, Dz, L, x, y, z, f, ghm, p_u, p_v, p_w,
                                            gradghm, H, nsteps, s)
                      : run_noalloc<float>(n, nnbr, gh0, dt, idx, Dx, Dy, Dz, L, x, y, z, f, ghm, p_u, p_v, p_w,
                                           gradghm, H, nsteps, s);
}
