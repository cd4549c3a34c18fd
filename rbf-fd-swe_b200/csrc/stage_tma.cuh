// Fused RK4 stage kernel, bulk-copy pipelined (plain form, FP64 / FP32).
//
// Same math and lane split as stage_kernel.cuh, restructured around B200's
// bulk copy engine.  Persistent CTAs run one producer warp and TILE/4 consumer
// warps over tiles of TILE consecutive nodes: 64-node tiles with one CTA per SM,
// 32-node tiles with two or 16-node tiles with four CTAs per SM (more producers
// in flight per SM; the library times the three at init).  For every tile the producer issues six
// cp.async.bulk copies (global -> shared, completing on an mbarrier) into one
// of kStages ring slots: the tile's packed weights (TILE x 1 KB in FP64),
// packed stencil indices, pointwise records, own state rows, and the H / D rows
// for stages 1-3 -- every contiguous per-node stream of the stage.  Consumers
// wait on the slot's mbarrier, gather the neighbour states through L1/L2 (the
// state arrays are L2-resident; a tile's neighbours are scattered rows, which
// suits plain loads better than many small bulk copies), run the stencil sums,
// reduction and pointwise/RK combine with every other operand in shared memory,
// store their outputs and release the slot.  Launched with programmatic
// dependent launch: the first tile's weights, indices and pointwise records are
// requested before griddepcontrol.wait, so they load while the previous stage
// finishes; every read of a state array comes after the wait.  Every wait is
// bounded; a timeout sets an error word and the kernel drains its outstanding
// copies and returns.
#pragma once

#include "stage_kernel.cuh"
#include "tcgen05.cuh"

namespace swe {


template <int TILE>
struct TmaShape {
    static constexpr int kTile = TILE;                     // nodes per tile
    static constexpr int kConsumerWarps = TILE / 4;        // 4 nodes per warp
    static constexpr int kThreads = 32 * (kConsumerWarps + 1);
    static constexpr int kCtasPerSm = 64 / TILE;
};
constexpr uint64_t kTmaWaitLimitNs = 2000000000ull;   // a slot wait gives up after 2 s

namespace tma {
using tc::bulk_g2s;
__device__ __forceinline__ void arrive_expect_tx(uint64_t* b, uint32_t tx) { tc::mbar_arrive_expect_tx(b, tx); }
__device__ __forceinline__ void arrive(uint64_t* b) { tc::mbar_arrive(b); }
}  // namespace tma

template <typename T, int TILE>
struct TmaLayout {
    static constexpr int kTmaTile = TILE;
    static constexpr int kWn = kSlots * 4 * (int)sizeof(T);     // weight bytes per node
    static constexpr int kIdxn = kSlots * 4;                      // index bytes per node
    static constexpr int kPtn = kPointStride * (int)sizeof(T);   // pointwise bytes per node
    static constexpr int kRow = 4 * (int)sizeof(T);               // one state row
    static constexpr int oW = 0, oIdx = oW + kTmaTile * kWn, oPt = oIdx + kTmaTile * kIdxn,
                         oOwn = oPt + kTmaTile * kPtn, oH = oOwn + kTmaTile * kRow, oD = oH + kTmaTile * kRow;
    static constexpr int kSlotBytes = ((oD + kTmaTile * kRow) + 127) / 128 * 128;
    static constexpr int kStages = (sizeof(T) == 8) ? 2 : 4;   // 180 KB (FP64) / 196 KB (FP32) per SM
    static constexpr int kSmem = kStages * kSlotBytes;
};

template <typename T>
struct TmaArgs {
    StageArgs<T> s;
    int ntiles;
    int* err;
};

template <typename T, int MODE, int TILE>
__global__ void __launch_bounds__(TmaShape<TILE>::kThreads, TmaShape<TILE>::kCtasPerSm)
    stage_tma_kernel(const TmaArgs<T> ta) {
    using Lay = TmaLayout<T, TILE>;
    constexpr int kTmaTile = TILE;
    constexpr int kTmaConsumerWarps = TmaShape<TILE>::kConsumerWarps;
    const StageArgs<T>& a = ta.s;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[Lay::kStages], empty[Lay::kStages];
    __shared__ __align__(16) T red[kTmaConsumerWarps][4][16];
    __shared__ int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < Lay::kStages; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], kTmaConsumerWarps);
        }
        s_abort = 0;
        tc::fence_mbar_init();
    }
    __syncthreads();
    const bool need_hd = MODE == kStage1 || MODE == kStage2 || MODE == kStage3;

    if (warp == kTmaConsumerWarps) {
        // ---------------- producer: lanes 0-5 each issue one stream ----------------
        int it = 0, issued = 0;
        for (int tile = blockIdx.x; tile < ta.ntiles; tile += gridDim.x, ++it) {
            const int s = it % Lay::kStages;
            int wait_ok = 1;
            if (lane == 0 && it >= Lay::kStages)
                wait_ok = tc::mbar_wait_timed(&empty[s], ((it / Lay::kStages) - 1) & 1, kTmaWaitLimitNs);
            wait_ok = __shfl_sync(0xffffffffu, wait_ok, 0);
            if (!wait_ok || *(volatile int*)&s_abort) {
                if (lane == 0) { atomicExch(ta.err, 1); s_abort = 1; }
                break;
            }
            unsigned char* slot = smem + s * Lay::kSlotBytes;
            const long n0 = (long)tile * kTmaTile;
            const int nn = (int)min((long)kTmaTile, (long)a.n - n0);
            if (lane == 0) {
                const uint32_t tx = nn * (Lay::kWn + Lay::kIdxn + Lay::kPtn + Lay::kRow) + (need_hd ? 2 * nn * Lay::kRow : 0);
                tma::arrive_expect_tx(&full[s], tx);
            }
            __syncwarp();
            // static streams (never written by a stage) first: for the first tile they
            // load while the previous stage is still finishing
            switch (lane) {
                case 0: tma::bulk_g2s(slot + Lay::oW, a.W + n0 * kSlotChunks * Quad<T>::kUnits * 8, nn * Lay::kWn,
                                      &full[s]); break;
                case 1: tma::bulk_g2s(slot + Lay::oIdx, a.idx + n0 * 8, nn * Lay::kIdxn, &full[s]); break;
                case 2: tma::bulk_g2s(slot + Lay::oPt, a.PT + n0 * kPointStride, nn * Lay::kPtn, &full[s]); break;
                default: break;
            }
            if (it == 0) {
                pdl_wait();
                pdl_trigger();
            }
            switch (lane) {
                case 3: tma::bulk_g2s(slot + Lay::oOwn, a.Kin + 4L * (n0 + a.pid0), nn * Lay::kRow, &full[s]); break;
                case 4: if (need_hd) tma::bulk_g2s(slot + Lay::oH, a.H + 4L * n0, nn * Lay::kRow, &full[s]); break;
                case 5: if (need_hd) tma::bulk_g2s(slot + Lay::oD, a.D + 4L * n0, nn * Lay::kRow, &full[s]); break;
                default: break;
            }
            ++issued;
        }
        // drain: every issued slot must have landed before the CTA exits
        if (lane == 0)
            for (int j = max(0, issued - Lay::kStages); j < issued; ++j)
                tc::mbar_wait_timed(&full[j % Lay::kStages], (j / Lay::kStages) & 1, kTmaWaitLimitNs);
        return;
    }

// ---------------- consumers ----------------
    const int g = lane >> 3, k = lane & 7;
    constexpr int U = Quad<T>::kUnits;
    pdl_wait();            // neighbour states come from the previous stage
    pdl_trigger();
    int it = 0;
    for (int tile = blockIdx.x; tile < ta.ntiles; tile += gridDim.x, ++it) {
        const int s = it % Lay::kStages;
        const bool ok = tc::mbar_wait_timed(&full[s], (it / Lay::kStages) & 1, kTmaWaitLimitNs);
        if (!ok || *(volatile int*)&s_abort) {
            if (lane == 0) { atomicExch(ta.err, 2); s_abort = 1; }
            break;
        }
        const unsigned char* slot = smem + s * Lay::kSlotBytes;
        const uint4* Ws = reinterpret_cast<const uint4*>(slot + Lay::oW);
        const int t = warp * 4 + g;                       // node within the tile
        const long i = (long)tile * kTmaTile + t;
        const bool valid = i < a.n;
        const int tt = valid ? t : 0;
        const int4 nb = *reinterpret_cast<const int4*>(slot + Lay::oIdx + (tt * 8 + k) * 16);
        const int nbr[4] = {nb.x, nb.y, nb.z, nb.w};
        T kg[kSlotChunks][4];
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m) Quad<T>::load_row(a.Kin + 4L * nbr[m], kg[m]);
        T acc[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[q] = T(0);
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m) {
            T w[4], kv[4];
            const uint4* wu = Ws + ((tt * kSlotChunks + m) * U) * 8 + k;
            if constexpr (sizeof(T) == 8) {
                const double2 w0 = *reinterpret_cast<const double2*>(wu);
                const double2 w1 = *reinterpret_cast<const double2*>(wu + 8);
                w[0] = w0.x; w[1] = w0.y; w[2] = w1.x; w[3] = w1.y;
            } else {
                const float4 w0 = *reinterpret_cast<const float4*>(wu);
                w[0] = w0.x; w[1] = w0.y; w[2] = w0.z; w[3] = w0.w;
            }
#pragma unroll
            for (int f = 0; f < 4; ++f) kv[f] = kg[m][f];
#pragma unroll
            for (int op = 0; op < 4; ++op)
#pragma unroll
                for (int f = 0; f < 4; ++f) acc[op * 4 + f] += w[op] * kv[f];
        }
        T r0, r1;
        reduce_scatter8(acc, k, r0, r1);
        red[warp][g][2 * k] = r0;
        red[warp][g][2 * k + 1] = r1;
        __syncwarp();
        if (k == 0 && valid) {
            T sm[16], q[4], F[4];
#pragma unroll
            for (int x = 0; x < 16; ++x) sm[x] = red[warp][g][x];
            const T* own = reinterpret_cast<const T*>(slot + Lay::oOwn) + 4 * t;
#pragma unroll
            for (int x = 0; x < 4; ++x) q[x] = own[x];
            pointwise_rhs(sm, q, reinterpret_cast<const T*>(slot + Lay::oPt) + t * kPointStride, a.gh0, F);
            if (MODE == kEvalOnly) {
                Quad<T>::store_row(a.F + 4 * i, F);
            } else if (MODE == kStage0) {
                T kn[4];
#pragma unroll
                for (int x = 0; x < 4; ++x) kn[x] = Quad<T>::axpy(q[x], a.c, F[x]);
                Quad<T>::store_row(a.D + 4 * i, F);
                Quad<T>::store_row(a.Kout + 4 * i, kn);
            } else {
                const T* hs = reinterpret_cast<const T*>(slot + Lay::oH) + 4 * t;
                const T* ds = reinterpret_cast<const T*>(slot + Lay::oD) + 4 * t;
                T h[4], d[4];
#pragma unroll
                for (int x = 0; x < 4; ++x) { h[x] = hs[x]; d[x] = ds[x]; }
                if (MODE == kStage1 || MODE == kStage2) {
                    T kn[4];
#pragma unroll
                    for (int x = 0; x < 4; ++x) {
                        d[x] = Quad<T>::axpy(d[x], T(2), F[x]);
                        kn[x] = Quad<T>::axpy(h[x], a.c, F[x]);
                    }
                    Quad<T>::store_row(a.D + 4 * i, d);
                    Quad<T>::store_row(a.Kout + 4 * i, kn);
                } else {
#pragma unroll
                    for (int x = 0; x < 4; ++x) {
                        d[x] = Quad<T>::axpy(d[x], T(1), F[x]);
                        h[x] = Quad<T>::update_h(h[x], a.dt6, d[x]);
                    }
                    Quad<T>::store_row(a.H + 4 * i, h);
                }
            }
        }
        __syncwarp();
        if (lane == 0) tma::arrive(&empty[s]);
    }
}

}  // namespace swe
