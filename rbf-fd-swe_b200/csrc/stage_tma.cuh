// Fused RK4 stage kernel, TMA-pipelined (plain form, FP64 / FP32).
//
// Same math and lane split as stage_kernel.cuh, restructured for B200's bulk
// copy engine.  A persistent CTA per SM runs one producer warp and 8 consumer
// warps over tiles of 32 consecutive nodes.  For every tile the producer
// issues cp.async.bulk copies (global -> shared, completing on an mbarrier)
// into one of kStages ring slots:
//   * the tile's packed weights (32 x 1 KB FP64) and pointwise records,
//   * its 16-bit window-local stencil indices,
//   * the tile's own state rows, and H / D rows for stages 1-3,
//   * the neighbour window: the state rows the tile's stencils touch, as up to
//     kMaxRanges contiguous row ranges of the RCM-ordered state, precomputed
//     at init.  In RCM order a 32-node tile's ~290 neighbour rows fall into
//     7-11 runs (at most 37 on the icosahedral grids up to N = 655362) once
//     gaps of up to 8 rows are bridged, about 310 rows (at most 468) in all.
// Consumers wait on the slot's mbarrier, run the stencil sums, reduction and
// pointwise/RK combine entirely from shared memory, store their outputs, and
// release the slot.  Every wait is bounded; a timeout sets an error word and
// the kernel drains its outstanding copies and returns.
#pragma once

#include "stage_kernel.cuh"
#include "tcgen05.cuh"

namespace swe {

constexpr int kTmaTile = 32;           // nodes per tile
constexpr int kMaxRanges = 40;         // contiguous row ranges per neighbour window (<= 64)
constexpr int kWinRows = 512;          // max rows per neighbour window
constexpr int kTmaConsumerWarps = 8;
constexpr int kTmaThreads = 32 * (kTmaConsumerWarps + 1);
constexpr uint32_t kTmaWaitTries = 1u << 24;

namespace tma {
__device__ __forceinline__ void arrive_expect_tx(uint64_t* b, uint32_t tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(b)), "r"(tx)
                 : "memory");
}
__device__ __forceinline__ void arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(b)) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            tc::smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(tc::smem_u32(mbar))
        : "memory");
}
}  // namespace tma

template <typename T>
struct TmaLayout {
    static constexpr int kW = kTmaTile * kSlots * 4 * (int)sizeof(T);    // weights
    static constexpr int kIdx = kTmaTile * kSlots * 2;                     // uint16 local indices
    static constexpr int kPt = kTmaTile * kPointStride * (int)sizeof(T);  // pointwise
    static constexpr int kRow = 4 * (int)sizeof(T);                       // one state row
    static constexpr int kRows = kTmaTile * kRow;                         // own / H / D rows
    static constexpr int kWin = kWinRows * kRow;
    static constexpr int oW = 0, oIdx = oW + kW, oPt = oIdx + kIdx, oOwn = oPt + kPt, oH = oOwn + kRows,
                         oD = oH + kRows, oWin = oD + kRows;
    static constexpr int kSlotBytes = ((oWin + kWin) + 127) / 128 * 128;
    static constexpr int kStages = (sizeof(T) == 8) ? 3 : 5;
    static constexpr int kSmem = kStages * kSlotBytes;
};

template <typename T>
struct TmaArgs {
    StageArgs<T> s;
    int ntiles;
    const uint16_t* idxl;   // [n][8 lanes][4] window-local indices
    const int2* ranges;     // [ntiles][1 + kMaxRanges]: {count, rows} then {start, nrows}
    int* err;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(kTmaThreads, 1) stage_tma_kernel(const TmaArgs<T> ta) {
    using Lay = TmaLayout<T>;
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
        // ---------------- producer (whole warp issues) ----------------
        // The tile's range list is loaded by all lanes at once, window offsets
        // come from a warp prefix sum, lane 0 posts the expected bytes and
        // every lane issues its share of the bulk copies.  complete_tx may
        // precede expect_tx inside a phase: the phase cannot close before
        // lane 0's single arrive.
        int it = 0, issued = 0;
        for (int tile = blockIdx.x; tile < ta.ntiles; tile += gridDim.x, ++it) {
            const int s = it % Lay::kStages;
            int wait_ok = 1;
            if (lane == 0 && it >= Lay::kStages)
                wait_ok = tc::mbar_wait_bounded(&empty[s], ((it / Lay::kStages) - 1) & 1, kTmaWaitTries);
            wait_ok = __shfl_sync(0xffffffffu, wait_ok, 0);
            if (!wait_ok || *(volatile int*)&s_abort) {
                if (lane == 0) { atomicExch(ta.err, 1); s_abort = 1; }
                break;
            }
            unsigned char* slot = smem + s * Lay::kSlotBytes;
            const long n0 = (long)tile * kTmaTile;
            const int nn = (int)min((long)kTmaTile, (long)a.n - n0);
            const int2* tab = ta.ranges + (long)tile * (1 + kMaxRanges);
            const int2 hdr = __ldg(tab);
            // ranges r = lane and r = lane + 32 (kMaxRanges <= 64)
            int2 r0 = make_int2(0, 0), r1 = make_int2(0, 0);
            if (lane < hdr.x) r0 = __ldg(tab + 1 + lane);
            if (lane + 32 < hdr.x) r1 = __ldg(tab + 1 + lane + 32);
            int p0 = r0.y, p1 = r1.y;                       // inclusive prefix sums of the lengths
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t0 = __shfl_up_sync(0xffffffffu, p0, o);
                const int t1 = __shfl_up_sync(0xffffffffu, p1, o);
                if (lane >= o) { p0 += t0; p1 += t1; }
            }
            const int first_total = __shfl_sync(0xffffffffu, p0, 31);
            const int off0 = p0 - r0.y, off1 = first_total + p1 - r1.y;
            if (lane == 0) {
                const uint32_t tx = nn * (kSlots * 4 * sizeof(T) + kSlots * 2 + kPointStride * sizeof(T) + Lay::kRow) +
                                    (need_hd ? 2 * nn * Lay::kRow : 0) + hdr.y * Lay::kRow;
                tma::arrive_expect_tx(&full[s], tx);
            }
            switch (lane) {
                case 0: tma::bulk_g2s(slot + Lay::oW, a.W + n0 * kSlotChunks * Quad<T>::kUnits * 8,
                                      nn * kSlots * 4 * sizeof(T), &full[s]); break;
                case 1: tma::bulk_g2s(slot + Lay::oIdx, ta.idxl + n0 * kSlots, nn * kSlots * 2, &full[s]); break;
                case 2: tma::bulk_g2s(slot + Lay::oPt, a.PT + n0 * kPointStride, nn * kPointStride * sizeof(T),
                                      &full[s]); break;
                case 3: tma::bulk_g2s(slot + Lay::oOwn, a.Kin + 4L * (n0 + a.pid0), nn * Lay::kRow, &full[s]); break;
                case 4: if (need_hd) tma::bulk_g2s(slot + Lay::oH, a.H + 4L * n0, nn * Lay::kRow, &full[s]); break;
                case 5: if (need_hd) tma::bulk_g2s(slot + Lay::oD, a.D + 4L * n0, nn * Lay::kRow, &full[s]); break;
                default: break;
            }
            if (lane < hdr.x)
                tma::bulk_g2s(slot + Lay::oWin + off0 * Lay::kRow, a.Kin + 4L * r0.x, r0.y * Lay::kRow, &full[s]);
            if (lane + 32 < hdr.x)
                tma::bulk_g2s(slot + Lay::oWin + off1 * Lay::kRow, a.Kin + 4L * r1.x, r1.y * Lay::kRow, &full[s]);
            ++issued;
        }
        // drain: every issued slot must have landed before the CTA exits
        if (lane == 0)
            for (int j = max(0, issued - Lay::kStages); j < issued; ++j)
                tc::mbar_wait_bounded(&full[j % Lay::kStages], (j / Lay::kStages) & 1, kTmaWaitTries);
        return;
    }

    // ---------------- consumers ----------------
    const int g = lane >> 3, k = lane & 7;
    constexpr int U = Quad<T>::kUnits;
    int it = 0;
    for (int tile = blockIdx.x; tile < ta.ntiles; tile += gridDim.x, ++it) {
        const int s = it % Lay::kStages;
        const bool ok = tc::mbar_wait_bounded(&full[s], (it / Lay::kStages) & 1, kTmaWaitTries);
        if (!ok || *(volatile int*)&s_abort) {
            if (lane == 0) { atomicExch(ta.err, 2); s_abort = 1; }
            break;
        }
        const unsigned char* slot = smem + s * Lay::kSlotBytes;
        const uint4* Ws = reinterpret_cast<const uint4*>(slot + Lay::oW);
        const T* win = reinterpret_cast<const T*>(slot + Lay::oWin);
        const int t = warp * 4 + g;                       // node within the tile
        const long i = (long)tile * kTmaTile + t;
        const bool valid = i < a.n;
        const int tt = valid ? t : 0;
        const ushort4 nb = *reinterpret_cast<const ushort4*>(slot + Lay::oIdx + (tt * 8 + k) * 8);
        const int nbr[4] = {nb.x, nb.y, nb.z, nb.w};
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
                const double2 k0 = *reinterpret_cast<const double2*>(win + 4 * nbr[m]);
                const double2 k1 = *reinterpret_cast<const double2*>(win + 4 * nbr[m] + 2);
                kv[0] = k0.x; kv[1] = k0.y; kv[2] = k1.x; kv[3] = k1.y;
            } else {
                const float4 w0 = *reinterpret_cast<const float4*>(wu);
                w[0] = w0.x; w[1] = w0.y; w[2] = w0.z; w[3] = w0.w;
                const float4 k0 = *reinterpret_cast<const float4*>(win + 4 * nbr[m]);
                kv[0] = k0.x; kv[1] = k0.y; kv[2] = k0.z; kv[3] = k0.w;
            }
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
