// Fused RK4 stage kernel, node-per-lane form (plain form, FP64 / FP32).
//
// Same stage semantics as stage_kernel.cuh (eval_RHS_swe plus the RK4 stage
// combine, swe_code/main/rk4_rbffd_swe.c:30-186 and :285-353), with a work split
// that needs little or no cross-lane reduction: each of a node's LPN lanes (1, 2
// or 4) sums the slots j = sub, sub + LPN, ... of the node serially -- with
// LPN = 1 that is the reference's own slot order -- and the LPN partial sums
// meet in a butterfly of log2(LPN) shuffle steps.  Lane sub 0 of every node then
// runs the pointwise part and the stage combine, so up to all 32 lanes of a warp
// are busy in the epilogue.
//
// The stencil weights and indices live in a second, tile-transposed copy
// (pack_stencils_kernel in pack.cuh): per 32-node tile, slot-major, node-minor,
// so one slot's weights of a warp's nodes are one contiguous 512-byte (FP64:
// two) or 16-byte-per-lane (FP32) row and one slot's indices a contiguous
// 128-byte row.  Weights and indices are streamed with L1 no-allocate loads; the
// neighbour gathers keep L1 to themselves.  One warp per unit of 32 / LPN nodes,
// no persistent loop: the hardware scheduler balances the tail.  MINB (4 or 5)
// is the register bound's CTAs per SM: 5 trades load depth for a grid that fits
// in one wave on mid-sized patches.  Programmatic dependent launch lets the next
// stage's CTAs take free SMs while the last wave of this stage finishes; every
// read of a state array comes after griddepcontrol.wait.  swe_cuda_init times
// the shapes (LPN x MINB x L2 prefetch) and keeps the fastest.
#pragma once

#include "stage_kernel.cuh"

namespace swe {

constexpr int kLaneThreads = 128;
constexpr int kLaneWarps = kLaneThreads / 32;
constexpr int kLaneTile = 32;      // nodes per transposed tile of the packed arrays

template <typename T>
struct LaneArgs {
    StageArgs<T> s;
    const uint4* Wl;   // [tile][slot][unit][32 nodes] 16-byte units (FP64: (Dx,Dy), (Dz,L); FP32: all four)
    const int* idxl;   // [tile][slot][32 nodes] gather rows
    const short* idxs; // the same as 16-bit offsets from the node's own row (clamped to n - 1)
    int l2_prefetch;   // 1: bulk L2 prefetch of each warp's contiguous blocks at its start
    int nnbr;          // stencil slots in use: slots nnbr.. hold zero weights (a lane's last one is not read)
};

namespace lane {

__device__ __forceinline__ int ld_stream(const int* p) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_stream(const short* p) {
    short v;
    asm volatile("ld.global.nc.L1::no_allocate.b16 %0, [%1];" : "=h"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double2 ld_stream(const double2* p) {
    double2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float4 ld_stream(const float4* p) {
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}
// the four weights (Dx, Dy, Dz, L) of one slot of node t; units of a slot are 32 x 16 bytes apart
__device__ __forceinline__ void weights(const uint4* u, double (&w)[4]) {
    const double2 a = ld_stream(reinterpret_cast<const double2*>(u));
    const double2 b = ld_stream(reinterpret_cast<const double2*>(u + kLaneTile));
    w[0] = a.x; w[1] = a.y; w[2] = b.x; w[3] = b.y;
}
__device__ __forceinline__ void weights(const uint4* u, float (&w)[4]) {
    const float4 a = ld_stream(reinterpret_cast<const float4*>(u));
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
}
}  // namespace lane

// I16: read the gather rows from the 16-bit offsets (half the index bytes); every
// patch whose stencil rows lie within 32767 rows of their node (any RCM-ordered grid)
template <typename T, int MODE, int LPN, int MINB, bool I16>
__global__ void __launch_bounds__(kLaneThreads, MINB) stage_lane_kernel(const LaneArgs<T> la) {
    static_assert(LPN == 1 || LPN == 2 || LPN == 4, "1, 2 or 4 lanes per node");
    constexpr int kNpw = 32 / LPN;          // nodes per warp
    constexpr int kJpl = kSlots / LPN;      // slots per lane
    constexpr int U = Quad<T>::kUnits;
    const StageArgs<T>& a = la.s;
    const int lane = threadIdx.x & 31;
    const int tl = lane % kNpw, sub = lane / kNpw;
    const long node0 = ((long)blockIdx.x * kLaneWarps + (threadIdx.x >> 5)) * kNpw;
    const int nvalid = (int)min((long)kNpw, (long)a.n - node0);
    // With l2_prefetch, one lane requests the warp's contiguous blocks into L2 up
    // front, so that the loads below wait on L2 rather than DRAM: this warp's share
    // of its tile's weight and index blocks (static: before the wait, overlapping
    // the previous stage), then its pointwise records and own / H / D rows.  On large
    // patches the extra requests compete with the demand loads; on small ones it
    // gains little now that the gather rows are read before the wait, so the
    // init-time timing keeps it only where it is clearly faster.
    constexpr uint32_t kTileW = kSlots * U * kLaneTile * 16, kTileI = kSlots * kLaneTile * (I16 ? 2 : 4);
    const bool pf = la.l2_prefetch != 0;
    if (pf && lane == 0 && nvalid > 0) {
        const long tb = node0 / kLaneTile;
        const int wt = (int)(node0 % kLaneTile) / kNpw;        // warp within its tile
        prefetch_l2_bulk(reinterpret_cast<const unsigned char*>(la.Wl) + tb * kTileW + wt * (kTileW / LPN), kTileW / LPN);
        const void* ib = I16 ? static_cast<const void*>(la.idxs) : static_cast<const void*>(la.idxl);
        prefetch_l2_bulk(reinterpret_cast<const unsigned char*>(ib) + tb * kTileI + wt * (kTileI / LPN), kTileI / LPN);
        prefetch_l2_bulk(a.PT + node0 * kPointStride, (uint32_t)(nvalid * kPointStride * sizeof(T)));
    }
    // a warp's nodes lie in one tile of the packed arrays (kNpw divides 32); nodes
    // past n in the last tile have zero weights and gather a valid row
    const long i = node0 + tl;
    const long tile = i / kLaneTile;
    const int t = (int)(i % kLaneTile);
    const int* ip = la.idxl + (tile * kSlots + sub) * kLaneTile + t;
    const short* sp = la.idxs + (tile * kSlots + sub) * kLaneTile + t;
    const int own = (int)min(i, (long)a.n - 1) + a.pid0;   // the row the 16-bit offsets start from
    // the gather rows are static: with 2 or 4 lanes per node (16 or 8 rows a lane), or
    // at 3 CTAs per SM (168 registers), they are read before the wait, so that the
    // gathers issue as soon as the previous stage's states are visible (32 rows a
    // lane in 96 or 128 registers would spill)
    constexpr bool kEarlyRows = LPN > 1 || MINB <= 3;
    auto row = [&](int jj) {
        return I16 ? own + lane::ld_stream(sp + jj * LPN * kLaneTile) : lane::ld_stream(ip + jj * LPN * kLaneTile);
    };
    int prow[kEarlyRows ? kJpl : 1];
    if (kEarlyRows && nvalid > 0) {
#pragma unroll
        for (int jj = 0; jj < kJpl; ++jj)
            prow[kEarlyRows ? jj : 0] = jj < kJpl - 1 || jj * LPN + sub < la.nnbr ? row(jj) : own;
    }
    pdl_wait();                // neighbour states and H / D come from the previous stage
    pdl_trigger();
    if (nvalid <= 0) return;
    if (pf && lane == 0) {
        const uint32_t rows = (uint32_t)(nvalid * 4 * sizeof(T));
        prefetch_l2_bulk(a.Kin + 4 * (node0 + a.pid0), rows);
        if (MODE != kStage0 && MODE != kEvalOnly) {
            prefetch_l2_bulk(a.H + 4 * node0, rows);
            prefetch_l2_bulk(a.D + 4 * node0, rows);
        }
    }
    const uint4* wp = la.Wl + (tile * kSlots + sub) * U * kLaneTile + t;
    T acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q] = T(0);
#pragma unroll
    for (int jj = 0; jj < kJpl; ++jj) {
        // a padding slot (zero weights) in a lane's last iteration moves no bytes (slot 31
        // of 31-neighbour stencils); a test in every iteration would keep the compiler
        // from issuing the other iterations' loads together
        if (jj == kJpl - 1 && jj * LPN + sub >= la.nnbr) continue;
        const int p = kEarlyRows ? prow[kEarlyRows ? jj : 0] : row(jj);
        T w[4], kv[4];
        lane::weights(wp + jj * LPN * U * kLaneTile, w);
        Quad<T>::load_row(a.Kin + 4L * p, kv);
#pragma unroll
        for (int op = 0; op < 4; ++op)
#pragma unroll
            for (int f = 0; f < 4; ++f) acc[op * 4 + f] += w[op] * kv[f];
    }
    if constexpr (LPN > 1) {
#pragma unroll
        for (int o = kNpw; o < 32; o <<= 1)
#pragma unroll
            for (int q = 0; q < 16; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    }
    if (sub != 0 || i >= a.n) return;
    T q[4], F[4];
    Quad<T>::load_row(a.Kin + 4L * (i + a.pid0), q);
    pointwise_rhs(acc, q, a.PT + i * kPointStride, a.gh0, F);
    if (MODE == kEvalOnly) {
        Quad<T>::store_row(a.F + 4 * i, F);
    } else if (MODE == kStage0) {
        // copy_fp_arr(D, F) and eval_K(H, K, F, dt/2): here K_in is H
        T kn[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) kn[x] = Quad<T>::axpy(q[x], a.c, F[x]);
        Quad<T>::store_row(a.D + 4 * i, F);
        Quad<T>::store_row(a.Kout + 4 * i, kn);
    } else {
        T h[4], d[4];
        Quad<T>::load_row_rw(a.H + 4 * i, h);
        Quad<T>::load_row_rw(a.D + 4 * i, d);
        if (MODE == kStage1 || MODE == kStage2) {
            // update_D(D, F, 2) and eval_K(H, K, F, c)
            T kn[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                d[x] = Quad<T>::axpy(d[x], T(2), F[x]);
                kn[x] = Quad<T>::axpy(h[x], a.c, F[x]);
            }
            Quad<T>::store_row(a.D + 4 * i, d);
            Quad<T>::store_row(a.Kout + 4 * i, kn);
        } else {
            // update_D(D, F, 1) and update_H(H, D, dt)
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                d[x] = Quad<T>::axpy(d[x], T(1), F[x]);
                h[x] = Quad<T>::update_h(h[x], a.dt6, d[x]);
            }
            Quad<T>::store_row(a.H + 4 * i, h);
        }
    }
}

}  // namespace swe
