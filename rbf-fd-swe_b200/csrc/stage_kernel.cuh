// Fused RK4 stage kernel of the plain form (FP64 or FP32).
//
// One launch computes, for every node i of the patch, the RBF-FD right-hand
// side of the reference's eval_RHS_swe (swe_code/main/rk4_rbffd_swe.c:189-362):
// sixteen stencil sums (Dx, Dy, Dz, L applied to u, v, w, h), the Coriolis and
// gravity terms, the projection P*rhs, hyperviscosity and the geopotential
// equation -- and then the RK4 stage combine of RK_substep (:30-72) with
// copy_fp_arr/update_D/eval_K/update_H (:74-186) folded into the same thread
// that produced F, so F never goes to memory in the time-stepping modes.
//
// Work split: a warp owns 4 nodes; each node is owned by 8 lanes; lane k of a
// node handles stencil slots j = k, k+8, k+16, k+24.  The device layout of the
// weights is "as consumed" (packed once at init): every 16-byte load of a warp
// covers 4 nodes x 128 contiguous bytes, and a lane's four stencil indices are
// one 16-byte load.  Neighbour states (one 32-byte FP64 / 16-byte FP32 row per
// node, node-major) are gathered through the read-only path.  The 8 partial
// sums of each of the 16 dot products are combined with a 3-step recursive-
// halving shuffle (14 exchanges per lane instead of 80 for naive butterflies),
// after which lane k holds sums 2k and 2k+1; they meet in shared memory and
// lane 0 of the node runs the pointwise part and the stage combine.  The
// operands of that epilogue (pointwise record, own state, H and D rows) are
// fetched by the node's 8 lanes together with the gather and staged in
// shared memory, and the next group's stencil indices are prefetched, so one
// global round trip (the neighbour gather) remains on each group's critical
// path.
#pragma once

#include "common.cuh"

namespace swe {

enum StageMode { kStage0 = 0, kStage1 = 1, kStage2 = 2, kStage3 = 3, kEvalOnly = 4 };

template <typename T>
struct StageArgs {
    int n;              // nodes to compute (compute_size)
    int pid0;           // compute_pid_s: row of node 0 in the gather source
    const T* Kin;       // gather source [rows][4]
    const int4* idx;    // [n][8] int4: slots (k, k+8, k+16, k+24) of lane k
    const uint4* W;     // packed weights, see pack_stencils_kernel (pack.cuh)
    const T* PT;        // [n][kPointStride] pointwise data
    T* H;               // [n][4] RK base state (stages) -- also the gather source of stage 0
    T* D;               // [n][4] RK accumulator
    T* Kout;            // [n][4] next stage state (stages 0-2)
    T* F;               // [n][4] RHS output (eval-only mode)
    T gh0;
    T c;                // stage coefficient: dt/2, dt/2, dt for stages 0-2
    double dt6;         // dt/6 (the reference forms it in double: rk4_rbffd_swe.c:115)
};

template <typename T>
struct Quad;  // the four weights (Dx, Dy, Dz, L) of one stencil slot

template <>
struct Quad<double> {
    static constexpr int kUnits = 2;  // 16-byte units per slot
    __device__ static void load(const uint4* W, long base, double (&w)[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(W + base));
        const double2 b = __ldg(reinterpret_cast<const double2*>(W + base + 8));
        w[0] = a.x; w[1] = a.y; w[2] = b.x; w[3] = b.y;
    }
    __device__ static void load_row(const double* p, double (&v)[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ static void load_row_rw(const double* p, double (&v)[4]) {
        const double2 a = reinterpret_cast<const double2*>(p)[0];
        const double2 b = reinterpret_cast<const double2*>(p)[1];
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ static void store_row(double* p, const double (&v)[4]) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
    // K = H + c*F, D + k*F: unfused multiply-add, as the reference's C computes it
    __device__ static double axpy(double h, double c, double f) { return __dadd_rn(h, __dmul_rn(c, f)); }
    // H += (dt/6) * D in double (rk4_rbffd_swe.c:115)
    __device__ static double update_h(double h, double dt6, double d) { return __dadd_rn(h, __dmul_rn(dt6, d)); }
};

template <>
struct Quad<float> {
    static constexpr int kUnits = 1;
    __device__ static void load(const uint4* W, long base, float (&w)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(W + base));
        w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    }
    __device__ static void load_row(const float* p, float (&v)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    __device__ static void load_row_rw(const float* p, float (&v)[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    __device__ static void store_row(float* p, const float (&v)[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
    __device__ static float axpy(float h, float c, float f) { return __fadd_rn(h, __fmul_rn(c, f)); }
    // The FP32 reference evaluates H + (dt/6.0)*D in double and rounds once.
    __device__ static float update_h(float h, double dt6, float d) {
        return __double2float_rn(__dadd_rn((double)h, __dmul_rn(dt6, (double)d)));
    }
};

// 8-lane recursive-halving reduce-scatter of 16 partial sums: on return lane
// k (0..7 within its group) holds the group totals of sums 2k and 2k+1.
template <typename T>
__device__ __forceinline__ void reduce_scatter8(const T (&a)[16], int k, T& r0, T& r1) {
    const unsigned full = 0xffffffffu;
    T h8[8], h4[4];
    const bool b2 = (k & 4) != 0, b1 = (k & 2) != 0, b0 = (k & 1) != 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const T send = b2 ? a[t] : a[8 + t];
        const T keep = b2 ? a[8 + t] : a[t];
        h8[t] = keep + __shfl_xor_sync(full, send, 4);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const T send = b1 ? h8[t] : h8[4 + t];
        const T keep = b1 ? h8[4 + t] : h8[t];
        h4[t] = keep + __shfl_xor_sync(full, send, 2);
    }
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const T send = b0 ? h4[t] : h4[2 + t];
        const T keep = b0 ? h4[2 + t] : h4[t];
        (t == 0 ? r0 : r1) = keep + __shfl_xor_sync(full, send, 1);
    }
}

// rk4_rbffd_swe.c:320-353 for one node, given its 16 stencil sums s[op*4+field]
// (op: Dx, Dy, Dz, L; field: u, v, w, h), its own state and pointwise record.
template <typename T>
__device__ __forceinline__ void pointwise_rhs(const T (&s)[16], const T (&q)[4], const T* __restrict__ pt,
                                              T gh0, T (&F)[4]) {
    const T du_dx = s[0], dv_dx = s[1], dw_dx = s[2], dh_dx = s[3];
    const T du_dy = s[4], dv_dy = s[5], dw_dy = s[6], dh_dy = s[7];
    const T du_dz = s[8], dv_dz = s[9], dw_dz = s[10], dh_dz = s[11];
    const T Lu = s[12], Lv = s[13], Lw = s[14], Lh = s[15];
    const T u = q[0], v = q[1], w = q[2], h = q[3];
    const T x = pt[PT_X], y = pt[PT_Y], z = pt[PT_Z], f = pt[PT_F], ghm = pt[PT_GHM];
    const T rhs_u = -((u * du_dx) + (v * du_dy) + (w * du_dz) + (f * ((y * w) - (z * v))) + dh_dx);
    const T rhs_v = -((u * dv_dx) + (v * dv_dy) + (w * dv_dz) + (f * ((z * u) - (x * w))) + dh_dy);
    const T rhs_w = -((u * dw_dx) + (v * dw_dy) + (w * dw_dz) + (f * ((x * v) - (y * u))) + dh_dz);
    F[0] = (pt[PT_PU] * rhs_u) + (pt[PT_PU + 1] * rhs_v) + (pt[PT_PU + 2] * rhs_w) + Lu;
    F[1] = (pt[PT_PV] * rhs_u) + (pt[PT_PV + 1] * rhs_v) + (pt[PT_PV + 2] * rhs_w) + Lv;
    F[2] = (pt[PT_PW] * rhs_u) + (pt[PT_PW + 1] * rhs_v) + (pt[PT_PW + 2] * rhs_w) + Lw;
    F[3] = -((u * (dh_dx - pt[PT_GG])) + (v * (dh_dy - pt[PT_GG + 1])) + (w * (dh_dz - pt[PT_GG + 2])) +
             ((h + gh0 - ghm) * (du_dx + dv_dy + dw_dz))) + Lh;
}

constexpr int kStageThreads = 256;
constexpr int kStageWarps = kStageThreads / 32;

template <typename T, int MODE>
__global__ void __launch_bounds__(kStageThreads, 2) stage_kernel(const StageArgs<T> a) {
    // per warp and node: 16 sums, then the epilogue operands staged by the
    // node's 8 lanes (pointwise record, own state, H and D rows)
    constexpr int kEp = kPointStride + 12;
    __shared__ __align__(16) T red[kStageWarps][4][16];
    __shared__ __align__(16) T ep[kStageWarps][4][kEp];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = lane >> 3;       // node of this lane within the warp
    const int k = lane & 7;        // lane within the node
    const long warps_total = (long)gridDim.x * kStageWarps;
    constexpr int U = Quad<T>::kUnits;
    constexpr bool kHD = MODE == kStage1 || MODE == kStage2 || MODE == kStage3;

    long base = ((long)blockIdx.x * kStageWarps + warp) * 4;
    // indices of the first group; later groups' indices are prefetched one
    // group ahead so that only the neighbour gather is on the critical path
    int4 nb = __ldg(a.idx + min(base + g, (long)a.n - 1) * 8 + k);
    for (; base < a.n; base += warps_total * 4) {
        const long i = base + g;
        const bool valid = i < a.n;
        const long ii = valid ? i : (long)a.n - 1;
        const int nbr[4] = {nb.x, nb.y, nb.z, nb.w};
        T kv[kSlotChunks][4];
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m) Quad<T>::load_row(a.Kin + 4L * nbr[m], kv[m]);
        T w[kSlotChunks][4];
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m) Quad<T>::load(a.W, ((ii * kSlotChunks + m) * U) * 8 + k, w[m]);
        // epilogue operands: lanes 0-4 fetch the pointwise record (4 values
        // each), lanes 5-7 the own state and the H and D rows
        {
            T* e = ep[warp][g];
            if (k < 5) {
                T p[4];
                Quad<T>::load_row(a.PT + ii * kPointStride + 4 * k, p);
#pragma unroll
                for (int x = 0; x < 4; ++x) e[4 * k + x] = p[x];
            } else if (k == 5) {
                T q[4];
                Quad<T>::load_row(a.Kin + 4L * (ii + a.pid0), q);
#pragma unroll
                for (int x = 0; x < 4; ++x) e[kPointStride + x] = q[x];
            } else if (kHD) {
                T r[4];
                Quad<T>::load_row_rw((k == 6 ? a.H : a.D) + 4 * ii, r);
#pragma unroll
                for (int x = 0; x < 4; ++x) e[kPointStride + 4 * (k - 5) + x] = r[x];
            }
        }
        const long nbase = base + warps_total * 4;
        if (nbase < a.n) nb = __ldg(a.idx + min(nbase + g, (long)a.n - 1) * 8 + k);

        T acc[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[t] = T(0);
#pragma unroll
        for (int m = 0; m < kSlotChunks; ++m)
#pragma unroll
            for (int op = 0; op < 4; ++op)
#pragma unroll
                for (int fld = 0; fld < 4; ++fld) acc[op * 4 + fld] += w[m][op] * kv[m][fld];

        T r0, r1;
        reduce_scatter8(acc, k, r0, r1);
        red[warp][g][2 * k] = r0;
        red[warp][g][2 * k + 1] = r1;
        __syncwarp();

        if (k == 0 && valid) {
            const T* e = ep[warp][g];
            T s[16];
#pragma unroll
            for (int t = 0; t < 16; ++t) s[t] = red[warp][g][t];
            T q[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) q[x] = e[kPointStride + x];
            T F[4];
            pointwise_rhs(s, q, e, a.gh0, F);
            if (MODE == kEvalOnly) {
                Quad<T>::store_row(a.F + 4 * i, F);
            } else if (MODE == kStage0) {
                // copy_fp_arr(D, F) and eval_K(H, K, F, dt/2): here K_in is H
                T kn[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) kn[t] = Quad<T>::axpy(q[t], a.c, F[t]);
                Quad<T>::store_row(a.D + 4 * i, F);
                Quad<T>::store_row(a.Kout + 4 * i, kn);
            } else if (MODE == kStage1 || MODE == kStage2) {
                // update_D(D, F, 2) and eval_K(H, K, F, c)
                T kn[4], d[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    d[t] = Quad<T>::axpy(e[kPointStride + 8 + t], T(2), F[t]);
                    kn[t] = Quad<T>::axpy(e[kPointStride + 4 + t], a.c, F[t]);
                }
                Quad<T>::store_row(a.D + 4 * i, d);
                Quad<T>::store_row(a.Kout + 4 * i, kn);
            } else {
                // update_D(D, F, 1) and update_H(H, D, dt)
                T h[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const T d = Quad<T>::axpy(e[kPointStride + 8 + t], T(1), F[t]);
                    h[t] = Quad<T>::update_h(e[kPointStride + 4 + t], a.dt6, d);
                }
                Quad<T>::store_row(a.H + 4 * i, h);
            }
        }
        __syncwarp();
    }
}

}  // namespace swe
