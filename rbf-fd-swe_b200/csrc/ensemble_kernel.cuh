// Batched-ensemble RK4 stage kernel on tcgen05 tensor cores (3xTF32).
//
// B ensemble members share one grid.  The state is stored member-innermost,
// [node][mf] with mf = 4*member + field, so a neighbour's state for all members
// is one contiguous row of 4B floats.  For a tile of T consecutive nodes (in
// RCM order) the stencil products of all members are one dense contraction
//
//     D[mf][4t+op] = sum_k  X[row_k][mf] * W[op](node t, row_k)
//
// over the tile's U unique neighbour rows k (U ~ 74 for T = 4, ~104 for T = 8
// on the icosahedral grids; W is zero where row_k is not in node t's stencil).
// M = mf (one 128-row half = 32 members per 128 threads), N = 4T (16 or 32),
// K = U padded to a multiple of 8.  Each unique row is gathered once per tile
// instead of once per stencil slot (31 times), which is what makes the tensor
// core pay here.
//
// Precision (3xTF32): every operand is split x ~ hi + lo, both rounded to
// nearest TF32 (|x - hi - lo| <= 2^-22 |x|), and D = A_hi B_hi + A_hi B_lo +
// A_lo B_hi is accumulated in FP32 in TMEM.  Before the split every gathered
// value is centred on the state of the tile's first node, c[mf]: the
// contraction runs on X - c, whose entries are the local variation of the
// fields rather than their magnitude, and c * sum_k w (FP64 row sums of the
// FP32 weights) is added back in the epilogue.  Derivative and
// hyperviscosity weights annihilate constants, so the added-back term is tiny
// and the cancellation that limits FP32 stencil sums mostly disappears.  The
// add-back uses the FP32 weights themselves (sum in FP64), not hi + lo, so the
// split's own rounding only ever multiplies the centred values.  The
// RK4 accumulation of h (base state and D register) is FP64; u, v, w and every
// stage state K are FP32.
//
// Per CTA (one tile x HPC halves): weights are scattered into the B operand
// (hi/lo) in shared memory; the A operand is filled 32 rows (one chunk) at a
// time by all threads (coalesced 512-byte row reads per half, TF32 split in
// registers); one thread issues the MMAs of the chunk and commits them to an
// mbarrier that every thread waits on (bounded) before the next chunk reuses
// the buffer.  The epilogue reads the accumulator with tcgen05.ld (TMEM lane =
// mf), exchanges the 4 fields of a member between 4 adjacent lanes, evaluates
// the pointwise part of eval_RHS_swe (rk4_rbffd_swe.c:320-353) and applies the
// RK_substep combine (:30-72) for its own (node, member, field).
#pragma once

#include "stage_kernel.cuh"
#include "tcgen05.cuh"

namespace swe {

template <int T>
struct EnsTile {
    static constexpr int kNodes = T;
    static constexpr int kN = 4 * T;                       // MMA N
    static constexpr int kKmax = (T == 4) ? 128 : 176;     // unique rows per tile, multiple of 8
    static constexpr int kChunk = 32;                      // A rows per chunk
    static constexpr int kABytes = 128 * kChunk * 4;       // one half, one of hi/lo: 16 KB
    static constexpr int kBBytes = kN * kKmax * 4;         // one of hi/lo
    static constexpr int kSboA = (kChunk / 4) * 128;       // bytes between 8-row groups of A
    static constexpr int kSboB = (kKmax / 4) * 128;
};

struct EnsArgs {
    int n;                 // nodes
    int ntiles;
    int mf;                // 4 * members (row length of the state arrays)
    const int* rows;       // [ntiles][kKmax] unique neighbour rows of each tile
    const int* kcount;     // [ntiles] number of unique rows
    const uint8_t* local;  // [ntiles][T][32] local row of (node t, slot j); 255 = unused
    const float4* W;       // [n][32] (Dx, Dy, Dz, L), slots >= nnbr zero
    const float4* PT;      // [n][5] pointwise record (20 floats)
    const float* Kin;      // gather source [n][mf]
    float* H32;            // [n][mf]  u, v, w base state (+ FP32 mirror of h)
    double* Hh;            // [n][members] h base state, FP64
    float* D32;            // [n][mf]  RK accumulator for u, v, w
    double* Dh;            // [n][members] RK accumulator for h, FP64
    float* Kout;           // [n][mf]  next stage state
    float* F;              // [n][mf]  eval-only output
    float gh0;
    double c;              // dt/2, dt/2, dt for stages 0-2
    double dt6;            // dt/6
    int* err;              // device error word (bounded-wait timeouts)
};

constexpr uint32_t kEnsWaitTries = 1u << 22;

template <int T, int HPC, int MODE>
__global__ void __launch_bounds__(128 * HPC, 1) ens_stage_kernel(const EnsArgs a) {
    using G = EnsTile<T>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* A_base = smem;                                      // [HPC][hi, lo][16 KB]
    unsigned char* B_hi = smem + HPC * 2 * G::kABytes;
    unsigned char* B_lo = B_hi + G::kBBytes;
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base_s;
    __shared__ int rows_s[G::kKmax];
    __shared__ double rowsum_s[T][4];

    const int tid = threadIdx.x;
    const int hh = tid >> 7;                 // half within the CTA
    const int m = tid & 127;                 // row within the half (TMEM lane)
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int tile = blockIdx.x;
    const int half = blockIdx.y * HPC + hh;
    const int col0 = half * 128;             // first mf of this half
    constexpr int kCols = (G::kN * HPC <= 32) ? 32 : 64;

    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_s, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_mbar_init();
    }
    const int K_u = a.kcount[tile];
    for (int k = tid; k < G::kKmax; k += 128 * HPC) rows_s[k] = a.rows[(long)tile * G::kKmax + k];

    // ---- B operand: zero, then scatter the tile's weights as TF32 hi/lo -------------
    {
        uint4* z = reinterpret_cast<uint4*>(B_hi);
        for (int t = tid; t < 2 * G::kBBytes / 16; t += 128 * HPC) z[t] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();
    // one warp per node t: lane j scatters slot j and the warp sums its weights
    for (int e = tid; e < T * 32; e += 128 * HPC) {
        const int t = e >> 5, j = e & 31;
        const long node = (long)tile * T + t;
        const int k = a.local[((long)tile * T + t) * 32 + j];
        double part[4] = {0.0, 0.0, 0.0, 0.0};
        if (node < a.n && k != 255) {
            const float4 w4 = __ldg(a.W + node * 32 + j);
            const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int op = 0; op < 4; ++op) {
                const int nrow = 4 * t + op;
                const uint32_t off = (nrow >> 3) * G::kSboB + (k >> 2) * 128 + (nrow & 7) * 16 + (k & 3) * 4;
                float hi, lo;
                tc::tf32_split(w[op], hi, lo);
                *reinterpret_cast<float*>(B_hi + off) = hi;
                *reinterpret_cast<float*>(B_lo + off) = lo;
                part[op] = (double)w[op];
            }
        }
#pragma unroll
        for (int op = 0; op < 4; ++op) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part[op] += __shfl_xor_sync(0xffffffffu, part[op], o);
        }
        if (j == 0) {
#pragma unroll
            for (int op = 0; op < 4; ++op) rowsum_s[t][op] = part[op];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    // ---- K loop: gather 32 unique rows, split, MMA ------------------------------------
    unsigned char* A_hi = A_base + hh * 2 * G::kABytes;
    unsigned char* A_lo = A_hi + G::kABytes;
    const int nchunks = (K_u + G::kChunk - 1) / G::kChunk;
    const int ksteps_total = (K_u + 7) / 8;
    const uint32_t idesc = tc::idesc_tf32(128, G::kN);
    uint32_t phase = 0;
    bool ok = true;
    // centre: the state of the tile's first node, for this thread's mf row
    const float cref = __ldg(a.Kin + (long)tile * T * a.mf + col0 + m);
    for (int c = 0; c < nchunks && ok; ++c) {
#pragma unroll 2
        for (int g4 = 0; g4 < G::kChunk / 4; ++g4) {
            float x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int k = c * G::kChunk + g4 * 4 + r;
                x[r] = (k < K_u) ? __ldg(a.Kin + (long)rows_s[k] * a.mf + col0 + m) - cref : 0.f;
            }
            float4 hi, lo;
            tc::tf32_split(x[0], hi.x, lo.x);
            tc::tf32_split(x[1], hi.y, lo.y);
            tc::tf32_split(x[2], hi.z, lo.z);
            tc::tf32_split(x[3], hi.w, lo.w);
            const uint32_t off = (m >> 3) * G::kSboA + g4 * 128 + (m & 7) * 16;
            *reinterpret_cast<float4*>(A_hi + off) = hi;
            *reinterpret_cast<float4*>(A_lo + off) = lo;
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const int s0 = c * (G::kChunk / 8);
            const int s1 = min(ksteps_total, s0 + G::kChunk / 8);
            for (int ks = s0; ks < s1; ++ks) {
                const int q = ks - s0;
                const uint64_t bh = tc::smem_desc(tc::smem_u32(B_hi + ks * 256), 128, G::kSboB);
                const uint64_t bl = tc::smem_desc(tc::smem_u32(B_lo + ks * 256), 128, G::kSboB);
#pragma unroll
                for (int h2 = 0; h2 < HPC; ++h2) {
                    unsigned char* ah = A_base + h2 * 2 * G::kABytes;
                    const uint64_t dah = tc::smem_desc(tc::smem_u32(ah + q * 256), 128, G::kSboA);
                    const uint64_t dal = tc::smem_desc(tc::smem_u32(ah + G::kABytes + q * 256), 128, G::kSboA);
                    const uint32_t d = tmem + h2 * G::kN;
                    tc::mma_tf32(d, dah, bh, idesc, ks > 0 ? 1u : 0u);
                    tc::mma_tf32(d, dah, bl, idesc, 1u);
                    tc::mma_tf32(d, dal, bh, idesc, 1u);
                }
            }
            tc::mma_commit(&mbar);
        }
        __syncwarp();
        const bool done = tc::mbar_wait_bounded(&mbar, phase, kEnsWaitTries);
        // one verdict for the whole CTA, so that no thread leaves the loop alone
        ok = __syncthreads_and(done) != 0;
        if (!ok && tid == 0) atomicExch(a.err, 1);
        phase ^= 1;
        tc::fence_after_sync();
    }

    // ---- epilogue ---------------------------------------------------------------------------
    if (ok) {
        float acc[G::kN];
        const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + hh * G::kN;
#pragma unroll
        for (int c16 = 0; c16 < G::kN / 16; ++c16) {
            float v[16];
            tc::tmem_ld16(taddr + c16 * 16, v);
            tc::tmem_wait_ld();
#pragma unroll
            for (int t = 0; t < 16; ++t) acc[c16 * 16 + t] = v[t];
        }
        // add back the centre: D += c * sum_k B
#pragma unroll
        for (int t = 0; t < T; ++t)
#pragma unroll
            for (int op = 0; op < 4; ++op)
                acc[4 * t + op] = (float)((double)acc[4 * t + op] + (double)cref * rowsum_s[t][op]);
        const int fld = m & 3;
        const int mf = col0 + m;
        const int member = mf >> 2;
        const int members = a.mf >> 2;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            const long node = (long)tile * T + t;
            if (node >= a.n) break;                       // uniform across the CTA
            float S[16];
#pragma unroll
            for (int op = 0; op < 4; ++op)
#pragma unroll
                for (int f2 = 0; f2 < 4; ++f2)
                    S[op * 4 + f2] = __shfl_sync(0xffffffffu, acc[4 * t + op], (lane & ~3) | f2);
            const float4 q4 = __ldg(reinterpret_cast<const float4*>(a.Kin + node * a.mf + (mf & ~3)));
            const float q[4] = {q4.x, q4.y, q4.z, q4.w};
            float pt[kPointStride];
#pragma unroll
            for (int p = 0; p < 5; ++p) {
                const float4 v = __ldg(a.PT + node * 5 + p);
                pt[4 * p] = v.x; pt[4 * p + 1] = v.y; pt[4 * p + 2] = v.z; pt[4 * p + 3] = v.w;
            }
            float F[4];
            pointwise_rhs<float>(S, q, pt, a.gh0, F);
            const float f = fld == 0 ? F[0] : fld == 1 ? F[1] : fld == 2 ? F[2] : F[3];
            const long e = node * a.mf + mf;
            const long eh = node * members + member;
            if (MODE == kEvalOnly) {
                a.F[e] = f;
            } else if (fld < 3) {
                const float c32 = (float)a.c;
                if (MODE == kStage0) {
                    a.D32[e] = f;
                    a.Kout[e] = __fadd_rn(q[fld], __fmul_rn(c32, f));
                } else if (MODE == kStage1 || MODE == kStage2) {
                    a.D32[e] = __fadd_rn(a.D32[e], __fmul_rn(2.f, f));
                    a.Kout[e] = __fadd_rn(a.H32[e], __fmul_rn(c32, f));
                } else {
                    const float d = __fadd_rn(a.D32[e], f);
                    a.H32[e] = __double2float_rn((double)a.H32[e] + a.dt6 * (double)d);
                }
            } else {
                const double fd = (double)f;
                if (MODE == kStage0) {
                    a.Dh[eh] = fd;
                    a.Kout[e] = __double2float_rn(a.Hh[eh] + a.c * fd);
                } else if (MODE == kStage1 || MODE == kStage2) {
                    a.Dh[eh] = a.Dh[eh] + 2.0 * fd;
                    a.Kout[e] = __double2float_rn(a.Hh[eh] + a.c * fd);
                } else {
                    const double d = a.Dh[eh] + fd;
                    const double h = a.Hh[eh] + a.dt6 * d;
                    a.Hh[eh] = h;
                    a.H32[e] = __double2float_rn(h);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kCols);
    }
}

}  // namespace swe
