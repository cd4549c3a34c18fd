// Batched-ensemble RK4 stage kernel on tcgen05 tensor cores (3xTF32).
//
// B ensemble members share one grid.  The state is stored member-innermost,
// [node][mf] with mf = 4*member + field, so a neighbour's state for all members
// is one contiguous row of 4B floats.  Nodes are grouped into tiles of 32
// consecutive nodes of a space-filling-curve order (compact patches: about 126
// unique neighbour rows per tile on the icosahedral grids).  For one tile the
// stencil products of a block of MPC members are one dense contraction
//
//     D[32*op + t][mf] = sum_k  W_op(node t, row_k) * (X[row_k][mf] - c[mf])
//
// M = 128 (4 operators Dx, Dy, Dz, L x 32 nodes), N = 4*MPC member-fields,
// K = the tile's unique neighbour rows (W is zero where row_k is not in node
// t's stencil).  Each unique row is gathered once per tile instead of once per
// stencil slot.
//
// Precision (3xTF32): both operands are split x ~ hi + lo, each rounded to
// nearest TF32 (|x - hi - lo| <= 2^-22 |x|), and D = A_hi B_hi + A_hi B_lo +
// A_lo B_hi accumulates in FP32 in tensor memory.  The gathered states are
// centred on the state of one node of the tile (c[mf]) before the split;
// c * sum_k W (row sums of the FP32 weights, summed in FP64) is added back in
// the epilogue.  Derivative and hyperviscosity weights annihilate constants,
// so the added-back term is small and the cancellation that limits FP32
// stencil sums mostly disappears.  The RK4 accumulation of h (base state and
// D register) is FP64; u, v, w and every stage state K are FP32.
//
// Persistent, warp-specialised CTA (one per SM; it owns all of tensor memory):
//   * converter warps (MPC/8): for each 16-row chunk of K they gather the rows
//     (16-byte loads, one chunk ahead), centre and split them into the B
//     operand, and build the matching A chunk from the tile's weight entries
//     sorted by chunk (zero, then scatter hi/lo); a ring of kEnsStages slots
//     hands chunks to
//   * the MMA warp: one thread issues 2 k-steps x 3 MMAs (128 x N x 8) per
//     chunk into one of two TMEM accumulators and commits each chunk to the
//     slot's "empty" barrier and each tile to the accumulator's "full" barrier;
//   * 8 epilogue warps (two per TMEM lane quarter): tcgen05.ld the accumulator
//     32 columns at a time, transpose (op, node) rows to (node, member) sets
//     through shared memory, add the centre back, evaluate the pointwise part
//     of eval_RHS_swe (rk4_rbffd_swe.c:320-353) and apply the RK_substep
//     combine (:30-72) for one (node, member) per thread, while the MMA warp
//     already fills the other accumulator.
// Every mbarrier wait is bounded; a timeout sets an error word and a shared
// abort flag that makes every role leave its loop.
#pragma once

#include "stage_kernel.cuh"
#include "tcgen05.cuh"

namespace swe {

constexpr int kEnsTileNodes = 32;   // nodes per tile (M = 4 * 32)
constexpr int kEnsKc = 16;          // neighbour rows per pipeline chunk
constexpr int kEnsStages = 3;       // ring slots
constexpr int kEnsEpiWarps = 8;
constexpr int kEnsMaxEntPerChunk = kEnsKc * kEnsTileNodes;   // every (row, node) pair once
constexpr uint32_t kEnsWaitTries = 1u << 22;

template <int MPC>
struct EnsCfg {
    static constexpr int kN = 4 * MPC;                     // MMA N: member-fields per CTA
    static constexpr int kConvWarps = MPC / 8;             // (kEnsKc / 4) * MPC converter threads
    static constexpr int kConvThreads = 32 * kConvWarps;
    static constexpr int kMmaWarp = kConvWarps;
    static constexpr int kEpiWarp0 = kConvWarps + 1;
    static constexpr int kThreads = 32 * (kConvWarps + 1 + kEnsEpiWarps);
    static constexpr int kEntPerThread = kEnsMaxEntPerChunk / kConvThreads;
    static constexpr int kSboA = (kEnsKc / 4) * 128;       // A: 8-row groups of 16-byte core rows
    static constexpr int kSboB = (kEnsKc / 4) * 128 + 16;  // B: odd 16-byte stride, conflict-free stores
    static constexpr int kAHalf = (128 / 8) * kSboA;       // one of hi / lo
    static constexpr int kBHalf = (kN / 8) * kSboB;
    static constexpr int kStageBytes = ((2 * kAHalf + 2 * kBHalf) + 127) / 128 * 128;
    static constexpr int kXchStride = 36;                  // floats per (op, node) row; 9 x 16 B
    static constexpr int kXchGroupFloats = 4 * kEnsTileNodes * kXchStride;
    static constexpr int kSmem = kEnsStages * kStageBytes + 2 * kXchGroupFloats * 4;
    static constexpr int kTmemCols = (2 * kN <= 256) ? 256 : 512;
    static_assert(kEnsMaxEntPerChunk % kConvThreads == 0, "entries per thread");
    static_assert(kN % 64 == 0 || kN == 32, "epilogue column chunks");
};

struct EnsArgs {
    int n;                 // nodes
    int ntiles;
    int units;             // ntiles * (members / MPC)
    int members;
    int mf;                // 4 * members (row length of the state arrays)
    const int* row_off;    // [ntiles + 1] offsets into rows, multiples of kEnsKc
    const int* rows;       // unique neighbour rows of each tile, ascending; -1 pads
    const int* ent_off;    // [rows / kEnsKc + 1] weight entries of each chunk
    const int* ent_tk;     // entry: node t | (row within chunk) << 8
    const float4* ent_w;   // entry: (Dx, Dy, Dz, L) weight
    const int* centre;     // [ntiles] node whose state centres the tile
    const float4* PT;      // [n][5] pointwise record (20 floats)
    const float4* RS;      // [n] row sums of the four operators
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

namespace ens {

__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// Named barrier with an AND reduction: every participant gets the same verdict.
__device__ __forceinline__ bool named_and(int id, int nthreads, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(b)) : "memory");
}
__device__ __forceinline__ float4 ldg_f4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// Bounded wait that also gives up as soon as another role has aborted.
__device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, volatile int* abort_s, int* err, int code) {
    for (uint32_t t = 0; t < kEnsWaitTries; ++t) {
        if (tc::mbar_try_wait(b, parity)) return true;
        if (*abort_s) return false;
    }
    *abort_s = 1;
    atomicExch(err, code);
    return false;
}

// Position of a converter in its CTA's sequence of (work unit, chunk) steps.
struct Pos {
    int u, gc, gc_end;     // unit, global chunk id, end of the unit's chunks
    bool valid;
};

__device__ __forceinline__ Pos first_pos(const EnsArgs& a, int halves) {
    Pos p;
    p.u = blockIdx.x;
    p.valid = p.u < a.units;
    if (p.valid) {
        const int tile = p.u / halves;
        p.gc = __ldg(a.row_off + tile) / kEnsKc;
        p.gc_end = __ldg(a.row_off + tile + 1) / kEnsKc;
    }
    return p;
}

__device__ __forceinline__ Pos next_pos(Pos p, const EnsArgs& a, int halves) {
    if (!p.valid) return p;
    if (++p.gc < p.gc_end) return p;
    p.u += gridDim.x;
    p.valid = p.u < a.units;
    if (p.valid) {
        const int tile = p.u / halves;
        p.gc = __ldg(a.row_off + tile) / kEnsKc;
        p.gc_end = __ldg(a.row_off + tile + 1) / kEnsKc;
    }
    return p;
}

}  // namespace ens

template <int MPC, int MODE>
__global__ void __launch_bounds__(EnsCfg<MPC>::kThreads, 1) ens_stage_kernel(const EnsArgs a) {
    using C = EnsCfg<MPC>;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full_bar[kEnsStages], empty_bar[kEnsStages];
    __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], fin_bar;
    __shared__ uint32_t tmem_s;
    __shared__ int abort_s;
    volatile int* abort_v = &abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int halves = a.members / MPC;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kEnsStages; ++s) {
            tc::mbar_init(&full_bar[s], C::kConvWarps);
            tc::mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&accf_bar[b], 1);
            tc::mbar_init(&acce_bar[b], kEnsEpiWarps);
        }
        tc::mbar_init(&fin_bar, 1);
        abort_s = 0;
        tc::fence_mbar_init();
    }
    if (warp == C::kMmaWarp) {
        tc::tmem_alloc(&tmem_s, C::kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_s;

    if (warp < C::kConvWarps) {
        // =============================== converters ===============================
        const int ct = threadIdx.x;              // 0 .. 4*MPC-1
        const int quad = ct % MPC;               // member within the CTA's block
        const int kg = ct / MPC;                 // rows 4kg .. 4kg+3 of each chunk
        ens::Pos p0 = ens::first_pos(a, halves);
        ens::Pos p1 = ens::next_pos(p0, a, halves);
        // stage "x" (current): rows loaded; stage "i" (next): row indices loaded
        int4 idx0 = make_int4(-1, -1, -1, -1), idx1 = make_int4(-1, -1, -1, -1);
        int e00 = 0, e01 = 0, e10 = 0, e11 = 0;
        if (p0.valid) {
            idx0 = __ldg(reinterpret_cast<const int4*>(a.rows + p0.gc * kEnsKc + 4 * kg));
            e00 = __ldg(a.ent_off + p0.gc);
            e01 = __ldg(a.ent_off + p0.gc + 1);
        }
        if (p1.valid) {
            idx1 = __ldg(reinterpret_cast<const int4*>(a.rows + p1.gc * kEnsKc + 4 * kg));
            e10 = __ldg(a.ent_off + p1.gc);
            e11 = __ldg(a.ent_off + p1.gc + 1);
        }
        auto load_rows = [&](const ens::Pos& p, const int4& id, float4 (&x)[4]) {
            const long col = (long)(p.u % halves) * C::kN + 4 * quad;
            const int r[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                x[i] = r[i] >= 0 ? ens::ldg_f4(a.Kin + (long)r[i] * a.mf + col) : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        auto load_ent = [&](int e0, int e1, int (&tk)[C::kEntPerThread], float4 (&w)[C::kEntPerThread]) {
#pragma unroll
            for (int q = 0; q < C::kEntPerThread; ++q) {
                const int e = e0 + ct + q * C::kConvThreads;
                tk[q] = e < e1 ? __ldg(a.ent_tk + e) : -1;
                w[q] = e < e1 ? __ldg(a.ent_w + e) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        auto load_centre = [&](const ens::Pos& p) {
            const int tile = p.u / halves;
            const long col = (long)(p.u % halves) * C::kN + 4 * quad;
            return ens::ldg_f4(a.Kin + (long)__ldg(a.centre + tile) * a.mf + col);
        };
        float4 x0[4], x1[4];
        int tk0[C::kEntPerThread], tk1[C::kEntPerThread];
        float4 w0[C::kEntPerThread], w1[C::kEntPerThread];
        float4 cen0 = make_float4(0.f, 0.f, 0.f, 0.f), cen1 = cen0;
        if (p0.valid) {
            load_rows(p0, idx0, x0);
            load_ent(e00, e01, tk0, w0);
            cen0 = load_centre(p0);
        }
        int g = 0;
        while (p0.valid) {
            // look ahead: rows and entries of p1, indices of p2
            ens::Pos p2 = ens::next_pos(p1, a, halves);
            int4 idx2 = make_int4(-1, -1, -1, -1);
            int e20 = 0, e21 = 0;
            if (p1.valid) {
                load_rows(p1, idx1, x1);
                load_ent(e10, e11, tk1, w1);
                cen1 = (p1.u != p0.u) ? load_centre(p1) : cen0;
            }
            if (p2.valid) {
                idx2 = __ldg(reinterpret_cast<const int4*>(a.rows + p2.gc * kEnsKc + 4 * kg));
                e20 = __ldg(a.ent_off + p2.gc);
                e21 = __ldg(a.ent_off + p2.gc + 1);
            }
            // ---- fill ring slot s with chunk p0 ----
            const int s = g % kEnsStages;
            const bool got = ens::wait(&empty_bar[s], ((g / kEnsStages) & 1) ^ 1, abort_v, a.err, 3);
            unsigned char* slot = smem + s * C::kStageBytes;
            unsigned char* A_hi = slot;
            unsigned char* A_lo = slot + C::kAHalf;
            unsigned char* B_hi = slot + 2 * C::kAHalf;
            unsigned char* B_lo = B_hi + C::kBHalf;
            if (got) {
                uint4* z = reinterpret_cast<uint4*>(A_hi);
                for (int q = ct; q < 2 * C::kAHalf / 16; q += C::kConvThreads) z[q] = make_uint4(0, 0, 0, 0);
            }
            // zeroing done by every converter before any scatter; one verdict for all of them
            if (!ens::named_and(1, C::kConvThreads, got && !*abort_v)) break;
#pragma unroll
            for (int q = 0; q < C::kEntPerThread; ++q) {
                if (tk0[q] < 0) continue;
                const int t = tk0[q] & 0xff, kk = tk0[q] >> 8;
                const float w[4] = {w0[q].x, w0[q].y, w0[q].z, w0[q].w};
#pragma unroll
                for (int op = 0; op < 4; ++op) {
                    const int r = 32 * op + t;
                    const uint32_t off = (r >> 3) * C::kSboA + (kk >> 2) * 128 + (r & 7) * 16 + (kk & 3) * 4;
                    float hi, lo;
                    tc::tf32_split(w[op], hi, lo);
                    *reinterpret_cast<float*>(A_hi + off) = hi;
                    *reinterpret_cast<float*>(A_lo + off) = lo;
                }
            }
            {
                // B: 4 rows x 4 member-fields; each member-field's 4 rows are one 16-byte core row
                const float xv[4][4] = {{x0[0].x, x0[0].y, x0[0].z, x0[0].w},
                                        {x0[1].x, x0[1].y, x0[1].z, x0[1].w},
                                        {x0[2].x, x0[2].y, x0[2].z, x0[2].w},
                                        {x0[3].x, x0[3].y, x0[3].z, x0[3].w}};
                const int4 idr = idx0;
                const bool live[4] = {idr.x >= 0, idr.y >= 0, idr.z >= 0, idr.w >= 0};
                const float cv[4] = {cen0.x, cen0.y, cen0.z, cen0.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int nrow = 4 * quad + j;
                    float4 hi, lo;
                    float y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) y[i] = live[i] ? xv[i][j] - cv[j] : 0.f;
                    tc::tf32_split(y[0], hi.x, lo.x);
                    tc::tf32_split(y[1], hi.y, lo.y);
                    tc::tf32_split(y[2], hi.z, lo.z);
                    tc::tf32_split(y[3], hi.w, lo.w);
                    const uint32_t off = (nrow >> 3) * C::kSboB + kg * 128 + (nrow & 7) * 16;
                    *reinterpret_cast<float4*>(B_hi + off) = hi;
                    *reinterpret_cast<float4*>(B_lo + off) = lo;
                }
            }
            tc::fence_async_smem();
            __syncwarp();
            if (lane == 0) ens::mbar_arrive(&full_bar[s]);
            ++g;
            // rotate
            p0 = p1; p1 = p2;
            idx0 = idx1; idx1 = idx2;
            e10 = e20; e11 = e21;
#pragma unroll
            for (int i = 0; i < 4; ++i) x0[i] = x1[i];
#pragma unroll
            for (int q = 0; q < C::kEntPerThread; ++q) { tk0[q] = tk1[q]; w0[q] = w1[q]; }
            cen0 = cen1;
        }
    } else if (warp == C::kMmaWarp) {
        // =============================== MMA issuer ===============================
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_tf32(128, C::kN);
            int g = 0, it = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < a.units && ok; u += gridDim.x, ++it) {
                const int ab = it & 1;
                if (!ens::wait(&acce_bar[ab], ((it >> 1) & 1) ^ 1, abort_v, a.err, 4)) { ok = false; break; }
                tc::fence_after_sync();
                const int tile = u / halves;
                const int gc0 = __ldg(a.row_off + tile) / kEnsKc, gc1 = __ldg(a.row_off + tile + 1) / kEnsKc;
                const uint32_t d = tmem + ab * C::kN;
                for (int gc = gc0; gc < gc1; ++gc, ++g) {
                    const int s = g % kEnsStages;
                    if (!ens::wait(&full_bar[s], (g / kEnsStages) & 1, abort_v, a.err, 5)) { ok = false; break; }
                    tc::fence_after_sync();
                    unsigned char* slot = smem + s * C::kStageBytes;
                    const uint32_t a_hi = tc::smem_u32(slot), a_lo = a_hi + C::kAHalf;
                    const uint32_t b_hi = a_hi + 2 * C::kAHalf, b_lo = b_hi + C::kBHalf;
#pragma unroll
                    for (int ks = 0; ks < kEnsKc / 8; ++ks) {
                        const uint64_t dah = tc::smem_desc(a_hi + ks * 256, 128, C::kSboA);
                        const uint64_t dal = tc::smem_desc(a_lo + ks * 256, 128, C::kSboA);
                        const uint64_t dbh = tc::smem_desc(b_hi + ks * 256, 128, C::kSboB);
                        const uint64_t dbl = tc::smem_desc(b_lo + ks * 256, 128, C::kSboB);
                        tc::mma_tf32(d, dah, dbh, idesc, (gc > gc0 || ks > 0) ? 1u : 0u);
                        tc::mma_tf32(d, dah, dbl, idesc, 1u);
                        tc::mma_tf32(d, dal, dbh, idesc, 1u);
                    }
                    tc::mma_commit(&empty_bar[s]);
                }
                if (!ok) break;
                tc::mma_commit(&accf_bar[ab]);
            }
            // every MMA this thread issued has completed before tensor memory is freed
            // (this wait ignores the abort flag: it only ends when they have)
            tc::mma_commit(&fin_bar);
            if (!tc::mbar_wait_bounded(&fin_bar, 0, kEnsWaitTries)) {
                *abort_v = 1;
                atomicExch(a.err, 6);
            }
        }
        __syncwarp();
    } else {
        // =============================== epilogue ===============================
        const int e = warp - C::kEpiWarp0;       // 0..7
        const int grp = e >> 2;                  // column chunks alternate between the two groups
        const int op = warp & 3;                 // TMEM lane quarter = operator
        const int gt = threadIdx.x - 32 * (C::kEpiWarp0 + 4 * grp);   // 0..127 within the group
        float* xch = reinterpret_cast<float*>(smem + kEnsStages * C::kStageBytes) + grp * C::kXchGroupFloats;
        const int members = a.members;
        const float c32 = (float)a.c;
        int it = 0;
        for (int u = blockIdx.x; u < a.units; u += gridDim.x, ++it) {
            const int ab = it & 1;
            const bool got = ens::wait(&accf_bar[ab], (it >> 1) & 1, abort_v, a.err, 7);
            if (!ens::named_and(2 + grp, 128, got && !*abort_v)) break;
            tc::fence_after_sync();
            const int tile = u / halves;
            const int col0 = (u % halves) * C::kN;
            const long cnode = __ldg(a.centre + tile);
            for (int ch = grp; ch < C::kN / 32; ch += 2) {
                float v[32];
                {
                    const uint32_t taddr = tmem + ((uint32_t)(32 * op) << 16) + ab * C::kN + ch * 32;
                    float v0[16], v1[16];
                    tc::tmem_ld16(taddr, v0);
                    tc::tmem_ld16(taddr + 16, v1);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 16; ++q) { v[q] = v0[q]; v[16 + q] = v1[q]; }
                }
                float* row = xch + (op * 32 + lane) * C::kXchStride;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    *reinterpret_cast<float4*>(row + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                ens::named_sync(2 + grp, 128);
#pragma unroll
                for (int pi = 0; pi < 2; ++pi) {
                    const int pr = gt + 128 * pi;
                    const int t = pr >> 3, bm = pr & 7;
                    const long node = (long)tile * kEnsTileNodes + t;
                    if (node >= a.n) continue;
                    const int mfb = col0 + ch * 32 + 4 * bm;      // first mf of this member
                    const int member = mfb >> 2;
                    float S[16];
#pragma unroll
                    for (int o = 0; o < 4; ++o) {
                        const float4 sv = *reinterpret_cast<const float4*>(xch + (o * 32 + t) * C::kXchStride + 4 * bm);
                        S[4 * o] = sv.x; S[4 * o + 1] = sv.y; S[4 * o + 2] = sv.z; S[4 * o + 3] = sv.w;
                    }
                    const float4 cen = ens::ldg_f4(a.Kin + cnode * a.mf + mfb);
                    const float4 rs4 = __ldg(a.RS + node);
                    const float cf[4] = {cen.x, cen.y, cen.z, cen.w};
                    const float rs[4] = {rs4.x, rs4.y, rs4.z, rs4.w};
#pragma unroll
                    for (int o = 0; o < 4; ++o)
#pragma unroll
                        for (int f = 0; f < 4; ++f) S[4 * o + f] = fmaf(cf[f], rs[o], S[4 * o + f]);
                    const float4 q4 = ens::ldg_f4(a.Kin + node * a.mf + mfb);
                    const float q[4] = {q4.x, q4.y, q4.z, q4.w};
                    float pt[kPointStride];
#pragma unroll
                    for (int pp = 0; pp < 5; ++pp) {
                        const float4 pv = __ldg(a.PT + node * 5 + pp);
                        pt[4 * pp] = pv.x; pt[4 * pp + 1] = pv.y; pt[4 * pp + 2] = pv.z; pt[4 * pp + 3] = pv.w;
                    }
                    float F[4];
                    pointwise_rhs<float>(S, q, pt, a.gh0, F);
                    const long e4 = node * a.mf + mfb;
                    const long eh = node * members + member;
                    if (MODE == kEvalOnly) {
                        *reinterpret_cast<float4*>(a.F + e4) = make_float4(F[0], F[1], F[2], F[3]);
                    } else if (MODE == kStage0) {
                        // K = H + c F (q is the base state here); D = F
                        const double fh = (double)F[3];
                        const double hb = a.Hh[eh];
                        *reinterpret_cast<float4*>(a.D32 + e4) = make_float4(F[0], F[1], F[2], 0.f);
                        a.Dh[eh] = fh;
                        *reinterpret_cast<float4*>(a.Kout + e4) =
                            make_float4(__fadd_rn(q[0], __fmul_rn(c32, F[0])), __fadd_rn(q[1], __fmul_rn(c32, F[1])),
                                        __fadd_rn(q[2], __fmul_rn(c32, F[2])), __double2float_rn(hb + a.c * fh));
                    } else if (MODE == kStage1 || MODE == kStage2) {
                        const double fh = (double)F[3];
                        const double hb = a.Hh[eh];
                        const float4 h4 = *reinterpret_cast<const float4*>(a.H32 + e4);
                        const float4 d4 = *reinterpret_cast<const float4*>(a.D32 + e4);
                        *reinterpret_cast<float4*>(a.D32 + e4) =
                            make_float4(__fadd_rn(d4.x, __fmul_rn(2.f, F[0])), __fadd_rn(d4.y, __fmul_rn(2.f, F[1])),
                                        __fadd_rn(d4.z, __fmul_rn(2.f, F[2])), 0.f);
                        a.Dh[eh] = a.Dh[eh] + 2.0 * fh;
                        *reinterpret_cast<float4*>(a.Kout + e4) =
                            make_float4(__fadd_rn(h4.x, __fmul_rn(c32, F[0])), __fadd_rn(h4.y, __fmul_rn(c32, F[1])),
                                        __fadd_rn(h4.z, __fmul_rn(c32, F[2])), __double2float_rn(hb + a.c * fh));
                    } else {
                        const float4 h4 = *reinterpret_cast<const float4*>(a.H32 + e4);
                        const float4 d4 = *reinterpret_cast<const float4*>(a.D32 + e4);
                        const float du = __fadd_rn(d4.x, F[0]), dv = __fadd_rn(d4.y, F[1]), dw = __fadd_rn(d4.z, F[2]);
                        const double dh = a.Dh[eh] + (double)F[3];
                        const double h = a.Hh[eh] + a.dt6 * dh;
                        a.Hh[eh] = h;
                        *reinterpret_cast<float4*>(a.H32 + e4) =
                            make_float4(__double2float_rn((double)h4.x + a.dt6 * (double)du),
                                        __double2float_rn((double)h4.y + a.dt6 * (double)dv),
                                        __double2float_rn((double)h4.z + a.dt6 * (double)dw), __double2float_rn(h));
                    }
                }
                ens::named_sync(2 + grp, 128);
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) ens::mbar_arrive(&acce_bar[ab]);
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (warp == C::kMmaWarp) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, C::kTmemCols);
    }
}

}  // namespace swe
