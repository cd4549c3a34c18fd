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
//     (16-byte loads issued one chunk ahead into a ping-pong register set),
//     centre and split them into the B operand, and write the matching A chunk
//     densely, one 16-byte core row (4 chunk rows of one operator and node) per
//     store, from a map of chunk rows to stencil slots; a ring of kEnsStages
//     slots hands chunks to
//   * the MMA warp: one thread issues 2 k-steps x 3 MMAs (128 x N x 8) per
//     chunk into one of two TMEM accumulators and commits each chunk to the
//     slot's "empty" barrier and each tile to the accumulator's "full" barrier;
//   * 8 epilogue warps (two per TMEM lane quarter): tcgen05.ld the accumulator
//     32 columns at a time, transpose (op, node) rows to (node, member) sets
//     through shared memory, add the centre back, evaluate the pointwise part
//     of eval_RHS_swe (rk4_rbffd_swe.c:320-353) and apply the RK_substep
//     combine (:30-72) for one (node, member) per thread, while the tensor
//     cores already fill the other accumulator.
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
constexpr uint32_t kEnsWaitTries = 1u << 22;

template <int MPC>
struct EnsCfg {
    static constexpr int kN = 4 * MPC;                     // MMA N: member-fields per CTA
    static constexpr int kConvWarps = MPC / 8;             // (kEnsKc / 4) * MPC converter threads
    static constexpr int kConvThreads = 32 * kConvWarps;
    static constexpr int kMmaWarp = kConvWarps;
    static constexpr int kEpiWarp0 = kConvWarps + 1;
    static constexpr int kThreads = 32 * (kConvWarps + 1 + kEnsEpiWarps);
    static constexpr int kOpp = 256 / kConvThreads;          // operator pairs per converter (A build)
    static constexpr int kSboA = (kEnsKc / 4) * 128;       // A: 8-row groups of 16-byte core rows
    static constexpr int kSboB = (kEnsKc / 4) * 128 + 16;  // B: odd 16-byte stride, conflict-free stores
    static constexpr int kAHalf = (128 / 8) * kSboA;       // one of hi / lo
    static constexpr int kBHalf = (kN / 8) * kSboB;
    static constexpr int kStageBytes = ((2 * kAHalf + 2 * kBHalf) + 127) / 128 * 128;
    static constexpr int kXchStride = 36;                  // floats per (op, node) row; 9 x 16 B
    static constexpr int kXchGroupFloats = 4 * kEnsTileNodes * kXchStride;
    static constexpr int kTbRs = kEnsTileNodes * kPointStride * 4;   // per-tile buffer: PT, row sums, centre
    static constexpr int kTbCen = kTbRs + kEnsTileNodes * 16;
    static constexpr int kTileBuf = (kTbCen + kN * 4 + 127) / 128 * 128;
    static constexpr int kSmem = kEnsStages * kStageBytes + 2 * kXchGroupFloats * 4 + 2 * kTileBuf;
    static constexpr int kTmemCols = (2 * kN <= 256) ? 256 : 512;
    static_assert(kOpp == 1 || kOpp == 2, "A build covers 32 nodes x 4 row groups x 2 operator pairs");
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
    const uint32_t* jmap;  // [chunk][row group][node t]: stencil slot of each of the 4 rows, 255 = none
    const float4* W;       // [n][32] (Dx, Dy, Dz, L) per stencil slot
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
using tc::mbar_arrive;
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

// Position of a converter in its CTA's sequence of (work unit, chunk) steps;
// the chunk range of the following unit is fetched one unit ahead.
struct Cursor {
    int u, ti;               // unit, and its position in this CTA's sequence of units
    int gc, gc0, gc_end;     // global chunk id, first and end chunk of the unit
    int nx_gc, nx_end;     // chunk range of unit u + gridDim.x
    bool valid;
};

__device__ __forceinline__ void unit_range(const EnsArgs& a, int u, int halves, int& g0, int& g1) {
    if (u < a.units) {
        const int tile = u / halves;
        g0 = __ldg(a.row_off + tile) / kEnsKc;
        g1 = __ldg(a.row_off + tile + 1) / kEnsKc;
    } else {
        g0 = g1 = 0;
    }
}

__device__ __forceinline__ Cursor first_cursor(const EnsArgs& a, int halves) {
    Cursor p;
    p.u = blockIdx.x;
    p.ti = 0;
    p.valid = p.u < a.units;
    unit_range(a, p.u, halves, p.gc, p.gc_end);
    p.gc0 = p.gc;
    unit_range(a, p.u + gridDim.x, halves, p.nx_gc, p.nx_end);
    return p;
}

__device__ __forceinline__ Cursor next_cursor(Cursor p, const EnsArgs& a, int halves) {
    if (!p.valid) return p;
    if (++p.gc < p.gc_end) return p;
    p.u += gridDim.x;
    ++p.ti;
    p.valid = p.u < a.units;
    p.gc = p.gc0 = p.nx_gc;
    p.gc_end = p.nx_end;
    unit_range(a, p.u + gridDim.x, halves, p.nx_gc, p.nx_end);
    return p;
}

// Indices of one step (row ids for the B operand, stencil slots for the A operand).
struct Fetch {
    int4 idx = make_int4(-1, -1, -1, -1);
    uint32_t jj = 0xffffffffu;
    int u = -1;
};

// Streamed operands of one epilogue chunk (two (node, member) pairs per thread).
struct EpiSet {
    float4 own[2], h32[2], d32[2];
    double hh[2], dh[2];
};

// Operands of one step held in registers.
template <int OPP>
struct ConvSet {
    float4 x[4];           // 4 gathered rows x 4 member-fields
    float4 cen;            // centre state of the same member-fields
    int live;              // bit i: row i is a real row
    float2 w[OPP][4];      // weights of the operator pairs for the 4 chunk rows
};

}  // namespace ens

template <int MPC, int MODE>
__global__ void __launch_bounds__(EnsCfg<MPC>::kThreads, 1) ens_stage_kernel(const EnsArgs a) {
    using C = EnsCfg<MPC>;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full_bar[kEnsStages], empty_bar[kEnsStages];
    __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], tile_bar[2], fin_bar;
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
            tc::mbar_init(&tile_bar[b], 1);
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
        // B operand: rows 4kg..4kg+3 of each chunk x member-fields 4quad..4quad+3
        const int quad = ct % MPC;
        const int kg = ct / MPC;
        // A operand: node t, rows 4akg..4akg+3 of each chunk, operator pairs opp0 .. opp0+kOpp-1
        const int at = ct & 31;
        const int akg = (ct >> 5) & 3;
        const int opp0 = (ct >> 7) * C::kOpp;
        ens::Cursor cur = ens::first_cursor(a, halves);
        ens::Fetch fx;                 // indices of the step after the current one
        ens::ConvSet<C::kOpp> sa, sb;  // operands of the current / next step (ping-pong)
        auto fetch_idx = [&](const ens::Cursor& p, ens::Fetch& f) {
            if (!p.valid) return;
            f.idx = __ldg(reinterpret_cast<const int4*>(a.rows + p.gc * kEnsKc + 4 * kg));
            f.jj = __ldg(a.jmap + (p.gc * 4 + akg) * 32 + at);
            f.u = p.u;
        };
        auto fetch_ops = [&](const ens::Cursor& p, const ens::Fetch& f, ens::ConvSet<C::kOpp>& o, const float4& cen_prev,
                             int u_prev) {
            if (!p.valid) return;
            const int tile = p.u / halves;
            const long col = (long)(p.u % halves) * C::kN + 4 * quad;
            const int r[4] = {f.idx.x, f.idx.y, f.idx.z, f.idx.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
                o.x[i] = r[i] >= 0 ? ens::ldg_f4(a.Kin + (long)r[i] * a.mf + col) : make_float4(0.f, 0.f, 0.f, 0.f);
            o.live = (r[0] >= 0 ? 1 : 0) | (r[1] >= 0 ? 2 : 0) | (r[2] >= 0 ? 4 : 0) | (r[3] >= 0 ? 8 : 0);
            o.cen = (p.u != u_prev) ? ens::ldg_f4(a.Kin + (long)__ldg(a.centre + tile) * a.mf + col) : cen_prev;
            const long node = (long)tile * kEnsTileNodes + at;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint32_t j = (f.jj >> (8 * i)) & 0xffu;
#pragma unroll
                for (int q = 0; q < C::kOpp; ++q)
                    o.w[q][i] = j != 0xffu ? __ldg(reinterpret_cast<const float2*>(a.W + node * 32 + j) + opp0 + q)
                                           : make_float2(0.f, 0.f);
            }
        };
        int g = 0;
        auto step = [&](ens::ConvSet<C::kOpp>& o, ens::ConvSet<C::kOpp>& nx, int u_cur) -> bool {
            // look ahead: operands of the next step, indices of the one after
            ens::Cursor nxt = ens::next_cursor(cur, a, halves);
            fetch_ops(nxt, fx, nx, o.cen, u_cur);
            ens::Cursor nxt2 = ens::next_cursor(nxt, a, halves);
            fetch_idx(nxt2, fx);
            const int s = g % kEnsStages;
            if (!ens::wait(&empty_bar[s], ((g / kEnsStages) & 1) ^ 1, abort_v, a.err, 3)) return false;
            unsigned char* slot = smem + s * C::kStageBytes;
            unsigned char* A_hi = slot;
            unsigned char* A_lo = slot + C::kAHalf;
            unsigned char* B_hi = slot + 2 * C::kAHalf;
            unsigned char* B_lo = B_hi + C::kBHalf;
            // A: one 16-byte core row (4 chunk rows) of (operator, node) per operator handled
#pragma unroll
            for (int q = 0; q < C::kOpp; ++q)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = 32 * (2 * (opp0 + q) + h) + at;
                    float4 hi, lo;
                    tc::tf32_split(h ? o.w[q][0].y : o.w[q][0].x, hi.x, lo.x);
                    tc::tf32_split(h ? o.w[q][1].y : o.w[q][1].x, hi.y, lo.y);
                    tc::tf32_split(h ? o.w[q][2].y : o.w[q][2].x, hi.z, lo.z);
                    tc::tf32_split(h ? o.w[q][3].y : o.w[q][3].x, hi.w, lo.w);
                    const uint32_t off = (r >> 3) * C::kSboA + akg * 128 + (r & 7) * 16;
                    *reinterpret_cast<float4*>(A_hi + off) = hi;
                    *reinterpret_cast<float4*>(A_lo + off) = lo;
                }
            // B: 4 rows x 4 member-fields; each member-field's 4 rows are one 16-byte core row
            {
                const float xv[4][4] = {{o.x[0].x, o.x[0].y, o.x[0].z, o.x[0].w},
                                        {o.x[1].x, o.x[1].y, o.x[1].z, o.x[1].w},
                                        {o.x[2].x, o.x[2].y, o.x[2].z, o.x[2].w},
                                        {o.x[3].x, o.x[3].y, o.x[3].z, o.x[3].w}};
                const float cv[4] = {o.cen.x, o.cen.y, o.cen.z, o.cen.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int nrow = 4 * quad + j;
                    float4 hi, lo;
                    float y[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) y[i] = ((o.live >> i) & 1) ? xv[i][j] - cv[j] : 0.f;
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
            cur = nxt;
            return true;
        };
        if (cur.valid) {
            ens::Fetch f0;
            fetch_idx(cur, f0);
            fetch_ops(cur, f0, sa, sa.cen, -1);
            fetch_idx(ens::next_cursor(cur, a, halves), fx);
        }
        // two steps per trip so that the ping-pong sets never need copying
        while (cur.valid) {
            int u = cur.u;
            if (!step(sa, sb, u)) break;
            if (!cur.valid) break;
            u = cur.u;
            if (!step(sb, sa, u)) break;
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
                    const uint32_t a_hi = tc::smem_u32(smem + s * C::kStageBytes), a_lo = a_hi + C::kAHalf;
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
        const int et = threadIdx.x - 32 * C::kEpiWarp0;   // 0..255
        const int grp = e >> 2;                  // column chunks alternate between the two groups
        const int op = warp & 3;                 // TMEM lane quarter = operator
        const int gt = et & 127;                 // thread within the group
        float* xch = reinterpret_cast<float*>(smem + kEnsStages * C::kStageBytes) + grp * C::kXchGroupFloats;
        unsigned char* tbuf = smem + kEnsStages * C::kStageBytes + 2 * C::kXchGroupFloats * 4;
        const int members = a.members;
        const float c32 = (float)a.c;
        constexpr bool kHD = MODE == kStage1 || MODE == kStage2 || MODE == kStage3;
        // per-tile pointwise records, row sums and centre row: bulk copies into tbuf[it & 1]
        auto issue_tile = [&](int u, int b) {
            const int tile = u / halves;
            const int nn = min(kEnsTileNodes, a.n - tile * kEnsTileNodes);
            unsigned char* tb = tbuf + b * C::kTileBuf;
            tc::mbar_arrive_expect_tx(&tile_bar[b], nn * (kPointStride * 4 + 16) + C::kN * 4);
            tc::bulk_g2s(tb, a.PT + (long)tile * kEnsTileNodes * 5, nn * kPointStride * 4, &tile_bar[b]);
            tc::bulk_g2s(tb + C::kTbRs, a.RS + (long)tile * kEnsTileNodes, nn * 16, &tile_bar[b]);
            tc::bulk_g2s(tb + C::kTbCen, a.Kin + (long)__ldg(a.centre + tile) * a.mf + (u % halves) * C::kN,
                         C::kN * 4, &tile_bar[b]);
        };
        // streamed per-(node, member) operands of one chunk for this thread's two pairs
        auto fetch = [&](int u, int ch, ens::EpiSet& o) {
            if (u >= a.units) return;
            const int tile = u / halves;
            const int col0 = (u % halves) * C::kN;
#pragma unroll
            for (int pi = 0; pi < 2; ++pi) {
                const int pr = gt + 128 * pi;
                const long node = (long)tile * kEnsTileNodes + (pr >> 3);
                if (node >= a.n) continue;
                const int mfb = col0 + ch * 32 + 4 * (pr & 7);
                const long e4 = node * a.mf + mfb;
                const long eh = node * members + (mfb >> 2);
                o.own[pi] = ens::ldg_f4(a.Kin + e4);
                if (MODE != kEvalOnly) o.hh[pi] = __ldg(a.Hh + eh);
                if (kHD) {
                    o.h32[pi] = ens::ldg_f4(a.H32 + e4);
                    o.d32[pi] = ens::ldg_f4(a.D32 + e4);
                    o.dh[pi] = __ldg(a.Dh + eh);
                }
            }
        };
        // one 32-column chunk: accumulator -> exchange -> (node, member) epilogue
        auto chunk = [&](int u, int it, int ch, const ens::EpiSet& o) {
            const int ab = it & 1;
            const int tile = u / halves;
            const int col0 = (u % halves) * C::kN;
            const float* tb = reinterpret_cast<const float*>(tbuf + (it & 1) * C::kTileBuf);
            {
                const uint32_t taddr = tmem + ((uint32_t)(32 * op) << 16) + ab * C::kN + ch * 32;
                float v0[16], v1[16];
                tc::tmem_ld16(taddr, v0);
                tc::tmem_ld16(taddr + 16, v1);
                tc::tmem_wait_ld();
                float* row = xch + (op * 32 + lane) * C::kXchStride;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    *reinterpret_cast<float4*>(row + 4 * q) = make_float4(v0[4 * q], v0[4 * q + 1], v0[4 * q + 2], v0[4 * q + 3]);
                    *reinterpret_cast<float4*>(row + 16 + 4 * q) =
                        make_float4(v1[4 * q], v1[4 * q + 1], v1[4 * q + 2], v1[4 * q + 3]);
                }
            }
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
                for (int o2 = 0; o2 < 4; ++o2) {
                    const float4 sv = *reinterpret_cast<const float4*>(xch + (o2 * 32 + t) * C::kXchStride + 4 * bm);
                    S[4 * o2] = sv.x; S[4 * o2 + 1] = sv.y; S[4 * o2 + 2] = sv.z; S[4 * o2 + 3] = sv.w;
                }
                const float4 cen = *reinterpret_cast<const float4*>(tb + C::kTbCen / 4 + (mfb - col0));
                const float4 rs4 = *reinterpret_cast<const float4*>(tb + C::kTbRs / 4 + 4 * t);
                const float cf[4] = {cen.x, cen.y, cen.z, cen.w};
                const float rs[4] = {rs4.x, rs4.y, rs4.z, rs4.w};
#pragma unroll
                for (int o2 = 0; o2 < 4; ++o2)
#pragma unroll
                    for (int f = 0; f < 4; ++f) S[4 * o2 + f] = fmaf(cf[f], rs[o2], S[4 * o2 + f]);
                const float q[4] = {o.own[pi].x, o.own[pi].y, o.own[pi].z, o.own[pi].w};
                float F[4];
                pointwise_rhs<float>(S, q, tb + t * kPointStride, a.gh0, F);
                const long e4 = node * a.mf + mfb;
                const long eh = node * members + member;
                if (MODE == kEvalOnly) {
                    *reinterpret_cast<float4*>(a.F + e4) = make_float4(F[0], F[1], F[2], F[3]);
                } else if (MODE == kStage0) {
                    // K = H + c F (q is the base state here); D = F
                    const double fh = (double)F[3];
                    *reinterpret_cast<float4*>(a.D32 + e4) = make_float4(F[0], F[1], F[2], 0.f);
                    a.Dh[eh] = fh;
                    *reinterpret_cast<float4*>(a.Kout + e4) =
                        make_float4(__fadd_rn(q[0], __fmul_rn(c32, F[0])), __fadd_rn(q[1], __fmul_rn(c32, F[1])),
                                    __fadd_rn(q[2], __fmul_rn(c32, F[2])), __double2float_rn(o.hh[pi] + a.c * fh));
                } else if (MODE == kStage1 || MODE == kStage2) {
                    const double fh = (double)F[3];
                    const float4 h4 = o.h32[pi], d4 = o.d32[pi];
                    *reinterpret_cast<float4*>(a.D32 + e4) =
                        make_float4(__fadd_rn(d4.x, __fmul_rn(2.f, F[0])), __fadd_rn(d4.y, __fmul_rn(2.f, F[1])),
                                    __fadd_rn(d4.z, __fmul_rn(2.f, F[2])), 0.f);
                    a.Dh[eh] = o.dh[pi] + 2.0 * fh;
                    *reinterpret_cast<float4*>(a.Kout + e4) =
                        make_float4(__fadd_rn(h4.x, __fmul_rn(c32, F[0])), __fadd_rn(h4.y, __fmul_rn(c32, F[1])),
                                    __fadd_rn(h4.z, __fmul_rn(c32, F[2])), __double2float_rn(o.hh[pi] + a.c * fh));
                } else {
                    const float4 h4 = o.h32[pi], d4 = o.d32[pi];
                    const float du = __fadd_rn(d4.x, F[0]), dv = __fadd_rn(d4.y, F[1]), dw = __fadd_rn(d4.z, F[2]);
                    const double dh = o.dh[pi] + (double)F[3];
                    const double h = o.hh[pi] + a.dt6 * dh;
                    a.Hh[eh] = h;
                    *reinterpret_cast<float4*>(a.H32 + e4) =
                        make_float4(__double2float_rn((double)h4.x + a.dt6 * (double)du),
                                    __double2float_rn((double)h4.y + a.dt6 * (double)dv),
                                    __double2float_rn((double)h4.z + a.dt6 * (double)dw), __double2float_rn(h));
                }
            }
            ens::named_sync(2 + grp, 128);
        };
        constexpr int kCh = C::kN / 64;          // chunks per group per tile
        ens::EpiSet sa;
        if (et == 0 && blockIdx.x < a.units) issue_tile(blockIdx.x, 0);
        int it = 0;
        for (int u = blockIdx.x; u < a.units; u += gridDim.x, ++it) {
            const int ab = it & 1;
            const bool got = ens::wait(&accf_bar[ab], (it >> 1) & 1, abort_v, a.err, 7) &&
                             ens::wait(&tile_bar[it & 1], (it >> 1) & 1, abort_v, a.err, 8);
            // every epilogue thread is done with the previous tile (and its tile buffer)
            if (!ens::named_and(4, 32 * kEnsEpiWarps, got && !*abort_v)) break;
            tc::fence_after_sync();
            if (et == 0 && u + (int)gridDim.x < a.units) {
                tc::fence_async_smem();   // the buffer's earlier reads come before the copy's writes
                issue_tile(u + gridDim.x, (it + 1) & 1);
            }
#pragma unroll 1
            for (int c = 0; c < kCh; ++c) {
                // streamed operands first: their latency overlaps the accumulator read and exchange
                const int ch = grp + 2 * c;
                fetch(u, ch, sa);
                chunk(u, it, ch, sa);
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
