// Batched-ensemble RK4 stage kernel on tcgen05 tensor cores (3xTF32 or split BF16).
//
// B ensemble members share one grid.  The state is stored member-innermost,
// [node][mf] with mf = 4*member + field, so a neighbour's state for all members
// is one contiguous row of 4B floats.  Nodes are grouped into tiles of 32
// consecutive nodes of a space-filling-curve order (compact patches: about 126
// unique neighbour rows per tile on the icosahedral grids).  For one tile the
// stencil products of a block of MPC members are one dense contraction
//
//     D[row(op, t)][mf] = sum_k  W_op(node t, row_k) * (X[row_k][mf] - c[mf])
//
// M = 128 (4 operators Dx, Dy, Dz, L x 32 nodes; row(op, t) = ens_a_row puts the
// four operators of a node in adjacent rows), N = 4*MPC member-fields,
// K = the tile's unique neighbour rows (W is zero where row_k is not in node
// t's stencil).  Each unique row is gathered once per tile instead of once per
// stencil slot.
//
// Precision: both operands are split x ~ hi + lo, and D = A_hi B_hi + A_hi B_lo
// + A_lo B_hi accumulates in FP32 in tensor memory; the split is 3xTF32
// (|x - hi - lo| <= 2^-21 |x| as the tensor core reads it), split FP16 with
// power-of-two scales (2^-22) or split BF16 (2^-17), see ens_operands.cuh.  The
// gathered states are centred on the state of one node of the tile (c[mf]) before
// the split, and c * sum_k W (row sums of the FP64 weights) is added back: with
// 3xTF32 and split FP16 by the MMA itself, through one more K row whose B values
// are c and whose A weights are the row sums; with split BF16 in the epilogue.  Derivative and
// hyperviscosity weights annihilate constants, so the added-back term is small
// and the cancellation that limits FP32 stencil sums mostly disappears.  The RK4
// accumulation of h (base state and D register) is FP64; u, v, w and every stage
// state K are FP32.
//
// Persistent, warp-specialised CTA (one per SM; it owns all of tensor memory):
//   * converter warps (MPC/8): for each 16-row chunk of K they gather the rows
//     as async copies into a staging buffer issued two chunks ahead, three
//     buffers deep, so that no register waits on a gather (16 bytes a row for
//     3xTF32, 8 for the 16-bit splits), and centre and split them into the B
//     operand;
//   * the A producer warp: the A chunks are static, so they are split once at
//     init into an image of the slot's A part (per precision); one thread streams
//     each chunk's image into its slot with one bulk copy (and prefetches the
//     image two chunks ahead into L2);
//   * a ring of slots (2 for 3xTF32, whose staging takes the third slot's shared
//     memory; 5 for the 16-bit splits) hands chunks to the MMA warp: one thread issues the chunk's 3
//     products (128 x N x 16) into one of two TMEM accumulators once the
//     converters and the A copy have filled the slot, and commits each chunk to
//     the slot's "empty" barrier and each tile to the accumulator's "full" barrier;
//   * 8 epilogue warps (two per TMEM lane quarter, each quarter holding T/4
//     nodes with their four operators): each warp tcgen05.ld's its quarter 32
//     columns at a time, transposes its (node, operator) rows to (node, member)
//     sets through its own shared-memory rows (no barrier between warps),
//     evaluates the pointwise part of eval_RHS_swe (rk4_rbffd_swe.c:320-353)
//     and applies the RK_substep combine (:30-72) for one (node, member) per
//     thread and pair, while the tensor cores already fill the other accumulator.
// Every mbarrier wait is bounded; a timeout sets an error word and a shared
// abort flag that makes every role leave its loop.
#pragma once

#include "ens_operands.cuh"
#include "stage_kernel.cuh"
#include "tcgen05.cuh"

namespace swe {

constexpr int kEnsEpiWarps = 8;
constexpr uint32_t kEnsWaitTries = 1u << 22;              // final MMA drain: polls
constexpr uint32_t kEnsWaitHintNs = 20000;                 // one sleeping try: up to 20 us
constexpr uint64_t kEnsWaitLimitNs = 2000000000ull;        // a wait gives up after 2 s

template <int T, int MPC, int PREC>
struct EnsCfg {
    using Op = ens::Operands<T, MPC, PREC>;
    static constexpr int kT = T;                           // nodes per tile
    static constexpr int kN = 4 * MPC;                     // MMA N: member-fields per CTA
    static constexpr int kConvWarps = MPC / 8;             // 4 * MPC converter threads
    static constexpr int kConvThreads = 32 * kConvWarps;
    static constexpr int kMmaWarp = kConvWarps;
    static constexpr int kEpiWarp0 = kConvWarps + 1;
    static constexpr int kProdWarp = kEpiWarp0 + kEnsEpiWarps;   // A operand producer
    static constexpr int kThreads = 32 * (kConvWarps + 2 + kEnsEpiWarps);
    static constexpr int kStages = Op::kStages;            // ring slots
    static constexpr int kStageBytes = Op::kStageBytes;
    static constexpr int kXchStride = 36;                  // floats per (op, node) row; 9 x 16 B
    // an epilogue warp's exchange rows (16-node tiles only: 32-node tiles read their
    // sums straight from tensor memory)
    static constexpr int kXchWarpFloats = T == 32 ? 0 : T * kXchStride;
    static constexpr int kTbRs = T * kPointStride * 4;     // per-tile buffer: PT, row sums, centre
    static constexpr int kTbCen = kTbRs + T * 16;
    static constexpr int kPairs = T / 16;                  // (node, member) pairs per epilogue thread and chunk
    static constexpr int kTbAi = kTbCen + kN * 4;          // FP16 operands: the tile's A-row inverse scales
    static constexpr int kTileBuf = (kTbAi + T * 16 + 127) / 128 * 128;
    static constexpr int kStgOff = kStages * kStageBytes + kEnsEpiWarps * kXchWarpFloats * 4 + 2 * kTileBuf;
    static constexpr int kSmem = kStgOff + Op::kStgDepth * Op::kStgBytes;
    static constexpr int kTmemCols = (2 * kN <= 256) ? 256 : 512;
    static_assert(kConvThreads == Op::kConvThreads, "converter thread count");
    static_assert(kSmem + 1024 <= 227 * 1024, "dynamic shared memory beside the barriers fits 227 KB");
    static_assert(kN % 64 == 0, "epilogue column chunks");
};

struct EnsArgs {
    int n;                 // nodes
    int ntiles;
    int units;             // ntiles * (members / MPC)
    int members;
    int mf;                // 4 * members (row length of the state arrays)
    const int* row_off;    // [ntiles + 1] offsets into rows, multiples of kEnsKc
    const int* rows;       // unique neighbour rows of each tile, ascending; padded with the centring node
    const unsigned char* Aimg;   // [chunk] A operand image (hi, then lo) in the slot's layout
    const int* centre;     // [ntiles] node whose state centres the tile
    const float4* PT;      // [n][5] pointwise record (20 floats)
    const float4* RS;      // [n] row sums of the four operators
    const float4* AI;      // [n] FP16 operands: 2^-k of each A row's scale (Dx, Dy, Dz, L)
    const unsigned* bmax;  // FP16 operands: the state fields' largest |value| (FP32 bits) of the state read
    unsigned* bmax_next;   // FP16 operands: the maxima of the state stage 3 writes (stage 2 clears them,
                           // stage 3 raises them by atomicMax, the next stage 0 reads them)
    unsigned* bmax_pub;    // FP16 operands, stage 0: where it copies the maxima it read for stages 1-3
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

// Bounded wait that also gives up as soon as another role has aborted.  Each try
// sleeps in hardware (suspend-time hint) rather than spinning, so waiting warps
// leave the issue slots to the working ones; the bound is wall time.
__device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, volatile int* abort_s, int* err, int code) {
    if (tc::mbar_try_wait(b, parity)) return true;
    const uint64_t t0 = tc::globaltimer_ns();
    for (;;) {
        if (tc::mbar_try_wait_hint(b, parity, kEnsWaitHintNs)) return true;
        if (*abort_s) return false;
        if (tc::globaltimer_ns() - t0 > kEnsWaitLimitNs) break;
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

// Streamed operands of one epilogue chunk (two (node, member) pairs per thread).
struct EpiSet {
    float4 own[2], h32[2], d32[2];
    double hh[2], dh[2];
};

}  // namespace ens

template <int T, int MPC, int MODE, int PREC>
__global__ void __launch_bounds__(EnsCfg<T, MPC, PREC>::kThreads, 1) ens_stage_kernel(const EnsArgs a) {
    using C = EnsCfg<T, MPC, PREC>;
    using Op = typename C::Op;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full_bar[C::kStages], empty_bar[C::kStages], afull_bar[C::kStages];
    __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], tile_bar[2], fin_bar;
    __shared__ uint32_t tmem_s;
    __shared__ int abort_s;
    volatile int* abort_v = &abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int halves = a.members / MPC;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::kStages; ++s) {
            tc::mbar_init(&full_bar[s], C::kConvWarps);
            tc::mbar_init(&empty_bar[s], 1);
            tc::mbar_init(&afull_bar[s], 1);
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
    // split FP16: the field maxima hand over from step to step without another launch --
    // stage 0 copies the ones it reads (the previous stage 3's) to where stages 1-3 read
    // them, and stage 2 clears the slot stage 3 fills.  No launch reads a slot that the
    // same launch writes.
    if constexpr (PREC == kFp16x3) {
        if (blockIdx.x == 0 && threadIdx.x < 4) {
            if constexpr (MODE == kStage0) a.bmax_pub[threadIdx.x] = a.bmax[threadIdx.x];
            if constexpr (MODE == kStage2) a.bmax_next[threadIdx.x] = 0u;
        }
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
        // FP16 operands: this thread's two fields (f0, f0 + 1) and their scales
        float2 sc = make_float2(1.f, 1.f);
        if constexpr (PREC == kFp16x3) {
            const int f0 = typename Op::Thread(threadIdx.x).col() & 3;
            sc = make_float2(ens::fp16_field_scale(a.bmax, f0, false), ens::fp16_field_scale(a.bmax, f0 + 1, false));
        }
        // staged gathers: chunk g + 2's rows are in flight (cp.async) while chunk g is
        // built from its staging buffer
        const typename Op::Thread th(threadIdx.x);
        const int ct = threadIdx.x;
        unsigned char* stg0 = smem + C::kStgOff;
        // chunk g's gathers are issued two steps ahead as async copies into staging
        // buffer g % 3; the centre row of a new unit is loaded into a register then too
        ens::Cursor cur = ens::first_cursor(a, halves);
        ens::Cursor c1 = ens::next_cursor(cur, a, halves);
        ens::Cursor c2 = ens::next_cursor(c1, a, halves);
        typename Op::Fetch f2, f3;     // indices of chunks g + 2 and g + 3
        using Cen = typename Op::Cen;
        Cen cen0{}, cen1{}, cen2{};    // centres of chunks g, g+1, g+2
        // returns the centre state of chunk p's unit (a new unit loads it; else prev)
        auto issue = [&](const ens::Cursor& p, const typename Op::Fetch& f, int slot, Cen prev) {
            Cen c = prev;
            if (p.valid) {
                const int tile = p.u / halves;
                const long col = (long)(p.u % halves) * C::kN + th.col();
                Op::stage_issue(stg0 + slot * Op::kStgBytes, ct, a.Kin, a.mf, col, f);
                if (p.gc == p.gc0) c = Op::load_cen(a.Kin + (long)__ldg(a.centre + tile) * a.mf + col);
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            return c;
        };
        if (cur.valid) {
            typename Op::Fetch f0, f1;
            Op::fetch_idx(a.rows, cur.gc, th, f0);
            if (c1.valid) Op::fetch_idx(a.rows, c1.gc, th, f1);
            if (c2.valid) Op::fetch_idx(a.rows, c2.gc, th, f2);
            cen0 = issue(cur, f0, 0, cen0);
            cen1 = issue(c1, f1, 1, cen0);
        }
        int g = 0;
        while (cur.valid) {
            // chunk g + 2's gathers, chunk g + 3's indices
            cen2 = issue(c2, f2, (g + 2) % 3, cen1);
            const ens::Cursor c3 = ens::next_cursor(c2, a, halves);
            if (c3.valid) Op::fetch_idx(a.rows, c3.gc, th, f3);
            asm volatile("cp.async.wait_group 2;" ::: "memory");
            const int s = g % C::kStages;
            if (!ens::wait(&empty_bar[s], ((g / C::kStages) & 1) ^ 1, abort_v, a.err, 3)) break;
            typename Op::Set o;
            Op::stage_read(stg0 + (g % 3) * Op::kStgBytes, ct, cen0, o);
            Op::build(smem + s * C::kStageBytes, th, o, sc, cur.gc + 1 == cur.gc_end);
            tc::fence_async_smem();
            __syncwarp();
            if (lane == 0) ens::mbar_arrive(&full_bar[s]);
            ++g;
            cur = c1;
            c1 = c2;
            c2 = c3;
            f2 = f3;
            cen0 = cen1;
            cen1 = cen2;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp == C::kMmaWarp) {
        // =============================== MMA issuer ===============================
        if (lane == 0) {
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
                    const int s = g % C::kStages;
                    if (!ens::wait(&full_bar[s], (g / C::kStages) & 1, abort_v, a.err, 5)) { ok = false; break; }
                    if (!ens::wait(&afull_bar[s], (g / C::kStages) & 1, abort_v, a.err, 9)) { ok = false; break; }
                    tc::fence_after_sync();
                    Op::issue(tc::smem_u32(smem + s * C::kStageBytes), d, gc == gc0);
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
    } else if (warp == C::kProdWarp) {
        // =========================== A operand producer ===========================
        {
            if (lane == 0) {
                constexpr uint32_t kABytes = Op::kABytes;
                ens::Cursor cur = ens::first_cursor(a, halves);
                ens::Cursor pf = ens::next_cursor(ens::next_cursor(cur, a, halves), a, halves);
                int g = 0;
                while (cur.valid) {
                    const int s = g % C::kStages;
                    if (!ens::wait(&empty_bar[s], ((g / C::kStages) & 1) ^ 1, abort_v, a.err, 10)) break;
                    tc::mbar_arrive_expect_tx(&afull_bar[s], kABytes);
                    tc::bulk_g2s(smem + s * C::kStageBytes, a.Aimg + (size_t)cur.gc * kABytes, kABytes, &afull_bar[s]);
                    if (pf.valid) prefetch_l2_bulk(a.Aimg + (size_t)pf.gc * kABytes, kABytes);
                    ++g;
                    cur = ens::next_cursor(cur, a, halves);
                    pf = ens::next_cursor(pf, a, halves);
                }
                // the copies of the last chunks land before the CTA ends, consumed or not
                for (int k = g > C::kStages ? g - C::kStages : 0; k < g; ++k)
                    tc::mbar_wait_bounded(&afull_bar[k % C::kStages], (k / C::kStages) & 1, kEnsWaitTries);
            }
        }
        __syncwarp();
    } else {
        // =============================== epilogue ===============================
        const int e = warp - C::kEpiWarp0;       // 0..7
        const int et = threadIdx.x - 32 * C::kEpiWarp0;   // 0..255
        const int grp = e >> 2;                  // column chunks alternate between the two groups
        const int qt = warp & 3;                 // TMEM lane quarter: tile nodes qt T/4 .. qt T/4 + T/4 - 1
        // this warp's exchange rows: one per TMEM lane (node, operator) of its quarter
        float* xch = reinterpret_cast<float*>(smem + C::kStages * C::kStageBytes) + e * C::kXchWarpFloats;
        unsigned char* tbuf = smem + C::kStages * C::kStageBytes + kEnsEpiWarps * C::kXchWarpFloats * 4;
        const int members = a.members;
        const float c32 = (float)a.c;
        // FP16 operands: the state fields' inverse scales
        float binv[4] = {1.f, 1.f, 1.f, 1.f};
        if constexpr (PREC == kFp16x3) {
#pragma unroll
            for (int f = 0; f < 4; ++f) binv[f] = ens::fp16_field_scale(a.bmax, f, true);
        }
        constexpr bool kHD = MODE == kStage1 || MODE == kStage2 || MODE == kStage3;
        // per-tile pointwise records (and, for split BF16, whose accumulator lacks the
        // add-back, the row sums and centre row): bulk copies into tbuf[it & 1]
        auto issue_tile = [&](int u, int b) {
            const int tile = u / halves;
            const int nn = min(T, a.n - tile * T);
            unsigned char* tb = tbuf + b * C::kTileBuf;
            constexpr bool kAddBack = PREC == kBf16x3;
            constexpr bool kScaled = PREC == kFp16x3;
            tc::mbar_arrive_expect_tx(&tile_bar[b], nn * kPointStride * 4 + (kAddBack ? nn * 16 + C::kN * 4 : 0) +
                                                        (kScaled ? nn * 16 : 0));
            tc::bulk_g2s(tb, a.PT + (long)tile * T * 5, nn * kPointStride * 4, &tile_bar[b]);
            if constexpr (kAddBack) {
                tc::bulk_g2s(tb + C::kTbRs, a.RS + (long)tile * T, nn * 16, &tile_bar[b]);
                tc::bulk_g2s(tb + C::kTbCen, a.Kin + (long)__ldg(a.centre + tile) * a.mf + (u % halves) * C::kN,
                             C::kN * 4, &tile_bar[b]);
            }
            if constexpr (kScaled) tc::bulk_g2s(tb + C::kTbAi, a.AI + (long)tile * T, nn * 16, &tile_bar[b]);
        };
        // this thread's pair pi of a chunk: tile node pair_node(pi) and chunk member
        // pair_member(pi).  32-node tiles: node qt 8 + lane / 4, members lane % 4 and
        // lane % 4 + 4 (the columns tmem_ld16x256 gives the thread, ens_b_col);
        // 16-node tiles: node qt 4 + (p >> 3), member p & 7, with p = lane + 32 pi.
        auto pair_node = [&](int pi) { return T == 32 ? qt * 8 + (lane >> 2) : qt * (T / 4) + ((lane + 32 * pi) >> 3); };
        auto pair_member = [&](int pi) { return T == 32 ? (lane & 3) + 4 * pi : (lane + 32 * pi) & 7; };
        // streamed per-(node, member) operands of one chunk for this thread's pairs
        auto fetch = [&](int u, int ch, ens::EpiSet& o) {
            if (u >= a.units) return;
            const int tile = u / halves;
            const int col0 = (u % halves) * C::kN;
#pragma unroll
            for (int pi = 0; pi < C::kPairs; ++pi) {
                const long node = (long)tile * T + pair_node(pi);
                if (node >= a.n) continue;
                const int mfb = col0 + ch * 32 + 4 * pair_member(pi);
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
        // split FP16, stage 3: the largest |value| of each field this thread writes, for
        // the next step's field scales
        unsigned hmax[4] = {0u, 0u, 0u, 0u};
        // one 32-column chunk: accumulator -> exchange -> (node, member) epilogue
        auto chunk = [&](int u, int it, int ch, ens::EpiSet& o) {
            const int ab = it & 1;
            const int tile = u / halves;
            const int col0 = (u % halves) * C::kN;
            const float* tb = reinterpret_cast<const float*>(tbuf + (it & 1) * C::kTileBuf);
            const uint32_t taddr = tmem + ((uint32_t)(32 * qt) << 16) + ab * C::kN + ch * 32;
            float v0[16], v1[16];
            if constexpr (T == 32) {
                // no exchange: lanes 0..15 of the quarter hold operators 0 and 1 of its
                // 8 nodes, lanes 16..31 operators 2 and 3 (ens_a_row), and a 16x256b
                // load hands each thread both members' 16 sums (ens_b_col)
                fetch(u, ch, o);
                tc::tmem_ld16x256(taddr, v0);
                tc::tmem_ld16x256(taddr + (16u << 16), v1);
                tc::tmem_wait_ld();
            } else {
                tc::tmem_ld16(taddr, v0);
                tc::tmem_ld16(taddr + 16, v1);
                tc::tmem_wait_ld();
                // lane 4 j + op of the quarter holds operator op of the quarter's node j
                // (ens_a_row); with M = 64 only lanes 0..15 hold rows
                if (lane < T) {
                    float* row = xch + lane * C::kXchStride;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        *reinterpret_cast<float4*>(row + 4 * q) =
                            make_float4(v0[4 * q], v0[4 * q + 1], v0[4 * q + 2], v0[4 * q + 3]);
                        *reinterpret_cast<float4*>(row + 16 + 4 * q) =
                            make_float4(v1[4 * q], v1[4 * q + 1], v1[4 * q + 2], v1[4 * q + 3]);
                    }
                }
                // the streamed operands are requested after the exchange stores: issued
                // before them, the loads hold the stores up in the load/store queue
                fetch(u, ch, o);
                __syncwarp();
            }
#pragma unroll
            for (int pi = 0; pi < C::kPairs; ++pi) {
                const int t = pair_node(pi);
                const long node = (long)tile * T + t;
                if (node >= a.n) continue;
                const int bm = pair_member(pi);
                const int mfb = col0 + ch * 32 + 4 * bm;      // first mf of this member
                const int member = mfb >> 2;
                float S[16];
                if constexpr (T == 32) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const int k = 2 * (f >> 1) + pi, b = f & 1;
                        S[f] = v0[4 * k + b];
                        S[4 + f] = v0[4 * k + 2 + b];
                        S[8 + f] = v1[4 * k + b];
                        S[12 + f] = v1[4 * k + 2 + b];
                    }
                } else {
                    const int j = (lane + 32 * pi) >> 3;
#pragma unroll
                    for (int o2 = 0; o2 < 4; ++o2) {
                        const float4 sv =
                            *reinterpret_cast<const float4*>(xch + (4 * j + o2) * C::kXchStride + 4 * bm);
                        S[4 * o2] = sv.x; S[4 * o2 + 1] = sv.y; S[4 * o2 + 2] = sv.z; S[4 * o2 + 3] = sv.w;
                    }
                }
                if constexpr (PREC == kFp16x3) {
                    // divide out the A row's and the state field's power-of-two scales (exact)
                    const float4 ai4 = *reinterpret_cast<const float4*>(tb + C::kTbAi / 4 + 4 * t);
                    const float ai[4] = {ai4.x, ai4.y, ai4.z, ai4.w};
#pragma unroll
                    for (int o2 = 0; o2 < 4; ++o2)
#pragma unroll
                        for (int f = 0; f < 4; ++f) S[4 * o2 + f] *= ai[o2] * binv[f];
                }
                if constexpr (PREC == kBf16x3) {
                    // the centre term c * sum_k W (3xTF32 and split FP16 accumulate it in
                    // their add-back row)
                    const float4 cen = *reinterpret_cast<const float4*>(tb + C::kTbCen / 4 + (mfb - col0));
                    const float4 rs4 = *reinterpret_cast<const float4*>(tb + C::kTbRs / 4 + 4 * t);
                    const float cf[4] = {cen.x, cen.y, cen.z, cen.w};
                    const float rs[4] = {rs4.x, rs4.y, rs4.z, rs4.w};
#pragma unroll
                    for (int o2 = 0; o2 < 4; ++o2)
#pragma unroll
                        for (int f = 0; f < 4; ++f) S[4 * o2 + f] = fmaf(cf[f], rs[o2], S[4 * o2 + f]);
                }
                const float q[4] = {o.own[pi].x, o.own[pi].y, o.own[pi].z, o.own[pi].w};
                float pt[kPointStride];
#pragma unroll
                for (int pp = 0; pp < kPointStride / 4; ++pp) {
                    const float4 pv = *reinterpret_cast<const float4*>(tb + t * kPointStride + 4 * pp);
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
                    const float4 hn = make_float4(__double2float_rn((double)h4.x + a.dt6 * (double)du),
                                                  __double2float_rn((double)h4.y + a.dt6 * (double)dv),
                                                  __double2float_rn((double)h4.z + a.dt6 * (double)dw),
                                                  __double2float_rn(h));
                    *reinterpret_cast<float4*>(a.H32 + e4) = hn;
                    if constexpr (PREC == kFp16x3) {
                        hmax[0] = max(hmax[0], __float_as_uint(fabsf(hn.x)));
                        hmax[1] = max(hmax[1], __float_as_uint(fabsf(hn.y)));
                        hmax[2] = max(hmax[2], __float_as_uint(fabsf(hn.z)));
                        hmax[3] = max(hmax[3], __float_as_uint(fabsf(hn.w)));
                    }
                }
            }
            if constexpr (T != 32) __syncwarp();   // the exchange rows are rewritten by the next chunk
        };
        constexpr int kCh = C::kN / 64;          // chunks per group per tile
        ens::EpiSet sa;
        // pend: the iteration whose tile copy thread 0 has issued and not yet seen land
        int pend = -1;
        if (et == 0 && blockIdx.x < a.units) {
            issue_tile(blockIdx.x, 0);
            pend = 0;
        }
        int it = 0;
        for (int u = blockIdx.x; u < a.units; u += gridDim.x, ++it) {
            const int ab = it & 1;
            const bool got = ens::wait(&accf_bar[ab], (it >> 1) & 1, abort_v, a.err, 7) &&
                             ens::wait(&tile_bar[it & 1], (it >> 1) & 1, abort_v, a.err, 8);
            if (got && pend == it) pend = -1;
            // every epilogue thread is done with the previous tile (and its tile buffer)
            if (!ens::named_and(4, 32 * kEnsEpiWarps, got && !*abort_v)) break;
            tc::fence_after_sync();
            if (et == 0 && u + (int)gridDim.x < a.units) {
                tc::fence_async_smem();   // the buffer's earlier reads come before the copy's writes
                issue_tile(u + gridDim.x, (it + 1) & 1);
                pend = it + 1;
            }
#pragma unroll 1
            for (int c = 0; c < kCh; ++c) chunk(u, it, grp + 2 * c, sa);
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) ens::mbar_arrive(&acce_bar[ab]);
        }
        if constexpr (MODE == kStage3 && PREC == kFp16x3) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const unsigned w = __reduce_max_sync(0xffffffffu, hmax[f]);
                if (lane == 0 && w) atomicMax(a.bmax_next + f, w);
            }
        }
        // after an abort, a tile copy still in flight lands before the CTA ends
        if (pend >= 0) tc::mbar_wait_bounded(&tile_bar[pend & 1], (pend >> 1) & 1, kEnsWaitTries);
    }

    tc::fence_before_sync();
    __syncthreads();
    if (warp == C::kMmaWarp) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, C::kTmemCols);
    }
}

}  // namespace swe
