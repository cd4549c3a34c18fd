// Operand policies of the batched-ensemble kernel: how the converter threads
// gather one 16-row chunk of a tile's neighbour rows and split them into hi / lo
// parts in the tensor core's shared-memory layout (the B operand), where the A
// (weight) operand's image sits in the slot, and how the MMA thread issues the
// chunk's three products.
//
//   Tf32x3: kind::tf32, hi = tf32(x) rounded to nearest, lo = x - hi kept in
//           FP32 and read by the tensor core at TF32 precision
//           (|x - hi - lo| <= 2^-21 |x|), 2 k-steps of K = 8 per chunk.
//   Bf16x3: kind::f16 with BF16 operands, hi = bf16(x), lo = bf16(x - hi)
//           (|x - hi - lo| <= 2^-17 |x|), one k-step of K = 16 per chunk;
//           half the shared-memory bytes of Tf32x3 and twice the tensor rate.
//   Fp16x3: the same with FP16 operands, which carry TF32's 11-bit significand:
//           |x - hi - lo| <= 2^-22 |x| within FP16's range.  Power-of-two scales
//           bring each A row (node, operator) and each state field into that range
//           (weights: the row's largest at 2^13..2^14; state: the field's largest
//           value at 2^11..2^12, taken again after every step, so that centred values
//           stay below 2^13 and a field can grow 8-fold within a step before FP16
//           overflows); the epilogue divides them out exactly.  The centre add-back
//           rides in the MMA as in Tf32x3.
//
// Padding rows of a tile's neighbour list name the tile's centring node, so their
// centred values are exactly zero (their weights are zero as well).  Every tile has
// at least one: with 3xTF32 its last padding row is the add-back row (see build).
//
// Both are K-major without swizzle: 8-row x 16-byte core matrices, LBO = 128
// (the next core matrix along K), SBO = the stride between 8-row groups.  The
// B (state) operand's SBO is padded by 16 bytes so that the converters'
// 16-byte stores of consecutive member-fields fall in distinct bank groups.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>


#include "tcgen05.cuh"

namespace swe {

constexpr int kEnsTileNodes = 32;   // nodes per tile of the default shape (M = 4 operators x 32 nodes)
constexpr int kEnsKc = 16;          // neighbour rows per pipeline chunk

enum EnsPrecision { kTf32x3 = 0, kBf16x3 = 1, kFp16x3 = 2 };

// Row of the A operand (and TMEM lane of the accumulator) that holds operator op of
// tile node t.  Each 32-lane quarter of tensor memory holds T/4 consecutive tile nodes,
// so that one epilogue warp reads all four operators of its nodes:
//   T = 32: operator op of quarter node j in lane j + 8 op.  A 16x256b load of lanes
//           0..15 then gives thread i operators 0 and 1 of node i / 4, and one of lanes
//           16..31 operators 2 and 3 (tmem_ld16x256);
//   T = 16 (M = 64, lanes 0..15 of each quarter): the four operators of a node in
//           adjacent lanes 4 j + op, read with 32x32b loads and exchanged through
//           shared memory.
template <int T>
__host__ __device__ constexpr int ens_a_row(int op, int t) {
    return T == 32 ? 32 * (t / 8) + 8 * op + (t % 8) : T * (t / (T / 4)) + 4 * (t % (T / 4)) + op;
}
template <int T>
__host__ __device__ constexpr int ens_a_row_op(int r) { return T == 32 ? (r & 31) >> 3 : r & 3; }
template <int T>
__host__ __device__ constexpr int ens_a_row_node(int r) {
    return T == 32 ? (r >> 5) * 8 + (r & 7) : (r / T) * (T / 4) + ((r % T) >> 2);
}

// Column of the B operand (and of the accumulator) within a 32-column chunk that holds
// field f of chunk member m (0..7).  T = 32: thread i's columns in a 16x256b load,
// 8 k + 2 (i % 4) + b, are fields 0..3 of members i % 4 and i % 4 + 4 (member
// i % 4 + 4 (k & 1), field 2 (k >> 1) + b).  T = 16: member-major, 4 m + f.
template <int T>
__host__ __device__ constexpr int ens_b_col(int m, int f) {
    return T == 32 ? 8 * (2 * (f >> 1) + (m >> 2)) + 2 * (m & 3) + (f & 1) : 4 * m + f;
}

struct EnsArgs;

namespace ens {

__device__ __forceinline__ float4 ldg_f4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float2 ldg_f2(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }

// hi = bf16(a, b) (round to nearest even), lo = bf16 of the remainders; packed pairs, a in the low half.
__device__ __forceinline__ uint32_t bf16x2_split(float a, float b, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    lo = *reinterpret_cast<const uint32_t*>(&l);
    return *reinterpret_cast<const uint32_t*>(&h);
}
// the same with FP16 halves
__device__ __forceinline__ uint32_t f16x2_split(float a, float b, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    lo = *reinterpret_cast<const uint32_t*>(&l);
    return *reinterpret_cast<const uint32_t*>(&h);
}
template <bool F16>
__device__ __forceinline__ uint32_t half2_split(float a, float b, uint32_t& lo) {
    return F16 ? f16x2_split(a, b, lo) : bf16x2_split(a, b, lo);
}

// Scale of state field f for the FP16 operands: 2^e with the field's largest |value|
// (max_bits[f], an FP32 bit pattern; the velocity fields 0-2 share their largest) at
// 2^11..2^12; 1 when that is zero.  inverse: 2^-e.
__host__ __device__ inline float fp16_field_scale(const unsigned* max_bits, int f, bool inverse) {
    unsigned m = max_bits[3];
    if (f < 3) {
        m = max_bits[0] > max_bits[1] ? max_bits[0] : max_bits[1];
        m = m > max_bits[2] ? m : max_bits[2];
    }
    const int ex = (int)((m >> 23) & 0xff);      // biased exponent of the largest value
    int e = ex == 0 ? 0 : 11 - (ex - 127);
    e = e < -60 ? -60 : (e > 60 ? 60 : e);
    // 2^e as an FP32 bit pattern (|e| <= 60 stays normal)
    const unsigned bits = (unsigned)((inverse ? -e : e) + 127) << 23;
    float r;
    memcpy(&r, &bits, sizeof(r));
    return r;
}

template <int T, int MPC, int PREC>
struct Operands;

// --------------------------------------------------------------------------------------
// 3xTF32, tiles of T = 32 or 16 nodes (M = 4T = 128 or 64).  The A (weight) operand of
// every chunk is static: it is split once at init into an image of the slot's A part
// (a_offset below) and streamed into the slot by one bulk copy per chunk.  B thread:
// member-fields 4q..4q+3 of rows 4kg..4kg+3.
// --------------------------------------------------------------------------------------
template <int T, int MPC>
struct Operands<T, MPC, kTf32x3> {
    static constexpr int kN = 4 * MPC;
    static constexpr int kM = 4 * T;
    static constexpr int kConvThreads = 4 * MPC;
    static constexpr int kSboA = (kEnsKc / 4) * 128;
    static constexpr int kSboB = (kEnsKc / 4) * 128 + 16;
    static constexpr int kAHalf = (kM / 8) * kSboA;
    static constexpr int kBHalf = (kN / 8) * kSboB;
    static constexpr int kABytes = 2 * kAHalf;                     // one chunk's A image: hi, then lo
    static constexpr int kStageBytes = ((2 * kAHalf + 2 * kBHalf) + 127) / 128 * 128;
    static constexpr int kStages = 2;
    // staged gathers: per converter thread and chunk, 4 rows x 16 B of state in
    // structure-of-arrays order (row-major over threads) so that each warp's
    // shared-memory accesses are contiguous
    static constexpr int kStgBytes = 4 * kConvThreads * 16;
    static constexpr int kStgDepth = 3;                            // chunks in flight: g, g+1, g+2
    static_assert(T == 16 || T == 32, "tiles of 16 or 32 nodes");

    // Byte offset, within A_hi (and A_lo), of the 16-byte core row holding the weights
    // of operator-node row r (r = T op + t) for the chunk rows 4 akg .. 4 akg + 3.
    __host__ __device__ static constexpr int a_offset(int r, int akg) {
        return (r >> 3) * kSboA + akg * 128 + (r & 7) * 16;
    }

    struct Thread {
        int quad, kg;
        __device__ explicit Thread(int ct) : quad(ct % MPC), kg(ct / MPC) {}
        __device__ int col() const { return 4 * quad; }
    };
    struct Fetch {
        int4 idx = make_int4(-1, -1, -1, -1);
    };
    struct Set {
        float4 x[4];          // 4 gathered rows x 4 member-fields
        float4 cen;           // centre state of the same member-fields
    };
    using Cen = float4;
    __device__ static Cen load_cen(const float* p) { return ldg_f4(p); }

    __device__ static void fetch_idx(const int* rows, int gc, const Thread& th, Fetch& f) {
        f.idx = __ldg(reinterpret_cast<const int4*>(rows + gc * kEnsKc + 4 * th.kg));
    }
    // cp.async of this thread's 4 gathered rows of one chunk into staging buffer `stg`
    __device__ static void stage_issue(unsigned char* stg, int ct, const float* Kin, int mf, long col,
                                       const Fetch& f) {
        const int r[4] = {f.idx.x, f.idx.y, f.idx.z, f.idx.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t dst = tc::smem_u32(stg + (i * kConvThreads + ct) * 16);
            const float* src = Kin + (long)r[i] * mf + col;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
        }
    }
    __device__ static void stage_read(const unsigned char* stg, int ct, const float4& cen, Set& o) {
#pragma unroll
        for (int i = 0; i < 4; ++i) o.x[i] = *reinterpret_cast<const float4*>(stg + (i * kConvThreads + ct) * 16);
        o.cen = cen;
    }
    // The B operand of one chunk: centred rows split into hi and lo.  Row 15 of a
    // unit's last chunk (last = true) is its add-back row: it carries the centre state
    // itself, not centred, and its A weights are the operators' row sums, so the
    // accumulator receives c * sum_k W with the stencil sums.
    __device__ static void build(unsigned char* slot, const Thread& th, const Set& o, float2, bool last) {
        unsigned char* B_hi = slot + 2 * kAHalf;
        unsigned char* B_lo = B_hi + kBHalf;
        const bool keep15 = last && th.kg == 3;
        // B: each member-field's 4 rows are one 16-byte core row
        const float xv[4][4] = {{o.x[0].x, o.x[0].y, o.x[0].z, o.x[0].w},
                                {o.x[1].x, o.x[1].y, o.x[1].z, o.x[1].w},
                                {o.x[2].x, o.x[2].y, o.x[2].z, o.x[2].w},
                                {o.x[3].x, o.x[3].y, o.x[3].z, o.x[3].w}};
        const float cv[4] = {o.cen.x, o.cen.y, o.cen.z, o.cen.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int nrow = 32 * (th.quad >> 3) + ens_b_col<T>(th.quad & 7, j);
            float4 hi, lo;
            float y[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) y[i] = xv[i][j] - cv[j];
            if (keep15) y[3] = xv[3][j];
            tc::tf32_split_lo_fp32(y[0], hi.x, lo.x);
            tc::tf32_split_lo_fp32(y[1], hi.y, lo.y);
            tc::tf32_split_lo_fp32(y[2], hi.z, lo.z);
            tc::tf32_split_lo_fp32(y[3], hi.w, lo.w);
            const uint32_t off = (nrow >> 3) * kSboB + th.kg * 128 + (nrow & 7) * 16;
            *reinterpret_cast<float4*>(B_hi + off) = hi;
            *reinterpret_cast<float4*>(B_lo + off) = lo;
        }
    }
    // The chunk's products A_hi B_hi + A_hi B_lo + A_lo B_hi into accumulator d.
    __device__ static void issue(uint32_t slot, uint32_t d, bool first) {
        constexpr uint32_t idesc = tc::idesc_tf32(kM, kN);
        const uint32_t a_hi = slot, a_lo = slot + kAHalf, b_hi = slot + 2 * kAHalf, b_lo = b_hi + kBHalf;
#pragma unroll
        for (int ks = 0; ks < kEnsKc / 8; ++ks) {
            const uint64_t dah = tc::smem_desc(a_hi + ks * 256, 128, kSboA);
            const uint64_t dal = tc::smem_desc(a_lo + ks * 256, 128, kSboA);
            const uint64_t dbh = tc::smem_desc(b_hi + ks * 256, 128, kSboB);
            const uint64_t dbl = tc::smem_desc(b_lo + ks * 256, 128, kSboB);
            tc::mma_tf32(d, dah, dbh, idesc, (!first || ks > 0) ? 1u : 0u);
            tc::mma_tf32(d, dah, dbl, idesc, 1u);
            tc::mma_tf32(d, dal, dbh, idesc, 1u);
        }
    }
};

// --------------------------------------------------------------------------------------
// split BF16 and FP16 (F16), tiles of 32 nodes.  B thread: columns 2p, 2p+1 (fields f,
// f + 1 of one member, ens_b_col) of rows 8kh..8kh+7.  The A operand comes from an image
// split once at init (a_offset), like 3xTF32's.
// --------------------------------------------------------------------------------------
template <int MPC, bool F16>
struct HalfOperands {
    // staged gathers (cp.async, 8 bytes a row): per converter thread and chunk, 8 rows x
    // 2 member-fields in structure-of-arrays order, three chunks in flight
    static constexpr int kStgDepth = 3, kStgBytes = 8 * 4 * MPC * 8;
    static constexpr int kN = 4 * MPC;
    static constexpr int kConvThreads = 4 * MPC;
    static constexpr int kSboA = (kEnsKc / 8) * 128;
    static constexpr int kSboB = (kEnsKc / 8) * 128 + 16;
    static constexpr int kAHalf = (128 / 8) * kSboA;
    static constexpr int kBHalf = (kN / 8) * kSboB;
    static constexpr int kABytes = 2 * kAHalf;                     // one chunk's A image: hi, then lo
    static constexpr int kStageBytes = ((2 * kAHalf + 2 * kBHalf) + 127) / 128 * 128;
    static constexpr int kStages = 5;

    // Byte offset, within A_hi (and A_lo), of the 16-byte core row holding the weights
    // of A row r for the chunk rows 8 akh .. 8 akh + 7.
    __host__ __device__ static constexpr int a_offset(int r, int akh) {
        return (r >> 3) * kSboA + akh * 128 + (r & 7) * 16;
    }

    struct Thread {
        int p, kh;
        __device__ explicit Thread(int ct) : p(ct % (kN / 2)), kh(ct / (kN / 2)) {}
        // member-field (state column) of B column 2p: within its 32-column chunk,
        // 2p = 8 k + 2 i holds member i + 4 (k & 1), fields 2 (k >> 1) and + 1
        __device__ int col() const {
            const int k = (p >> 2) & 3, i = p & 3;
            return 32 * (p >> 4) + 4 * (i + 4 * (k & 1)) + 2 * (k >> 1);
        }
    };
    struct Fetch {
        int4 idx[2] = {make_int4(-1, -1, -1, -1), make_int4(-1, -1, -1, -1)};
    };
    struct Set {
        float2 x[8];          // 8 gathered rows x 2 member-fields
        float2 cen;
    };
    using Cen = float2;
    __device__ static Cen load_cen(const float* p) { return ldg_f2(p); }

    __device__ static void fetch_idx(const int* rows, int gc, const Thread& th, Fetch& f) {
        const int4* r = reinterpret_cast<const int4*>(rows + gc * kEnsKc + 8 * th.kh);
        f.idx[0] = __ldg(r);
        f.idx[1] = __ldg(r + 1);
    }
    // cp.async of this thread's 8 gathered rows of one chunk into staging buffer `stg`
    __device__ static void stage_issue(unsigned char* stg, int ct, const float* Kin, int mf, long col,
                                       const Fetch& f) {
        const int r[8] = {f.idx[0].x, f.idx[0].y, f.idx[0].z, f.idx[0].w,
                          f.idx[1].x, f.idx[1].y, f.idx[1].z, f.idx[1].w};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t dst = tc::smem_u32(stg + (i * kConvThreads + ct) * 8);
            const float* src = Kin + (long)r[i] * mf + col;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
        }
    }
    __device__ static void stage_read(const unsigned char* stg, int ct, const float2& cen, Set& o) {
#pragma unroll
        for (int i = 0; i < 8; ++i) o.x[i] = *reinterpret_cast<const float2*>(stg + (i * kConvThreads + ct) * 8);
        o.cen = cen;
    }
    // the B operand of one chunk: centred rows (times the thread's two field scales sc,
    // F16 only) split into hi and lo, each member-field's 8 rows one 16-byte core row.
    // F16: row 15 of a unit's last chunk (last = true) is its add-back row, as in
    // 3xTF32: it carries the centre state itself, and the image's weights there are the
    // operators' row sums.
    __device__ static void build(unsigned char* slot, const Thread& th, const Set& o, float2 sc, bool last) {
        const bool keep15 = F16 && last && th.kh == 1;
        unsigned char* B_hi = slot + 2 * kAHalf;
        unsigned char* B_lo = B_hi + kBHalf;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const float c = j ? o.cen.y : o.cen.x;
            const float m = j ? sc.y : sc.x;
            float y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) y[i] = F16 ? ((j ? o.x[i].y : o.x[i].x) - c) * m : (j ? o.x[i].y : o.x[i].x) - c;
            if (keep15) y[7] = (j ? o.x[7].y : o.x[7].x) * m;
            uint4 hi, lo;
            hi.x = half2_split<F16>(y[0], y[1], lo.x);
            hi.y = half2_split<F16>(y[2], y[3], lo.y);
            hi.z = half2_split<F16>(y[4], y[5], lo.z);
            hi.w = half2_split<F16>(y[6], y[7], lo.w);
            const int nrow = 2 * th.p + j;
            const uint32_t off = (nrow >> 3) * kSboB + th.kh * 128 + (nrow & 7) * 16;
            *reinterpret_cast<uint4*>(B_hi + off) = hi;
            *reinterpret_cast<uint4*>(B_lo + off) = lo;
        }
    }
    __device__ static void issue(uint32_t slot, uint32_t d, bool first) {
        constexpr uint32_t idesc = F16 ? tc::idesc_f16(128, kN) : tc::idesc_bf16(128, kN);
        const uint32_t a_hi = slot, a_lo = slot + kAHalf, b_hi = slot + 2 * kAHalf, b_lo = b_hi + kBHalf;
        const uint64_t dah = tc::smem_desc(a_hi, 128, kSboA);
        const uint64_t dal = tc::smem_desc(a_lo, 128, kSboA);
        const uint64_t dbh = tc::smem_desc(b_hi, 128, kSboB);
        const uint64_t dbl = tc::smem_desc(b_lo, 128, kSboB);
        tc::mma_f16(d, dah, dbh, idesc, first ? 0u : 1u);
        tc::mma_f16(d, dah, dbl, idesc, 1u);
        tc::mma_f16(d, dal, dbh, idesc, 1u);
    }
};

template <int MPC>
struct Operands<32, MPC, kBf16x3> : HalfOperands<MPC, false> {};
template <int MPC>
struct Operands<32, MPC, kFp16x3> : HalfOperands<MPC, true> {};

}  // namespace ens
}  // namespace swe
