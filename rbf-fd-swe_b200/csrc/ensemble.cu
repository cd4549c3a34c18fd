// Batched-ensemble form: swe_ens_* entry points of include/swe_b200.h.
//
// B members (32 or 64) share one grid.  The library orders nodes along a
// Hilbert curve on the six faces of the cube around the sphere, so that 32
// consecutive nodes form a compact patch, and builds per-tile tables once:
// the tile's unique neighbour rows (ascending, padded to 16-row chunks), the
// stencil slot (if any) of every (tile node, chunk row) pair, the node that
// centres it, and the operators' row sums.  All member states stay device-resident; each RK4
// stage is one persistent tcgen05 kernel (ensemble_kernel.cuh).  An autotuner
// times each members-per-CTA variant on the live state and keeps the fastest;
// whole steps replay a captured CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "ensemble_kernel.cuh"

namespace swe {
namespace {

// Hilbert index of (x, y) on a 2^bits grid: the classic quadrant walk that
// rotates / reflects the lower bits at every level.
uint64_t hilbert_index(uint32_t x, uint32_t y, int bits) {
    const uint32_t n = 1u << bits;
    uint64_t d = 0;
    for (uint32_t s = n >> 1; s > 0; s >>= 1) {
        const uint32_t rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = n - 1 - x;
                y = n - 1 - y;
            }
            std::swap(x, y);
        }
    }
    return d;
}

// mapping[new] = old: nodes sorted by (cube face, Hilbert index of the
// equal-angle face coordinates, old index).
std::vector<int> curve_order(int n, const double* x, const double* y, const double* z) {
    constexpr int kBits = 16;
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; ++i) {
        const double c[3] = {x[i], y[i], z[i]};
        int ax = 0;
        for (int d = 1; d < 3; ++d)
            if (std::fabs(c[d]) > std::fabs(c[ax])) ax = d;
        const int face = 2 * ax + (c[ax] > 0.0 ? 1 : 0);
        const double m = std::fabs(c[ax]) > 0.0 ? std::fabs(c[ax]) : 1.0;
        const int o0 = ax == 0 ? 1 : 0, o1 = ax == 2 ? 1 : 2;
        uint32_t q[2];
        const double uv[2] = {c[o0] / m, c[o1] / m};
        for (int d = 0; d < 2; ++d) {
            double a = std::atan(uv[d]) * (4.0 / 3.14159265358979323846);   // [-1, 1]
            a = std::min(1.0, std::max(-1.0, a));
            q[d] = (uint32_t)((a + 1.0) * 0.5 * (double)((1u << kBits) - 1) + 0.5);
        }
        key[i] = ((uint64_t)face << 40) | hilbert_index(q[0], q[1], kBits);
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    return order;
}

// Per-tile tables (node indices in the curve order).
struct TileTables {
    int ntiles = 0, nchunks = 0, max_rows = 0;
    std::vector<int> row_off, rows, centre;
    std::vector<uint32_t> jmap;   // [chunk][row group][node t] 4 stencil slots (255 = none)
};

TileTables build_tiles(int T, int n, int nnbr, const std::vector<int>& ridx, const std::vector<double>& X) {
    TileTables tb;
    tb.ntiles = (n + T - 1) / T;
    tb.row_off.assign(tb.ntiles + 1, 0);
    tb.centre.assign(tb.ntiles, 0);
    std::vector<int> u;
    std::vector<uint8_t> slot;   // [t][k] stencil slot of row k in node t's stencil
    for (int tile = 0; tile < tb.ntiles; ++tile) {
        const int n0 = tile * T, n1 = std::min(n, n0 + T);
        u.clear();
        for (int i = n0; i < n1; ++i)
            for (int j = 0; j < nnbr; ++j) u.push_back(ridx[(size_t)i * nnbr + j]);
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        tb.max_rows = std::max(tb.max_rows, (int)u.size());
        // at least one padding row: the last one is the 3xTF32 add-back row
        const int nch = ((int)u.size() + 1 + kEnsKc - 1) / kEnsKc;
        const int kpad = nch * kEnsKc;
        // padding rows: the centring node (chosen below), whose centred state is exactly 0
        const size_t pad0 = tb.rows.size() + u.size();
        for (int k = 0; k < kpad; ++k) tb.rows.push_back(k < (int)u.size() ? u[k] : -1);
        tb.row_off[tile + 1] = (int)tb.rows.size();
        slot.assign((size_t)T * kpad, 0xff);
        for (int i = n0; i < n1; ++i)
            for (int j = 0; j < nnbr; ++j) {
                const int k = (int)(std::lower_bound(u.begin(), u.end(), ridx[(size_t)i * nnbr + j]) - u.begin());
                slot[(size_t)(i - n0) * kpad + k] = (uint8_t)j;
            }
        for (int c = 0; c < nch; ++c)
            for (int g = 0; g < 4; ++g)
                for (int t = 0; t < T; ++t) {
                    uint32_t v = 0;
                    for (int i = 0; i < 4; ++i) v |= (uint32_t)slot[(size_t)t * kpad + c * kEnsKc + 4 * g + i] << (8 * i);
                    tb.jmap.push_back(v);
                }
        // centre: the tile node nearest the tile's centroid
        double cx = 0, cy = 0, cz = 0;
        for (int i = n0; i < n1; ++i) { cx += X[3 * i]; cy += X[3 * i + 1]; cz += X[3 * i + 2]; }
        cx /= (n1 - n0); cy /= (n1 - n0); cz /= (n1 - n0);
        double best = 1e300;
        for (int i = n0; i < n1; ++i) {
            const double d = (X[3 * i] - cx) * (X[3 * i] - cx) + (X[3 * i + 1] - cy) * (X[3 * i + 1] - cy) +
                             (X[3 * i + 2] - cz) * (X[3 * i + 2] - cz);
            if (d < best) { best = d; tb.centre[tile] = i; }
        }
        for (size_t k = pad0; k < tb.rows.size(); ++k) tb.rows[k] = tb.centre[tile];
    }
    tb.nchunks = (int)tb.rows.size() / kEnsKc;
    return tb;
}

// A kernel variant: tile shape (nodes per tile) and members per CTA.
struct Variant {
    int tile = 32;
    int mpc = 32;
    bool usable = false;
};

// Device copies of one tile shape's tables.
struct DevTables {
    int ntiles = 0, max_rows = 0, nchunks = 0;
    int *row_off = nullptr, *rows = nullptr, *centre = nullptr;
    uint32_t* jmap = nullptr;
    unsigned char* aimg = nullptr;   // [chunk] 3xTF32 A operand image (hi, then lo), 512 T bytes a chunk
    unsigned char* aimg_bf16 = nullptr;   // 32-node tiles: [chunk] split-BF16 A operand image, 8 KB a chunk
    unsigned char* aimg_f16 = nullptr;    // 32-node tiles: [chunk] FP16 A operand image (rows scaled), 8 KB a chunk
};
constexpr int kEnsShapes = 2;          // tiles of 32 and 16 nodes
constexpr int kEnsShapeNodes[kEnsShapes] = {32, 16};
constexpr int kEnsVariants = 4;        // (32, 64), (32, 32), (16, 64), (16, 32)

// The 3xTF32 A operand of every chunk, split once (the weights are static): one
// thread per (chunk, A row r = ens_a_row(op, t), row group akg) writes the 4 chunk
// rows' weights of that row as one 16-byte core row of the hi image and one of the
// lo image (zero where a chunk row is not in node t's stencil).  Row 15 of a tile's
// last chunk is the add-back row: its weights are the operators' row sums.
template <int T>
__global__ void ens_build_aimg(const uint32_t* __restrict__ jmap, const int* __restrict__ chunk_tile,
                              const int* __restrict__ row_off, const float4* __restrict__ W,
                              const float4* __restrict__ RS, int n, int nchunks, unsigned char* __restrict__ img) {
    using Op = ens::Operands<T, 32, kTf32x3>;   // the A layout does not depend on the members per CTA
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nchunks * 16 * T) return;
    const int akg = (int)(t & 3);
    const int r = (int)((t >> 2) % (4 * T));
    const long gc = (t >> 2) / (4 * T);
    const int op = ens_a_row_op<T>(r), at = ens_a_row_node<T>(r);
    const int tile = chunk_tile[gc];
    const long node = (long)tile * T + at;
    const uint32_t jj = jmap[(gc * 4 + akg) * T + at];
    float v[4];
    for (int i = 0; i < 4; ++i) {
        const uint32_t j = (jj >> (8 * i)) & 0xffu;
        v[i] = (j != 0xffu && node < n) ? reinterpret_cast<const float*>(W + node * 32 + j)[op] : 0.f;
    }
    if (akg == 3 && (gc + 1) * kEnsKc == row_off[tile + 1] && node < n)
        v[3] = reinterpret_cast<const float*>(RS + node)[op];
    float4 hi, lo;
    tc::tf32_split_lo_fp32(v[0], hi.x, lo.x);
    tc::tf32_split_lo_fp32(v[1], hi.y, lo.y);
    tc::tf32_split_lo_fp32(v[2], hi.z, lo.z);
    tc::tf32_split_lo_fp32(v[3], hi.w, lo.w);
    unsigned char* base = img + (size_t)gc * Op::kABytes + Op::a_offset(r, akg);
    *reinterpret_cast<float4*>(base) = hi;
    *reinterpret_cast<float4*>(base + Op::kAHalf) = lo;
}

// The split-BF16 A operand of every chunk (32-node tiles): one thread per (chunk, A row
// r, row half akh) writes the 8 chunk rows' weights of that row as one 16-byte core row
// of BF16 pairs for hi and one for lo.  The add-back row stays zero: split BF16 adds
// the centre term back in the epilogue.
__global__ void ens_build_aimg_bf16(const uint32_t* __restrict__ jmap, const int* __restrict__ chunk_tile,
                                    const float4* __restrict__ W, int n, int nchunks, unsigned char* __restrict__ img) {
    using Op = ens::Operands<32, 32, kBf16x3>;   // the A layout does not depend on the members per CTA
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nchunks * 256) return;
    const int akh = (int)(t & 1);
    const int r = (int)((t >> 1) & 127);
    const long gc = t >> 8;
    const int op = ens_a_row_op<32>(r), at = ens_a_row_node<32>(r);
    const long node = (long)chunk_tile[gc] * 32 + at;
    float v[8];
    for (int h = 0; h < 2; ++h) {
        const uint32_t jj = jmap[(gc * 4 + 2 * akh + h) * 32 + at];
        for (int i = 0; i < 4; ++i) {
            const uint32_t j = (jj >> (8 * i)) & 0xffu;
            v[4 * h + i] = (j != 0xffu && node < n) ? reinterpret_cast<const float*>(W + node * 32 + j)[op] : 0.f;
        }
    }
    uint4 hi, lo;
    hi.x = ens::bf16x2_split(v[0], v[1], lo.x);
    hi.y = ens::bf16x2_split(v[2], v[3], lo.y);
    hi.z = ens::bf16x2_split(v[4], v[5], lo.z);
    hi.w = ens::bf16x2_split(v[6], v[7], lo.w);
    unsigned char* base = img + (size_t)gc * Op::kABytes + Op::a_offset(r, akh);
    *reinterpret_cast<uint4*>(base) = hi;
    *reinterpret_cast<uint4*>(base + Op::kAHalf) = lo;
}

static_assert(ens::Operands<32, 64, kTf32x3>::kABytes == 512 * 32 && ens::Operands<16, 64, kTf32x3>::kABytes == 512 * 16,
              "3xTF32 A image: 512 bytes per tile node and chunk");
static_assert(ens::Operands<32, 64, kBf16x3>::kABytes == 8192, "split-BF16 A image: 8 KB per chunk");

// The FP16 A operand of every chunk (32-node tiles): as ens_build_aimg_bf16, with each
// A row's weights times its power-of-two scale AS[node][op] (the row's largest weight at
// 2^13..2^14) before the split, so that hi and lo stay in FP16's normal range.  Row 15
// of a tile's last chunk is the add-back row, as in ens_build_aimg: its weights are the
// operators' row sums (scaled the same way).
__global__ void ens_build_aimg_f16(const uint32_t* __restrict__ jmap, const int* __restrict__ chunk_tile,
                                   const int* __restrict__ row_off, const float4* __restrict__ W,
                                   const float4* __restrict__ RS, const float4* __restrict__ AS, int n, int nchunks,
                                   unsigned char* __restrict__ img) {
    using Op = ens::Operands<32, 32, kFp16x3>;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nchunks * 256) return;
    const int akh = (int)(t & 1);
    const int r = (int)((t >> 1) & 127);
    const long gc = t >> 8;
    const int op = ens_a_row_op<32>(r), at = ens_a_row_node<32>(r);
    const long node = (long)chunk_tile[gc] * 32 + at;
    const float scale = node < n ? reinterpret_cast<const float*>(AS + node)[op] : 1.f;
    float v[8];
    for (int h = 0; h < 2; ++h) {
        const uint32_t jj = jmap[(gc * 4 + 2 * akh + h) * 32 + at];
        for (int i = 0; i < 4; ++i) {
            const uint32_t j = (jj >> (8 * i)) & 0xffu;
            v[4 * h + i] =
                (j != 0xffu && node < n) ? reinterpret_cast<const float*>(W + node * 32 + j)[op] * scale : 0.f;
        }
    }
    const int tile = chunk_tile[gc];
    if (akh == 1 && (gc + 1) * kEnsKc == row_off[tile + 1] && node < n)
        v[7] = reinterpret_cast<const float*>(RS + node)[op] * scale;
    uint4 hi, lo;
    hi.x = ens::f16x2_split(v[0], v[1], lo.x);
    hi.y = ens::f16x2_split(v[2], v[3], lo.y);
    hi.z = ens::f16x2_split(v[4], v[5], lo.z);
    hi.w = ens::f16x2_split(v[6], v[7], lo.w);
    unsigned char* base = img + (size_t)gc * Op::kABytes + Op::a_offset(r, akh);
    *reinterpret_cast<uint4*>(base) = hi;
    *reinterpret_cast<uint4*>(base + Op::kAHalf) = lo;
}

// The largest |value| of each of the four state fields of an FP32 state [node][4 m + f]
// (count values), as FP32 bit patterns (non-negative floats order as their bits): the
// FP16 operands' field scales.  out[0..3] must start at zero.
__global__ void ens_field_max(const float* __restrict__ X, long count, unsigned* __restrict__ out) {
    unsigned m[4] = {0u, 0u, 0u, 0u};
    const long q = count / 4;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < q; e += (long)gridDim.x * blockDim.x) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(X) + e);
        m[0] = max(m[0], __float_as_uint(fabsf(v.x)));
        m[1] = max(m[1], __float_as_uint(fabsf(v.y)));
        m[2] = max(m[2], __float_as_uint(fabsf(v.z)));
        m[3] = max(m[3], __float_as_uint(fabsf(v.w)));
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const unsigned w = __reduce_max_sync(0xffffffffu, m[f]);
        if ((threadIdx.x & 31) == 0 && w) atomicMax(out + f, w);
    }
}

__global__ void ens_invariants_kernel(const float* __restrict__ H32, const double* __restrict__ Hh,
                                      const float4* __restrict__ PT, int n, int members, double gh0,
                                      double* __restrict__ out) {
    // thread (member b = tid % members, node lane = tid / members) strides over nodes
    const int b = threadIdx.x % members;
    const int lanes = blockDim.x / members;
    const int nl = threadIdx.x / members;
    double mass = 0.0, energy = 0.0;
    if (nl < lanes) {
        for (long i = (long)blockIdx.x * lanes + nl; i < n; i += (long)gridDim.x * lanes) {
            const float* r = H32 + i * 4L * members + 4L * b;
            const double u = r[0], v = r[1], w = r[2];
            const double phi = Hh[i * members + b] + gh0;
            const double ghm = (double)reinterpret_cast<const float*>(PT + i * 5)[PT_GHM];
            const double thick = phi - ghm;
            mass += thick;
            energy += 0.5 * thick * (u * u + v * v + w * w) + 0.5 * phi * phi;
        }
    }
    atomicAdd(out + 2 * b, mass);
    atomicAdd(out + 2 * b + 1, energy);
}

// host [members][n][4] FP64 (natural order) <-> device arrays (RCM order)
__global__ void ens_scatter_state(const double* __restrict__ Hin, const int* __restrict__ perm, int n,
                                  int members, float* __restrict__ H32, double* __restrict__ Hh) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * members * 4) return;
    const int f = t & 3;
    const long bi = t >> 2;
    const int b = (int)(bi % members);
    const long i = bi / members;                 // device (RCM) node
    const double v = Hin[((long)b * n + perm[i]) * 4 + f];
    H32[i * 4L * members + 4L * b + f] = (float)v;
    if (f == 3 && Hh) Hh[i * members + b] = v;
}

__global__ void ens_gather_state(const float* __restrict__ H32, const double* __restrict__ Hh,
                                 const int* __restrict__ perm, int n, int members, double* __restrict__ Hout) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * members * 4) return;
    const int f = t & 3;
    const long bi = t >> 2;
    const int b = (int)(bi % members);
    const long i = bi / members;
    const double v = (f == 3 && Hh) ? Hh[i * members + b] : (double)H32[i * 4L * members + 4L * b + f];
    Hout[((long)b * n + perm[i]) * 4 + f] = v;
}

struct Ensemble {
    bool ready = false;
    int members = 0, n = 0, nnbr = 0, mf = 0, nsm = 148;
    double gh0 = 0, dt = 0;
    std::vector<int> perm_h;
    int* perm = nullptr;
    float4* PT = nullptr;
    float4* RS = nullptr;
    float *H32 = nullptr, *D32 = nullptr, *Ka = nullptr, *Kb = nullptr, *F = nullptr, *Kx = nullptr;
    double *Hh = nullptr, *Dh = nullptr, *io = nullptr, *inv = nullptr;
    float* bkH32 = nullptr;
    double* bkHh = nullptr;
    int* err = nullptr;
    // tile tables, one set per tile shape (32 and 16 nodes)
    DevTables tabs[kEnsShapes];
    float4* W = nullptr;         // raw FP32 weights [n][32], only while the A images are built
    float4* AI = nullptr;        // [n] FP16 operands: inverse power-of-two scale of each A row
    unsigned* bmax = nullptr;    // [12] FP16 operands: field maxima of the stepped state, of eval_rhs's, and of
                                 // the state stage 3 writes
    Variant var[kEnsVariants];   // (tile nodes, members per CTA): (32, 64), (32, 32), (16, 64), (16, 32)
    int chosen = -1;
    int prec = kTf32x3;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool timing = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool timed = false;
    double tune_ms[kEnsVariants] = {-1, -1, -1, -1};

    static int shape_of(int tile) { return tile == 32 ? 0 : 1; }

    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        void* ps[] = {perm, PT, RS, AI, bmax, H32, D32, Ka, Kb, F, Kx, Hh, Dh, io, inv, bkH32, bkHh, err, W};
        for (void* p : ps) if (p) cudaFree(p);
        for (DevTables& t : tabs) {
            void* tp[] = {t.row_off, t.rows, t.centre, t.jmap, t.aimg, t.aimg_bf16, t.aimg_f16};
            for (void* p : tp) if (p) cudaFree(p);
            t = DevTables{};
        }
        perm = nullptr; PT = nullptr; RS = nullptr; AI = nullptr; bmax = nullptr;
        H32 = D32 = Ka = Kb = F = Kx = nullptr;
        Hh = Dh = io = inv = nullptr; bkH32 = nullptr; bkHh = nullptr; err = nullptr;
        W = nullptr;
        for (auto& v : var) v = Variant{};
        for (auto& e : ev) { if (e) cudaEventDestroy(e); e = nullptr; }
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        chosen = -1;
        for (double& t : tune_ms) t = -1;
        ready = false;
    }

    EnsArgs args(int mode, int tile, int mpc) const {
        const DevTables& tb = tabs[shape_of(tile)];
        EnsArgs a{};
        a.n = n;
        a.ntiles = tb.ntiles;
        a.members = members;
        a.units = tb.ntiles * (members / mpc);
        a.mf = mf;
        a.row_off = tb.row_off; a.rows = tb.rows;
        a.Aimg = prec == kBf16x3 ? tb.aimg_bf16 : prec == kFp16x3 ? tb.aimg_f16 : tb.aimg;
        a.AI = AI;
        // the field maxima of the state the stage reads: the stepped state, or eval_rhs's
        // split FP16 field maxima: [0..3] what stages 1-3 read (stage 0 copies them in),
        // [4..7] eval_rhs's state, [8..11] the stepped state's (set_state, stage 3)
        a.bmax = mode == 0 ? bmax + 8 : (mode >= 1 && mode <= 3 ? bmax : bmax + 4);
        a.bmax_next = bmax + 8;
        a.bmax_pub = bmax;
        a.centre = tb.centre;
        a.PT = PT;
        a.RS = RS;
        a.H32 = H32; a.Hh = Hh; a.D32 = D32; a.Dh = Dh; a.F = F;
        a.gh0 = (float)gh0;
        a.dt6 = dt / 6.0;
        a.err = err;
        switch (mode) {
            case 0: a.Kin = H32; a.Kout = Ka; a.c = dt / 2.0; break;
            case 1: a.Kin = Ka; a.Kout = Kb; a.c = dt / 2.0; break;
            case 2: a.Kin = Kb; a.Kout = Ka; a.c = dt; break;
            case 3: a.Kin = Ka; a.Kout = nullptr; a.c = dt; break;
            default: a.Kin = Kx; a.Kout = nullptr; a.c = 0.0; break;
        }
        return a;
    }

    template <int T, int MPC, int PREC>
    void launch_v(int mode) {
        using C = EnsCfg<T, MPC, PREC>;
        const EnsArgs a = args(mode, T, MPC);
        const int grid = std::min(a.units, nsm);
        switch (mode) {
            case 0: ens_stage_kernel<T, MPC, kStage0, PREC><<<grid, C::kThreads, C::kSmem, stream>>>(a); break;
            case 1: ens_stage_kernel<T, MPC, kStage1, PREC><<<grid, C::kThreads, C::kSmem, stream>>>(a); break;
            case 2: ens_stage_kernel<T, MPC, kStage2, PREC><<<grid, C::kThreads, C::kSmem, stream>>>(a); break;
            case 3: ens_stage_kernel<T, MPC, kStage3, PREC><<<grid, C::kThreads, C::kSmem, stream>>>(a); break;
            default: ens_stage_kernel<T, MPC, kEvalOnly, PREC><<<grid, C::kThreads, C::kSmem, stream>>>(a); break;
        }
    }

    // split BF16 has 32-node tiles only: usable() keeps it off the 16-node variants
    bool usable(int vi) const { return var[vi].usable && (prec == kTf32x3 || var[vi].tile == 32); }

    void launch(int vi, int mode) {
        const Variant& v = var[vi];
        if (prec == kFp16x3) {
            if (v.mpc == 64) launch_v<32, 64, kFp16x3>(mode);
            else launch_v<32, 32, kFp16x3>(mode);
        } else if (prec == kBf16x3) {
            if (v.mpc == 64) launch_v<32, 64, kBf16x3>(mode);
            else launch_v<32, 32, kBf16x3>(mode);
        } else if (v.tile == 32) {
            if (v.mpc == 64) launch_v<32, 64, kTf32x3>(mode);
            else launch_v<32, 32, kTf32x3>(mode);
        } else {
            if (v.mpc == 64) launch_v<16, 64, kTf32x3>(mode);
            else launch_v<16, 32, kTf32x3>(mode);
        }
        count_launch();
    }

    template <int T, int MPC, int PREC>
    static int set_attrs() {
        const int sm = EnsCfg<T, MPC, PREC>::kSmem;
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, MPC, kStage0, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, MPC, kStage1, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, MPC, kStage2, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, MPC, kStage3, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, MPC, kEvalOnly, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        return SWE_OK;
    }

    int build_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        cudaGraph_t g;
        SWE_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < 4; ++s) launch(chosen, s);
        SWE_CUDA_TRY(cudaStreamEndCapture(stream, &g));
        cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
            graph = nullptr;
            return SWE_ERR_CUDA;
        }
        return SWE_OK;
    }

    // the four field maxima of FP32 state X into out[0..3] (the FP16 operands' scales)
    int field_max(const float* X, unsigned* out) {
        const long count = (long)n * mf;
        SWE_CUDA_TRY(cudaMemsetAsync(out, 0, 4 * sizeof(unsigned), stream));
        const int blocks = (int)std::min<long>(std::max<long>(1, (count / 4 + 255) / 256), 4L * nsm);
        ens_field_max<<<blocks, 256, 0, stream>>>(X, count, out);
        count_launch();
        SWE_CUDA_TRY(cudaGetLastError());
        return SWE_OK;
    }

    int check_err() {
        int h = 0;
        SWE_CUDA_TRY(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SWE_CUDA_TRY(cudaStreamSynchronize(stream));
        if (h) {
            set_error("ensemble kernel: a bounded mbarrier wait ran out (code %d)", h);
            return SWE_ERR_TIMEOUT;
        }
        return SWE_OK;
    }
};

Ensemble g_ens;

int ens_ready() {
    if (!g_ens.ready) {
        set_error("swe_ens_init has not been called");
        return SWE_ERR_STATE;
    }
    return SWE_OK;
}

int tune(Ensemble& E) {
    // time every usable variant on one RK4 step of the live state, restore the state
    const size_t b32 = (size_t)E.n * E.mf * sizeof(float), b64 = (size_t)E.n * E.members * sizeof(double);
    SWE_CUDA_TRY(cudaMemcpyAsync(E.bkH32, E.H32, b32, cudaMemcpyDeviceToDevice, E.stream));
    SWE_CUDA_TRY(cudaMemcpyAsync(E.bkHh, E.Hh, b64, cudaMemcpyDeviceToDevice, E.stream));
    cudaEvent_t e0, e1;
    SWE_CUDA_TRY(cudaEventCreate(&e0));
    SWE_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_i = -1;
    for (int vi = 0; vi < kEnsVariants; ++vi) {
        E.tune_ms[vi] = -1.0;
        if (!E.usable(vi)) continue;
        for (int w = 0; w < 2; ++w)
            for (int s = 0; s < 4; ++s) E.launch(vi, s);
        SWE_CUDA_TRY(cudaEventRecord(e0, E.stream));
        const int reps = 3;
        for (int r = 0; r < reps; ++r)
            for (int s = 0; s < 4; ++s) E.launch(vi, s);
        SWE_CUDA_TRY(cudaEventRecord(e1, E.stream));
        SWE_CUDA_TRY(cudaEventSynchronize(e1));
        SWE_CUDA_TRY(cudaGetLastError());
        float ms = 0.f;
        SWE_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        ms /= reps;
        E.tune_ms[vi] = ms;
        if (ms < best) { best = ms; best_i = vi; }
        SWE_CUDA_TRY(cudaMemcpyAsync(E.H32, E.bkH32, b32, cudaMemcpyDeviceToDevice, E.stream));
        SWE_CUDA_TRY(cudaMemcpyAsync(E.Hh, E.bkHh, b64, cudaMemcpyDeviceToDevice, E.stream));
        // the restored state's field maxima, which the steps above moved on
        SWE_TRY(E.field_max(E.H32, E.bmax + 8));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SWE_TRY(E.check_err());
    if (best_i < 0) {
        set_error("no usable ensemble kernel variant");
        return SWE_ERR_ARG;
    }
    E.chosen = best_i;
    return E.build_graph();
}

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" {

int swe_ens_init(int members, int n, int nnbr, double gh0, double dt, const int* idx, const double* Dx,
                 const double* Dy, const double* Dz, const double* L, const double* x, const double* y,
                 const double* z, const double* f, const double* ghm, const double* p_u, const double* p_v,
                 const double* p_w, const double* gradghm) {
    if (members != 32 && members != 64) { set_error("swe_ens_init: members must be 32 or 64, got %d", members); return SWE_ERR_ARG; }
    if (n <= 0 || nnbr <= 0 || nnbr > 32) { set_error("swe_ens_init: need n > 0 and 1 <= nnbr <= 32"); return SWE_ERR_ARG; }
    if (!idx || !Dx || !Dy || !Dz || !L || !x || !y || !z || !f || !ghm || !p_u || !p_v || !p_w || !gradghm) {
        set_error("swe_ens_init: null array");
        return SWE_ERR_ARG;
    }
    if ((double)n * 4 * members >= 4294967296.0) {
        set_error("swe_ens_init: %d nodes x %d members exceed the 2^32 state values a stage indexes", n, members);
        return SWE_ERR_ARG;
    }
    for (long e = 0; e < (long)n * nnbr; ++e)
        if (idx[e] < 0 || idx[e] >= n) { set_error("swe_ens_init: idx[%ld] = %d out of range", e, idx[e]); return SWE_ERR_INDEX; }
    Ensemble& E = g_ens;
    E.release();
    E.members = members;
    E.n = n;
    E.nnbr = nnbr;
    E.mf = 4 * members;
    E.gh0 = gh0;
    E.dt = dt;
    {
        int dev = 0;
        SWE_CUDA_TRY(cudaGetDevice(&dev));
        SWE_CUDA_TRY(cudaDeviceGetAttribute(&E.nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    // curve order (mapping[new] = old) and the renumbered stencils
    E.perm_h = curve_order(n, x, y, z);
    std::vector<int> inv(n), ridx((size_t)n * nnbr);
    for (int i = 0; i < n; ++i) inv[E.perm_h[i]] = i;
    for (long i = 0; i < n; ++i)
        for (int j = 0; j < nnbr; ++j) ridx[i * nnbr + j] = inv[idx[(long)E.perm_h[i] * nnbr + j]];
    // Static data in FP32, curve order.  The operator row sums that add the centre
    // back (c * sum_k W) are summed from the FP64 weights: the weights themselves are
    // rounded to FP32, which moves each row sum by up to 2^-24 sum_k |W|, and a row sum
    // taken from the rounded weights would add that error times the full state value
    // c at every node and stage.  With the FP64 sums only the centred part sum_k W (X -
    // c), which is small, sees the rounded weights; the operators' annihilation of
    // constants holds to FP64 accuracy (the h error of the batched form after 1000
    // steps drops several-fold).
    std::vector<float> w((size_t)n * 32 * 4, 0.f), pt((size_t)n * kPointStride, 0.f), rs((size_t)n * 4);
    std::vector<float> as((size_t)n * 4), ai((size_t)n * 4);
    std::vector<double> X((size_t)n * 3);
    for (long i = 0; i < n; ++i) {
        const long o = E.perm_h[i];
        double sum[4] = {0, 0, 0, 0};
        for (int j = 0; j < nnbr; ++j) {
            float* q = &w[((size_t)i * 32 + j) * 4];
            const double wd[4] = {Dx[o * nnbr + j], Dy[o * nnbr + j], Dz[o * nnbr + j], L[o * nnbr + j]};
            for (int op = 0; op < 4; ++op) {
                q[op] = (float)wd[op];
                sum[op] += wd[op];
            }
        }
        for (int op = 0; op < 4; ++op) rs[i * 4 + op] = (float)sum[op];
        // FP16 operands: each A row's scale 2^k puts its largest weight at 2^13..2^14
        for (int op = 0; op < 4; ++op) {
            float m = 0.f;
            for (int j = 0; j < nnbr; ++j) m = std::max(m, std::fabs(w[((size_t)i * 32 + j) * 4 + op]));
            int ex = 0;
            if (m > 0.f) std::frexp(m, &ex);
            const int k = m > 0.f ? std::min(60, std::max(-60, 14 - ex)) : 0;
            as[i * 4 + op] = std::ldexp(1.f, k);
            ai[i * 4 + op] = std::ldexp(1.f, -k);
        }
        float* r = &pt[(size_t)i * kPointStride];
        r[PT_X] = (float)x[o]; r[PT_Y] = (float)y[o]; r[PT_Z] = (float)z[o]; r[PT_F] = (float)f[o];
        r[PT_GHM] = (float)ghm[o];
        for (int c = 0; c < 3; ++c) {
            r[PT_PU + c] = (float)p_u[o * 3 + c]; r[PT_PV + c] = (float)p_v[o * 3 + c];
            r[PT_PW + c] = (float)p_w[o * 3 + c]; r[PT_GG + c] = (float)gradghm[o * 3 + c];
        }
        X[3 * i] = x[o]; X[3 * i + 1] = y[o]; X[3 * i + 2] = z[o];
    }
    TileTables tbs[kEnsShapes];
    for (int sh = 0; sh < kEnsShapes; ++sh) tbs[sh] = build_tiles(kEnsShapeNodes[sh], n, nnbr, ridx, X);
    SWE_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
    const size_t s32 = (size_t)n * E.mf * sizeof(float), s64 = (size_t)n * members * sizeof(double);
    auto upload = [](auto** dst, const auto& vec) -> int {
        const size_t bytes = vec.size() * sizeof(vec[0]);
        SWE_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(bytes, 16)));
        if (bytes) SWE_CUDA_TRY(cudaMemcpy(*dst, vec.data(), bytes, cudaMemcpyHostToDevice));
        return SWE_OK;
    };
    SWE_TRY(upload(&E.perm, E.perm_h));
    SWE_TRY(upload(reinterpret_cast<float**>(&E.PT), pt));
    SWE_TRY(upload(reinterpret_cast<float**>(&E.RS), rs));
    SWE_TRY(upload(reinterpret_cast<float**>(&E.AI), ai));
    float4* ascale = nullptr;    // the A-row scales themselves, while the FP16 image is built
    SWE_TRY(upload(reinterpret_cast<float**>(&ascale), as));
    for (int sh = 0; sh < kEnsShapes; ++sh) {
        DevTables& d = E.tabs[sh];
        d.ntiles = tbs[sh].ntiles;
        d.max_rows = tbs[sh].max_rows;
        d.nchunks = tbs[sh].nchunks;
        SWE_TRY(upload(&d.row_off, tbs[sh].row_off));
        SWE_TRY(upload(&d.rows, tbs[sh].rows));
        SWE_TRY(upload(&d.jmap, tbs[sh].jmap));
        SWE_TRY(upload(&d.centre, tbs[sh].centre));
    }
    SWE_TRY(upload(reinterpret_cast<float**>(&E.W), w));
    // A images: 3xTF32 for both tile shapes (about 4 KB per node for 32-node tiles,
    // 3 KB for 16-node tiles) and split BF16 for 32-node tiles (2 KB per node), built
    // on the device from the tables and the weights
    for (int sh = 0; sh < kEnsShapes; ++sh) {
        const int T = kEnsShapeNodes[sh];
        const TileTables& tb = tbs[sh];
        std::vector<int> chunk_tile(tb.nchunks);
        for (int tile = 0; tile < tb.ntiles; ++tile)
            for (int c = tb.row_off[tile] / kEnsKc; c < tb.row_off[tile + 1] / kEnsKc; ++c) chunk_tile[c] = tile;
        int* dct = nullptr;
        SWE_TRY(upload(&dct, chunk_tile));
        const size_t bytes = (size_t)tb.nchunks * 512 * T;
        const int rc = [&]() -> int {
            SWE_CUDA_TRY(cudaMalloc(&E.tabs[sh].aimg, std::max<size_t>(bytes, 16)));
            const long work = (long)tb.nchunks * 16 * T;
            const int blocks = (int)std::max<long>(1, (work + 255) / 256);
            DevTables& d = E.tabs[sh];
            if (T == 32) {
                ens_build_aimg<32><<<blocks, 256, 0, E.stream>>>(d.jmap, dct, d.row_off, E.W, E.RS, n, tb.nchunks, d.aimg);
                SWE_CUDA_TRY(cudaMalloc(&d.aimg_bf16, std::max<size_t>((size_t)tb.nchunks * 8192, 16)));
                const long wb = (long)tb.nchunks * 256;
                ens_build_aimg_bf16<<<(int)std::max<long>(1, (wb + 255) / 256), 256, 0, E.stream>>>(d.jmap, dct, E.W, n,
                                                                                               tb.nchunks, d.aimg_bf16);
                SWE_CUDA_TRY(cudaMalloc(&d.aimg_f16, std::max<size_t>((size_t)tb.nchunks * 8192, 16)));
                ens_build_aimg_f16<<<(int)std::max<long>(1, (wb + 255) / 256), 256, 0, E.stream>>>(
                    d.jmap, dct, d.row_off, E.W, E.RS, ascale, n, tb.nchunks, d.aimg_f16);
            } else {
                ens_build_aimg<16><<<blocks, 256, 0, E.stream>>>(d.jmap, dct, d.row_off, E.W, E.RS, n, tb.nchunks, d.aimg);
            }
            SWE_CUDA_TRY(cudaGetLastError());
            SWE_CUDA_TRY(cudaStreamSynchronize(E.stream));
            return SWE_OK;
        }();
        cudaFree(dct);
        if (rc != SWE_OK) { cudaFree(ascale); return rc; }
    }
    // the stage kernels read only the images: the raw weights are not kept
    cudaFree(E.W);
    E.W = nullptr;
    cudaFree(ascale);
    for (float** p : {&E.H32, &E.D32, &E.Ka, &E.Kb, &E.F, &E.Kx, &E.bkH32}) SWE_CUDA_TRY(cudaMalloc(p, s32));
    for (double** p : {&E.Hh, &E.Dh, &E.bkHh}) SWE_CUDA_TRY(cudaMalloc(p, s64));
    SWE_CUDA_TRY(cudaMalloc(&E.io, (size_t)n * members * 4 * sizeof(double)));
    SWE_CUDA_TRY(cudaMalloc(&E.inv, 2 * members * sizeof(double)));
    SWE_CUDA_TRY(cudaMalloc(&E.err, sizeof(int)));
    SWE_CUDA_TRY(cudaMemset(E.err, 0, sizeof(int)));
    for (float* p : {E.H32, E.D32, E.Ka, E.Kb, E.F, E.Kx}) SWE_CUDA_TRY(cudaMemset(p, 0, s32));
    for (double* p : {E.Hh, E.Dh}) SWE_CUDA_TRY(cudaMemset(p, 0, s64));
    const int shapes[kEnsVariants][2] = {{32, 64}, {32, 32}, {16, 64}, {16, 32}};
    for (int vi = 0; vi < kEnsVariants; ++vi) {
        E.var[vi].tile = shapes[vi][0];
        E.var[vi].mpc = shapes[vi][1];
        E.var[vi].usable = members % shapes[vi][1] == 0;
    }
    SWE_TRY((Ensemble::set_attrs<32, 32, kTf32x3>()));
    SWE_TRY((Ensemble::set_attrs<32, 64, kTf32x3>()));
    SWE_TRY((Ensemble::set_attrs<16, 32, kTf32x3>()));
    SWE_TRY((Ensemble::set_attrs<16, 64, kTf32x3>()));
    SWE_TRY((Ensemble::set_attrs<32, 32, kBf16x3>()));
    SWE_TRY((Ensemble::set_attrs<32, 64, kBf16x3>()));
    SWE_TRY((Ensemble::set_attrs<32, 32, kFp16x3>()));
    SWE_TRY((Ensemble::set_attrs<32, 64, kFp16x3>()));
    SWE_CUDA_TRY(cudaMalloc(&E.bmax, 12 * sizeof(unsigned)));
    SWE_CUDA_TRY(cudaMemset(E.bmax, 0, 12 * sizeof(unsigned)));
    E.prec = kTf32x3;
    E.ready = true;
    // default choice until tuned: 32-node tiles, all members in one CTA
    E.chosen = E.var[0].usable ? 0 : 1;
    return E.build_graph();
}

int swe_ens_set_state(const double* H) {
    SWE_TRY(ens_ready());
    if (!H) { set_error("swe_ens_set_state: null H"); return SWE_ERR_ARG; }
    Ensemble& E = g_ens;
    const long total = (long)E.n * E.members * 4;
    SWE_CUDA_TRY(cudaMemcpyAsync(E.io, H, total * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    ens_scatter_state<<<ceil_div(total, 256), 256, 0, E.stream>>>(E.io, E.perm, E.n, E.members, E.H32, E.Hh);
    count_launch();
    SWE_TRY(E.field_max(E.H32, E.bmax + 8));
    SWE_CUDA_TRY(cudaGetLastError());
    return SWE_OK;
}

int swe_ens_get_state(double* H) {
    SWE_TRY(ens_ready());
    if (!H) { set_error("swe_ens_get_state: null H"); return SWE_ERR_ARG; }
    Ensemble& E = g_ens;
    const long total = (long)E.n * E.members * 4;
    ens_gather_state<<<ceil_div(total, 256), 256, 0, E.stream>>>(E.H32, E.Hh, E.perm, E.n, E.members, E.io);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    SWE_CUDA_TRY(cudaMemcpyAsync(H, E.io, total * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    return E.check_err();
}

int swe_ens_eval_rhs(const double* K, double* Fh) {
    SWE_TRY(ens_ready());
    if (!K || !Fh) { set_error("swe_ens_eval_rhs: null K or F"); return SWE_ERR_ARG; }
    Ensemble& E = g_ens;
    const long total = (long)E.n * E.members * 4;
    SWE_CUDA_TRY(cudaMemcpyAsync(E.io, K, total * sizeof(double), cudaMemcpyHostToDevice, E.stream));
    ens_scatter_state<<<ceil_div(total, 256), 256, 0, E.stream>>>(E.io, E.perm, E.n, E.members, E.Kx, nullptr);
    count_launch();
    SWE_TRY(E.field_max(E.Kx, E.bmax + 4));
    E.launch(E.chosen, kEvalOnly);
    ens_gather_state<<<ceil_div(total, 256), 256, 0, E.stream>>>(E.F, nullptr, E.perm, E.n, E.members, E.io);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    SWE_CUDA_TRY(cudaMemcpyAsync(Fh, E.io, total * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    return E.check_err();
}

int swe_ens_step(int nsteps) {
    SWE_TRY(ens_ready());
    if (nsteps < 0) { set_error("swe_ens_step: nsteps < 0"); return SWE_ERR_ARG; }
    Ensemble& E = g_ens;
    if (E.timing) {
        for (auto& e : E.ev) if (!e) SWE_CUDA_TRY(cudaEventCreate(&e));
        SWE_CUDA_TRY(cudaEventRecord(E.ev[0], E.stream));
    }
    for (int s = 0; s < nsteps; ++s) SWE_CUDA_TRY(cudaGraphLaunch(E.graph, E.stream));
    count_launch(4LL * nsteps);
    if (E.timing) {
        SWE_CUDA_TRY(cudaEventRecord(E.ev[1], E.stream));
        E.timed = true;
    }
    return SWE_OK;
}

int swe_ens_stage(int substep_id) {
    SWE_TRY(ens_ready());
    if (substep_id < 0 || substep_id > 3) { set_error("swe_ens_stage: substep_id %d not in 0..3", substep_id); return SWE_ERR_ARG; }
    g_ens.launch(g_ens.chosen, substep_id);
    SWE_CUDA_TRY(cudaGetLastError());
    return SWE_OK;
}

int swe_ens_tune(double* ms_per_step) {
    SWE_TRY(ens_ready());
    SWE_TRY(tune(g_ens));
    if (ms_per_step)
        for (int vi = 0; vi < kEnsVariants; ++vi) ms_per_step[vi] = g_ens.tune_ms[vi];
    return SWE_OK;
}

int swe_ens_use_variant(int tile_nodes, int members_per_cta) {
    SWE_TRY(ens_ready());
    if (tile_nodes != 32 && tile_nodes != 16) {
        set_error("swe_ens_use_variant: tiles have 32 or 16 nodes, got %d", tile_nodes);
        return SWE_ERR_ARG;
    }
    if (members_per_cta != 32 && members_per_cta != 64) {
        set_error("swe_ens_use_variant: members per CTA must be 32 or 64, got %d", members_per_cta);
        return SWE_ERR_ARG;
    }
    for (int vi = 0; vi < kEnsVariants; ++vi) {
        const Variant& v = g_ens.var[vi];
        if (v.tile != tile_nodes || v.mpc != members_per_cta) continue;
        if (!v.usable) {
            set_error("swe_ens_use_variant: %d members per CTA does not divide %d members", members_per_cta,
                      g_ens.members);
            return SWE_ERR_ARG;
        }
        if (!g_ens.usable(vi)) {
            set_error("swe_ens_use_variant: split BF16 runs on 32-node tiles only");
            return SWE_ERR_ARG;
        }
        g_ens.chosen = vi;
        return g_ens.build_graph();
    }
    set_error("swe_ens_use_variant: no variant (%d, %d)", tile_nodes, members_per_cta);
    return SWE_ERR_ARG;
}

int swe_ens_config(int* out) {
    SWE_TRY(ens_ready());
    if (!out) { set_error("swe_ens_config: null out"); return SWE_ERR_ARG; }
    const Variant& v = g_ens.var[g_ens.chosen];
    const DevTables& tb = g_ens.tabs[Ensemble::shape_of(v.tile)];
    out[0] = v.tile;
    out[1] = v.mpc;
    out[2] = tb.max_rows;
    out[3] = tb.ntiles;
    out[4] = g_ens.prec;
    out[5] = tb.nchunks;
    return SWE_OK;
}

int swe_ens_set_precision(int precision) {
    SWE_TRY(ens_ready());
    if (precision != kTf32x3 && precision != kBf16x3 && precision != kFp16x3) {
        set_error("swe_ens_set_precision: %d is none of 0 (3xTF32), 1 (split BF16), 2 (split FP16)", precision);
        return SWE_ERR_ARG;
    }
    SWE_CUDA_TRY(cudaStreamSynchronize(g_ens.stream));
    g_ens.prec = precision;
    // split FP16 reads the field maxima of the current state, which the other precisions
    // do not keep up to date while they step
    if (precision == kFp16x3) SWE_TRY(g_ens.field_max(g_ens.H32, g_ens.bmax + 8));
    for (double& t : g_ens.tune_ms) t = -1.0;
    // the 16-bit splits have 32-node tiles only: keep the members per CTA, move to 32-node tiles
    if (!g_ens.usable(g_ens.chosen))
        for (int vi = 0; vi < kEnsVariants; ++vi)
            if (g_ens.var[vi].tile == 32 && g_ens.var[vi].mpc == g_ens.var[g_ens.chosen].mpc) g_ens.chosen = vi;
    return g_ens.build_graph();
}

int swe_ens_invariants(double* out) {
    SWE_TRY(ens_ready());
    if (!out) { set_error("swe_ens_invariants: null out"); return SWE_ERR_ARG; }
    Ensemble& E = g_ens;
    SWE_CUDA_TRY(cudaMemsetAsync(E.inv, 0, 2 * E.members * sizeof(double), E.stream));
    const int threads = 256;
    ens_invariants_kernel<<<std::min(ceil_div(E.n, threads / E.members), 592), threads, 0, E.stream>>>(
        E.H32, E.Hh, E.PT, E.n, E.members, E.gh0, E.inv);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    SWE_CUDA_TRY(cudaMemcpyAsync(out, E.inv, 2 * E.members * sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    SWE_CUDA_TRY(cudaStreamSynchronize(E.stream));
    const double area = 4.0 * 3.14159265358979323846 / (double)E.n;
    for (int t = 0; t < 2 * E.members; ++t) out[t] *= area;
    // NaN/Inf watchdog per member: one non-finite value in a member's state makes its sums non-finite
    for (int b = 0; b < E.members; ++b)
        if (!std::isfinite(out[2 * b]) || !std::isfinite(out[2 * b + 1])) {
            set_error("swe_ens_invariants: member %d's state holds NaN or Inf", b);
            return SWE_ERR_NONFINITE;
        }
    return SWE_OK;
}

int swe_ens_sync(void) {
    SWE_TRY(ens_ready());
    SWE_CUDA_TRY(cudaStreamSynchronize(g_ens.stream));
    return g_ens.check_err();
}

int swe_ens_set_timing(int enabled) {
    SWE_TRY(ens_ready());
    SWE_CUDA_TRY(cudaStreamSynchronize(g_ens.stream));
    g_ens.timing = enabled != 0;
    g_ens.timed = false;
    return SWE_OK;
}

int swe_ens_last_timings(double* out) {
    SWE_TRY(ens_ready());
    if (!out) { set_error("swe_ens_last_timings: null out"); return SWE_ERR_ARG; }
    SWE_CUDA_TRY(cudaStreamSynchronize(g_ens.stream));
    out[0] = 0.0;
    if (g_ens.timed) {
        float ms = 0.f;
        SWE_CUDA_TRY(cudaEventElapsedTime(&ms, g_ens.ev[0], g_ens.ev[1]));
        out[0] = ms * 1e-3;
    }
    return SWE_OK;
}

void* swe_ens_stream(void) { return g_ens.ready ? (void*)g_ens.stream : nullptr; }

int swe_ens_finalize(void) {
    if (g_ens.stream) cudaStreamSynchronize(g_ens.stream);
    g_ens.release();
    return SWE_OK;
}

}  // extern "C"
