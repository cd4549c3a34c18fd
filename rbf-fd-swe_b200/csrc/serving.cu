// Serving form: swe_srv_* entry points of include/swe_b200.h.
//
// Forecast requests (a grid, 1-32 members, a number of RK4 steps, initial
// states) arrive while others run.  A host scheduler thread admits them as
// device memory frees up (first fit in one arena of the configured HBM budget),
// uploads their states on a copy stream, and appends their work to a queue:
// round-robin over the active requests, one RK4 stage (node chunks x blocks of
// two members) per request per round, at most two steps ahead of a request's
// progress, so that new requests join the mix at once.  One persistent kernel --
// one CTA per SM slot -- claims work items from that queue (kept in device
// memory and published by copies on the copy stream, so nothing polls across
// PCIe), waits (bounded) until the chunks its stencils reach have completed the
// request's previous stage, runs the plain form's fused FP64 stage math on the
// chunk for its members, and publishes completion counters; the last item of
// a request raises its completion flag in host memory.  Each work item runs the
// plain form's node-per-lane split (stage_lane.cuh): two lanes per node over a
// tile-transposed copy of the grid's weights and indices, each weight and index
// loaded once for the item's two members; every member's sums run in the same
// order as for a member alone, so a request's result does not depend on what it
// was mixed with.
//
// Waits are bounded (%globaltimer): an idle kernel exits after a while (the
// scheduler relaunches it when work arrives) and a dependency that is never
// met ends the kernel with an error flag instead of hanging the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "stage_kernel.cuh"
#include "stage_lane.cuh"
#include "pack.cuh"

namespace swe {
namespace srv {

struct Item {            // one queue entry (16 bytes)
    int slot;            // request slot
    int q;               // stage index within the request: step * 4 + stage
    int chunk;           // node chunk [chunk * chunk_nodes, ...)
    int member;          // first ensemble member of the item's block (kSrvMB members)
};

struct alignas(16) ReqDesc {   // device table entry of an admitted request
    const uint4* W;      // grid: packed weights
    const int4* idx;     // grid: packed stencil indices
    const double* PT;    // grid: pointwise records
    const uint4* Wl;     // grid: tile-transposed weights (node-per-lane split)
    const int* idxl;     // grid: tile-transposed stencil indices
    int n;               // nodes
    int nnbr;            // stencil slots in use (slot 31 of 31-neighbour stencils is padding)
    int members;
    int chunk_nodes;     // nodes per work item
    int per_stage;       // items per stage: chunks x member blocks
    int nchunks;         // node chunks of the grid
    int reach;           // chunks a chunk's stencils reach on either side
    int* cdone;          // [members][nchunks]: stages completed by each chunk of each member
    int total;           // items of the whole request
    int id;              // request id (written into the completion flag)
    int cancelled;
    double gh0, dt;
    double* H;           // [members][n][4]
    double* Ka;
    double* Kb;
    double* D;
};

struct Shared {          // host-mapped block the kernel writes (posted stores only)
    volatile int error;            // kernel-side error code
    volatile int error_request;    // request whose dependency wait ran out (error 2)
    volatile long long progress;   // items completed (approximate mirror)
};

struct DevCtl {          // device-resident control words the host sets by async copies
    long long tail;      // items published by the host
    int stop;            // host asks the kernel to exit
    int pad;
    unsigned long long dep_ns;   // dependency wait limit
};

constexpr int kThreads = kStageThreads;         // 8 warps x 4 nodes
static_assert(sizeof(ReqDesc) % 16 == 0 && sizeof(ReqDesc) / 16 <= kStageThreads, "descriptor copy");
constexpr unsigned long long kIdleNs = 20ull * 1000 * 1000;          // idle exit after 20 ms
constexpr unsigned long long kDepNs = 10ull * 1000 * 1000 * 1000;    // default dependency wait limit 10 s

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void load_row_cg(const double* p, double (&v)[4]) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// One warp, 16 nodes [base, base + 16) of one member and one stage, two lanes per
// node: the node-per-lane stage kernel's math and data movement (stage_lane.cuh),
// with L2-coherent loads of everything the kernel itself writes (states change
// between stages inside one launch).  Nodes at or past `end` belong to another
// work item (or pad the last tile): they are computed on valid rows and not stored.
constexpr int kSrvLpn = 2, kSrvNpw = 32 / kSrvLpn;
constexpr int kSrvMB = 2;   // members per work item: each weight and index is loaded once for them
static_assert(kSrvMB == 2, "serve_kernel dispatches blocks of one or two members");
// pointwise RHS and RK combine of node i of one member
__device__ __forceinline__ void serve_epilogue(const ReqDesc& r, int stage, long i, const double (&acc)[16], double* __restrict__ Hm,
                               const double* __restrict__ Kin, double* __restrict__ Kout, double* __restrict__ Dm) {
    double q[4], F[4];
    load_row_cg(Kin + 4 * i, q);
    pointwise_rhs(acc, q, r.PT + i * kPointStride, r.gh0, F);
    const double dt = r.dt;
    if (stage == 0) {
        double kn[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) kn[x] = Quad<double>::axpy(q[x], dt / 2.0, F[x]);
        Quad<double>::store_row(Dm + 4 * i, F);
        Quad<double>::store_row(Kout + 4 * i, kn);
    } else {
        double h[4], d[4];
        load_row_cg(Hm + 4 * i, h);
        load_row_cg(Dm + 4 * i, d);
        if (stage < 3) {
            const double c = stage == 1 ? dt / 2.0 : dt;
            double kn[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                d[x] = Quad<double>::axpy(d[x], 2.0, F[x]);
                kn[x] = Quad<double>::axpy(h[x], c, F[x]);
            }
            Quad<double>::store_row(Dm + 4 * i, d);
            Quad<double>::store_row(Kout + 4 * i, kn);
        } else {
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                d[x] = Quad<double>::axpy(d[x], 1.0, F[x]);
                h[x] = Quad<double>::update_h(h[x], dt / 6.0, d[x]);
            }
            Quad<double>::store_row(Hm + 4 * i, h);
        }
    }
}

// MB members m = 0 .. MB-1 of one request; member m's arrays start at + m * moff
template <int MB>
__device__ void serve_lanes(const ReqDesc& r, int stage, long base, long end, long moff, double* __restrict__ Hm,
                            double* __restrict__ Kam, double* __restrict__ Kbm, double* __restrict__ Dm, int lane) {
    const double* Kin = stage == 0 ? Hm : stage == 1 ? Kam : stage == 2 ? Kbm : Kam;
    double* Kout = stage == 0 ? Kam : stage == 1 ? Kbm : Kam;
    const int tl = lane % kSrvNpw, sub = lane / kSrvNpw;
    const long i = base + tl;
    const long tile = i / kLaneTile;
    const int t = (int)(i % kLaneTile);
    const int* ip = r.idxl + (tile * kSlots + sub) * kLaneTile + t;
    const uint4* wp = r.Wl + (tile * kSlots + sub) * 2 * kLaneTile + t;
    double acc[MB][16];
#pragma unroll
    for (int m = 0; m < MB; ++m)
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[m][q] = 0.0;
#pragma unroll
    for (int jj = 0; jj < kSlots / kSrvLpn; ++jj) {
        // a padding slot (zero weights) in a lane's last iteration moves no bytes
        if (jj == kSlots / kSrvLpn - 1 && jj * kSrvLpn + sub >= r.nnbr) continue;
        const int p = lane::ld_stream(ip + jj * kSrvLpn * kLaneTile);
        double w[4];
        lane::weights(wp + jj * kSrvLpn * 2 * kLaneTile, w);
#pragma unroll
        for (int m = 0; m < MB; ++m) {
            double kv[4];
            load_row_cg(Kin + m * moff + 4L * p, kv);
#pragma unroll
            for (int op = 0; op < 4; ++op)
#pragma unroll
                for (int f = 0; f < 4; ++f) acc[m][op * 4 + f] += w[op] * kv[f];
        }
    }
#pragma unroll
    for (int m = 0; m < MB; ++m)
#pragma unroll
        for (int o = kSrvNpw; o < 32; o <<= 1)
#pragma unroll
            for (int q = 0; q < 16; ++q) acc[m][q] += __shfl_xor_sync(0xffffffffu, acc[m][q], o);
    if (sub != 0 || i >= end) return;
#pragma unroll
    for (int m = 0; m < MB; ++m)
        serve_epilogue(r, stage, i, acc[m], Hm + m * moff, Kin + m * moff, Kout + m * moff, Dm + m * moff);
}

// Exit is collective: the first CTA that has found the queue empty for kIdleNs
// raises *exiting; from then on no CTA claims work (items already claimed are
// finished), so every launch runs at full width and the host relaunches, with
// *exiting cleared, once the kernel has ended and work is queued again.
// The queue, its tail and the stop word live in device memory (the host
// publishes them with copies on its copy stream), so polling CTAs never read
// host memory across PCIe; the kernel only posts stores to host memory
// (completion flags and counters).
__global__ void __launch_bounds__(kThreads, 2)
serve_kernel(Shared* ctl, const DevCtl* dctl, const Item* __restrict__ ring, long long ring_cap,
             unsigned long long* head, const ReqDesc* __restrict__ reqs, int* done, int* flags, int* mdone,
             unsigned long long* items_done, int* exiting, int* kerr) {
    __shared__ long long s_pos;
    __shared__ Item s_item;
    __shared__ int s_ok;
    __shared__ ReqDesc s_req;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long idle_since = globaltimer();
    while (true) {
        if (threadIdx.x == 0) {
            long long got = -1;
            while (true) {
                if (*(volatile const int*)&dctl->stop || *(volatile int*)kerr || *(volatile int*)exiting) break;
                const unsigned long long h = *(volatile unsigned long long*)head;
                const long long t = *(volatile const long long*)&dctl->tail;
                if ((long long)h < t) {
                    if (atomicCAS(head, h, h + 1) == h) { got = (long long)h; break; }
                    continue;
                }
                if (globaltimer() - idle_since > kIdleNs) {           // idle: end this launch everywhere
                    atomicExch(exiting, 1);
                    break;
                }
                __nanosleep(2000);
            }
            s_pos = got;
            if (got >= 0) {
                const int4 v = __ldcg(reinterpret_cast<const int4*>(ring + got % ring_cap));
                s_item.slot = v.x;
                s_item.q = v.y;
                s_item.chunk = v.z;
                s_item.member = v.w;
            }
        }
        __syncthreads();
        if (s_pos < 0) return;
        const Item it = s_item;
        // slots are reused by later requests: read the descriptor through L2
        if (threadIdx.x < (int)(sizeof(ReqDesc) / 16))
            reinterpret_cast<uint4*>(&s_req)[threadIdx.x] =
                __ldcg(reinterpret_cast<const uint4*>(reqs + it.slot) + threadIdx.x);
        __syncthreads();
        const ReqDesc& r = s_req;
        // dependency: the member's chunks within reach of this one (the rows its
        // stencils read) have completed the previous stage.  That also orders the
        // writes: a chunk's stage q overwrites the K buffer stage q - 2 wrote, and its
        // neighbours finished reading that buffer in stage q - 1.
        const int mb = min(kSrvMB, r.members - it.member);   // members of this item
        if (threadIdx.x == 0) {
            s_ok = 1;
            const int* cd = r.cdone + (long)it.member * r.nchunks;
            const int c_lo = max(0, it.chunk - r.reach), c_hi = min(r.nchunks - 1, it.chunk + r.reach);
            const unsigned long long limit = *(volatile const unsigned long long*)&dctl->dep_ns;
            const unsigned long long t0 = globaltimer();
            // plain loads (served by L2) with exponential backoff
            unsigned ns = 64;
            auto ready = [&]() {
                for (int m = 0; m < mb; ++m)
                    for (int c = c_lo; c <= c_hi; ++c)
                        if (*(volatile const int*)(cd + (long)m * r.nchunks + c) < it.q) return false;
                return true;
            };
            while (!ready()) {
                if (*(volatile const int*)&dctl->stop) { s_ok = 0; break; }
                if (globaltimer() - t0 > limit) {
                    s_ok = 0;
                    if (atomicExch(kerr, 2) == 0) ctl->error_request = r.id;
                    ctl->error = 2;
                    break;
                }
                __nanosleep(ns);
                ns = ns < 4096 ? 2 * ns : ns;
            }
            __threadfence();
        }
        __syncthreads();
        if (!s_ok) return;
        if (!r.cancelled) {
            const int stage = it.q & 3;
            const long off = 4L * r.n * it.member;
            const long begin = (long)it.chunk * r.chunk_nodes;
            const long end = min((long)r.n, begin + r.chunk_nodes);
            // chunks start on 32-node tiles, so a warp's 16 nodes lie in one tile
            const long moff = 4L * r.n;
            for (long base = begin + warp * (long)kSrvNpw; base < end; base += kStageWarps * (long)kSrvNpw) {
                if (mb == kSrvMB)
                    serve_lanes<kSrvMB>(r, stage, base, end, moff, r.H + off, r.Ka + off, r.Kb + off, r.D + off, lane);
                else
                    serve_lanes<1>(r, stage, base, end, moff, r.H + off, r.Ka + off, r.Kb + off, r.D + off, lane);
            }
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            // this chunk of these members has completed stage index q
            for (int m = 0; m < mb; ++m)
                *(volatile int*)(r.cdone + (long)(it.member + m) * r.nchunks + it.chunk) = it.q + 1;
            __threadfence();
            const int c = atomicAdd(done + it.slot, 1) + 1;
            const unsigned long long d = atomicAdd(items_done, 1ull) + 1;
            if ((d & 63) == 0) ctl->progress = (long long)d;
            // the scheduler paces its appends on a per-request mirror in host memory,
            // pushed out when a stage's worth of items has completed
            if (c % r.per_stage == 0) {
                ((volatile int*)mdone)[it.slot] = c;
                __threadfence_system();
            }
            if (c == r.total) {
                __threadfence_system();
                ((volatile int*)flags)[it.slot] = r.id;
                __threadfence_system();
            }
        }
        idle_since = globaltimer();
    }
}

// ---------------------------------------------------------------------------
// Host side

struct Grid {
    int n, nnbr;
    int reach = 0;          // work-item chunks a chunk's stencils reach on either side
    double gh0, dt;
    void* W = nullptr;
    int* idx = nullptr;
    void* PT = nullptr;
    void* Wl = nullptr;     // tile-transposed copies for the node-per-lane split
    int* idxl = nullptr;
};

struct Request {
    int id, grid, members, nsteps, slot = -1;
    size_t offset = 0, bytes = 0;
    size_t state_bytes = 0;              // members * n * 4 doubles
    std::vector<double> host;            // pageable copy of the states (when the pinned pool is full)
    double* pinned = nullptr;            // states in the pinned pool (initial, later final)
    size_t pin_off = 0;
    cudaEvent_t ev = nullptr;            // completion of its current upload / download
    int next_stage = 0;                  // stage indices (4 per RK4 step) appended so far
    long long appended = 0;              // items appended so far
    enum State { PENDING, UPLOADING, RUNNING, DRAINING, DONE, CANCELLED, FAILED } state = PENDING;
    long long withhold_q = -1;           // test hook: stage index whose first item is never queued
    double t_submit = 0, t_admit = 0, t_done = 0;
    bool cancel_req = false;
};

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Server {
    bool running = false;
    int device = 0, sms = 0, per_sm = 0, max_slots = 0;
    size_t budget = 0, in_use = 0, peak = 0;
    char* arena = nullptr;
    std::map<size_t, size_t> free_blocks;         // offset -> size
    char* pin = nullptr;                          // pinned staging pool for state transfers
    size_t pin_size = 0;
    std::map<size_t, size_t> pin_free;
    Shared* ctl = nullptr;                        // mapped (kernel -> host)
    DevCtl* dctl = nullptr;                       // device (host -> kernel by copies)
    DevCtl* hctl = nullptr;                       // pinned staging of dctl
    Item* ring = nullptr;                         // device queue
    Item* ring_h = nullptr;                       // pinned staging of the queue
    int* kerr = nullptr;                          // device error word
    long long ring_cap = 0, tail = 0, published = 0;
    int* flags = nullptr;                         // mapped [max_slots]
    int* mdone = nullptr;                         // mapped [max_slots]: items done per slot
    unsigned long long* head = nullptr;           // device
    unsigned long long* items_done = nullptr;     // device
    int* exiting = nullptr;                       // device
    ReqDesc* reqs_d = nullptr;                    // device
    int* done_d = nullptr;                        // device
    std::vector<int> free_slots;
    std::vector<Grid> grids;
    std::map<int, Request> requests;
    std::deque<int> pending;
    std::vector<int> active;                      // slots order for round-robin
    int next_id = 0;
    long long failures = 0;                       // dependency-wait failures recovered from
    long long withhold_next_q = -1;               // test hook armed for the next submission
    cudaStream_t kstream = nullptr, cstream = nullptr, pstream = nullptr;
    long long launches = 0, admitted = 0, completed = 0;
    std::thread worker;
    std::mutex mu;
    std::atomic<bool> quit{false};
    std::string fatal;
    bool trace = getenv("SWE_SRV_TRACE") != nullptr;   // scheduler trace on stderr
    double t0 = now_s(), last_trace = 0.0;

    // first-fit allocation in a free list (offset -> size)
    static bool fl_alloc(std::map<size_t, size_t>& fl, size_t bytes, size_t& off) {
        for (auto it = fl.begin(); it != fl.end(); ++it) {
            if (it->second >= bytes) {
                off = it->first;
                const size_t rest = it->second - bytes;
                const size_t noff = it->first + bytes;
                fl.erase(it);
                if (rest) fl[noff] = rest;
                return true;
            }
        }
        return false;
    }
    static void fl_release(std::map<size_t, size_t>& fl, size_t off, size_t bytes) {
        auto it = fl.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != fl.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            fl.erase(nx);
        }
        if (it != fl.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                fl.erase(it);
            }
        }
    }
    bool alloc(size_t bytes, size_t& off) {
        if (!fl_alloc(free_blocks, bytes, off)) return false;
        in_use += bytes;
        peak = std::max(peak, in_use);
        return true;
    }
    void release(size_t off, size_t bytes) {
        in_use -= bytes;
        fl_release(free_blocks, off, bytes);
    }
    // pinned staging of one request's states (falls back to pageable memory)
    void stage_host(Request& r, const double* src) {
        const size_t b = (r.state_bytes + 255) / 256 * 256;
        if (pin && fl_alloc(pin_free, b, r.pin_off)) {
            r.pinned = reinterpret_cast<double*>(pin + r.pin_off);
            if (src) memcpy(r.pinned, src, r.state_bytes);
        } else {
            r.pinned = nullptr;
            if (src) r.host.assign(src, src + r.state_bytes / sizeof(double));
            else r.host.resize(r.state_bytes / sizeof(double));
        }
    }
    void unstage_host(Request& r) {
        if (r.pinned) fl_release(pin_free, r.pin_off, (r.state_bytes + 255) / 256 * 256);
        r.pinned = nullptr;
        std::vector<double>().swap(r.host);
    }
    const double* host_states(const Request& r) const { return r.pinned ? r.pinned : r.host.data(); }

    static size_t state_bytes(int n, int members) {
        const size_t one = (size_t)n * 4 * sizeof(double) * members;
        const size_t prog = (size_t)members * ((n + chunk_nodes(n) - 1) / chunk_nodes(n)) * sizeof(int);
        return ((one + 255) / 256 * 256) * 4 + (prog + 255) / 256 * 256;   // H, Ka, Kb, D, chunk progress
    }
    // nodes per work item: about 2048 (tens of microseconds of FP64 stage work),
    // fewer on small grids so that they still split into several items
    static int chunk_nodes(int n) {
        int c = std::min(2048, std::max(256, n / 8));
        c = (c + 31) / 32 * 32;
        return std::min(c, n);
    }
    static constexpr int kLookaheadStages = 8;   // two RK4 steps

    bool kernel_running() { return cudaStreamQuery(kstream) == cudaErrorNotReady; }

    void launch_kernel() {
        cudaMemsetAsync(exiting, 0, sizeof(int), kstream);
        serve_kernel<<<sms * std::max(per_sm, 1), kThreads, 0, kstream>>>(ctl, dctl, ring, ring_cap, head, reqs_d,
                                                                         done_d, flags, mdone, items_done, exiting,
                                                                         kerr);
        ++launches;
        count_launch();
    }

    static int member_blocks(int members) { return (members + kSrvMB - 1) / kSrvMB; }
    int items_per_stage(const Request& r) const {
        const int n = grids[r.grid].n, cn = chunk_nodes(n);
        return ((n + cn - 1) / cn) * member_blocks(r.members);
    }

    // append the next stage index (chunks x member blocks, chunk-major) of request r
    void append_stage(Request& r) {
        const Grid& G = grids[r.grid];
        const int cn = chunk_nodes(G.n);
        const int nch = (G.n + cn - 1) / cn;
        const int q = r.next_stage;
        for (int c = 0; c < nch; ++c)
            for (int mb = 0; mb < r.members; mb += kSrvMB) {
                if (q == r.withhold_q && c == 0 && mb == 0) {    // test hook: never queued
                    ++r.appended;
                    continue;
                }
                Item& it = ring_h[tail % ring_cap];
                it.slot = r.slot;
                it.q = q;
                it.chunk = c;
                it.member = mb;
                ++tail;
                ++r.appended;
            }
        ++r.next_stage;
    }

    int admit(Request& r) {
        size_t off;
        if (free_slots.empty() || !alloc(r.bytes, off)) return 0;
        const Grid& G = grids[r.grid];
        r.offset = off;
        r.slot = free_slots.back();
        free_slots.pop_back();
        const size_t one = ((size_t)G.n * 4 * sizeof(double) * r.members + 255) / 256 * 256;
        ReqDesc d{};
        d.W = reinterpret_cast<const uint4*>(G.W);
        d.idx = reinterpret_cast<const int4*>(G.idx);
        d.PT = reinterpret_cast<const double*>(G.PT);
        d.Wl = reinterpret_cast<const uint4*>(G.Wl);
        d.idxl = G.idxl;
        d.n = G.n;
        d.nnbr = G.nnbr;
        d.members = r.members;
        d.chunk_nodes = chunk_nodes(G.n);
        d.nchunks = (G.n + d.chunk_nodes - 1) / d.chunk_nodes;
        d.reach = G.reach;
        d.per_stage = d.nchunks * member_blocks(r.members);
        d.cdone = reinterpret_cast<int*>(arena + off + 4 * one);
        d.total = d.per_stage * 4 * r.nsteps;
        d.id = r.id;
        d.cancelled = 0;
        d.gh0 = G.gh0;
        d.dt = G.dt;
        d.H = reinterpret_cast<double*>(arena + off);
        d.Ka = reinterpret_cast<double*>(arena + off + one);
        d.Kb = reinterpret_cast<double*>(arena + off + 2 * one);
        d.D = reinterpret_cast<double*>(arena + off + 3 * one);
        int zero = 0;
        flags[r.slot] = -1;
        mdone[r.slot] = 0;
        // descriptor and counter first, then the states; work is queued once
        // the upload event has completed (pass()), so the GPU keeps running
        // other requests meanwhile
        cudaMemcpyAsync(reqs_d + r.slot, &d, sizeof(d), cudaMemcpyHostToDevice, cstream);
        cudaMemcpyAsync(done_d + r.slot, &zero, sizeof(int), cudaMemcpyHostToDevice, cstream);
        cudaMemsetAsync(d.cdone, 0, sizeof(int) * (size_t)d.nchunks * r.members, cstream);
        cudaMemcpyAsync(d.H, host_states(r), r.state_bytes, cudaMemcpyHostToDevice, cstream);
        if (cudaEventRecord(r.ev, cstream) != cudaSuccess) {
            fatal = "request upload failed";
            return -1;
        }
        r.state = Request::UPLOADING;
        active.push_back(r.id);
        ++admitted;
        return 1;
    }

    // the kernel has finished the request: copy its final states back (async)
    void drain(Request& r) {
        cudaMemcpyAsync(const_cast<double*>(host_states(r)), arena + r.offset, r.state_bytes,
                        cudaMemcpyDeviceToHost, cstream);
        cudaEventRecord(r.ev, cstream);
        r.state = Request::DRAINING;
    }
    void retire(Request& r, Request::State st) {
        release(r.offset, r.bytes);
        free_slots.push_back(r.slot);
        r.slot = -1;
        r.t_done = now_s();
        r.state = st;
        if (st != Request::DONE) unstage_host(r);
        ++completed;
    }

    // copy the new queue entries, then the tail, to the device (copy stream)
    void publish() {
        long long from = published;
        while (from < tail) {
            const long long s0 = from % ring_cap;
            const long long cnt = std::min(tail - from, ring_cap - s0);
            cudaMemcpyAsync(ring + s0, ring_h + s0, cnt * sizeof(Item), cudaMemcpyHostToDevice, pstream);
            from += cnt;
        }
        hctl->tail = tail;
        cudaMemcpyAsync(&dctl->tail, &hctl->tail, sizeof(long long), cudaMemcpyHostToDevice, pstream);
        cudaStreamSynchronize(pstream);
        published = tail;
    }

    // A dependency wait ran out (error 2): the kernel stops claiming work, and it
    // ends once its other waits, bounded by the same limit, have ended.  Items it
    // skipped are lost, so every request whose work was queued (RUNNING) fails;
    // uploads in flight, drains and pending requests carry on.  The queue and its
    // counters start again from zero, and the next pass relaunches the kernel.
    void recover_from_dependency_timeout() {
        for (size_t a = 0; a < active.size();) {
            Request& r = requests[active[a]];
            if (r.state == Request::RUNNING) {
                retire(r, Request::FAILED);
                active.erase(active.begin() + a);
            } else {
                ++a;
            }
        }
        tail = published = 0;
        hctl->tail = 0;
        cudaMemcpyAsync(&dctl->tail, &hctl->tail, sizeof(long long), cudaMemcpyHostToDevice, cstream);
        cudaMemsetAsync(head, 0, sizeof(unsigned long long), cstream);
        cudaMemsetAsync(items_done, 0, sizeof(unsigned long long), cstream);
        cudaMemsetAsync(kerr, 0, sizeof(int), cstream);
        if (cudaStreamSynchronize(cstream) != cudaSuccess) {
            fatal = "serving: reset after a dependency timeout failed";
            return;
        }
        ctl->progress = 0;
        ctl->error = 0;
        ++failures;
    }

    // one scheduler pass (called with mu held)
    void pass() {
        if (ctl->error) {
            if (ctl->error != 2) {
                fatal = "serving kernel error";
                return;
            }
            if (kernel_running()) return;
            recover_from_dependency_timeout();
            if (!fatal.empty()) return;
        }
        // uploads done -> running; kernel done -> draining; drained -> done
        for (size_t a = 0; a < active.size();) {
            Request& r = requests[active[a]];
            bool gone = false;
            if (r.state == Request::UPLOADING && cudaEventQuery(r.ev) == cudaSuccess) {
                r.state = Request::RUNNING;
                r.t_admit = now_s();
            }
            if (r.state == Request::RUNNING && ((volatile int*)flags)[r.slot] == r.id) {
                if (r.cancel_req) { retire(r, Request::CANCELLED); gone = true; }
                else drain(r);
            }
            if (r.state == Request::DRAINING && cudaEventQuery(r.ev) == cudaSuccess) {
                retire(r, Request::DONE);
                gone = true;
            }
            if (gone) active.erase(active.begin() + a);
            else ++a;
        }
        // admissions: FIFO, later requests may overtake one that does not fit yet
        for (auto it = pending.begin(); it != pending.end();) {
            Request& r = requests[*it];
            const int st = admit(r);
            if (st < 0) return;
            if (st == 1) it = pending.erase(it);
            else ++it;
        }
        // work: round-robin, one stage per request per round, so that other
        // requests' stages sit between a request's stage and the next one that
        // depends on it; at most kLookaheadStages stages queued or in flight per
        // request (so that CTAs waiting on a request's previous stage stay few)
        const long long done_items = ctl->progress;
        bool appended = false;
        for (int round = 0; round < kLookaheadStages; ++round) {
            bool any = false;
            for (int id : active) {
                Request& r = requests[id];
                if (r.state != Request::RUNNING || r.next_stage >= 4 * r.nsteps) continue;
                const int ips = items_per_stage(r);
                const long long outstanding = r.appended - ((volatile int*)mdone)[r.slot];
                if (outstanding >= (long long)kLookaheadStages * ips) continue;
                if (tail + ips > ring_cap + done_items - 1024) break;       // ring full
                append_stage(r);
                any = appended = true;
            }
            if (!any) break;
        }
        if (appended) publish();
        const bool work = tail > (long long)ctl->progress || !active.empty();
        if (ctl->error) return;                  // handled by the next pass
        const bool was_running = kernel_running();
        if (work && !was_running) launch_kernel();
        if (trace) {
            const double t = now_s() - t0;
            if (t - last_trace > 0.002 || (work && !was_running)) {
                last_trace = t;
                fprintf(stderr, "[srv %.4f] tail %lld progress %lld active %zu pending %zu launches %lld%s",
                        t, tail, (long long)ctl->progress, active.size(), pending.size(), launches,
                        (work && !was_running) ? " RELAUNCH" : "");
                for (int id : active) {
                    const Request& r = requests[id];
                    fprintf(stderr, " | r%d st%d stage %d/%d app %lld done %d", id, (int)r.state, r.next_stage, 4 * r.nsteps,
                            r.appended, r.slot >= 0 ? ((volatile int*)mdone)[r.slot] : -1);
                }
                fprintf(stderr, "\n");
            }
        }
    }

    void loop() {
        while (!quit.load()) {
            {
                std::lock_guard<std::mutex> lock(mu);
                if (fatal.empty()) pass();
            }
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
};

Server* g_srv = nullptr;

}  // namespace srv
}  // namespace swe

using namespace swe;
using namespace swe::srv;

extern "C" {

int swe_srv_start(double budget_bytes, int max_requests) {
    if (g_srv) { set_error("swe_srv_start: server already running"); return SWE_ERR_STATE; }
    if (budget_bytes < (1 << 20) || max_requests <= 0 || max_requests > 4096) {
        set_error("swe_srv_start: need budget >= 1 MiB and 1 <= max_requests <= 4096");
        return SWE_ERR_ARG;
    }
    Server* S = new Server();
    S->budget = (size_t)budget_bytes;
    S->max_slots = max_requests;
    cudaError_t e;
    auto fail = [&](const char* what) {
        set_error("swe_srv_start: %s: %s", what, cudaGetErrorString(e));
        delete S;
        return SWE_ERR_CUDA;
    };
    if ((e = cudaGetDevice(&S->device)) != cudaSuccess) return fail("cudaGetDevice");
    cudaDeviceGetAttribute(&S->sms, cudaDevAttrMultiProcessorCount, S->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&S->per_sm, serve_kernel, kThreads, 0);
    if ((e = cudaMalloc(&S->arena, S->budget)) != cudaSuccess) {
        set_error("swe_srv_start: cannot reserve the %.3g-byte HBM budget: %s", budget_bytes, cudaGetErrorString(e));
        delete S;
        return SWE_ERR_NOMEM;
    }
    S->free_blocks[0] = S->budget;
    S->ring_cap = 1LL << 22;
    if ((e = cudaHostAlloc(&S->ctl, sizeof(Shared), cudaHostAllocMapped)) != cudaSuccess) return fail("cudaHostAlloc");
    if ((e = cudaMalloc(&S->ring, sizeof(Item) * S->ring_cap)) != cudaSuccess) return fail("cudaMalloc ring");
    if ((e = cudaHostAlloc(&S->ring_h, sizeof(Item) * S->ring_cap, cudaHostAllocDefault)) != cudaSuccess) return fail("cudaHostAlloc ring");
    if ((e = cudaHostAlloc(&S->hctl, sizeof(DevCtl), cudaHostAllocDefault)) != cudaSuccess) return fail("cudaHostAlloc ctl");
    if ((e = cudaMalloc(&S->dctl, sizeof(DevCtl))) != cudaSuccess) return fail("cudaMalloc ctl");
    if ((e = cudaMalloc(&S->kerr, sizeof(int))) != cudaSuccess) return fail("cudaMalloc err");
    memset(S->hctl, 0, sizeof(DevCtl));
    S->hctl->dep_ns = kDepNs;
    cudaMemcpy(S->dctl, S->hctl, sizeof(DevCtl), cudaMemcpyHostToDevice);
    cudaMemset(S->kerr, 0, sizeof(int));
    if ((e = cudaHostAlloc(&S->flags, sizeof(int) * max_requests, cudaHostAllocMapped)) != cudaSuccess) return fail("cudaHostAlloc flags");
    if ((e = cudaHostAlloc(&S->mdone, sizeof(int) * max_requests, cudaHostAllocMapped)) != cudaSuccess) return fail("cudaHostAlloc mdone");
    for (int i = 0; i < max_requests; ++i) S->mdone[i] = 0;
    memset((void*)S->ctl, 0, sizeof(Shared));
    for (int i = 0; i < max_requests; ++i) S->flags[i] = -1;
    if ((e = cudaMalloc(&S->head, sizeof(unsigned long long))) != cudaSuccess) return fail("cudaMalloc head");
    if ((e = cudaMalloc(&S->items_done, sizeof(unsigned long long))) != cudaSuccess) return fail("cudaMalloc counter");
    if ((e = cudaMalloc(&S->reqs_d, sizeof(ReqDesc) * max_requests)) != cudaSuccess) return fail("cudaMalloc table");
    if ((e = cudaMalloc(&S->done_d, sizeof(int) * max_requests)) != cudaSuccess) return fail("cudaMalloc done");
    if ((e = cudaMalloc(&S->exiting, sizeof(int))) != cudaSuccess) return fail("cudaMalloc exiting");
    cudaMemset(S->head, 0, sizeof(unsigned long long));
    cudaMemset(S->items_done, 0, sizeof(unsigned long long));
    cudaMemset(S->reqs_d, 0, sizeof(ReqDesc) * max_requests);
    cudaMemset(S->done_d, 0, sizeof(int) * max_requests);
    cudaStreamCreateWithFlags(&S->kstream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&S->cstream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&S->pstream, cudaStreamNonBlocking);
    // pinned staging pool for state transfers: a quarter of the budget, 64 MiB .. 4 GiB
    S->pin_size = std::min<size_t>(std::max<size_t>(S->budget / 4, (size_t)64 << 20), (size_t)4 << 30);
    if (cudaHostAlloc(&S->pin, S->pin_size, cudaHostAllocDefault) == cudaSuccess) S->pin_free[0] = S->pin_size;
    else { S->pin = nullptr; cudaGetLastError(); }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail("setup");
    for (int i = max_requests - 1; i >= 0; --i) S->free_slots.push_back(i);
    S->running = true;
    g_srv = S;
    S->worker = std::thread([S]() {
        cudaSetDevice(S->device);
        S->loop();
    });
    return SWE_OK;
}

int swe_srv_add_grid(int n, int nnbr, double gh0, double dt, const int* idx, const double* Dx, const double* Dy,
                     const double* Dz, const double* L, const double* x, const double* y, const double* z,
                     const double* f, const double* ghm, const double* p_u, const double* p_v, const double* p_w,
                     const double* gradghm) {
    if (!g_srv) { set_error("swe_srv_add_grid: server not started"); return -SWE_ERR_STATE; }
    if (n <= 0 || nnbr <= 0 || nnbr > kSlots) { set_error("swe_srv_add_grid: bad sizes"); return -SWE_ERR_ARG; }
    // packed on the device exactly as the plain form packs a patch in the default
    // layout (node order as given, rows of nnbr stencil slots)
    CallerLayout cl;
    cl.layout = 0;
    cl.S = 1;
    cl.pnbr = nnbr;
    PackedStatic<double> ps;
    const int st = pack_static_device<double>(cl, n, n, 0, nnbr, Dx, Dy, Dz, L, idx, x, y, z, f, ghm, p_u, p_v, p_w,
                                              gradghm, ps);
    if (st != SWE_OK) return -st;
    Grid G;
    G.n = n; G.nnbr = nnbr; G.gh0 = gh0; G.dt = dt;
    // how many work-item chunks a chunk's stencils reach on either side
    {
        const int cn = Server::chunk_nodes(n);
        for (long i = 0; i < n; ++i)
            for (int j = 0; j < nnbr; ++j) {
                const int dc = std::abs(idx[i * nnbr + j] / cn - (int)(i / cn));
                G.reach = std::max(G.reach, dc);
            }
    }
    G.W = ps.W;
    G.idx = ps.idx;
    G.PT = ps.PT;
    G.Wl = ps.Wl;
    G.idxl = ps.idxl;
    // the 16-bit offsets are not read here: a second index path in the persistent
    // kernel raises its register demand past the 128 it runs at
    cudaFree(ps.idxs);
    std::lock_guard<std::mutex> lock(g_srv->mu);
    g_srv->grids.push_back(G);
    return (int)g_srv->grids.size() - 1;
}

int swe_srv_submit(int grid, int members, int nsteps, const double* H0) {
    if (!g_srv) { set_error("swe_srv_submit: server not started"); return -SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    if (!S.fatal.empty()) { set_error("%s", S.fatal.c_str()); return -SWE_ERR_TIMEOUT; }
    if (grid < 0 || grid >= (int)S.grids.size()) { set_error("swe_srv_submit: unknown grid %d", grid); return -SWE_ERR_ARG; }
    if (members < 1 || members > 32 || nsteps < 1 || !H0) {
        set_error("swe_srv_submit: need 1 <= members <= 32, nsteps >= 1 and initial states");
        return -SWE_ERR_ARG;
    }
    const Grid& G = S.grids[grid];
    Request r;
    r.id = S.next_id++;
    r.grid = grid;
    r.members = members;
    r.nsteps = nsteps;
    r.bytes = Server::state_bytes(G.n, members);
    if (r.bytes > S.budget) {
        set_error("swe_srv_submit: request needs %zu bytes, more than the whole budget", r.bytes);
        return -SWE_ERR_NOMEM;
    }
    r.state_bytes = (size_t)members * G.n * 4 * sizeof(double);
    S.stage_host(r, H0);
    if (cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming) != cudaSuccess) {
        S.unstage_host(r);
        set_error("swe_srv_submit: cudaEventCreate failed");
        return -SWE_ERR_CUDA;
    }
    r.t_submit = now_s();
    r.withhold_q = S.withhold_next_q;
    S.withhold_next_q = -1;
    S.requests[r.id] = std::move(r);
    S.pending.push_back(S.requests.rbegin()->first);
    return S.requests.rbegin()->first;
}

int swe_srv_poll(int id, double* times) {
    if (!g_srv) { set_error("swe_srv_poll: server not started"); return -SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    if (!S.fatal.empty()) { set_error("%s", S.fatal.c_str()); return -SWE_ERR_TIMEOUT; }
    auto it = S.requests.find(id);
    if (it == S.requests.end()) { set_error("swe_srv_poll: unknown request %d", id); return -SWE_ERR_ARG; }
    const Request& r = it->second;
    if (times) {
        times[0] = r.t_admit > 0 ? r.t_admit - r.t_submit : -1.0;
        times[1] = r.t_done > 0 ? r.t_done - r.t_submit : -1.0;
    }
    switch (r.state) {
        case Request::DONE: return 1;
        case Request::CANCELLED: return 2;
        case Request::FAILED:
            set_error("swe_srv_poll: request %d failed: a dependency wait in the serving kernel ran out", id);
            return -SWE_ERR_TIMEOUT;
        default: return 0;
    }
}

int swe_srv_set_dep_limit(double seconds) {
    if (!g_srv) { set_error("swe_srv_set_dep_limit: server not started"); return SWE_ERR_STATE; }
    if (!(seconds >= 1e-3 && seconds <= 3600.0)) {
        set_error("swe_srv_set_dep_limit: limit %g s outside 1 ms .. 1 h", seconds);
        return SWE_ERR_ARG;
    }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    S.hctl->dep_ns = (unsigned long long)(seconds * 1e9);
    SWE_CUDA_TRY(cudaMemcpyAsync(&S.dctl->dep_ns, &S.hctl->dep_ns, sizeof(unsigned long long),
                                 cudaMemcpyHostToDevice, S.cstream));
    SWE_CUDA_TRY(cudaStreamSynchronize(S.cstream));
    return SWE_OK;
}

int swe_srv_test_withhold(int id, int stage_index) {
    if (!g_srv) { set_error("swe_srv_test_withhold: server not started"); return SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    if (id < 0) {                       // arm the hook for the next submission
        if (stage_index < 0) { set_error("swe_srv_test_withhold: negative stage index"); return SWE_ERR_ARG; }
        S.withhold_next_q = stage_index;
        return SWE_OK;
    }
    auto it = S.requests.find(id);
    if (it == S.requests.end()) { set_error("swe_srv_test_withhold: unknown request %d", id); return SWE_ERR_ARG; }
    Request& r = it->second;
    if (stage_index < r.next_stage || stage_index >= 4 * r.nsteps) {
        set_error("swe_srv_test_withhold: stage index %d already queued or past the request's end", stage_index);
        return SWE_ERR_ARG;
    }
    r.withhold_q = stage_index;
    return SWE_OK;
}

int swe_srv_fetch(int id, double* H) {
    if (!g_srv) { set_error("swe_srv_fetch: server not started"); return SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    auto it = S.requests.find(id);
    if (it == S.requests.end()) { set_error("swe_srv_fetch: unknown request %d", id); return SWE_ERR_ARG; }
    Request& r = it->second;
    if (r.state != Request::DONE) { set_error("swe_srv_fetch: request %d has not completed", id); return SWE_ERR_STATE; }
    if (H) memcpy(H, S.host_states(r), r.state_bytes);
    S.unstage_host(r);
    if (r.ev) cudaEventDestroy(r.ev);
    S.requests.erase(it);
    return SWE_OK;
}

int swe_srv_cancel(int id) {
    if (!g_srv) { set_error("swe_srv_cancel: server not started"); return SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    auto it = S.requests.find(id);
    if (it == S.requests.end()) { set_error("swe_srv_cancel: unknown request %d", id); return SWE_ERR_ARG; }
    Request& r = it->second;
    r.cancel_req = true;
    if (r.state == Request::PENDING) {
        S.pending.erase(std::remove(S.pending.begin(), S.pending.end(), id), S.pending.end());
        r.state = Request::CANCELLED;
        r.t_done = now_s();
        S.unstage_host(r);
        return SWE_OK;
    }
    if (r.state == Request::RUNNING && r.slot >= 0) {
        // the kernel skips the compute of a cancelled request's remaining items
        const int one = 1;
        cudaMemcpyAsync(&S.reqs_d[r.slot].cancelled, &one, sizeof(int), cudaMemcpyHostToDevice, S.cstream);
        cudaStreamSynchronize(S.cstream);
        // the rest of its steps still have to pass through the queue to retire it
    }
    return SWE_OK;
}

int swe_srv_stats(double* out) {
    if (!g_srv) { set_error("swe_srv_stats: server not started"); return SWE_ERR_STATE; }
    Server& S = *g_srv;
    std::lock_guard<std::mutex> lock(S.mu);
    out[0] = (double)S.launches;
    out[1] = (double)S.admitted;
    out[2] = (double)S.completed;
    out[3] = (double)S.in_use;
    out[4] = (double)S.peak;
    out[5] = (double)S.budget;
    out[6] = (double)S.ctl->progress;
    out[7] = (double)S.pending.size();
    out[8] = (double)S.active.size();
    out[9] = (double)S.failures;
    return SWE_OK;
}

int swe_srv_stop(void) {
    if (!g_srv) return SWE_OK;
    Server* S = g_srv;
    S->quit = true;
    if (S->worker.joinable()) S->worker.join();
    S->hctl->stop = 1;
    cudaMemcpyAsync(&S->dctl->stop, &S->hctl->stop, sizeof(int), cudaMemcpyHostToDevice, S->cstream);
    cudaStreamSynchronize(S->cstream);
    cudaStreamSynchronize(S->pstream);
    cudaStreamSynchronize(S->kstream);
    cudaStreamSynchronize(S->cstream);
    for (auto& G : S->grids) {
        cudaFree(G.W);
        cudaFree(G.idx);
        cudaFree(G.PT);
        cudaFree(G.Wl);
        cudaFree(G.idxl);
    }
    cudaFree(S->arena);
    cudaFree(S->head);
    cudaFree(S->items_done);
    cudaFree(S->reqs_d);
    cudaFree(S->done_d);
    cudaFree(S->exiting);
    cudaFreeHost((void*)S->ctl);
    cudaFree(S->ring);
    cudaFreeHost(S->ring_h);
    cudaFreeHost(S->hctl);
    cudaFree(S->dctl);
    cudaFree(S->kerr);
    cudaFreeHost(S->flags);
    cudaFreeHost(S->mdone);
    for (auto& kv : S->requests)
        if (kv.second.ev) cudaEventDestroy(kv.second.ev);
    if (S->pin) cudaFreeHost(S->pin);
    cudaStreamDestroy(S->kstream);
    cudaStreamDestroy(S->cstream);
    cudaStreamDestroy(S->pstream);
    const bool err = !S->fatal.empty();
    std::string msg = S->fatal;
    delete S;
    g_srv = nullptr;
    if (err) { set_error("%s", msg.c_str()); return SWE_ERR_TIMEOUT; }
    return SWE_OK;
}

}  // extern "C"
