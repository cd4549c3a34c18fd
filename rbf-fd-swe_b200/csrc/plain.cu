// Plain drop-in form: the swe_cuda_* entry points of include/swe_b200.h.
//
// Host side of the fused stage kernel: canonicalisation of the caller's
// (reference-layout) static data into the device layout, device-resident RK
// registers H, K (ping-pong), D, the four stage launches of RK_substep
// (swe_code/main/rk4_rbffd_swe.c:30-72) and a captured CUDA graph for whole
// steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "stage_kernel.cuh"
#include "history.cuh"
#include "stage_tma.cuh"
#include "stage_lane.cuh"
#include "pack.cuh"

namespace swe {

static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

void count_launch(long long n) { g_launches += n; }

// ---------------------------------------------------------------------------
// Device helpers ---------------------------------------------------------------

// caller layout (SVM_LIN_ID) <-> node-major rows; dir 0: caller -> canonical
template <typename T>
__global__ void permute_state_kernel(const T* __restrict__ src, T* __restrict__ dst, long rows,
                                     CallerLayout cl, int dir) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows * 4) return;
    const long p = t >> 2, sv = t & 3;
    const long c = cl.svm(p, sv);
    if (dir == 0) dst[t] = src[c];
    else dst[c] = src[t];
}

// FP64 mass/energy sums over n nodes (equal areas 4*pi/n).
template <typename T>
__global__ void invariants_kernel(const T* __restrict__ H, const T* __restrict__ PT, int n, double gh0,
                                  double* __restrict__ out) {
    double mass = 0.0, energy = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double u = H[4 * i], v = H[4 * i + 1], w = H[4 * i + 2], h = H[4 * i + 3];
        const double phi = h + gh0;
        const double thick = phi - (double)PT[i * kPointStride + PT_GHM];
        mass += thick;
        energy += 0.5 * thick * (u * u + v * v + w * w) + 0.5 * phi * phi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mass += __shfl_xor_sync(0xffffffffu, mass, o);
        energy += __shfl_xor_sync(0xffffffffu, energy, o);
    }
    __shared__ double sm[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sm[0][warp] = mass; sm[1][warp] = energy; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        mass = lane < nw ? sm[0][lane] : 0.0;
        energy = lane < nw ? sm[1][lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            mass += __shfl_xor_sync(0xffffffffu, mass, o);
            energy += __shfl_xor_sync(0xffffffffu, energy, o);
        }
        if (lane == 0) { atomicAdd(out, mass); atomicAdd(out + 1, energy); }
    }
}

// ---------------------------------------------------------------------------
// Plain solver ---------------------------------------------------------------

struct Plain {
    bool ready = false;
    int fsize = 8, n = 0, rows = 0, pid0 = 0, nnbr = 0;
    CallerLayout cl;
    double gh0 = 0, dt = 0;
    void *W = nullptr, *PT = nullptr, *H = nullptr, *Ka = nullptr, *Kb = nullptr, *D = nullptr, *F = nullptr,
         *Kx = nullptr, *raw = nullptr, *Wl = nullptr;
    int* idx = nullptr;
    int* idxl = nullptr;            // node-per-lane kernel: tile-transposed weights / indices
    short* idxs = nullptr;          // the same indices as 16-bit offsets from each node's own row
    bool idxs_fit = false;          // every offset fits 16 bits
    bool idxs_ok = false;           // the kernel reads idxs (idxs_fit, unless 32-bit indices were asked for)
    int* halo_send = nullptr;       // patch rows this rank sends / receives (swe_cuda_halo_setup)
    int* halo_recv = nullptr;
    int n_send = 0, n_recv = 0;
    double* inv = nullptr;
    int* err = nullptr;             // pipelined kernel: bounded-wait error word
    int* err_host = nullptr;        // pinned copy of it, read back with the state
    bool err_pending = false;       // a pipelined launch since the error word was last read
    bool tma_ok = false;            // pipelined kernel set up
    int kernel_choice = 0;          // 0 = bulk-copy pipelined, 1 = register-streaming, 2 = node-per-lane kernel
    float tune_us[3] = {0.f, 0.f, 0.f};  // stage launch time of each kernel at init (its best shape)
    int lane_lpn = 1;               // node-per-lane kernel: lanes per node (1, 2, 4)
    int lane_pf = 0;                // node-per-lane kernel: bulk L2 prefetch at warp start
    int lane_minb = 4;              // node-per-lane kernel: CTAs per SM of its register bound (3, 4, 5)
    int tma_tile = 64;              // pipelined kernel: nodes per tile (64: 1 CTA/SM, 32: 2 CTAs/SM)
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int grid = 0;
    bool timing = false;
    std::vector<cudaEvent_t> ev;   // pairs (start, stop) of timed launches
    size_t ev_used = 0;
    double t_step_last = 0.0;
    cudaEvent_t step_ev[2] = {nullptr, nullptr};
    bool step_timed = false;

    size_t fbytes(long count) const { return (size_t)count * fsize; }

    HistoryWriter hist;             // history output (swe_hist_open)
    long long steps_done = 0;       // completed RK4 steps since the last swe_cuda_set_state

    void release() {
        hist.close();
        steps_done = 0;
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (void* p : {W, PT, H, Ka, Kb, D, F, Kx, raw, Wl, (void*)halo_send, (void*)halo_recv}) if (p) cudaFree(p);
        halo_send = halo_recv = nullptr;
        n_send = n_recv = 0;
        if (idx) cudaFree(idx);
        if (idxl) cudaFree(idxl);
        if (idxs) cudaFree(idxs);
        if (inv) cudaFree(inv);
        if (err) cudaFree(err);
        if (err_host) cudaFreeHost(err_host);
        err_host = nullptr;
        err_pending = false;
        W = PT = H = Ka = Kb = D = F = Kx = raw = Wl = nullptr;
        idx = nullptr;
        idxl = nullptr;
        idxs = nullptr;
        idxs_fit = idxs_ok = false;
        lane_lpn = 1;
        lane_pf = 0;
        lane_minb = 4;
        inv = nullptr;
        err = nullptr;
        tma_ok = false;
        kernel_choice = 0;
        tma_tile = 64;
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
        ev_used = 0;
        for (auto& e : step_ev) { if (e) cudaEventDestroy(e); e = nullptr; }
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        ready = false;
    }

    int timed_begin(cudaEvent_t* pair) {
        if (!timing) return SWE_OK;
        if (ev_used + 2 > ev.size()) {
            for (int t = 0; t < 64; ++t) {
                cudaEvent_t e;
                SWE_CUDA_TRY(cudaEventCreate(&e));
                ev.push_back(e);
            }
        }
        pair[0] = ev[ev_used];
        pair[1] = ev[ev_used + 1];
        ev_used += 2;
        SWE_CUDA_TRY(cudaEventRecord(pair[0], stream));
        return SWE_OK;
    }

    // The stage kernels index the compute rows 0..n-1 for everything they write (D, F,
    // K_out, H) and read the gather source at patch rows.  H and the K buffers hold the
    // whole patch, as the reference's do (eval_K and update_H write rows compute_pid_s +
    // i, rk4_rbffd_swe.c:86-158), so the kernels get H and K_out starting at the first
    // compute row; with no halo rows (compute_pid_s = 0) the offset is zero.
    template <typename T>
    StageArgs<T> args(int mode) const {
        StageArgs<T> a{};
        a.n = n;
        a.pid0 = pid0;
        a.idx = reinterpret_cast<const int4*>(idx);
        a.W = reinterpret_cast<const uint4*>(W);
        a.PT = reinterpret_cast<const T*>(PT);
        a.H = reinterpret_cast<T*>(H) + 4L * pid0;
        a.D = reinterpret_cast<T*>(D);
        a.F = reinterpret_cast<T*>(F);
        a.gh0 = (T)gh0;
        const T dtT = (T)dt;
        a.dt6 = (double)dtT / 6.0;
        T* ka = reinterpret_cast<T*>(Ka) + 4L * pid0;
        T* kb = reinterpret_cast<T*>(Kb) + 4L * pid0;
        switch (mode) {
            case 0: a.Kin = reinterpret_cast<const T*>(H); a.Kout = ka; a.c = (T)(dtT / 2.0); break;
            case 1: a.Kin = reinterpret_cast<const T*>(Ka); a.Kout = kb; a.c = (T)(dtT / 2.0); break;
            case 2: a.Kin = reinterpret_cast<const T*>(Kb); a.Kout = ka; a.c = dtT; break;
            case 3: a.Kin = reinterpret_cast<const T*>(Ka); a.Kout = nullptr; a.c = dtT; break;
            default: a.Kin = reinterpret_cast<const T*>(Kx); a.Kout = nullptr; a.c = T(0); break;
        }
        return a;
    }

    // the buffer substep `s` reads its gather source from: H, Ka, Kb, Ka
    void* stage_input(int s) const { return s == 0 ? H : s == 2 ? Kb : Ka; }

    bool use_tma() const { return tma_ok && kernel_choice == 0; }

    template <typename T, int TILE>
    void launch_tma(const StageArgs<T>& a, int mode) {
        using Sh = TmaShape<TILE>;
        const int ntiles = (n + TILE - 1) / TILE;
        const TmaArgs<T> ta{a, ntiles, err};
        const int g = std::max(1, std::min(ntiles, sms * Sh::kCtasPerSm));
        const int sm = TmaLayout<T, TILE>::kSmem;
        // programmatic dependent launch: the kernel loads its static streams before
        // griddepcontrol.wait (stage_tma.cuh)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g);
        cfg.blockDim = dim3(Sh::kThreads);
        cfg.dynamicSmemBytes = sm;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        switch (mode) {
            case 0: cudaLaunchKernelEx(&cfg, stage_tma_kernel<T, kStage0, TILE>, ta); break;
            case 1: cudaLaunchKernelEx(&cfg, stage_tma_kernel<T, kStage1, TILE>, ta); break;
            case 2: cudaLaunchKernelEx(&cfg, stage_tma_kernel<T, kStage2, TILE>, ta); break;
            case 3: cudaLaunchKernelEx(&cfg, stage_tma_kernel<T, kStage3, TILE>, ta); break;
            default: cudaLaunchKernelEx(&cfg, stage_tma_kernel<T, kEvalOnly, TILE>, ta); break;
        }
    }

    template <typename T, int LPN, int MINB>
    void launch_lane(const StageArgs<T>& a, int mode) {
        if (idxs_ok) launch_lane_i<T, LPN, MINB, true>(a, mode);
        else launch_lane_i<T, LPN, MINB, false>(a, mode);
    }
    template <typename T, int LPN, int MINB, bool I16>
    void launch_lane_i(const StageArgs<T>& a, int mode) {
        const LaneArgs<T> la{a, reinterpret_cast<const uint4*>(Wl), idxl, idxs, lane_pf, nnbr};
        const int units = ceil_div(n, kLaneTile / LPN);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ceil_div(units, kLaneWarps));
        cfg.blockDim = dim3(kLaneThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        switch (mode) {
            case 0: cudaLaunchKernelEx(&cfg, stage_lane_kernel<T, kStage0, LPN, MINB, I16>, la); break;
            case 1: cudaLaunchKernelEx(&cfg, stage_lane_kernel<T, kStage1, LPN, MINB, I16>, la); break;
            case 2: cudaLaunchKernelEx(&cfg, stage_lane_kernel<T, kStage2, LPN, MINB, I16>, la); break;
            case 3: cudaLaunchKernelEx(&cfg, stage_lane_kernel<T, kStage3, LPN, MINB, I16>, la); break;
            default: cudaLaunchKernelEx(&cfg, stage_lane_kernel<T, kEvalOnly, LPN, MINB, I16>, la); break;
        }
    }

    template <typename T>
    void launch_t(int mode) {
        const StageArgs<T> a = args<T>(mode);
        if (kernel_choice == 2) {
            if (lane_minb == 3) {
                if (lane_lpn == 4) launch_lane<T, 4, 3>(a, mode);
                else if (lane_lpn == 2) launch_lane<T, 2, 3>(a, mode);
                else launch_lane<T, 1, 3>(a, mode);
            } else if (lane_minb == 5) {
                if (lane_lpn == 4) launch_lane<T, 4, 5>(a, mode);
                else if (lane_lpn == 2) launch_lane<T, 2, 5>(a, mode);
                else launch_lane<T, 1, 5>(a, mode);
            } else {
                if (lane_lpn == 4) launch_lane<T, 4, 4>(a, mode);
                else if (lane_lpn == 2) launch_lane<T, 2, 4>(a, mode);
                else launch_lane<T, 1, 4>(a, mode);
            }
            return;
        }
        if (use_tma()) {
            err_pending = true;
            if (tma_tile == 32) launch_tma<T, 32>(a, mode);
            else if (tma_tile == 16) launch_tma<T, 16>(a, mode);
            else launch_tma<T, 64>(a, mode);
            return;
        }
        switch (mode) {
            case 0: stage_kernel<T, kStage0><<<grid, kStageThreads, 0, stream>>>(a); break;
            case 1: stage_kernel<T, kStage1><<<grid, kStageThreads, 0, stream>>>(a); break;
            case 2: stage_kernel<T, kStage2><<<grid, kStageThreads, 0, stream>>>(a); break;
            case 3: stage_kernel<T, kStage3><<<grid, kStageThreads, 0, stream>>>(a); break;
            default: stage_kernel<T, kEvalOnly><<<grid, kStageThreads, 0, stream>>>(a); break;
        }
    }

    int launch(int mode) {
        cudaEvent_t pair[2] = {nullptr, nullptr};
        SWE_TRY(timed_begin(pair));
        if (fsize == 8) launch_t<double>(mode);
        else launch_t<float>(mode);
        count_launch();
        SWE_CUDA_TRY(cudaGetLastError());
        if (pair[1]) SWE_CUDA_TRY(cudaEventRecord(pair[1], stream));
        return SWE_OK;
    }

    int build_graph() {
        cudaGraph_t g;
        SWE_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const bool was = timing;
        timing = false;
        for (int s = 0; s < 4; ++s) {
            if (fsize == 8) launch_t<double>(s);
            else launch_t<float>(s);
        }
        timing = was;
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
};

static Plain g_plain;

// Node-per-lane shape s in 0..17 (swe_cuda_select_kernel's 6 + s): lanes per node
// 1 / 2 / 4 = s % 3; s < 12: 5 CTAs per SM when (s / 3) % 2 (else 4), L2 prefetch
// when s >= 6; s >= 12: 3 CTAs per SM, L2 prefetch when s >= 15.
static void lane_shape(Plain& P, int s) {
    P.kernel_choice = 2;
    P.lane_lpn = 1 << (s % 3);
    if (s < 12) {
        P.lane_minb = (s / 3) % 2 ? 5 : 4;
        P.lane_pf = s >= 6 ? 1 : 0;
    } else {
        P.lane_minb = 3;
        P.lane_pf = s >= 15 ? 1 : 0;
    }
}

template <typename T, int TILE>
static int set_tma_attrs() {
    const int sm = TmaLayout<T, TILE>::kSmem;
    SWE_CUDA_TRY(cudaFuncSetAttribute(stage_tma_kernel<T, kStage0, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    SWE_CUDA_TRY(cudaFuncSetAttribute(stage_tma_kernel<T, kStage1, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    SWE_CUDA_TRY(cudaFuncSetAttribute(stage_tma_kernel<T, kStage2, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    SWE_CUDA_TRY(cudaFuncSetAttribute(stage_tma_kernel<T, kStage3, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    SWE_CUDA_TRY(cudaFuncSetAttribute(stage_tma_kernel<T, kEvalOnly, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    return SWE_OK;
}

template <typename T>
static int upload_static(Plain& P, const void* x, const void* y, const void* z, const void* f, const void* ghm,
                         const void* pu, const void* pv, const void* pw, const void* gg, const int* idx,
                         const void* Dx, const void* Dy, const void* Dz, const void* L) {
    // the caller's arrays go to the device once; every device layout is packed there (pack.cuh)
    PackedStatic<T> ps;
    SWE_TRY(pack_static_device<T>(P.cl, P.n, P.rows, P.pid0, P.nnbr, (const T*)Dx, (const T*)Dy, (const T*)Dz,
                                  (const T*)L, idx, (const T*)x, (const T*)y, (const T*)z, (const T*)f,
                                  (const T*)ghm, (const T*)pu, (const T*)pv, (const T*)pw, (const T*)gg, ps));
    P.W = ps.W;
    P.idx = ps.idx;
    P.Wl = ps.Wl;
    P.idxl = ps.idxl;
    P.idxs = ps.idxs;
    P.idxs_fit = P.idxs_ok = ps.idxs_ok;
    P.PT = ps.PT;
    P.tma_ok = true;
    {
        SWE_CUDA_TRY(cudaMalloc(&P.err, sizeof(int)));
        SWE_CUDA_TRY(cudaMemset(P.err, 0, sizeof(int)));
        SWE_CUDA_TRY(cudaHostAlloc(&P.err_host, sizeof(int), cudaHostAllocDefault));
        *P.err_host = 0;
        SWE_TRY((set_tma_attrs<T, 64>()));
        SWE_TRY((set_tma_attrs<T, 32>()));
        SWE_TRY((set_tma_attrs<T, 16>()));
    }
    return SWE_OK;
}

// Reads the pipelined kernel's bounded-wait error word: enqueues its copy into
// pinned memory and synchronises the stream once (callers that also read data
// back enqueue their copy first, so one synchronisation serves both).
static int check_tma_err() {
    Plain& P = g_plain;
    // only the pipelined kernel writes the word: read it back (one more small copy before
    // the synchronisation) only after such a launch
    if (!P.err || !P.err_host || !P.err_pending) {
        SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
        return SWE_OK;
    }
    SWE_CUDA_TRY(cudaMemcpyAsync(P.err_host, P.err, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    const int h = *P.err_host;
    P.err_pending = h != 0;   // a timeout stays reported until the word is cleared
    if (h) {
        set_error("stage kernel: a bounded wait on the bulk-copy pipeline ran out (code %d)", h);
        return SWE_ERR_TIMEOUT;
    }
    return SWE_OK;
}

static int require_ready() {
    if (!g_plain.ready) {
        set_error("swe_cuda_init has not been called");
        return SWE_ERR_STATE;
    }
    return SWE_OK;
}

static int permute_state(const void* src, void* dst, int dir);

// One RK4 step has been enqueued: count it and snapshot the state if the history is due.
static int after_step() {
    Plain& P = g_plain;
    ++P.steps_done;
    return P.hist.after_step(P.steps_done, P.stream, [&](void* dbuf) { return permute_state(P.H, dbuf, 1); });
}

static int permute_state(const void* src, void* dst, int dir) {
    Plain& P = g_plain;
    const long total = (long)P.rows * 4;
    const int threads = 256;
    const int blocks = ceil_div(total, threads);
    if (P.fsize == 8)
        permute_state_kernel<double><<<blocks, threads, 0, P.stream>>>((const double*)src, (double*)dst, P.rows, P.cl, dir);
    else
        permute_state_kernel<float><<<blocks, threads, 0, P.stream>>>((const float*)src, (float*)dst, P.rows, P.cl, dir);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    return SWE_OK;
}

}  // namespace swe

using namespace swe;

extern "C" {

const char* swe_cuda_last_error(void) { return g_err.c_str(); }

long long swe_b200_kernel_launches(void) { return g_launches.load(); }

int swe_cuda_select_device(int device) {
    SWE_CUDA_TRY(cudaSetDevice(device));
    return SWE_OK;
}

int swe_cuda_init(int fsize, int layout, int simd_length, int compute_size, int patch_size, int compute_pid_s,
                  int nnbr, int padded_nnbr, double gh0, double dt, const void* x, const void* y, const void* z,
                  const void* f, const void* ghm, const void* p_u, const void* p_v, const void* p_w,
                  const void* gradghm, const int* idx, const void* Dx, const void* Dy, const void* Dz,
                  const void* L) {
    if (fsize != 8 && fsize != 4) { set_error("fsize must be 8 or 4, got %d", fsize); return SWE_ERR_ARG; }
    if (layout & ~(SWE_LAYOUT_CFDL | SWE_LAYOUT_SFDL)) { set_error("unknown layout flags %d", layout); return SWE_ERR_ARG; }
    if (compute_size <= 0 || patch_size < compute_size || compute_pid_s < 0 ||
        compute_pid_s + compute_size > patch_size) {
        set_error("bad patch: compute_size %d patch_size %d compute_pid_s %d", compute_size, patch_size, compute_pid_s);
        return SWE_ERR_ARG;
    }
    if (nnbr <= 0 || nnbr > kSlots || padded_nnbr < nnbr) {
        set_error("nnbr %d / padded_nnbr %d unsupported (need 1 <= nnbr <= %d <= padded)", nnbr, padded_nnbr, kSlots);
        return SWE_ERR_ARG;
    }
    if (simd_length <= 0 || ((layout & SWE_LAYOUT_SFDL) && compute_size % simd_length) ||
        (!(layout & SWE_LAYOUT_CFDL) && patch_size % simd_length)) {
        set_error("tile width %d does not divide the padded sizes", simd_length);
        return SWE_ERR_ARG;
    }
    if (!x || !y || !z || !f || !ghm || !p_u || !p_v || !p_w || !gradghm || !idx || !Dx || !Dy || !Dz || !L) {
        set_error("null static array");
        return SWE_ERR_ARG;
    }
    Plain& P = g_plain;
    P.release();
    P.fsize = fsize;
    P.n = compute_size;
    P.rows = patch_size;
    P.pid0 = compute_pid_s;
    P.nnbr = nnbr;
    P.cl.layout = layout;
    P.cl.S = simd_length;
    P.cl.pnbr = padded_nnbr;
    P.gh0 = gh0;
    P.dt = dt;
    SWE_CUDA_TRY(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
    int st = fsize == 8 ? upload_static<double>(P, x, y, z, f, ghm, p_u, p_v, p_w, gradghm, idx, Dx, Dy, Dz, L)
                        : upload_static<float>(P, x, y, z, f, ghm, p_u, p_v, p_w, gradghm, idx, Dx, Dy, Dz, L);
    if (st != SWE_OK) { P.release(); return st; }
    const size_t srow = P.fbytes(4L * P.rows), scomp = P.fbytes(4L * P.n);
    SWE_CUDA_TRY(cudaMalloc(&P.H, srow));
    SWE_CUDA_TRY(cudaMalloc(&P.Ka, srow));
    SWE_CUDA_TRY(cudaMalloc(&P.Kb, srow));
    SWE_CUDA_TRY(cudaMalloc(&P.Kx, srow));
    SWE_CUDA_TRY(cudaMalloc(&P.raw, srow));
    SWE_CUDA_TRY(cudaMalloc(&P.D, scomp));
    SWE_CUDA_TRY(cudaMalloc(&P.F, scomp));
    SWE_CUDA_TRY(cudaMalloc(&P.inv, 2 * sizeof(double)));
    SWE_CUDA_TRY(cudaMemset(P.H, 0, srow));
    SWE_CUDA_TRY(cudaMemset(P.Ka, 0, srow));
    SWE_CUDA_TRY(cudaMemset(P.Kb, 0, srow));
    SWE_CUDA_TRY(cudaMemset(P.D, 0, scomp));
    int dev = 0, sms = 0, per_sm = 0;
    SWE_CUDA_TRY(cudaGetDevice(&dev));
    SWE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (fsize == 8)
        SWE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_kernel<double, kStage1>, kStageThreads, 0));
    else
        SWE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_kernel<float, kStage1>, kStageThreads, 0));
    const int want = ceil_div(P.n, 4 * kStageWarps);
    P.grid = std::max(1, std::min(want, sms * std::max(per_sm, 1)));
    P.sms = sms;
    P.ready = true;
    // Keep the fastest stage kernel for this patch: the pipelined kernel with 64-,
    // 32- or 16-node tiles, the register kernel, or the node-per-lane kernel with
    // 1, 2 or 4 lanes per node.  (The first two do identical arithmetic; the
    // node-per-lane kernel sums each node's slots in a different order.)
    {
        cudaEvent_t e0, e1;
        SWE_CUDA_TRY(cudaEventCreate(&e0));
        SWE_CUDA_TRY(cudaEventCreate(&e1));
        SWE_CUDA_TRY(cudaMemsetAsync(P.Kx, 0, srow, P.stream));
        // candidates 0-2: pipelined 64 / 32 / 16; 3: register; 4-21: node-per-lane
        // shape 6 + (c - 4) in swe_cuda_select_kernel's numbering
        constexpr int kLane0 = 4, kCand = kLane0 + 18;
        const int cand_tile[3] = {64, 32, 16};
        float us_c[kCand] = {};
        for (int c = 0; c < kCand; ++c) {
            if (c < 3) { P.kernel_choice = 0; P.tma_tile = cand_tile[c]; }
            else if (c == 3) P.kernel_choice = 1;
            else lane_shape(P, c - kLane0);
            // stages 0, 1 and 2 chained as a step chains them (none of them writes H):
            // one sequence to warm up, then three timed
            auto stages = [&]() {
                for (int s = 0; s < 3; ++s) { if (fsize == 8) P.launch_t<double>(s); else P.launch_t<float>(s); }
            };
            stages();
            SWE_CUDA_TRY(cudaEventRecord(e0, P.stream));
            for (int r = 0; r < 3; ++r) stages();
            SWE_CUDA_TRY(cudaEventRecord(e1, P.stream));
            SWE_CUDA_TRY(cudaEventSynchronize(e1));
            SWE_CUDA_TRY(cudaGetLastError());
            float ms = 0.f;
            SWE_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            us_c[c] = ms * 1e3f / 9.f;
        }
        count_launch(12 * kCand);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // the pipelined and node-per-lane kernels keep their fastest shapes, also
        // when another kernel wins
        int bt = 0, bl = kLane0;
        for (int c = 1; c < 3; ++c)
            if (us_c[c] < us_c[bt]) bt = c;
        // a shape with the L2 prefetch must beat the best one without by 3 %: timed
        // back to back the two come within a few per cent, while a step that starts
        // from a cold L2 runs 9 % faster without (N=40962)
        int bp = -1;
        for (int c = kLane0; c < kCand; ++c) {
            lane_shape(P, c - kLane0);
            if (P.lane_pf) { if (bp < 0 || us_c[c] < us_c[bp]) bp = c; }
            else if (us_c[c] < us_c[bl]) bl = c;
        }
        if (bp >= 0 && us_c[bp] < 0.97f * us_c[bl]) bl = bp;
        P.tma_tile = cand_tile[bt];
        lane_shape(P, bl - kLane0);
        P.tune_us[0] = us_c[bt];
        P.tune_us[1] = us_c[3];
        P.tune_us[2] = us_c[bl];
        int best = 0;
        for (int k = 1; k < 3; ++k)
            if (P.tune_us[k] < P.tune_us[best]) best = k;
        P.kernel_choice = best;
        SWE_TRY(check_tma_err());
    }
    if ((st = P.build_graph()) != SWE_OK) return st;
    return SWE_OK;
}

int swe_cuda_set_state(const void* Hh) {
    SWE_TRY(require_ready());
    if (!Hh) { set_error("null H"); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    const size_t bytes = P.fbytes(4L * P.rows);
    if (P.cl.layout & SWE_LAYOUT_CFDL) {
        // CFDL's SVM_LIN_ID is node-major [p][4], the device layout: no permutation
        SWE_CUDA_TRY(cudaMemcpyAsync(P.H, Hh, bytes, cudaMemcpyHostToDevice, P.stream));
    } else {
        SWE_CUDA_TRY(cudaMemcpyAsync(P.raw, Hh, bytes, cudaMemcpyHostToDevice, P.stream));
        SWE_TRY(permute_state(P.raw, P.H, 0));
    }
    // (the K ping-pong buffers need no copy: stage 0 gathers from H and writes K
    // before any stage reads it)
    P.steps_done = 0;
    return SWE_OK;
}

int swe_cuda_get_state(void* Hh) {
    SWE_TRY(require_ready());
    if (!Hh) { set_error("null H"); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    const size_t bytes = P.fbytes(4L * P.rows);
    if (P.cl.layout & SWE_LAYOUT_CFDL) {
        SWE_CUDA_TRY(cudaMemcpyAsync(Hh, P.H, bytes, cudaMemcpyDeviceToHost, P.stream));
    } else {
        SWE_TRY(permute_state(P.H, P.raw, 1));
        SWE_CUDA_TRY(cudaMemcpyAsync(Hh, P.raw, bytes, cudaMemcpyDeviceToHost, P.stream));
    }
    return check_tma_err();   // one synchronisation covers the state copy and the error word
}

int swe_cuda_eval_rhs(const void* K, void* Fh) {
    SWE_TRY(require_ready());
    if (!K || !Fh) { set_error("null K or F"); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    SWE_CUDA_TRY(cudaMemcpyAsync(P.raw, K, P.fbytes(4L * P.rows), cudaMemcpyHostToDevice, P.stream));
    SWE_TRY(permute_state(P.raw, P.Kx, 0));
    SWE_TRY(P.launch(kEvalOnly));
    // F has compute_size rows in the caller's SVM layout (compute-local ids)
    CallerLayout cl = P.cl;
    const long total = 4L * P.n;
    if (P.fsize == 8)
        permute_state_kernel<double><<<ceil_div(total, 256), 256, 0, P.stream>>>((const double*)P.F, (double*)P.raw, P.n, cl, 1);
    else
        permute_state_kernel<float><<<ceil_div(total, 256), 256, 0, P.stream>>>((const float*)P.F, (float*)P.raw, P.n, cl, 1);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    SWE_CUDA_TRY(cudaMemcpyAsync(Fh, P.raw, P.fbytes(total), cudaMemcpyDeviceToHost, P.stream));
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    return SWE_OK;
}

int swe_cuda_rk_substep(int substep_id) {
    SWE_TRY(require_ready());
    if (substep_id < 0 || substep_id > 3) { set_error("substep_id %d not in 0..3", substep_id); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    SWE_TRY(P.launch(substep_id));
    return substep_id == 3 ? after_step() : SWE_OK;
}

int swe_cuda_step(int nsteps) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    if (nsteps < 0) { set_error("nsteps < 0"); return SWE_ERR_ARG; }
    if (P.pid0 != 0 || P.rows != P.n) {
        set_error("swe_cuda_step runs whole steps without halo exchanges: a patch with halo rows steps by "
                  "swe_cuda_rk_substep, with swe_cuda_halo_pack / swe_cuda_halo_unpack between substeps");
        return SWE_ERR_ARG;
    }
    if (P.timing) {
        for (auto& e : P.step_ev) if (!e) SWE_CUDA_TRY(cudaEventCreate(&e));
        SWE_CUDA_TRY(cudaEventRecord(P.step_ev[0], P.stream));
    }
    if (P.use_tma()) P.err_pending = true;
    for (int s = 0; s < nsteps; ++s) {
        SWE_CUDA_TRY(cudaGraphLaunch(P.graph, P.stream));
        SWE_TRY(after_step());
    }
    count_launch(4LL * nsteps);
    if (P.timing) {
        SWE_CUDA_TRY(cudaEventRecord(P.step_ev[1], P.stream));
        P.step_timed = true;
    }
    return SWE_OK;
}

}  // extern "C"

// Halo rows of a patch (rows outside compute_pid_s .. compute_pid_s + compute_size - 1
// that the compute rows' stencils read): the caller exchanges them between substeps,
// as the reference's exchange_SVM_halos does after eval_K and update_H
// (rk4_rbffd_swe.c:86-158).  pack copies the listed patch rows of the buffer substep
// `substep_id` reads into a [count][4] device buffer; unpack writes such a buffer into
// the listed rows.  Row lists are set once by swe_cuda_halo_setup.
template <typename T>
__global__ void halo_copy_kernel(const int* __restrict__ rows, int count, const T* __restrict__ src, T* __restrict__ dst,
                                 int to_rows) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * 4) return;
    const int j = t >> 2, f = t & 3;
    const long r = rows[j];
    if (to_rows) dst[4 * r + f] = src[t];
    else dst[t] = src[4 * r + f];
}

static int halo_copy(int substep_id, void* ext, bool pack) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    if (substep_id < 0 || substep_id > 3) { set_error("substep_id %d not in 0..3", substep_id); return SWE_ERR_ARG; }
    const int count = pack ? P.n_send : P.n_recv;
    const int* rows = pack ? P.halo_send : P.halo_recv;
    if (count == 0) return SWE_OK;
    if (!ext) { set_error("swe_cuda_halo_%s: null buffer", pack ? "pack" : "unpack"); return SWE_ERR_ARG; }
    void* buf = P.stage_input(substep_id);
    const int threads = 256, blocks = ceil_div(4L * count, threads);
    if (P.fsize == 8)
        halo_copy_kernel<double><<<blocks, threads, 0, P.stream>>>(rows, count, (const double*)(pack ? buf : ext),
                                                                  (double*)(pack ? ext : buf), pack ? 0 : 1);
    else
        halo_copy_kernel<float><<<blocks, threads, 0, P.stream>>>(rows, count, (const float*)(pack ? buf : ext),
                                                                 (float*)(pack ? ext : buf), pack ? 0 : 1);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    return SWE_OK;
}

extern "C" {

int swe_cuda_halo_setup(const int* send_rows, int n_send, const int* recv_rows, int n_recv) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    if (n_send < 0 || n_recv < 0 || (n_send && !send_rows) || (n_recv && !recv_rows)) {
        set_error("swe_cuda_halo_setup: bad row lists");
        return SWE_ERR_ARG;
    }
    for (int j = 0; j < n_send; ++j)
        if (send_rows[j] < P.pid0 || send_rows[j] >= P.pid0 + P.n) {
            set_error("swe_cuda_halo_setup: send row %d (entry %d) is not a compute row %d..%d", send_rows[j], j,
                      P.pid0, P.pid0 + P.n - 1);
            return SWE_ERR_INDEX;
        }
    for (int j = 0; j < n_recv; ++j)
        if (recv_rows[j] < 0 || recv_rows[j] >= P.rows || (recv_rows[j] >= P.pid0 && recv_rows[j] < P.pid0 + P.n)) {
            set_error("swe_cuda_halo_setup: receive row %d (entry %d) is not a halo row of the %d-row patch",
                      recv_rows[j], j, P.rows);
            return SWE_ERR_INDEX;
        }
    if (P.halo_send) cudaFree(P.halo_send);
    if (P.halo_recv) cudaFree(P.halo_recv);
    P.halo_send = P.halo_recv = nullptr;
    P.n_send = P.n_recv = 0;
    SWE_CUDA_TRY(cudaMalloc(&P.halo_send, sizeof(int) * std::max(n_send, 1)));
    SWE_CUDA_TRY(cudaMalloc(&P.halo_recv, sizeof(int) * std::max(n_recv, 1)));
    if (n_send)
        SWE_CUDA_TRY(cudaMemcpyAsync(P.halo_send, send_rows, sizeof(int) * n_send, cudaMemcpyHostToDevice, P.stream));
    if (n_recv)
        SWE_CUDA_TRY(cudaMemcpyAsync(P.halo_recv, recv_rows, sizeof(int) * n_recv, cudaMemcpyHostToDevice, P.stream));
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    P.n_send = n_send;
    P.n_recv = n_recv;
    return SWE_OK;
}

int swe_cuda_halo_pack(int substep_id, void* send_buf) { return halo_copy(substep_id, send_buf, true); }
int swe_cuda_halo_unpack(int substep_id, const void* recv_buf) {
    return halo_copy(substep_id, const_cast<void*>(recv_buf), false);
}

int swe_cuda_sync(void) {
    SWE_TRY(require_ready());
    return check_tma_err();   // synchronises the stream
}

int swe_cuda_select_kernel(int which) {
    SWE_TRY(require_ready());
    if (which < 0 || which > 23) {
        set_error("swe_cuda_select_kernel: 0 (pipelined), 1 (register), 2 / 3 / 4 (pipelined, 64 / 32 / 16-node tiles), "
                  "5 (node-per-lane), 6-17 (node-per-lane shapes: 6 + lanes index (1/2/4 lanes per node) "
                  "+ 3 x (5 CTAs per SM) + 6 x (L2 prefetch)), 18-23 (the same at 3 CTAs per SM: 18 + lanes "
                  "index + 3 x (L2 prefetch)), got %d", which);
        return SWE_ERR_ARG;
    }
    Plain& P = g_plain;
    const bool piped = which == 0 || (which >= 2 && which <= 4);
    if (piped && !P.tma_ok) { set_error("swe_cuda_select_kernel: the pipelined kernel is not set up"); return SWE_ERR_STATE; }
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    P.kernel_choice = piped ? 0 : (which == 1 ? 1 : 2);
    if (which == 2) P.tma_tile = 64;
    if (which == 3) P.tma_tile = 32;
    if (which == 4) P.tma_tile = 16;
    if (which >= 6) lane_shape(P, which - 6);
    if (P.graph) cudaGraphExecDestroy(P.graph);
    P.graph = nullptr;
    return P.build_graph();
}

int swe_cuda_set_index_width(int bits) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    if (bits != 16 && bits != 32) {
        set_error("swe_cuda_set_index_width: 16 or 32, got %d", bits);
        return SWE_ERR_ARG;
    }
    if (bits == 16 && !P.idxs_fit) {
        set_error("swe_cuda_set_index_width: a stencil row lies more than 32767 rows from its node");
        return SWE_ERR_ARG;
    }
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    P.idxs_ok = bits == 16;
    if (P.graph) cudaGraphExecDestroy(P.graph);
    P.graph = nullptr;
    return P.build_graph();
}

int swe_cuda_kernel_info(int* out) {
    SWE_TRY(require_ready());
    if (!out) { set_error("null out"); return SWE_ERR_ARG; }
    out[0] = g_plain.kernel_choice;
    out[1] = g_plain.tma_ok ? g_plain.tma_tile : 0;
    out[2] = (int)(g_plain.tune_us[0] * 1000.f);   // nanoseconds per stage launch, pipelined
    out[3] = (int)(g_plain.tune_us[1] * 1000.f);   // register-streaming
    out[4] = g_plain.lane_lpn;
    out[5] = (int)(g_plain.tune_us[2] * 1000.f);   // node-per-lane
    out[6] = g_plain.lane_pf;
    out[7] = g_plain.lane_minb;
    out[8] = g_plain.idxs_ok ? 1 : 0;
    return SWE_OK;
}

int swe_cuda_set_timing(int enabled) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    P.timing = enabled != 0;
    P.ev_used = 0;
    P.step_timed = false;
    return SWE_OK;
}

int swe_cuda_last_timings(double* out) {
    SWE_TRY(require_ready());
    if (!out) { set_error("null out"); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    double total = 0.0;
    for (size_t e = 0; e < P.ev_used; e += 2) {
        float ms = 0.f;
        SWE_CUDA_TRY(cudaEventElapsedTime(&ms, P.ev[e], P.ev[e + 1]));
        total += ms * 1e-3;
    }
    out[0] = total;
    out[1] = (double)(P.ev_used / 2);
    out[2] = 0.0;
    if (P.step_timed) {
        float ms = 0.f;
        SWE_CUDA_TRY(cudaEventElapsedTime(&ms, P.step_ev[0], P.step_ev[1]));
        out[2] = ms * 1e-3;
    }
    P.ev_used = 0;
    return SWE_OK;
}

void* swe_cuda_stream(void) { return g_plain.ready ? (void*)g_plain.stream : nullptr; }

int swe_cuda_invariants(double* me) {
    SWE_TRY(require_ready());
    if (!me) { set_error("null out"); return SWE_ERR_ARG; }
    Plain& P = g_plain;
    SWE_CUDA_TRY(cudaMemsetAsync(P.inv, 0, 2 * sizeof(double), P.stream));
    const int blocks = std::min(ceil_div(P.n, 256), 1184);
    if (P.fsize == 8)
        invariants_kernel<double><<<blocks, 256, 0, P.stream>>>((const double*)P.H, (const double*)P.PT, P.n, P.gh0, P.inv);
    else
        invariants_kernel<float><<<blocks, 256, 0, P.stream>>>((const float*)P.H, (const float*)P.PT, P.n, (double)(float)P.gh0, P.inv);
    count_launch();
    SWE_CUDA_TRY(cudaGetLastError());
    SWE_CUDA_TRY(cudaMemcpyAsync(me, P.inv, 2 * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    SWE_CUDA_TRY(cudaStreamSynchronize(P.stream));
    const double area = 4.0 * 3.14159265358979323846 / (double)P.n;
    me[0] *= area;
    me[1] *= area;
    // NaN/Inf watchdog: one non-finite value anywhere in H makes a sum non-finite
    if (!std::isfinite(me[0]) || !std::isfinite(me[1])) {
        set_error("swe_cuda_invariants: the state holds NaN or Inf (mass %g, energy %g)", me[0], me[1]);
        return SWE_ERR_NONFINITE;
    }
    return SWE_OK;
}

int swe_hist_open(const char* path, int interval) {
    SWE_TRY(require_ready());
    Plain& P = g_plain;
    int dev = 0;
    SWE_CUDA_TRY(cudaGetDevice(&dev));
    return P.hist.open(path, interval, 4LL * P.rows, P.fsize, P.dt, P.cl.layout, P.cl.S, dev);
}

int swe_hist_close(void) {
    SWE_TRY(require_ready());
    SWE_CUDA_TRY(cudaStreamSynchronize(g_plain.stream));
    return g_plain.hist.close();
}

int swe_hist_stats(long long* out) {
    SWE_TRY(require_ready());
    if (!out) { set_error("swe_hist_stats: null out"); return SWE_ERR_ARG; }
    out[0] = g_plain.hist.active() ? 1 : 0;
    out[1] = g_plain.hist.records();
    out[2] = g_plain.hist.bytes();
    out[3] = g_plain.steps_done;
    return SWE_OK;
}

int swe_cuda_finalize(void) {
    if (g_plain.stream) cudaStreamSynchronize(g_plain.stream);
    g_plain.release();
    return SWE_OK;
}

}  // extern "C"
