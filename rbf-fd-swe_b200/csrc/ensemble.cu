// Batched-ensemble form: swe_ens_* entry points of include/swe_b200.h.
//
// B members (a multiple of 32, at most 64) share one grid.  The library
// orders nodes by the reference's RCM permutation (rcm/rcm.c:9-62, restated in
// host_layout.cu) so that tiles of consecutive nodes have compact neighbour
// sets, builds per-tile neighbour tables once, keeps all member states
// device-resident, and runs each RK4 stage as one tcgen05 kernel
// (ensemble_kernel.cuh).  An autotuner times every (tile nodes T, members per
// CTA) variant on the live state and keeps the fastest; whole steps replay a
// captured CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ensemble_kernel.cuh"

extern "C" int swe_host_rcm_mapping(int n, int nnbr, const int* idx, int* mapping);

namespace swe {
namespace {

// Per-tile neighbour tables for one tile size T.
struct Tables {
    bool ok = false;
    int ntiles = 0, kmax_seen = 0;
    int* rows = nullptr;
    int* kcount = nullptr;
    uint8_t* local = nullptr;
};

struct Variant {
    int T = 4, hpc = 1;
    bool usable = false;
};

template <int T>
bool build_tiles(int n, int nnbr, const std::vector<int>& idx, std::vector<int>& rows, std::vector<int>& kcount,
                 std::vector<uint8_t>& local, int& ntiles, int& kmax_seen) {
    using G = EnsTile<T>;
    ntiles = (n + T - 1) / T;
    rows.assign((size_t)ntiles * G::kKmax, -1);
    kcount.assign(ntiles, 0);
    local.assign((size_t)ntiles * T * 32, 255);
    std::vector<int> u;
    kmax_seen = 0;
    for (int tile = 0; tile < ntiles; ++tile) {
        u.clear();
        for (int t = 0; t < T; ++t) {
            const long node = (long)tile * T + t;
            if (node >= n) break;
            for (int j = 0; j < nnbr; ++j) u.push_back(idx[node * nnbr + j]);
        }
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        kmax_seen = std::max(kmax_seen, (int)u.size());
        if ((int)u.size() > G::kKmax) return false;
        kcount[tile] = (int)u.size();
        std::copy(u.begin(), u.end(), rows.begin() + (size_t)tile * G::kKmax);
        for (int t = 0; t < T; ++t) {
            const long node = (long)tile * T + t;
            if (node >= n) break;
            for (int j = 0; j < nnbr; ++j) {
                const int k = (int)(std::lower_bound(u.begin(), u.end(), idx[node * nnbr + j]) - u.begin());
                local[((size_t)tile * T + t) * 32 + j] = (uint8_t)k;
            }
        }
    }
    return true;
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
    int members = 0, n = 0, nnbr = 0, mf = 0, halves = 0;
    double gh0 = 0, dt = 0;
    std::vector<int> perm_h;
    int* perm = nullptr;
    float4* W = nullptr;
    float4* PT = nullptr;
    float *H32 = nullptr, *D32 = nullptr, *Ka = nullptr, *Kb = nullptr, *F = nullptr, *Kx = nullptr;
    double *Hh = nullptr, *Dh = nullptr, *io = nullptr, *inv = nullptr;
    float* bkH32 = nullptr;
    double* bkHh = nullptr;
    int* err = nullptr;
    Tables tab[2];        // T = 4, T = 8
    Variant var[4];       // (4,1) (4,2) (8,1) (8,2)
    int chosen = -1;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool timing = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool timed = false;
    double tune_ms[4] = {0, 0, 0, 0};

    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        void* ps[] = {perm, W, PT, H32, D32, Ka, Kb, F, Kx, Hh, Dh, io, inv, bkH32, bkHh, err};
        for (void* p : ps) if (p) cudaFree(p);
        perm = nullptr; W = nullptr; PT = nullptr; H32 = D32 = Ka = Kb = F = Kx = nullptr;
        Hh = Dh = io = inv = nullptr; bkH32 = nullptr; bkHh = nullptr; err = nullptr;
        for (auto& t : tab) {
            if (t.rows) cudaFree(t.rows);
            if (t.kcount) cudaFree(t.kcount);
            if (t.local) cudaFree(t.local);
            t = Tables{};
        }
        for (auto& v : var) v = Variant{};
        for (auto& e : ev) { if (e) cudaEventDestroy(e); e = nullptr; }
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        chosen = -1;
        ready = false;
    }

    EnsArgs args(int mode) const {
        EnsArgs a{};
        a.n = n;
        a.mf = mf;
        a.W = W;
        a.PT = PT;
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

    template <int T, int HPC>
    static size_t smem_bytes() {
        return (size_t)HPC * 2 * EnsTile<T>::kABytes + 2 * EnsTile<T>::kBBytes;
    }

    template <int T, int HPC>
    void launch_tv(int mode) {
        const Tables& tb = tab[T == 8];
        EnsArgs a = args(mode);
        a.rows = tb.rows;
        a.kcount = tb.kcount;
        a.local = tb.local;
        a.ntiles = tb.ntiles;
        const dim3 grid(tb.ntiles, halves / HPC);
        const size_t sm = smem_bytes<T, HPC>();
        switch (mode) {
            case 0: ens_stage_kernel<T, HPC, kStage0><<<grid, 128 * HPC, sm, stream>>>(a); break;
            case 1: ens_stage_kernel<T, HPC, kStage1><<<grid, 128 * HPC, sm, stream>>>(a); break;
            case 2: ens_stage_kernel<T, HPC, kStage2><<<grid, 128 * HPC, sm, stream>>>(a); break;
            case 3: ens_stage_kernel<T, HPC, kStage3><<<grid, 128 * HPC, sm, stream>>>(a); break;
            default: ens_stage_kernel<T, HPC, kEvalOnly><<<grid, 128 * HPC, sm, stream>>>(a); break;
        }
    }

    void launch(int vi, int mode) {
        const Variant& v = var[vi];
        if (v.T == 4 && v.hpc == 1) launch_tv<4, 1>(mode);
        else if (v.T == 4) launch_tv<4, 2>(mode);
        else if (v.hpc == 1) launch_tv<8, 1>(mode);
        else launch_tv<8, 2>(mode);
        count_launch();
    }

    template <int T, int HPC>
    static int set_attrs() {
        const int sm = (int)smem_bytes<T, HPC>();
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, HPC, kStage0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, HPC, kStage1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, HPC, kStage2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, HPC, kStage3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        SWE_CUDA_TRY(cudaFuncSetAttribute(ens_stage_kernel<T, HPC, kEvalOnly>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
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

    int check_err() {
        int h = 0;
        SWE_CUDA_TRY(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        SWE_CUDA_TRY(cudaStreamSynchronize(stream));
        if (h) {
            set_error("ensemble kernel: a bounded mbarrier wait for tensor-core completion ran out");
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
    for (int vi = 0; vi < 4; ++vi) {
        E.tune_ms[vi] = -1.0;
        if (!E.var[vi].usable) continue;
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
    Ensemble& E = g_ens;
    E.release();
    E.members = members;
    E.n = n;
    E.nnbr = nnbr;
    E.mf = 4 * members;
    E.halves = members / 32;
    E.gh0 = gh0;
    E.dt = dt;
    // RCM order (mapping[new] = old) and the renumbered stencils
    E.perm_h.assign(n, 0);
    SWE_TRY(swe_host_rcm_mapping(n, nnbr, idx, E.perm_h.data()));
    std::vector<int> inv(n), ridx((size_t)n * nnbr);
    for (int i = 0; i < n; ++i) inv[E.perm_h[i]] = i;
    for (long i = 0; i < n; ++i)
        for (int j = 0; j < nnbr; ++j) ridx[i * nnbr + j] = inv[idx[(long)E.perm_h[i] * nnbr + j]];
    // static data in FP32, RCM order
    std::vector<float> w((size_t)n * 32 * 4, 0.f), pt((size_t)n * kPointStride, 0.f);
    for (long i = 0; i < n; ++i) {
        const long o = E.perm_h[i];
        for (int j = 0; j < nnbr; ++j) {
            float* q = &w[((size_t)i * 32 + j) * 4];
            q[0] = (float)Dx[o * nnbr + j]; q[1] = (float)Dy[o * nnbr + j];
            q[2] = (float)Dz[o * nnbr + j]; q[3] = (float)L[o * nnbr + j];
        }
        float* r = &pt[(size_t)i * kPointStride];
        r[PT_X] = (float)x[o]; r[PT_Y] = (float)y[o]; r[PT_Z] = (float)z[o]; r[PT_F] = (float)f[o];
        r[PT_GHM] = (float)ghm[o];
        for (int c = 0; c < 3; ++c) {
            r[PT_PU + c] = (float)p_u[o * 3 + c]; r[PT_PV + c] = (float)p_v[o * 3 + c];
            r[PT_PW + c] = (float)p_w[o * 3 + c]; r[PT_GG + c] = (float)gradghm[o * 3 + c];
        }
    }
    SWE_CUDA_TRY(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
    const size_t s32 = (size_t)n * E.mf * sizeof(float), s64 = (size_t)n * members * sizeof(double);
    SWE_CUDA_TRY(cudaMalloc(&E.perm, n * sizeof(int)));
    SWE_CUDA_TRY(cudaMalloc(&E.W, w.size() * sizeof(float)));
    SWE_CUDA_TRY(cudaMalloc(&E.PT, pt.size() * sizeof(float)));
    for (float** p : {&E.H32, &E.D32, &E.Ka, &E.Kb, &E.F, &E.Kx, &E.bkH32}) SWE_CUDA_TRY(cudaMalloc(p, s32));
    for (double** p : {&E.Hh, &E.Dh, &E.bkHh}) SWE_CUDA_TRY(cudaMalloc(p, s64));
    SWE_CUDA_TRY(cudaMalloc(&E.io, (size_t)n * members * 4 * sizeof(double)));
    SWE_CUDA_TRY(cudaMalloc(&E.inv, 2 * members * sizeof(double)));
    SWE_CUDA_TRY(cudaMalloc(&E.err, sizeof(int)));
    SWE_CUDA_TRY(cudaMemset(E.err, 0, sizeof(int)));
    for (float* p : {E.H32, E.D32, E.Ka, E.Kb, E.F, E.Kx}) SWE_CUDA_TRY(cudaMemset(p, 0, s32));
    for (double* p : {E.Hh, E.Dh}) SWE_CUDA_TRY(cudaMemset(p, 0, s64));
    SWE_CUDA_TRY(cudaMemcpy(E.perm, E.perm_h.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    SWE_CUDA_TRY(cudaMemcpy(E.W, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
    SWE_CUDA_TRY(cudaMemcpy(E.PT, pt.data(), pt.size() * sizeof(float), cudaMemcpyHostToDevice));
    // tile tables for the two tile sizes
    {
        std::vector<int> rows, kcount;
        std::vector<uint8_t> local;
        for (int ti = 0; ti < 2; ++ti) {
            Tables& tb = E.tab[ti];
            tb.ok = ti == 0 ? build_tiles<4>(n, nnbr, ridx, rows, kcount, local, tb.ntiles, tb.kmax_seen)
                            : build_tiles<8>(n, nnbr, ridx, rows, kcount, local, tb.ntiles, tb.kmax_seen);
            if (!tb.ok) continue;
            SWE_CUDA_TRY(cudaMalloc(&tb.rows, rows.size() * sizeof(int)));
            SWE_CUDA_TRY(cudaMalloc(&tb.kcount, kcount.size() * sizeof(int)));
            SWE_CUDA_TRY(cudaMalloc(&tb.local, local.size()));
            SWE_CUDA_TRY(cudaMemcpy(tb.rows, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
            SWE_CUDA_TRY(cudaMemcpy(tb.kcount, kcount.data(), kcount.size() * sizeof(int), cudaMemcpyHostToDevice));
            SWE_CUDA_TRY(cudaMemcpy(tb.local, local.data(), local.size(), cudaMemcpyHostToDevice));
        }
    }
    if (!E.tab[0].ok && !E.tab[1].ok) {
        const int k4 = E.tab[0].kmax_seen, k8 = E.tab[1].kmax_seen;
        E.release();
        set_error("swe_ens_init: a tile's neighbour set exceeds the kernel limit (T=4: %d rows > %d; T=8: %d > %d)",
                  k4, EnsTile<4>::kKmax, k8, EnsTile<8>::kKmax);
        return SWE_ERR_ARG;
    }
    {
        const int Ts[4] = {4, 4, 8, 8}, hpcs[4] = {1, 2, 1, 2};
        for (int vi = 0; vi < 4; ++vi) {
            E.var[vi].T = Ts[vi];
            E.var[vi].hpc = hpcs[vi];
            E.var[vi].usable = E.tab[Ts[vi] == 8].ok && hpcs[vi] <= E.halves;
        }
    }
    SWE_TRY((Ensemble::set_attrs<4, 1>()));
    SWE_TRY((Ensemble::set_attrs<4, 2>()));
    SWE_TRY((Ensemble::set_attrs<8, 1>()));
    SWE_TRY((Ensemble::set_attrs<8, 2>()));
    E.ready = true;
    // default choice until tuned: T = 4, one half per CTA
    E.chosen = E.var[0].usable ? 0 : 2;
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
        for (int vi = 0; vi < 4; ++vi) ms_per_step[vi] = g_ens.tune_ms[vi];
    return SWE_OK;
}

int swe_ens_use_variant(int tile_nodes, int members_per_cta) {
    SWE_TRY(ens_ready());
    for (int vi = 0; vi < 4; ++vi) {
        const Variant& v = g_ens.var[vi];
        if (v.T == tile_nodes && 32 * v.hpc == members_per_cta) {
            if (!v.usable) {
                set_error("swe_ens_use_variant: (%d, %d) not usable for this grid / member count", tile_nodes, members_per_cta);
                return SWE_ERR_ARG;
            }
            g_ens.chosen = vi;
            return g_ens.build_graph();
        }
    }
    set_error("swe_ens_use_variant: no variant (%d nodes, %d members per CTA)", tile_nodes, members_per_cta);
    return SWE_ERR_ARG;
}

int swe_ens_config(int* out) {
    SWE_TRY(ens_ready());
    if (!out) { set_error("swe_ens_config: null out"); return SWE_ERR_ARG; }
    const Variant& v = g_ens.var[g_ens.chosen];
    out[0] = v.T;
    out[1] = 32 * v.hpc;
    out[2] = g_ens.tab[0].kmax_seen;
    out[3] = g_ens.tab[1].kmax_seen;
    return SWE_OK;
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
