// Node ordering on the device: swe_dev_rcm_mapping.
//
// The reference orders nodes by reverse Cuthill-McKee on the host
// (swe_code/rcm/rcm.c:9-62; restated in host_layout.cu): breadth-first from
// node 0, each visited node appending its not yet mapped stencil neighbours in
// increasing order of their count of still-unmapped neighbours.  That count
// changes after every append, so each step depends on all earlier ones and the
// exact permutation is sequential.
//
// This is the same breadth-first level structure built one level at a time, in
// parallel within a level, and reversed at the end:
//   * expand: every node of the current level offers itself as parent to its
//     unmapped stencil neighbours (slots 1..nnbr-1); a neighbour keeps the
//     smallest key (parent position in the order, slot), so children follow
//     their first parent, nearest stencil slot first; the first offer of each
//     neighbour appends it to the next level's list;
//   * sort: one CTA sorts the next level by key in shared memory (bitonic) and
//     writes it after the current level.
// Keys are (parent position, slot), not the reference's dynamic degree, so the
// permutation differs from the reference's; its bandwidth (max and mean over
// nodes of max - min stencil index, as rcm.c:68-96 prints it) is of the same
// size, which is what the gathers' locality depends on.  A level may hold at
// most kMaxLevel nodes (the breadth-first rings of a quasi-uniform spherical
// grid hold a few thousand up to N ~ 10^7).
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace swe {
namespace {

constexpr int kMaxLevel = 16384;         // nodes per breadth-first level
constexpr int kSortThreads = 1024;
constexpr unsigned long long kNoKey = ~0ull;

// Offers of the current level [lv0, lv1) of `order` to their unmapped neighbours.
__global__ void expand_level(int nnbr, const int* __restrict__ idx, const int* __restrict__ order, int lv0, int lv1,
                             const int* __restrict__ mapped, unsigned long long* __restrict__ key,
                             int* __restrict__ next, int* __restrict__ next_count, int* __restrict__ overflow) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)(lv1 - lv0) * (nnbr - 1);
    if (t >= total) return;
    const int p = lv0 + (int)(t / (nnbr - 1));
    const int j = 1 + (int)(t % (nnbr - 1));
    const int v = order[p];
    const int w = idx[(long)v * nnbr + j];
    if (mapped[w]) return;
    const unsigned long long k = ((unsigned long long)p << 8) | (unsigned)j;
    const unsigned long long old = atomicMin(key + w, k);
    if (old == kNoKey) {                      // first offer: w joins the next level
        const int slot = atomicAdd(next_count, 1);
        if (slot < kMaxLevel) next[slot] = w;
        else atomicExch(overflow, 1);
    }
}

// Sorts the next level (count nodes) by key and appends it to `order` at `base`;
// marks the nodes mapped.  One CTA.  Keys are unique ((parent position, slot) names
// one node), and with n < 2^24 a key and its node pack into one 64-bit word, key
// high: (key << 24) | node.
__global__ void __launch_bounds__(kSortThreads) place_level(const int* __restrict__ next, const int* __restrict__ next_count,
                                                            const unsigned long long* __restrict__ key,
                                                            int* __restrict__ order, int base, int* __restrict__ mapped) {
    extern __shared__ unsigned long long sk[];
    __shared__ int s_count;
    if (threadIdx.x == 0) s_count = min(*next_count, kMaxLevel);
    __syncthreads();
    const int count = s_count;
    int size = 1;
    while (size < count) size <<= 1;
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
        if (i < count) {
            const int w = next[i];
            sk[i] = (key[w] << 24) | (unsigned long long)w;
        } else {
            sk[i] = kNoKey;
        }
    }
    __syncthreads();
    for (int k = 2; k <= size; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < size; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const unsigned long long a = sk[i], b = sk[l];
                    if (((i & k) == 0) ? (a > b) : (a < b)) {
                        sk[i] = b;
                        sk[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const int w = (int)(sk[i] & 0xffffffull);
        order[base + i] = w;
        mapped[w] = 1;
    }
}

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" int swe_dev_rcm_mapping(int n, int nnbr, const int* idx, int* mapping) {
    if (n <= 0 || n >= (1 << 24) || nnbr < 2 || nnbr > kSlots || !idx || !mapping) {
        set_error("swe_dev_rcm_mapping: need 0 < n < 2^24, 2 <= nnbr <= %d and both arrays", kSlots);
        return SWE_ERR_ARG;
    }
    for (long t = 0; t < (long)n * nnbr; ++t)
        if (idx[t] < 0 || idx[t] >= n) {
            set_error("swe_dev_rcm_mapping: idx[%ld] = %d outside [0, %d)", t, idx[t], n);
            return SWE_ERR_INDEX;
        }
    int *d_idx = nullptr, *d_order = nullptr, *d_mapped = nullptr, *d_next = nullptr, *d_cnt = nullptr;
    unsigned long long* d_key = nullptr;
    cudaStream_t st = nullptr;
    int status = SWE_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        set_error("swe_dev_rcm_mapping: %s: %s", what, cudaGetErrorString(e));
        status = SWE_ERR_CUDA;
    };
    cudaError_t e;
    const size_t sort_smem = kMaxLevel * sizeof(unsigned long long);
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) { fail(e, "stream"); return status; }
    do {
        if ((e = cudaMalloc(&d_idx, sizeof(int) * (size_t)n * nnbr)) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&d_order, sizeof(int) * (size_t)n)) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&d_mapped, sizeof(int) * (size_t)n)) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&d_key, sizeof(unsigned long long) * (size_t)n)) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&d_next, sizeof(int) * kMaxLevel)) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaMalloc(&d_cnt, 2 * sizeof(int))) != cudaSuccess) { fail(e, "cudaMalloc"); break; }
        if ((e = cudaFuncSetAttribute(place_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sort_smem)) !=
            cudaSuccess) { fail(e, "cudaFuncSetAttribute"); break; }
        cudaMemcpyAsync(d_idx, idx, sizeof(int) * (size_t)n * nnbr, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_mapped, 0, sizeof(int) * (size_t)n, st);
        cudaMemsetAsync(d_key, 0xff, sizeof(unsigned long long) * (size_t)n, st);
        // level 0: node 0, as the reference's breadth-first search starts there
        const int zero = 0, one = 1;
        cudaMemcpyAsync(d_order, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_mapped, &one, sizeof(int), cudaMemcpyHostToDevice, st);
        int lv0 = 0, lv1 = 1;
        int h_cnt[2] = {0, 0};
        while (lv1 < n) {
            cudaMemsetAsync(d_cnt, 0, 2 * sizeof(int), st);
            const long work = (long)(lv1 - lv0) * (nnbr - 1);
            expand_level<<<ceil_div(work, 256), 256, 0, st>>>(nnbr, d_idx, d_order, lv0, lv1, d_mapped, d_key, d_next,
                                                              d_cnt, d_cnt + 1);
            place_level<<<1, kSortThreads, sort_smem, st>>>(d_next, d_cnt, d_key, d_order, lv1, d_mapped);
            count_launch(2);
            if ((e = cudaMemcpyAsync(h_cnt, d_cnt, 2 * sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                (e = cudaStreamSynchronize(st)) != cudaSuccess) { fail(e, "level"); break; }
            if (h_cnt[1]) {
                set_error("swe_dev_rcm_mapping: a breadth-first level holds more than %d nodes", kMaxLevel);
                status = SWE_ERR_ARG;
                break;
            }
            if (h_cnt[0] == 0) {
                set_error("swe_dev_rcm_mapping: stencil graph is not connected (%d of %d nodes reached)", lv1, n);
                status = SWE_ERR_ARG;
                break;
            }
            lv0 = lv1;
            lv1 += h_cnt[0];
        }
        if (status != SWE_OK) break;
        std::vector<int> cm(n);
        if ((e = cudaMemcpyAsync(cm.data(), d_order, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess) { fail(e, "readback"); break; }
        for (int i = 0; i < n; ++i) mapping[i] = cm[n - 1 - i];      // reversed: RCM
    } while (false);
    cudaFree(d_idx);
    cudaFree(d_order);
    cudaFree(d_mapped);
    cudaFree(d_key);
    cudaFree(d_next);
    cudaFree(d_cnt);
    cudaStreamDestroy(st);
    return status;
}
