// Shared helpers of the sm_100a library: status/error plumbing, launch
// counting, and the caller-layout index maps of the reference
// (swe_code/main/include/swe_config.h:21-54).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/swe_b200.h"

namespace swe {

void set_error(const char* fmt, ...);
void count_launch(long long n = 1);

#define SWE_CUDA_TRY(call)                                                                     \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::swe::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                             __LINE__);                                                        \
            return SWE_ERR_CUDA;                                                               \
        }                                                                                      \
    } while (0)

#define SWE_TRY(expr)               \
    do {                            \
        int st_ = (expr);           \
        if (st_ != SWE_OK) return st_; \
    } while (0)

// Caller-side layout of one patch (the reference's compile-time options).
struct CallerLayout {
    int layout = 0;   // SWE_LAYOUT_CFDL | SWE_LAYOUT_SFDL
    int S = 1;        // SIMD_LENGTH (tile width)
    int pnbr = 0;     // padded_Nnbr: row length of the DM arrays

    // DM_LIN_ID (swe_config.h:31-36)
    __host__ __device__ long dm(long i, long j) const {
        return (layout & SWE_LAYOUT_SFDL) ? (i / S) * S * pnbr + j * S + (i % S) : i * pnbr + j;
    }
    // VECT_LIN_ID (swe_config.h:31-36)
    __host__ __device__ long vect(long i, long c) const {
        return (layout & SWE_LAYOUT_SFDL) ? (i / S) * S * 3 + c * S + (i % S) : i * 3 + c;
    }
    // SVM_LIN_ID (swe_config.h:50-54)
    __host__ __device__ long svm(long p, long sv) const {
        return (layout & SWE_LAYOUT_CFDL) ? 4 * p + sv : (p / S) * S * 4 + sv * S + (p % S);
    }
};

// Device layout constants of the plain form.
constexpr int kSlots = 32;      // stencil slots per node (nnbr <= 32)
constexpr int kLanesPerNode = 8;
constexpr int kSlotChunks = kSlots / kLanesPerNode;   // 4 slots per lane
constexpr int kPointStride = 20;                      // per-node pointwise values (17 used)

// Pointwise record, per node: x y z f ghm pu0..2 pv0..2 pw0..2 gg0..2 (17)
enum PointField { PT_X = 0, PT_Y, PT_Z, PT_F, PT_GHM, PT_PU, PT_PV = PT_PU + 3, PT_PW = PT_PV + 3,
                  PT_GG = PT_PW + 3 };

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// Programmatic dependent launch.  The previous stage's writes are visible only
// after pdl_wait(); a CTA lets the next stage launch (pdl_trigger) only after its
// own wait, so at most two consecutive stages are ever resident together.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Bulk prefetch of a contiguous block into L2 (address and size 16-byte aligned);
// it completes on its own and costs the issuing thread no registers.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

}  // namespace swe
