// Internal declarations shared by the CUDA translation units of libb3gpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/b3gpu.h"

// ---------------------------------------------------------------------------
// Error reporting
// ---------------------------------------------------------------------------
void b3_set_error(const char* fmt, ...);

#define B3_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e__ = (call);                                              \
        if (e__ != cudaSuccess) {                                              \
            b3_set_error("%s:%d %s -> %s", __FILE__, __LINE__, #call,          \
                         cudaGetErrorString(e__));                             \
            return B3_ERR_CUDA;                                                \
        }                                                                      \
    } while (0)

#define B3_CHECK_LAUNCH()                                                      \
    do {                                                                       \
        cudaError_t e__ = cudaGetLastError();                                  \
        if (e__ != cudaSuccess) {                                              \
            b3_set_error("%s:%d launch -> %s", __FILE__, __LINE__,             \
                         cudaGetErrorString(e__));                             \
            return B3_ERR_CUDA;                                                \
        }                                                                      \
    } while (0)

#define B3_TRY(expr)                                                           \
    do {                                                                       \
        int s__ = (expr);                                                      \
        if (s__ != B3_OK) return s__;                                          \
    } while (0)

struct b3Context_t {
    int device = 0;
    int numSMs = 148;
    int maxSmemOptin = 0;
    // scratch for the primitive entry points (grown on demand)
    void* scratch = nullptr;
    size_t scratchBytes = 0;
    int ensureScratch(size_t bytes);
};

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// Device-wide primitives (implemented in primitives.cu). All take a device
// side element count (n_dev) so they can be captured in CUDA graphs without
// host synchronisation; n_max bounds the grid and scratch sizes.
// ---------------------------------------------------------------------------
namespace b3 {

// Polls of a device-side wait before it gives up (the Jacobi grid barrier's
// limit can be changed per world, b3_set_wait_limits).
constexpr int kDefaultSpinLimit = 1 << 22;

// Onesweep radix sort scratch: returns bytes for n_max elements.
size_t radix_scratch_bytes(int64_t n_max, int key_bits);
// Sort (keys, vals) of device count *n_dev (<= n_max). The sorted result
// ends in (keys_alt, vals_alt) when the number of passes is odd, else in
// (keys, vals); *result_in_alt tells which. vals may be null (keys only).
int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                     const int32_t* n_dev, int64_t n_max, int key_bits, void* scratch,
                     size_t scratch_bytes, int32_t* err_flag, cudaStream_t st, bool* result_in_alt,
                     int numSMs);

// Out-of-place sort: (keys_in, vals_in) are only read; the sorted result
// lands in (keys_out, vals_out); (keys_tmp, vals_tmp) hold the passes in
// between (unused for one pass). vals_in may be null (keys only).
int radix_sort_kv_out(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                      uint32_t* keys_tmp, uint32_t* vals_tmp, const int32_t* n_dev, int64_t n_max, int key_bits,
                      void* scratch, size_t scratch_bytes, int32_t* err_flag, cudaStream_t st, int numSMs);
// Interleaved (key, value) pairs (btSortData): result in kv_alt when
// *result_in_alt, else in kv.
int radix_sort_interleaved(uint2* kv, uint2* kv_alt, const int32_t* n_dev, int64_t n_max, int key_bits,
                           void* scratch, size_t scratch_bytes, int32_t* err_flag, cudaStream_t st,
                           bool* result_in_alt, int numSMs);

size_t scan_scratch_bytes(int64_t n_max);
// Exclusive scan of n_dev u32 values; total to d_total (may be null).
int exclusive_scan_u32(const uint32_t* src, uint32_t* dst, const int32_t* n_dev, int64_t n_max,
                       uint32_t* d_total, void* scratch, size_t scratch_bytes, int32_t* err_flag,
                       cudaStream_t st, int numSMs);

int fill_u32(uint32_t* dst, uint32_t v, int64_t n, cudaStream_t st);
int bound_search(const uint32_t* keys, const int32_t* n_dev, int64_t n_max, uint32_t* dst,
                 int64_t n_dst, int mode, cudaStream_t st);
int bound_search_interleaved(const uint2* kv, const int32_t* n_dev, int64_t n_max, uint32_t* dst, int64_t n_dst,
                             int mode, cudaStream_t st);

}  // namespace b3

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
namespace b3dev {

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bounded spin budget for every device-side wait: about 4M polls with a
// short back-off (well under a second), after which the waiter records an
// error and proceeds instead of hanging the GPU.
constexpr int kSpinLimit = b3::kDefaultSpinLimit;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace b3dev
#endif
