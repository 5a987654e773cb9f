// Exclusive prefix scan that allocates nothing.
//
// Some callers cannot allocate device memory: an engine or renderer that
// owns every GPU byte through its own pre-sized pool, a real-time loop that
// must not hit cudaMalloc (it can synchronise the device and stall other
// streams), or a plug-in host whose allocator belongs to another runtime.
// b3_prefix_scan_u32 takes its scratch from the context, which grows it
// with cudaMalloc. This entry point keeps its scratch in the file-scope
// device array below instead; the caller passes only the input and output.
//
// Limits and sharing:
//   * at most kStaticScanMaxN (16,777,216) elements per call; larger n is
//     rejected with B3_ERR_CAPACITY;
//   * the array lives on every GPU that loads the library, until exit;
//   * every call on a device uses the same array, and the array keeps the
//     last call's contents; each call clears the parts that must start at
//     zero (tile counter, tile status words, error flag, total) on the
//     stream before the scan, with a set-up kernel that takes n by value;
//   * the scan's look-back waits are bounded; a wait that gives up sets the
//     array's error flag, which the call copies to the caller's d_err
//     (1 = the result is not valid, 0 = a valid scan);
//   * two calls whose work overlaps on the GPU (different streams, or
//     different host threads) race on the array and give wrong results;
//     serialise them on one stream;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first
//     call before any stream capture.
#include "b3_internal.h"

#include <mutex>

namespace {

constexpr int64_t kStaticScanMaxN = 1 << 24;
constexpr int64_t kScanTileElems = 4096;  // k_scan_u32 tile (256 threads x 16)
constexpr size_t kHeaderBytes = 256;       // n, error flag, total
constexpr size_t kStaticScanBytes =
    kHeaderBytes + 256 + (size_t)(kStaticScanMaxN / kScanTileElems + 1) * 8;

__device__ __align__(256) unsigned char g_static_scan_scratch[kStaticScanBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

int static_scratch(int dev, void** ptr, int* sms) {
    if (dev < 0 || dev >= kMaxDevices) return B3_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scan_scratch);
        if (e != cudaSuccess || !p) {
            b3_set_error("cudaGetSymbolAddress(static scan scratch) -> %s", cudaGetErrorString(e));
            return B3_ERR_CUDA;
        }
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            b3_set_error("cudaDeviceGetAttribute -> %s", cudaGetErrorString(e));
            return B3_ERR_CUDA;
        }
        g_sms[dev] = n;
        g_ptr[dev] = p;
    }
    *ptr = g_ptr[dev];
    *sms = g_sms[dev];
    return B3_OK;
}

// Writes n and clears the error flag and the total (header words 0, 1, 2).
__global__ void k_static_scan_begin(int32_t* hdr, int32_t n) {
    hdr[0] = n;
    hdr[1] = 0;
    hdr[2] = 0;
}

// Copies the total and the error flag out of the array to the caller.
__global__ void k_static_scan_end(const int32_t* hdr, uint32_t* d_sum, int32_t* d_err) {
    if (d_sum) *d_sum = (uint32_t)hdr[2];
    if (d_err) *d_err = hdr[1] != 0 ? 1 : 0;
}

}  // namespace

extern "C" int b3_prefix_scan_u32_static(const uint32_t* d_src, uint32_t* d_dst, int64_t n, uint32_t* d_sum,
                                         int32_t* d_err, void* stream) {
    if (n < 0 || (n > 0 && (!d_src || !d_dst))) return B3_ERR_INVALID_ARG;
    if (n > kStaticScanMaxN) {
        b3_set_error("b3_prefix_scan_u32_static: n = %lld exceeds the static limit of %lld elements",
                     (long long)n, (long long)kStaticScanMaxN);
        return B3_ERR_CAPACITY;
    }
    int dev = 0;
    B3_CUDA(cudaGetDevice(&dev));
    void* base = nullptr;
    int sms = 0;
    B3_TRY(static_scratch(dev, &base, &sms));
    cudaStream_t st = as_stream(stream);
    unsigned char* b = (unsigned char*)base;
    int32_t* n_dev = (int32_t*)b;
    int32_t* err = (int32_t*)(b + 4);
    uint32_t* total = (uint32_t*)(b + 8);
    void* body = b + kHeaderBytes;
    const size_t body_bytes = kStaticScanBytes - kHeaderBytes;
    k_static_scan_begin<<<1, 1, 0, st>>>(n_dev, (int32_t)n);
    B3_CHECK_LAUNCH();
    B3_TRY(b3::exclusive_scan_u32(d_src, d_dst, n_dev, n, total, body, body_bytes, err, st, sms));
    if (d_sum || d_err) {
        k_static_scan_end<<<1, 1, 0, st>>>(n_dev, d_sum, d_err);
        B3_CHECK_LAUNCH();
    }
    return B3_OK;
}
