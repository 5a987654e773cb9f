// C ABI: context, errors and the primitive objects (fill, prefix scan,
// radix sort, bound search), each replacing the OpenCL object named in
// include/b3gpu.h.
#include "b3_internal.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>

static thread_local char g_err[1024] = "";

void b3_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char* b3_last_error(void) { return g_err; }

int b3Context_t::ensureScratch(size_t bytes) {
    if (bytes <= scratchBytes) return B3_OK;
    if (scratch) cudaFree(scratch);
    scratch = nullptr;
    scratchBytes = 0;
    B3_CUDA(cudaMalloc(&scratch, bytes));
    scratchBytes = bytes;
    return B3_OK;
}

extern "C" int b3_context_create(int device, b3Context* out) {
    if (!out) return B3_ERR_INVALID_ARG;
    *out = nullptr;
    if (device == -1) {
        b3Context c = new b3Context_t();
        c->device = -1;
        c->numSMs = 0;
        *out = c;
        return B3_OK;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        b3_set_error("no CUDA device");
        return B3_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return B3_ERR_INVALID_ARG;
    B3_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    B3_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        b3_set_error("device %s is sm_%d%d; this library is built for sm_100a", prop.name, prop.major,
                     prop.minor);
        return B3_ERR_NO_DEVICE;
    }
    b3Context c = new b3Context_t();
    c->device = device;
    c->numSMs = prop.multiProcessorCount;
    c->maxSmemOptin = (int)prop.sharedMemPerBlockOptin;
    *out = c;
    return B3_OK;
}

extern "C" int b3_context_destroy(b3Context ctx) {
    if (!ctx) return B3_OK;
    if (ctx->device < 0) {
        delete ctx;
        return B3_OK;
    }
    cudaSetDevice(ctx->device);
    if (ctx->scratch) cudaFree(ctx->scratch);
    delete ctx;
    return B3_OK;
}

extern "C" int b3_sync(b3Context ctx, void* stream) {
    if (!ctx) return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    B3_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return B3_OK;
}

extern "C" int b3_context_info(b3Context ctx, char* buf, int buflen) {
    if (!ctx || !buf || buflen <= 0) return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) {
        snprintf(buf, buflen, "b3gpu host-only context");
        return B3_OK;
    }
    cudaDeviceProp prop;
    B3_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    int drv = 0, rt = 0;
    cudaDriverGetVersion(&drv);
    cudaRuntimeGetVersion(&rt);
    snprintf(buf, buflen, "b3gpu sm_%d%d %s SMs=%d driver=%d runtime=%d", prop.major, prop.minor,
             prop.name, prop.multiProcessorCount, drv, rt);
    return B3_OK;
}

extern "C" int b3_fill_u32(b3Context ctx, uint32_t* d_dst, uint32_t value, int64_t n, int64_t offset,
                           void* stream) {
    if (!ctx || (n > 0 && !d_dst) || n < 0 || offset < 0) return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    return b3::fill_u32(d_dst + offset, value, n, as_stream(stream));
}

namespace b3 {
int fill_int2(int2* dst, int2 v, int64_t n, cudaStream_t st);
}

extern "C" int b3_fill_int2(b3Context ctx, int32_t* d_dst_int2, int32_t x, int32_t y, int64_t n,
                            int64_t offset, void* stream) {
    if (!ctx || (n > 0 && !d_dst_int2) || n < 0 || offset < 0) return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    return b3::fill_int2(reinterpret_cast<int2*>(d_dst_int2) + offset, make_int2(x, y), n,
                         as_stream(stream));
}

// scratch layout for primitive calls: [n (int32) at 0][pad to 256][payload]
static int prim_scratch(b3Context ctx, size_t payload, int64_t n, cudaStream_t st, int32_t** n_dev,
                        int32_t** err, void** body) {
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    B3_TRY(ctx->ensureScratch(256 + payload));
    *n_dev = (int32_t*)ctx->scratch;
    *err = *n_dev + 1;
    *body = (unsigned char*)ctx->scratch + 256;
    const int32_t hv[2] = {(int32_t)n, 0};
    B3_CUDA(cudaMemcpyAsync(ctx->scratch, hv, sizeof(hv), cudaMemcpyHostToDevice, st));
    return B3_OK;
}

static int check_err_flag(int32_t* err, cudaStream_t st) {
    int32_t e = 0;
    B3_CUDA(cudaMemcpyAsync(&e, err, sizeof(e), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    if (e) {
        b3_set_error("a bounded device wait gave up");
        return B3_ERR_TIMEOUT;
    }
    return B3_OK;
}

extern "C" int b3_prefix_scan_u32(b3Context ctx, const uint32_t* d_src, uint32_t* d_dst, int64_t n,
                                  uint32_t* d_sum, uint32_t* h_sum, void* stream) {
    if (!ctx || n < 0 || n > (int64_t)0x7fffffff || (n > 0 && (!d_src || !d_dst))) return B3_ERR_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    int32_t *n_dev, *err;
    void* body;
    const size_t sb = b3::scan_scratch_bytes(n);
    B3_TRY(prim_scratch(ctx, sb + 64, n, st, &n_dev, &err, &body));
    uint32_t* tot = (uint32_t*)((unsigned char*)body + sb);
    // in-place scans are safe: each tile reads its input before it writes
    B3_TRY(b3::exclusive_scan_u32(d_src, d_dst, n_dev, n, tot, body, sb, err, st, ctx->numSMs));
    if (d_sum) B3_CUDA(cudaMemcpyAsync(d_sum, tot, 4, cudaMemcpyDeviceToDevice, st));
    if (h_sum) {
        B3_CUDA(cudaMemcpyAsync(h_sum, tot, 4, cudaMemcpyDeviceToHost, st));
        return check_err_flag(err, st);
    }
    return B3_OK;
}

static int sort_impl(b3Context ctx, uint32_t* d_keys, uint32_t* d_values, int64_t n, int key_bits,
                     void* stream) {
    if (!ctx || n < 0 || n > (int64_t)0x3fffffff || key_bits < 1 || key_bits > 32 || (n > 0 && !d_keys))
        return B3_ERR_INVALID_ARG;
    if (n <= 1) return B3_OK;
    cudaStream_t st = as_stream(stream);
    const size_t rb = b3::radix_scratch_bytes(n, key_bits);
    const size_t alt = ((size_t)n * 4 + 255) / 256 * 256;
    int32_t *n_dev, *err;
    void* body;
    B3_TRY(prim_scratch(ctx, rb + 2 * alt, n, st, &n_dev, &err, &body));
    uint32_t* kalt = (uint32_t*)((unsigned char*)body + rb);
    uint32_t* valt = d_values ? (uint32_t*)((unsigned char*)body + rb + alt) : nullptr;
    bool in_alt = false;
    B3_TRY(b3::radix_sort_pairs(d_keys, d_values, kalt, valt, n_dev, n, key_bits, body, rb, err, st,
                                &in_alt, ctx->numSMs));
    if (in_alt) {
        B3_CUDA(cudaMemcpyAsync(d_keys, kalt, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st));
        if (d_values) B3_CUDA(cudaMemcpyAsync(d_values, valt, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st));
    }
    return B3_OK;
}

extern "C" int b3_radix_sort32_kv(b3Context ctx, uint32_t* d_keys, uint32_t* d_values, int64_t n,
                                  int key_bits, void* stream) {
    if (n > 0 && !d_values) return B3_ERR_INVALID_ARG;
    return sort_impl(ctx, d_keys, d_values, n, key_bits, stream);
}

extern "C" int b3_radix_sort32_keys(b3Context ctx, uint32_t* d_keys, int64_t n, int key_bits, void* stream) {
    return sort_impl(ctx, d_keys, nullptr, n, key_bits, stream);
}

extern "C" int b3_radix_sort32_kv_out(b3Context ctx, const uint32_t* d_keys_in, uint32_t* d_keys_out,
                                      const uint32_t* d_values_in, uint32_t* d_values_out, int64_t n, int key_bits,
                                      void* stream) {
    if (!ctx || n < 0 || n > (int64_t)0x3fffffff || key_bits < 1 || key_bits > 32 ||
        (n > 0 && (!d_keys_in || !d_keys_out)) || (n > 0 && (d_values_in == nullptr) != (d_values_out == nullptr)))
        return B3_ERR_INVALID_ARG;
    if (d_keys_in == d_keys_out || (d_values_in && d_values_in == d_values_out)) {
        b3_set_error("b3_radix_sort32_kv_out: the outputs must not be the inputs (use b3_radix_sort32_kv)");
        return B3_ERR_INVALID_ARG;
    }
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    if (n == 0) return B3_OK;
    cudaStream_t st = as_stream(stream);
    if (n == 1) {
        B3_CUDA(cudaMemcpyAsync(d_keys_out, d_keys_in, 4, cudaMemcpyDeviceToDevice, st));
        if (d_values_in) B3_CUDA(cudaMemcpyAsync(d_values_out, d_values_in, 4, cudaMemcpyDeviceToDevice, st));
        return B3_OK;
    }
    const size_t rb = b3::radix_scratch_bytes(n, key_bits);
    const size_t alt = ((size_t)n * 4 + 255) / 256 * 256;
    int32_t *n_dev, *err;
    void* body;
    B3_TRY(prim_scratch(ctx, rb + 2 * alt, n, st, &n_dev, &err, &body));
    uint32_t* ktmp = (uint32_t*)((unsigned char*)body + rb);
    uint32_t* vtmp = d_values_in ? (uint32_t*)((unsigned char*)body + rb + alt) : nullptr;
    return b3::radix_sort_kv_out(d_keys_in, d_values_in, d_keys_out, d_values_out, ktmp, vtmp, n_dev, n, key_bits,
                                 body, rb, err, st, ctx->numSMs);
}

extern "C" int b3_radix_sort32_sortdata(b3Context ctx, int32_t* d_key_values, int64_t n, int key_bits,
                                        void* stream) {
    if (!ctx || n < 0 || n > (int64_t)0x3fffffff || key_bits < 1 || key_bits > 32 || (n > 0 && !d_key_values))
        return B3_ERR_INVALID_ARG;
    if (((uintptr_t)d_key_values & 7) != 0) {
        b3_set_error("b3_radix_sort32_sortdata: the (key, value) array must be 8-byte aligned");
        return B3_ERR_INVALID_ARG;
    }
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    if (n <= 1) return B3_OK;
    cudaStream_t st = as_stream(stream);
    const size_t rb = b3::radix_scratch_bytes(n, key_bits);
    int32_t *n_dev, *err;
    void* body;
    B3_TRY(prim_scratch(ctx, rb + 8 * (size_t)n, n, st, &n_dev, &err, &body));
    uint2* kv = reinterpret_cast<uint2*>(d_key_values);
    uint2* alt = (uint2*)((unsigned char*)body + rb);  // rb is a multiple of 256
    bool in_alt = false;
    B3_TRY(b3::radix_sort_interleaved(kv, alt, n_dev, n, key_bits, body, rb, err, st, &in_alt, ctx->numSMs));
    if (in_alt) B3_CUDA(cudaMemcpyAsync(kv, alt, 8 * (size_t)n, cudaMemcpyDeviceToDevice, st));
    return B3_OK;
}

extern "C" int b3_bound_search(b3Context ctx, const uint32_t* d_sorted_keys, int64_t n_src,
                               uint32_t* d_dst, int64_t n_dst, int mode, void* stream) {
    if (!ctx || n_src < 0 || n_dst < 0 || mode < 0 || mode > 2 || (n_src > 0 && !d_sorted_keys) ||
        (n_dst > 0 && !d_dst) || n_src > (int64_t)0x7fffffff)
        return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    cudaStream_t st = as_stream(stream);
    if (mode == 2) B3_TRY(b3::fill_u32(d_dst, 0u, n_dst, st));
    if (n_src == 0) return B3_OK;
    int32_t *n_dev, *err;
    void* body;
    B3_TRY(prim_scratch(ctx, 0, n_src, st, &n_dev, &err, &body));
    return b3::bound_search(d_sorted_keys, n_dev, n_src, d_dst, n_dst, mode, st);
}

extern "C" int b3_bound_search_sortdata(b3Context ctx, const int32_t* d_sorted_key_values, int64_t n_src,
                                        uint32_t* d_dst, int64_t n_dst, int mode, void* stream) {
    if (!ctx || n_src < 0 || n_dst < 0 || mode < 0 || mode > 2 || (n_src > 0 && !d_sorted_key_values) ||
        (n_dst > 0 && !d_dst) || n_src > (int64_t)0x7fffffff || ((uintptr_t)d_sorted_key_values & 7) != 0)
        return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    cudaStream_t st = as_stream(stream);
    if (mode == 2) B3_TRY(b3::fill_u32(d_dst, 0u, n_dst, st));
    if (n_src == 0) return B3_OK;
    int32_t *n_dev, *err;
    void* body;
    B3_TRY(prim_scratch(ctx, 0, n_src, st, &n_dev, &err, &body));
    return b3::bound_search_interleaved(reinterpret_cast<const uint2*>(d_sorted_key_values), n_dev, n_src, d_dst,
                                        n_dst, mode, st);
}
