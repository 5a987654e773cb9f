// Sweep-and-prune broadphase for sm_100a (the default broadphase of
// gpu_rigidbody_pipeline2, P2/CLPhysicsDemo.cpp:17).
//
// Reference call tree (btGpuSapBroadphase::calculateOverlappingPairs,
// P2/btGpuSapBroadphase.cpp:97-485, GPU path):
//   initializeGpuAabbsFull          BB/broadphaseKernel.cl:293-331 (k_aabb_hash)
//   copyAabbsKernel                 BB/sap.cl:290-299 (small / large proxy arrays;
//                                   a proxy's max.w becomes its index in the full array)
//   flipFloatKernel                 BB/sap.cl:301-311 (FloatFlip of min.x, :272-278)
//   btRadixSort32CL                 BB/btRadixSort32CL.cpp:161-535 (stable)
//   scatterKernel                   BB/sap.cl:313-320
//   computePairsKernelTwoArrays     BB/sap.cl:65-90    large x small, all pairs
//   computePairsKernel              BB/sapFast.cl:48-150 small x later small while
//                                   min_j.x <= max_i.x
// Small proxies are the dynamic bodies, large proxies the static ones
// (P2/CLPhysicsDemo.cpp:558-568).
//
// B200 layout: the keys and the stable sort reuse the grid's key buffers
// and the onesweep sort; the sorted small proxies are copied into one
// contiguous (min, max) float4 array so each thread's sweep over later
// proxies reads consecutive 32-byte records. The reference appends pairs
// with atomics in an unspecified order; here every sorted proxy counts its
// pairs, a scan gives the offsets and a second pass writes them, so the
// pair list is deterministic: per sorted proxy i, its large-proxy pairs
// (large ids in body order) and then its later small proxies in sorted
// order.
//
// The reference's small-small test also skips a pair whose two max.w are
// both 0 (BB/sapFast.cl:39-41), meant as "both static"; after
// copyAabbsKernel max.w holds the proxy's index, so the skip can only
// apply to a proxy paired with itself, which the sweep never forms. The
// restatement keeps the test on the same values.
#include "b3_math.cuh"
#include "b3_world.h"

using namespace b3m;

namespace {

constexpr int kSapThreads = 256;

// FloatFlip (BB/sap.cl:272-278): order-preserving float -> uint32
__device__ __forceinline__ uint32_t float_flip(float f) {
    const uint32_t u = __float_as_uint(f);
    const uint32_t mask = (uint32_t)(-(int32_t)(u >> 31)) | 0x80000000u;
    return u ^ mask;
}

__device__ __forceinline__ float comp(float4 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// TestAabbAgainstAabb2 (BB/sap.cl:44-52, BB/sapFast.cl:37-48): inclusive,
// x, then z, then y
__device__ __forceinline__ bool aabb_overlap(float4 amn, float4 amx, float4 bmn, float4 bmx) {
    bool o = true;
    o = (amn.x > bmx.x || amx.x < bmn.x) ? false : o;
    o = (amn.z > bmx.z || amx.z < bmn.z) ? false : o;
    o = (amn.y > bmx.y || amx.y < bmn.y) ? false : o;
    return o;
}

// flipFloatKernel: key = FloatFlip(min.x) of small proxy s, value = body id
__global__ void k_sap_keys(const int* __restrict__ small, const int32_t* __restrict__ nDev,
                           const float4* __restrict__ aabbMin, uint32_t* __restrict__ keys,
                           uint32_t* __restrict__ vals) {
    const int n = *nDev;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int b = small[s];
        keys[s] = float_flip(aabbMin[b].x);
        vals[s] = (uint32_t)b;
    }
}

// scatterKernel + copyAabbsKernel: sorted (min, max) records; min.w is the
// body id (initializeGpuAabbsFull), max.w the proxy index (copyAabbsKernel),
// which for one proxy per body is the body id as well
__global__ void k_sap_scatter(const uint32_t* __restrict__ vals, const int32_t* __restrict__ nDev,
                              const float4* __restrict__ aabbMin, const float4* __restrict__ aabbMax,
                              float4* __restrict__ sorted) {
    const int n = *nDev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = (int)vals[i];
        float4 mx = aabbMax[b];
        mx.w = __int_as_float(b);
        sorted[2 * i] = aabbMin[b];
        sorted[2 * i + 1] = mx;
    }
}

// Pairs of sorted proxy i: the large proxies overlapping it, then the later
// small proxies up to the first whose min along axis exceeds i's max.
// COUNT writes counts[i]; otherwise the pairs go to offsets[i] onwards
// (those at or beyond cap are dropped).
template <bool COUNT>
__global__ void __launch_bounds__(kSapThreads)
k_sap_pairs(const float4* __restrict__ sorted, const int32_t* __restrict__ nDev, int axis,
            const float4* __restrict__ lgMin, const float4* __restrict__ lgMax, const int* __restrict__ large,
            int numLarge, uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
            int2* __restrict__ pairs, int cap) {
    const int n = *nDev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 mn = sorted[2 * i], mx = sorted[2 * i + 1];
        const int id = __float_as_int(mn.w);
        uint32_t c = 0;
        const uint32_t base = COUNT ? 0u : offsets[i];
        for (int l = 0; l < numLarge; ++l) {
            const int b = large[l];
            const float4 lmn = lgMin[b], lmx = lgMax[b];
            if (aabb_overlap(lmn, lmx, mn, mx)) {
                if (!COUNT && base + c < (uint32_t)cap) pairs[base + c] = make_int2(__float_as_int(lmn.w), id);
                ++c;
            }
        }
        const float test = comp(mx, axis);
        for (int j = i + 1; j < n; ++j) {
            const float4 jmn = sorted[2 * j];
            if (test < comp(jmn, axis)) break;
            const float4 jmx = sorted[2 * j + 1];
            if (__float_as_int(mx.w) == 0 && __float_as_int(jmx.w) == 0) continue;
            if (aabb_overlap(mn, mx, jmn, jmx)) {
                if (!COUNT && base + c < (uint32_t)cap) pairs[base + c] = make_int2(id, __float_as_int(jmn.w));
                ++c;
            }
        }
        if (COUNT) counts[i] = c;
    }
}

// total pairs (from the scan) -> stored count, capped, with the overflow;
// the step's pair counter as the grid broadphase reports it
__global__ void k_sap_finalize(int32_t* __restrict__ total, int cap, b3Counters* __restrict__ counters) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const uint32_t t = (uint32_t)*total;
        if (t > (uint32_t)cap) {
            atomicAdd(&counters->pairOverflow, (int)(t - (uint32_t)cap));
            *total = cap;
        }
        counters->numPairs = *total;
    }
}

int sap_grid(int numSMs, int n) { return std::max(1, std::min(numSMs * 8, (n + kSapThreads - 1) / kSapThreads)); }

}  // namespace

namespace b3 {

int launch_sap_sort(b3World_t* w, cudaStream_t st) {
    const int ns = w->numSmall;
    if (ns == 0) return B3_OK;
    auto& d = w->d;
    const int g = sap_grid(w->ctx->numSMs, ns);
    k_sap_keys<<<g, kSapThreads, 0, st>>>(d.sapSmall, d.scalars + S_NUM_SMALL, d.aabbMin, d.keys, d.vals);
    B3_CHECK_LAUNCH();
    bool alt = false;
    B3_TRY(radix_sort_pairs(d.keys, d.vals, d.keysAlt, d.valsAlt, d.scalars + S_NUM_SMALL, ns, 32, d.sortScratch,
                            d.sortScratchBytes, d.scalars + S_ERR, st, &alt, w->ctx->numSMs));
    if (alt) {
        B3_CUDA(cudaMemcpyAsync(d.keys, d.keysAlt, sizeof(uint32_t) * ns, cudaMemcpyDeviceToDevice, st));
        B3_CUDA(cudaMemcpyAsync(d.vals, d.valsAlt, sizeof(uint32_t) * ns, cudaMemcpyDeviceToDevice, st));
    }
    k_sap_scatter<<<g, kSapThreads, 0, st>>>(d.vals, d.scalars + S_NUM_SMALL, d.aabbMin, d.aabbMax, d.sapSorted);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int launch_sap_pairs(b3World_t* w, cudaStream_t st) {
    auto& d = w->d;
    B3_CUDA(cudaMemsetAsync(d.scalars + S_NUM_PAIRS, 0, sizeof(int32_t), st));
    const int ns = w->numSmall;
    if (ns == 0) return B3_OK;
    const int g = sap_grid(w->ctx->numSMs, ns);
    const int nl = (int)w->sapLargeHost.size();
    const int cap = w->cfg.maxPairs;
    k_sap_pairs<true><<<g, kSapThreads, 0, st>>>(d.sapSorted, d.scalars + S_NUM_SMALL, 0, d.aabbMin, d.aabbMax,
                                                 d.sapLarge, nl, d.sapCount, nullptr, nullptr, cap);
    B3_CHECK_LAUNCH();
    B3_TRY(exclusive_scan_u32(d.sapCount, d.sapOffset, d.scalars + S_NUM_SMALL, ns,
                              (uint32_t*)(d.scalars + S_NUM_PAIRS), d.scanScratch, d.scanScratchBytes,
                              d.scalars + S_ERR, st, w->ctx->numSMs));
    k_sap_pairs<false><<<g, kSapThreads, 0, st>>>(d.sapSorted, d.scalars + S_NUM_SMALL, 0, d.aabbMin, d.aabbMax,
                                                  d.sapLarge, nl, nullptr, d.sapOffset, d.pairs, cap);
    B3_CHECK_LAUNCH();
    k_sap_finalize<<<1, 32, 0, st>>>(d.scalars + S_NUM_PAIRS, cap, d.counters);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

}  // namespace b3

extern "C" int b3_sap_broadphase_calculate_overlapping_pairs(b3World w, void* stream) {
    if (!w) return B3_ERR_INVALID_ARG;
    if (!w->written || !w->sap) {
        b3_set_error("b3_sap_broadphase_calculate_overlapping_pairs: world not written or not created with "
                     "B3_WORLD_SAP_BROADPHASE");
        return B3_ERR_STATE;
    }
    if (w->ctx->device < 0) return B3_ERR_NO_DEVICE;
    B3_CUDA(cudaSetDevice(w->ctx->device));
    cudaStream_t st = as_stream(stream);
    B3_TRY(b3::launch_sap_sort(w, st));
    return b3::launch_sap_pairs(w, st);
}

extern "C" int b3_sap_compute_pairs(b3Context ctx, const float* d_sortedAabbs, int n, int axis, int32_t* d_pairs,
                                    int maxPairs, int32_t* d_count, void* stream) {
    if (!ctx || n < 0 || axis < 0 || axis > 2 || maxPairs < 0 || !d_count || (n > 0 && !d_sortedAabbs) ||
        (maxPairs > 0 && !d_pairs))
        return B3_ERR_INVALID_ARG;
    if (ctx->device < 0) return B3_ERR_NO_DEVICE;
    B3_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = as_stream(stream);
    if (n == 0) {
        B3_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int32_t), st));
        B3_CUDA(cudaStreamSynchronize(st));
        return B3_OK;
    }
    const size_t arr = ((size_t)(n + 1) * 4 + 255) / 256 * 256;
    const size_t sb = b3::scan_scratch_bytes(n);
    B3_TRY(ctx->ensureScratch(256 + 2 * arr + sb));
    unsigned char* base = (unsigned char*)ctx->scratch;
    int32_t* nDev = (int32_t*)base;
    int32_t* err = nDev + 1;
    uint32_t* counts = (uint32_t*)(base + 256);
    uint32_t* offsets = (uint32_t*)(base + 256 + arr);
    void* scan = base + 256 + 2 * arr;
    const int32_t hv[2] = {n, 0};
    B3_CUDA(cudaMemcpyAsync(nDev, hv, sizeof(hv), cudaMemcpyHostToDevice, st));
    const int g = sap_grid(ctx->numSMs, n);
    const float4* sorted = reinterpret_cast<const float4*>(d_sortedAabbs);
    k_sap_pairs<true><<<g, kSapThreads, 0, st>>>(sorted, nDev, axis, nullptr, nullptr, nullptr, 0, counts, nullptr,
                                                 nullptr, maxPairs);
    B3_CHECK_LAUNCH();
    B3_TRY(b3::exclusive_scan_u32(counts, offsets, nDev, n, (uint32_t*)d_count, scan, sb, err, st, ctx->numSMs));
    k_sap_pairs<false><<<g, kSapThreads, 0, st>>>(sorted, nDev, axis, nullptr, nullptr, nullptr, 0, nullptr, offsets,
                                                  reinterpret_cast<int2*>(d_pairs), maxPairs);
    B3_CHECK_LAUNCH();
    int32_t e = 0;
    B3_CUDA(cudaMemcpyAsync(&e, err, sizeof(e), cudaMemcpyDeviceToHost, st));
    B3_CUDA(cudaStreamSynchronize(st));
    if (e) {
        b3_set_error("b3_sap_compute_pairs: a bounded device wait gave up");
        return B3_ERR_TIMEOUT;
    }
    return B3_OK;
}
