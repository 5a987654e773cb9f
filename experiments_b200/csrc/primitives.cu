// GPU primitives for sm_100a: fill, single-pass exclusive scan, onesweep LSD
// radix sort (8-bit digits) and bound search.
//
// Replaces the reference's OpenCL primitive objects:
//   btFillCL         BB/btFillCL.cpp:42-110,   PR/Fill/FillKernels.cl:47-96
//   btPrefixScanCL   BB/btPrefixScanCL.cpp:46-126, PR/Scan/PrefixScanKernels.cl:38-154
//   btRadixSort32CL  BB/btRadixSort32CL.cpp:161-535, PR/Sort/RadixSort32Kernels.cl:271,337,797
//   btBoundSearchCL  BB/btBoundSearchCL.cpp:78-136, PR/Search/BoundSearchKernels.cl:42-104
//
// Design: the reference sorts 4 bits per pass (8 passes x 3 kernels each,
// fixed 120 work-groups). Here each pass is one onesweep kernel: tiles of
// 4096 keys take a tile id from an atomic counter, rank their keys stably
// with warp match (__match_any_sync) into per-warp shared histograms,
// publish per-digit tile counts and resolve their global offsets by
// decoupled look-back over preceding tiles, then stage the tile in shared
// memory in digit order so the scatter writes contiguous runs. One
// histogram kernel reads the keys once for all passes. Every look-back
// wait is bounded; a wait that gives up sets *err_flag.
#include "b3_internal.h"

#include <algorithm>

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys
constexpr int kRadix = 256;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPre = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int dev_n(const int32_t* n_dev) { return *n_dev; }

// Block-wide exclusive scan of one value per thread (blockDim = 256).
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t v, uint32_t* warp_tot,
                                                         uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = (lane < 8) ? warp_tot[lane] : 0u;
        uint32_t s = t;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < 8) warp_tot[lane] = s - t;  // exclusive warp offsets
        if (lane == 7 && total) *total = s;
    }
    __syncthreads();
    uint32_t r = warp_tot[warp] + x - v;
    __syncthreads();
    return r;
}

// ---------------------------------------------------------------------------
// Fill
// ---------------------------------------------------------------------------
__global__ void k_fill_u32(uint32_t* __restrict__ dst, uint32_t v, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}
__global__ void k_fill_int2(int2* __restrict__ dst, int2 v, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}

// ---------------------------------------------------------------------------
// Radix sort: one-read histogram for all passes
// ---------------------------------------------------------------------------
// Key i of a sort input: split arrays hold the keys contiguously; the
// interleaved form (btSortData, BB/btRadixSort32CL.h:7-11) holds (key, value)
// pairs, key first.
template <bool kPairs>
__device__ __forceinline__ uint32_t sort_key(const uint32_t* __restrict__ keys, int64_t i) {
    if (kPairs) return reinterpret_cast<const uint2*>(keys)[i].x;
    return keys[i];
}

template <bool kPairs>
__global__ void __launch_bounds__(kSortThreads)
k_radix_histogram(const uint32_t* __restrict__ keys, const int32_t* n_dev, int passes,
                  uint32_t* __restrict__ ghist /* [passes][256] */) {
    __shared__ uint32_t sh[4][kRadix];
    const int n = dev_n(n_dev);
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         i < ((int64_t)n + 31) / 32 * 32; i += stride) {
        const bool valid = i < n;
        const uint32_t k = valid ? sort_key<kPairs>(keys, i) : 0u;
        for (int p = 0; p < passes; ++p) {
            const uint32_t d = valid ? ((k >> (8 * p)) & 0xFFu) : 0x100u;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const int leader = __ffs(peers) - 1;
            if (valid && (int)(threadIdx.x & 31) == leader) atomicAdd(&sh[p][d], __popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
        uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&ghist[i], c);
    }
}

// ---------------------------------------------------------------------------
// Radix sort: one onesweep pass
// ---------------------------------------------------------------------------
struct SortSmem {
    uint32_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t warpCnt[kSortWarps][kRadix];
    uint32_t tileStart[kRadix];
    uint32_t gbase[kRadix];   // global digit base + preceding tiles
    uint32_t warpTot[8];
    int tile;
};

// kPairs: keys_in / keys_out hold interleaved (key, value) pairs and the
// value pointers are unused.
template <bool kPairs>
__global__ void __launch_bounds__(kSortThreads)
k_onesweep_pass(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                const int32_t* n_dev, int shift, const uint32_t* __restrict__ ghist_pass,
                uint32_t* __restrict__ status /* [tiles][256] */, int32_t* __restrict__ tile_counter,
                int32_t* __restrict__ err_flag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem& S = *reinterpret_cast<SortSmem*>(smem_raw);
    const int n = dev_n(n_dev);
    const int num_tiles = (n + kSortTile - 1) / kSortTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool has_vals = kPairs || vals_in != nullptr;

    for (;;) {
        if (threadIdx.x == 0) S.tile = atomicAdd(tile_counter, 1);
        __syncthreads();
        const int tile = S.tile;
        if (tile >= num_tiles) break;
        const int64_t tile_base = (int64_t)tile * kSortTile;
        const int tile_n = (int)min((int64_t)kSortTile, (int64_t)n - tile_base);

        for (int d = threadIdx.x; d < kSortWarps * kRadix; d += kSortThreads)
            (&S.warpCnt[0][0])[d] = 0;
        __syncthreads();

        // Load (striped within each warp: lane l, item i -> w*32*I + i*32 + l)
        uint32_t k[kSortItems], v[kSortItems];
        uint32_t rank[kSortItems];
#pragma unroll
        for (int i = 0; i < kSortItems; ++i) {
            const int idx = warp * 32 * kSortItems + i * 32 + lane;
            if (idx < tile_n) {
                if (kPairs) {
                    const uint2 kv = reinterpret_cast<const uint2*>(keys_in)[tile_base + idx];
                    k[i] = kv.x;
                    v[i] = kv.y;
                } else {
                    k[i] = keys_in[tile_base + idx];
                    v[i] = has_vals ? vals_in[tile_base + idx] : 0u;
                }
            } else {
                k[i] = 0xFFFFFFFFu;
                v[i] = 0u;
            }
        }
        // Stable warp ranking with match-any peer groups.
        const uint32_t lt = b3dev::lanemask_lt();
#pragma unroll
        for (int i = 0; i < kSortItems; ++i) {
            const int idx = warp * 32 * kSortItems + i * 32 + lane;
            const bool valid = idx < tile_n;
            const uint32_t d = valid ? ((k[i] >> shift) & 0xFFu) : 0x100u;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            uint32_t base = valid ? S.warpCnt[warp][d] : 0u;
            rank[i] = base + __popc(peers & lt);
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) S.warpCnt[warp][d] = base + __popc(peers);
            __syncwarp();
        }
        __syncthreads();

        // Per-digit totals, warp prefixes, tile-local digit starts.
        const int d = threadIdx.x;  // one digit per thread (256 threads)
        uint32_t cnt = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t t = S.warpCnt[w][d];
            S.warpCnt[w][d] = cnt;
            cnt += t;
        }
        // Publish this tile's aggregate for digit d, then look back.
        uint32_t* my = status + (int64_t)tile * kRadix + d;
        uint32_t excl = 0;
        if (tile == 0) {
            b3dev::st_release_u32(my, kFlagPre | cnt);
        } else {
            b3dev::st_release_u32(my, kFlagAgg | cnt);
            int t = tile - 1;
            while (t >= 0) {
                const uint32_t* p = status + (int64_t)t * kRadix + d;
                uint32_t s = 0;
                int spins = 0;
                while (((s = b3dev::ld_acquire_u32(p)) & (kFlagAgg | kFlagPre)) == 0) {
                    if (++spins > b3dev::kSpinLimit) {
                        atomicExch(err_flag, 1);
                        break;
                    }
                    __nanosleep(32);
                }
                excl += s & kValMask;
                if (s & kFlagPre) break;
                if ((s & (kFlagAgg | kFlagPre)) == 0) break;  // gave up
                --t;
            }
            b3dev::st_release_u32(my, kFlagPre | (excl + cnt));
        }
        const uint32_t gdig = ghist_pass[d];
        const uint32_t gexcl = block_excl_scan_256(gdig, S.warpTot, nullptr);
        const uint32_t tstart = block_excl_scan_256(cnt, S.warpTot, nullptr);
        S.tileStart[d] = tstart;
        S.gbase[d] = gexcl + excl;
        __syncthreads();

        // Stage the tile in digit order.
#pragma unroll
        for (int i = 0; i < kSortItems; ++i) {
            const int idx = warp * 32 * kSortItems + i * 32 + lane;
            if (idx < tile_n) {
                const uint32_t dd = (k[i] >> shift) & 0xFFu;
                const uint32_t pos = S.tileStart[dd] + S.warpCnt[warp][dd] + rank[i];
                S.keys[pos] = k[i];
                S.vals[pos] = v[i];
            }
        }
        __syncthreads();
        // Scatter contiguous digit runs.
        for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
            const uint32_t kk = S.keys[j];
            const uint32_t dd = (kk >> shift) & 0xFFu;
            const uint32_t dst = S.gbase[dd] + (j - S.tileStart[dd]);
            if (kPairs) {
                reinterpret_cast<uint2*>(keys_out)[dst] = make_uint2(kk, S.vals[j]);
            } else {
                keys_out[dst] = kk;
                if (has_vals) vals_out[dst] = S.vals[j];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Exclusive scan with decoupled look-back
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kScanThreads)
k_scan_u32(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const int32_t* n_dev,
           unsigned long long* __restrict__ status, int32_t* __restrict__ tile_counter,
           uint32_t* __restrict__ d_total, int32_t* __restrict__ err_flag) {
    __shared__ uint32_t sm[kScanTile + kScanTile / 32];
    __shared__ uint32_t warp_tot[8];
    __shared__ uint32_t tile_excl;
    __shared__ int tile_sh;
    const int n = dev_n(n_dev);
    const int num_tiles = (n + kScanTile - 1) / kScanTile;
    const unsigned long long FA = 1ull << 32, FP = 2ull << 32;
    for (;;) {
        if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1);
        __syncthreads();
        const int tile = tile_sh;
        if (tile >= num_tiles) break;
        const int64_t base = (int64_t)tile * kScanTile;
        const int tn = (int)min((int64_t)kScanTile, (int64_t)n - base);
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const int j = i * kScanThreads + threadIdx.x;
            sm[j + j / 32] = (j < tn) ? src[base + j] : 0u;
        }
        __syncthreads();
        uint32_t loc[kScanItems];
        uint32_t run = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const int j = threadIdx.x * kScanItems + i;
            loc[i] = run;
            run += sm[j + j / 32];
        }
        const uint32_t texcl = block_excl_scan_256(run, warp_tot, nullptr);
        if (threadIdx.x == kScanThreads - 1) warp_tot[0] = texcl + run;  // tile aggregate
        __syncthreads();
        const uint32_t agg = warp_tot[0];
        if (threadIdx.x == 0) {
            unsigned long long* my = status + tile;
            uint32_t excl = 0;
            if (tile == 0) {
                b3dev::st_release_u64(my, FP | agg);
            } else {
                b3dev::st_release_u64(my, FA | agg);
                int t = tile - 1;
                while (t >= 0) {
                    unsigned long long s = 0;
                    int spins = 0;
                    while (((s = b3dev::ld_acquire_u64(status + t)) >> 32) == 0) {
                        if (++spins > b3dev::kSpinLimit) {
                            atomicExch(err_flag, 1);
                            break;
                        }
                        __nanosleep(32);
                    }
                    excl += (uint32_t)s;
                    if ((s >> 32) == 2) break;
                    if ((s >> 32) == 0) break;
                    --t;
                }
                b3dev::st_release_u64(my, FP | (unsigned long long)(uint32_t)(excl + agg));
            }
            tile_excl = excl;
            if (tile == num_tiles - 1 && d_total) *d_total = excl + agg;
        }
        __syncthreads();
        const uint32_t off = tile_excl + texcl;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const int j = threadIdx.x * kScanItems + i;
            sm[j + j / 32] = off + loc[i];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const int j = i * kScanThreads + threadIdx.x;
            if (j < tn) dst[base + j] = sm[j + j / 32];
        }
        __syncthreads();
    }
    (void)n;
}

__global__ void k_scan_empty_total(const int32_t* n_dev, uint32_t* d_total) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && *n_dev <= 0 && d_total) *d_total = 0;
}

// ---------------------------------------------------------------------------
// Bound search over sorted keys
// ---------------------------------------------------------------------------
// kPairs: the sorted input is interleaved (key, value) pairs (btSortData).
template <bool kPairs>
__global__ void k_bound_lower(const uint32_t* __restrict__ keys, const int32_t* n_dev,
                              uint32_t* __restrict__ dst, int64_t n_dst) {
    const int n = dev_n(n_dev);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = sort_key<kPairs>(keys, i);
        if ((i == 0 || sort_key<kPairs>(keys, i - 1) != k) && k < (uint64_t)n_dst) dst[k] = (uint32_t)i;
    }
}
// kPairs also follows SearchSortDataUpperKernel (PR/Search/BoundSearchKernels.cl:66-86)
// where no key 0 is present: its first work item compares the first key
// with 0 and writes dst[0] = 0.
template <bool kPairs>
__global__ void k_bound_upper(const uint32_t* __restrict__ keys, const int32_t* n_dev,
                              uint32_t* __restrict__ dst, int64_t n_dst) {
    const int n = dev_n(n_dev);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = sort_key<kPairs>(keys, i);
        if ((i == n - 1 || sort_key<kPairs>(keys, i + 1) != k) && k < (uint64_t)n_dst) dst[k] = (uint32_t)(i + 1);
        if (kPairs && i == 0 && k != 0u && n_dst > 0) dst[0] = 0u;
    }
}
template <bool kPairs>
__global__ void k_bound_count(const uint32_t* __restrict__ keys, const int32_t* n_dev,
                              uint32_t* __restrict__ dst, int64_t n_dst) {
    const int n = dev_n(n_dev);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = sort_key<kPairs>(keys, i);
        if ((i == 0 || sort_key<kPairs>(keys, i - 1) != k) && k < (uint64_t)n_dst) {
            int64_t j = i;
            // run length by binary search for the first index with a larger key
            int64_t lo = i + 1, hi = n;
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (sort_key<kPairs>(keys, mid) == k) lo = mid + 1; else hi = mid;
            }
            dst[k] = (uint32_t)(lo - j);
        }
    }
}

int grid_for(int64_t n, int threads, int numSMs, int perSM = 8) {
    int64_t g = (n + threads - 1) / threads;
    g = std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)numSMs * perSM));
    return (int)g;
}

}  // namespace

namespace b3 {

static inline int sort_passes(int key_bits) { return (key_bits + 7) / 8; }

size_t radix_scratch_bytes(int64_t n_max, int key_bits) {
    const int P = sort_passes(key_bits);
    const int64_t tiles = (n_max + kSortTile - 1) / kSortTile;
    // [counters 64 B][ghist P*256*4][status P*tiles*256*4]
    return 256 + (size_t)P * kRadix * 4 + (size_t)P * (size_t)std::max<int64_t>(tiles, 1) * kRadix * 4;
}

// Passes of one sort: pass 0 reads (kin, vin) and writes buffer A, pass 1
// reads A and writes B, and so on; the result is in A when the pass count
// is odd, else in B. The input may be A or B itself (in-place sorts).
template <bool kPairs>
static int radix_sort_core(const uint32_t* kin, const uint32_t* vin, uint32_t* kA, uint32_t* vA, uint32_t* kB,
                           uint32_t* vB, const int32_t* n_dev, int64_t n_max, int key_bits, void* scratch,
                           size_t scratch_bytes, int32_t* err_flag, cudaStream_t st, int numSMs) {
    if (key_bits < 1 || key_bits > 32) return B3_ERR_INVALID_ARG;
    const int P = sort_passes(key_bits);
    const size_t need = radix_scratch_bytes(n_max, key_bits);
    if (scratch_bytes < need) return B3_ERR_CAPACITY;
    const int64_t tiles = std::max<int64_t>(1, (n_max + kSortTile - 1) / kSortTile);
    unsigned char* s = (unsigned char*)scratch;
    int32_t* counters = (int32_t*)s;                    // P tile counters
    uint32_t* ghist = (uint32_t*)(s + 256);             // P x 256
    uint32_t* status = ghist + (size_t)P * kRadix;      // P x tiles x 256
    B3_CUDA(cudaMemsetAsync(scratch, 0, need, st));
    if (n_max <= 0) return B3_OK;
    const int hgrid = grid_for(n_max, kSortThreads, numSMs, 4);
    k_radix_histogram<kPairs><<<hgrid, kSortThreads, 0, st>>>(kin, n_dev, P, ghist);
    B3_CHECK_LAUNCH();
    const size_t smem = sizeof(SortSmem);
    static bool attr_set = false;
    if (!attr_set) {
        B3_CUDA(cudaFuncSetAttribute(k_onesweep_pass<kPairs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        attr_set = true;
    }
    // Persistent grid: resident blocks only, so every tile whose result a
    // later tile waits for is held by a running block.
    int occ = 1;
    B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_onesweep_pass<kPairs>, kSortThreads, smem));
    occ = std::max(1, occ);
    const int pgrid = (int)std::min<int64_t>(tiles, (int64_t)numSMs * occ);
    const uint32_t* ki = kin;
    const uint32_t* vi = vin;
    for (int p = 0; p < P; ++p) {
        uint32_t* ko = (p & 1) ? kB : kA;
        uint32_t* vo = (p & 1) ? vB : vA;
        k_onesweep_pass<kPairs><<<pgrid, kSortThreads, smem, st>>>(
            ki, vi, ko, vo, n_dev, 8 * p, ghist + (size_t)p * kRadix, status + (size_t)p * tiles * kRadix,
            counters + p, err_flag);
        B3_CHECK_LAUNCH();
        ki = ko;
        vi = vo;
    }
    return B3_OK;
}

int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                     const int32_t* n_dev, int64_t n_max, int key_bits, void* scratch,
                     size_t scratch_bytes, int32_t* err_flag, cudaStream_t st, bool* result_in_alt,
                     int numSMs) {
    *result_in_alt = n_max > 0 && (sort_passes(key_bits) & 1) != 0;
    return radix_sort_core<false>(keys, vals, keys_alt, vals ? vals_alt : nullptr, keys, vals, n_dev, n_max,
                                  key_bits, scratch, scratch_bytes, err_flag, st, numSMs);
}

int radix_sort_kv_out(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                      uint32_t* keys_tmp, uint32_t* vals_tmp, const int32_t* n_dev, int64_t n_max, int key_bits,
                      void* scratch, size_t scratch_bytes, int32_t* err_flag, cudaStream_t st, int numSMs) {
    // the first pass writes the buffer that makes the last pass land in out
    const bool odd = (sort_passes(key_bits) & 1) != 0;
    uint32_t* kA = odd ? keys_out : keys_tmp;
    uint32_t* vA = odd ? vals_out : vals_tmp;
    uint32_t* kB = odd ? keys_tmp : keys_out;
    uint32_t* vB = odd ? vals_tmp : vals_out;
    return radix_sort_core<false>(keys_in, vals_in, kA, vals_in ? vA : nullptr, kB, vals_in ? vB : nullptr,
                                  n_dev, n_max, key_bits, scratch, scratch_bytes, err_flag, st, numSMs);
}

int radix_sort_interleaved(uint2* kv, uint2* kv_alt, const int32_t* n_dev, int64_t n_max, int key_bits,
                           void* scratch, size_t scratch_bytes, int32_t* err_flag, cudaStream_t st,
                           bool* result_in_alt, int numSMs) {
    *result_in_alt = n_max > 0 && (sort_passes(key_bits) & 1) != 0;
    uint32_t* a = reinterpret_cast<uint32_t*>(kv_alt);
    uint32_t* b = reinterpret_cast<uint32_t*>(kv);
    return radix_sort_core<true>(b, nullptr, a, nullptr, b, nullptr, n_dev, n_max, key_bits, scratch, scratch_bytes,
                                 err_flag, st, numSMs);
}

size_t scan_scratch_bytes(int64_t n_max) {
    const int64_t tiles = std::max<int64_t>(1, (n_max + kScanTile - 1) / kScanTile);
    return 256 + (size_t)tiles * 8;
}

int exclusive_scan_u32(const uint32_t* src, uint32_t* dst, const int32_t* n_dev, int64_t n_max,
                       uint32_t* d_total, void* scratch, size_t scratch_bytes, int32_t* err_flag,
                       cudaStream_t st, int numSMs) {
    const size_t need = scan_scratch_bytes(n_max);
    if (scratch_bytes < need) return B3_ERR_CAPACITY;
    B3_CUDA(cudaMemsetAsync(scratch, 0, need, st));
    int32_t* counter = (int32_t*)scratch;
    unsigned long long* status = (unsigned long long*)((unsigned char*)scratch + 256);
    if (d_total) {
        k_scan_empty_total<<<1, 32, 0, st>>>(n_dev, d_total);
        B3_CHECK_LAUNCH();
    }
    if (n_max <= 0) return B3_OK;
    const int64_t tiles = std::max<int64_t>(1, (n_max + kScanTile - 1) / kScanTile);
    int occ = 1;
    B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_scan_u32, kScanThreads, 0));
    occ = std::max(1, occ);
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)numSMs * occ);
    k_scan_u32<<<grid, kScanThreads, 0, st>>>(src, dst, n_dev, status, counter, d_total, err_flag);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int fill_u32(uint32_t* dst, uint32_t v, int64_t n, cudaStream_t st) {
    if (n <= 0) return B3_OK;
    k_fill_u32<<<grid_for(n, 256, 148, 16), 256, 0, st>>>(dst, v, n);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

template <bool kPairs>
static int bound_search_t(const uint32_t* keys, const int32_t* n_dev, int64_t n_max, uint32_t* dst,
                          int64_t n_dst, int mode, cudaStream_t st) {
    if (n_max <= 0) return B3_OK;
    const int g = grid_for(n_max, 256, 148, 16);
    if (mode == 0) k_bound_lower<kPairs><<<g, 256, 0, st>>>(keys, n_dev, dst, n_dst);
    else if (mode == 1) k_bound_upper<kPairs><<<g, 256, 0, st>>>(keys, n_dev, dst, n_dst);
    else k_bound_count<kPairs><<<g, 256, 0, st>>>(keys, n_dev, dst, n_dst);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int bound_search(const uint32_t* keys, const int32_t* n_dev, int64_t n_max, uint32_t* dst,
                 int64_t n_dst, int mode, cudaStream_t st) {
    return bound_search_t<false>(keys, n_dev, n_max, dst, n_dst, mode, st);
}

int bound_search_interleaved(const uint2* kv, const int32_t* n_dev, int64_t n_max, uint32_t* dst, int64_t n_dst,
                             int mode, cudaStream_t st) {
    return bound_search_t<true>(reinterpret_cast<const uint32_t*>(kv), n_dev, n_max, dst, n_dst, mode, st);
}

int fill_int2(int2* dst, int2 v, int64_t n, cudaStream_t st) {
    if (n <= 0) return B3_OK;
    k_fill_int2<<<grid_for(n, 256, 148, 16), 256, 0, st>>>(dst, v, n);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

}  // namespace b3
