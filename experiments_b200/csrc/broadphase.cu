// Uniform-grid broadphase for sm_100a.
//
// Reference call tree (btGridBroadphaseCl::calculateOverlappingPairs,
// BB/btGridBroadphaseCL.cpp:135-238):
//   initializeGpuAabbsFull   BB/broadphaseKernel.cl:293-331
//   kCalcHashAABB            G3/bt3dGridBroadphaseOCL.cl:4-48
//   RadixSort32              BB/btRadixSort32CL.cpp:161-535
//   kClearCellStart/kFindCellStart  G3/bt3dGridBroadphaseOCL.cl:50-87
//   kFindOverlappingPairs + findPairsInCell  G3/bt3dGridBroadphaseOCL.cl:89-215
//   countOverlappingpairs / scan / squeezePairCaches  BB/computeAabbKernelOCL.cl:40-111
//
// B200 layout:
//   * k_aabb_hash fuses the world AABB, the cell hash and setupBodies'
//     gravity update (BB/broadphaseKernel.cl:163-213) into one pass over the
//     float4 body streams; the AABB arithmetic uses non-contracting
//     intrinsics so keys are bit-reproducible.
//   * Cell starts live in a (stamp, index) table indexed by the full key,
//     so no per-step clear of the 128^3 cell array is needed (the reference
//     clears 2M cells per step).
//   * k_find_pairs searches the 27 neighbour cells exactly like
//     findPairsInCell (bucket cap, id(other) < id(self), inclusive AABB test),
//     adds a pass over the world's large bodies (kFindPairsLarge precedent,
//     G3/bt3dGridBroadphaseOCL.cl:218-275), and compacts the pairs in the
//     same kernel: each 128-body tile scans its counts in shared memory and
//     resolves its output offset by decoupled look-back. No persistent pair
//     cache: every step emits all overlapping candidate pairs, which is the
//     reference's output whenever its per-body cap is not reached.
#include "b3_math.cuh"
#include "b3_world.h"

using namespace b3m;

namespace {

constexpr int kAabbThreads = 256;
constexpr int kPairTile = 128;        // bodies per tile, one thread per body
constexpr int kWarpPairTile = 32;     // bodies per tile of the warp-per-body search
constexpr int kWarpPairThreads = 128; // its CTA: four warps of eight bodies each

struct GridParams {
    float invCell;
    int dimX, dimY, dimZ;
    int cellBits;
    int maxBodiesPerCell;
    int maxPairsPerBody;
    int maxPairs;
    int numSmall;
};

__device__ __forceinline__ int grid_coord(float c, float inv, int dim) {
    return ((int)floorf(mrn(c, inv))) & (dim - 1);
}

__global__ void __launch_bounds__(kAabbThreads)
k_aabb_hash(b3::BodiesDev B, const float4* __restrict__ localAabb, GridParams g, float3 gdt,
            const int* __restrict__ smallSlot, float4* __restrict__ aabbMin,
            float4* __restrict__ aabbMax, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
            int applyGravity) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n) return;
    const float4 p = B.pos[i];
    const float4 q = B.quat[i];
    const int col = B.collidable[i];
    const float invMass = B.invMass[i];
    const float4 lmn = localAabb[2 * col], lmx = localAabb[2 * col + 1];
    // initializeGpuAabbsFull (BB/broadphaseKernel.cl:309-330)
    const float4 he = make_float4(mrn(srn(lmx.x, lmn.x), 0.5f), mrn(srn(lmx.y, lmn.y), 0.5f),
                                  mrn(srn(lmx.z, lmn.z), 0.5f), 0.f);
    const float4 lc = make_float4(mrn(arn(lmx.x, lmn.x), 0.5f), mrn(arn(lmx.y, lmn.y), 0.5f),
                                  mrn(arn(lmx.z, lmn.z), 0.5f), 0.f);
    float4 wc = qt_rotate_rn(q, lc);
    wc.x = arn(wc.x, p.x);
    wc.y = arn(wc.y, p.y);
    wc.z = arn(wc.z, p.z);
    // |R| from qtGetRotationMatrix (BB/broadphaseKernel.cl:91-113)
    const float x2 = mrn(q.x, q.x), y2 = mrn(q.y, q.y), z2 = mrn(q.z, q.z);
    const float tx = mrn(2.f, q.x), ty = mrn(2.f, q.y), tw = mrn(2.f, q.w);
    const float4 r0 = make_float4(fabsf(srn(srn(1.f, mrn(2.f, y2)), mrn(2.f, z2))),
                                  fabsf(srn(mrn(tx, q.y), mrn(tw, q.z))),
                                  fabsf(arn(mrn(tx, q.z), mrn(tw, q.y))), 0.f);
    const float4 r1 = make_float4(fabsf(arn(mrn(tx, q.y), mrn(tw, q.z))),
                                  fabsf(srn(srn(1.f, mrn(2.f, x2)), mrn(2.f, z2))),
                                  fabsf(srn(mrn(ty, q.z), mrn(tw, q.x))), 0.f);
    const float4 r2 = make_float4(fabsf(srn(mrn(tx, q.z), mrn(tw, q.y))),
                                  fabsf(arn(mrn(ty, q.z), mrn(tw, q.x))),
                                  fabsf(srn(srn(1.f, mrn(2.f, x2)), mrn(2.f, y2))), 0.f);
    const float ex = dot3_rn(r0, he), ey = dot3_rn(r1, he), ez = dot3_rn(r2, he);
    const float4 mn = make_float4(srn(wc.x, ex), srn(wc.y, ey), srn(wc.z, ez), __int_as_float(i));
    const float4 mx = make_float4(arn(wc.x, ex), arn(wc.y, ey), arn(wc.z, ez),
                                  __int_as_float(invMass == 0.f ? 0 : 1));
    aabbMin[i] = mn;
    aabbMax[i] = mx;
    // setupBodiesKernel gravity (BB/broadphaseKernel.cl:175-183)
    if (applyGravity && invMass != 0.f) {
        float4 v = B.linVel[i];
        v.x += gdt.x;
        v.y += gdt.y;
        v.z += gdt.z;
        B.linVel[i] = v;
    }
    // kCalcHashAABB (G3/bt3dGridBroadphaseOCL.cl:26-48)
    const int slot = smallSlot[i];
    if (slot >= 0) {
        const float cx = mrn(arn(mn.x, mx.x), 0.5f);
        const float cy = mrn(arn(mn.y, mx.y), 0.5f);
        const float cz = mrn(arn(mn.z, mx.z), 0.5f);
        const int gx = grid_coord(cx, g.invCell, g.dimX);
        const int gy = grid_coord(cy, g.invCell, g.dimY);
        const int gz = grid_coord(cz, g.invCell, g.dimZ);
        const uint32_t h = (uint32_t)(gz * g.dimY * g.dimX + gy * g.dimX + gx);
        keys[slot] = ((uint32_t)B.worldId[i] << g.cellBits) | h;
        vals[slot] = (uint32_t)i;
    }
}

// kFindCellStart (G3/bt3dGridBroadphaseOCL.cl:61-87) into a stamped table.
__global__ void k_cell_start(const uint32_t* __restrict__ keys, int n, const int32_t* stamp_dev,
                             uint2* __restrict__ table) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) table[k] = make_uint2((uint32_t)*stamp_dev, (uint32_t)i);
}

__device__ __forceinline__ bool aabb_overlap(float4 mn0, float4 mx0, float4 mn1, float4 mx1) {
    return (mn0.x <= mx1.x) && (mn1.x <= mx0.x) && (mn0.y <= mx1.y) && (mn1.y <= mx0.y) &&
           (mn0.z <= mx1.z) && (mn1.z <= mx0.z);
}

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = (lane < nw) ? warp_tot[lane] : 0u;
        uint32_t s = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_tot[lane] = s - t;
        if (lane == nw - 1) *total = s;
    }
    __syncthreads();
    const uint32_t r = warp_tot[warp] + x - v;
    __syncthreads();
    return r;
}

// Output offset of one pair tile by decoupled look-back over the tiles before
// it (flag 1 = aggregate, 2 = inclusive prefix); the last tile publishes the
// pair count, clamped to maxPairs with the excess counted as pair overflow.
// Called by one thread of the tile.
__device__ uint32_t tile_lookback(int tile, int num_tiles, uint32_t agg, const GridParams& g,
                                  unsigned long long* __restrict__ status, int32_t* __restrict__ numPairs,
                                  b3Counters* __restrict__ counters, int32_t* __restrict__ err_flag) {
    const unsigned long long FA = 1ull << 32, FP = 2ull << 32;
    uint32_t excl = 0;
    if (tile == 0) {
        b3dev::st_release_u64(status, FP | agg);
    } else {
        b3dev::st_release_u64(status + tile, FA | agg);
        int t = tile - 1;
        while (t >= 0) {
            unsigned long long s = 0;
            int spins = 0;
            while (((s = b3dev::ld_acquire_u64(status + t)) >> 32) == 0) {
                if (++spins > b3dev::kSpinLimit) {
                    atomicExch(err_flag, 1);
                    atomicAdd(&counters->timeouts, 1);
                    break;
                }
                __nanosleep(32);
            }
            excl += (uint32_t)s;
            if ((s >> 32) != 1) break;
            --t;
        }
        b3dev::st_release_u64(status + tile, FP | (unsigned long long)(excl + agg));
    }
    if (tile == num_tiles - 1) {
        const uint32_t total = excl + agg;
        *numPairs = (int32_t)min(total, (uint32_t)g.maxPairs);
        if (total > (uint32_t)g.maxPairs) atomicAdd(&counters->pairOverflow, (int)(total - (uint32_t)g.maxPairs));
        counters->numPairs = (int32_t)min(total, (uint32_t)g.maxPairs);
    }
    return excl;
}

__global__ void __launch_bounds__(kPairTile)
k_find_pairs(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
             const float4* __restrict__ aabbMin, const float4* __restrict__ aabbMax,
             const uint2* __restrict__ table, const int32_t* stamp_dev,
             const int* __restrict__ largeStart, const int* __restrict__ largeList, GridParams g,
             int2* __restrict__ pairs, int32_t* __restrict__ numPairs,
             unsigned long long* __restrict__ status, int32_t* __restrict__ tile_counter,
             b3Counters* __restrict__ counters, int32_t* __restrict__ err_flag) {
    extern __shared__ int pbuf[];  // [kPairTile][maxPairsPerBody]
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t tile_total, tile_excl;
    __shared__ int tile_sh;
    const int n = g.numSmall;
    const int num_tiles = (n + kPairTile - 1) / kPairTile;
    const uint32_t stamp = (uint32_t)*stamp_dev;
    const int cap = g.maxPairsPerBody - 1;  // curr_max (G3/bt3dGridBroadphaseOCL.cl:129)
    for (;;) {
        if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1);
        __syncthreads();
        const int tile = tile_sh;
        if (tile >= num_tiles) break;
        const int i = tile * kPairTile + threadIdx.x;
        int cnt = 0;
        int* buf = pbuf + threadIdx.x * g.maxPairsPerBody;
        int ovf = 0, covf = 0;
        if (i < n) {
            const uint32_t key = keys[i];
            const uint32_t self = vals[i];
            const uint32_t world = key >> g.cellBits;
            const float4 mn0 = aabbMin[self], mx0 = aabbMax[self];
            const float cx = mrn(arn(mn0.x, mx0.x), 0.5f);
            const float cy = mrn(arn(mn0.y, mx0.y), 0.5f);
            const float cz = mrn(arn(mn0.z, mx0.z), 0.5f);
            const int gx = grid_coord(cx, g.invCell, g.dimX);
            const int gy = grid_coord(cy, g.invCell, g.dimY);
            const int gz = grid_coord(cz, g.invCell, g.dimZ);
            bool full = false;
            for (int dz = -1; dz <= 1; ++dz) {
                const int zz = (gz + dz) & (g.dimZ - 1);
                for (int dy = -1; dy <= 1; ++dy) {
                    const int yy = (gy + dy) & (g.dimY - 1);
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int xx = (gx + dx) & (g.dimX - 1);
                        const uint32_t h = (world << g.cellBits) |
                                           (uint32_t)(zz * g.dimY * g.dimX + yy * g.dimX + xx);
                        const uint2 e = table[h];
                        if (e.x != stamp) continue;
                        const int start = (int)e.y;
                        const int end = min(start + g.maxBodiesPerCell, n);
                        int j = start;
                        for (; j < end; ++j) {
                            if (keys[j] != h) break;
                            const uint32_t other = vals[j];
                            if (other < self) {
                                if (aabb_overlap(mn0, mx0, aabbMin[other], aabbMax[other])) {
                                    if (cnt >= cap) {
                                        ovf++;
                                        full = true;
                                        break;
                                    }
                                    buf[cnt++] = (int)other;
                                }
                            }
                        }
                        if (!full && j == end && end < n && keys[end] == h) covf++;
                        full = false;
                    }
                }
            }
            // large bodies of this world
            const int l0 = largeStart[world], l1 = largeStart[world + 1];
            for (int l = l0; l < l1; ++l) {
                const int L = largeList[l];
                if (aabb_overlap(mn0, mx0, aabbMin[L], aabbMax[L])) {
                    if (cnt >= cap) {
                        ovf++;
                        break;
                    }
                    buf[cnt++] = L;
                }
            }
        }
        // tile compaction with decoupled look-back
        const uint32_t texcl = block_excl_scan((uint32_t)cnt, warp_tot, &tile_total);
        if (threadIdx.x == 0)
            tile_excl = tile_lookback(tile, num_tiles, tile_total, g, status, numPairs, counters, err_flag);
        if (ovf) atomicAdd(&counters->pairOverflow, ovf);
        if (covf) atomicAdd(&counters->cellOverflow, covf);
        __syncthreads();
        if (i < n) {
            const uint32_t self = vals[i];
            const uint32_t base = tile_excl + texcl;
            for (int c = 0; c < cnt; ++c) {
                const uint32_t o = base + c;
                if (o < (uint32_t)g.maxPairs) pairs[o] = make_int2((int)self, buf[c]);
            }
        }
        __syncthreads();
    }
}

// Warp-cooperative form of k_find_pairs with the same output: one warp per
// body, lane l < 27 scanning neighbour cell l in findPairsInCell's z, y, x
// order (G3/bt3dGridBroadphaseOCL.cl:170-206). Each lane counts its cell's
// candidates (id(other) < id(self), inclusive AABB overlap) over the whole
// bucket, four entries per load batch; a warp scan of the counts gives every
// cell the pair count of the cells before it, and from that the sequential
// cap semantics follow per cell: the cell keeps min(count, cap - before)
// pairs, counts one pair overflow when it has more, and counts one cell
// overflow when it has none and its bucket holds more than maxBodiesPerCell
// bodies. Kept pairs are written from a 64-position candidate mask (a rescan
// covers candidates further into a bucket). The large bodies follow in
// 32-wide ballots with the same cap rule. Tiles of 32 bodies (eight per
// warp) are compacted like k_find_pairs' 128-body tiles, so the pair list,
// pair count and overflow counters are identical to it bit for bit.
__global__ void __launch_bounds__(kWarpPairThreads)
k_find_pairs_warp(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                  const float4* __restrict__ aabbMin, const float4* __restrict__ aabbMax,
                  const uint2* __restrict__ table, const int32_t* stamp_dev,
                  const int* __restrict__ largeStart, const int* __restrict__ largeList, GridParams g,
                  int2* __restrict__ pairs, int32_t* __restrict__ numPairs,
                  unsigned long long* __restrict__ status, int32_t* __restrict__ tile_counter,
                  b3Counters* __restrict__ counters, int32_t* __restrict__ err_flag) {
    extern __shared__ int pbuf[];  // [kWarpPairTile][maxPairsPerBody]
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t tile_total, tile_excl;
    __shared__ int tile_sh;
    __shared__ int cnts[kWarpPairTile];
    __shared__ uint32_t offs[kWarpPairTile];
    constexpr int kPerWarp = kWarpPairTile / (kWarpPairThreads / 32);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = g.numSmall;
    const int num_tiles = (n + kWarpPairTile - 1) / kWarpPairTile;
    const uint32_t stamp = (uint32_t)*stamp_dev;
    const int cap = g.maxPairsPerBody - 1;  // curr_max (G3/bt3dGridBroadphaseOCL.cl:129)
    const int dz = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dx = lane % 3 - 1;
    const uint32_t lanes_below = (1u << lane) - 1u;
    for (;;) {
        if (threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1);
        __syncthreads();
        const int tile = tile_sh;
        if (tile >= num_tiles) break;
        int ovf = 0, covf = 0;
        for (int b = 0; b < kPerWarp; ++b) {
            const int local = warp * kPerWarp + b;
            const int i = tile * kWarpPairTile + local;
            int cnt = 0;
            if (i < n) {  // warp-uniform
                const uint32_t key = keys[i];
                const uint32_t self = vals[i];
                const uint32_t world = key >> g.cellBits;
                const float4 mn0 = aabbMin[self], mx0 = aabbMax[self];
                const float cx = mrn(arn(mn0.x, mx0.x), 0.5f);
                const float cy = mrn(arn(mn0.y, mx0.y), 0.5f);
                const float cz = mrn(arn(mn0.z, mx0.z), 0.5f);
                int c = 0, start = 0, end = 0;
                uint32_t h = 0;
                bool active = false;
                unsigned long long mask = 0;  // candidate positions 0..63 of the bucket
                if (lane < 27) {
                    const int zz = (grid_coord(cz, g.invCell, g.dimZ) + dz) & (g.dimZ - 1);
                    const int yy = (grid_coord(cy, g.invCell, g.dimY) + dy) & (g.dimY - 1);
                    const int xx = (grid_coord(cx, g.invCell, g.dimX) + dx) & (g.dimX - 1);
                    h = (world << g.cellBits) | (uint32_t)(zz * g.dimY * g.dimX + yy * g.dimX + xx);
                    const uint2 e = table[h];
                    if (e.x == stamp) {
                        active = true;
                        start = (int)e.y;
                        end = min(start + g.maxBodiesPerCell, n);
                        for (int j = start; j < end; j += 4) {
                            bool in[4], cand[4];
                            uint32_t oo[4];
                            float4 amn[4], amx[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const int jj = j + u;
                                in[u] = false;
                                oo[u] = 0;
                                if (jj < end) {
                                    in[u] = keys[jj] == h;
                                    oo[u] = vals[jj];
                                }
                            }
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                cand[u] = in[u] && oo[u] < self;
                                amn[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                                amx[u] = amn[u];
                                if (cand[u]) {
                                    amn[u] = aabbMin[oo[u]];
                                    amx[u] = aabbMax[oo[u]];
                                }
                            }
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                if (cand[u] && aabb_overlap(mn0, mx0, amn[u], amx[u])) {
                                    const int pos = j + u - start;
                                    if (pos < 64) mask |= 1ull << pos;
                                    ++c;
                                }
                            }
                            if (!in[3]) break;  // keys are sorted: the bucket ended in this batch
                        }
                    }
                }
                // pairs of the cells before this one, and the cap rule per cell
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(full, incl, o);
                    if (lane >= o) incl += y;
                }
                const int before = min(incl - c, cap);
                const int room = cap - before;
                const int keep = min(c, room);
                const bool cell_ovf = c > room;
                ovf += cell_ovf ? 1 : 0;
                if (active && !cell_ovf && end < n && keys[end] == h) ++covf;
                cnt = min(__shfl_sync(full, incl, 31), cap);
                int* buf = pbuf + local * g.maxPairsPerBody;
                if (keep > 0) {
                    int w = 0;
                    unsigned long long m = mask;
                    while (m && w < keep) {
                        const int pos = __ffsll((long long)m) - 1;
                        m &= m - 1;
                        buf[before + w++] = (int)vals[start + pos];
                    }
                    for (int j = start + 64; j < end && w < keep; ++j) {
                        if (keys[j] != h) break;
                        const uint32_t other = vals[j];
                        if (other < self && aabb_overlap(mn0, mx0, aabbMin[other], aabbMax[other]))
                            buf[before + w++] = (int)other;
                    }
                }
                // large bodies of this world
                const int l0 = largeStart[world], l1 = largeStart[world + 1];
                for (int l = l0; l < l1; l += 32) {
                    const int ll = l + lane;
                    bool hit = false;
                    int L = 0;
                    if (ll < l1) {
                        L = largeList[ll];
                        hit = aabb_overlap(mn0, mx0, aabbMin[L], aabbMax[L]);
                    }
                    const uint32_t bm = __ballot_sync(full, hit);
                    const int rank = __popc(bm & lanes_below);
                    if (hit && cnt + rank < cap) buf[cnt + rank] = L;
                    const int nb = __popc(bm);
                    if (cnt + nb > cap) {
                        if (lane == 0) ++ovf;
                        cnt = cap;
                        break;
                    }
                    cnt += nb;
                }
            }
            if (lane == 0) cnts[local] = cnt;
        }
        __syncthreads();
        // tile compaction with decoupled look-back
        const uint32_t v = threadIdx.x < kWarpPairTile ? (uint32_t)cnts[threadIdx.x] : 0u;
        const uint32_t texcl = block_excl_scan(v, warp_tot, &tile_total);
        if (threadIdx.x < kWarpPairTile) offs[threadIdx.x] = texcl;
        if (threadIdx.x == 0)
            tile_excl = tile_lookback(tile, num_tiles, tile_total, g, status, numPairs, counters, err_flag);
        ovf = __reduce_add_sync(full, ovf);
        covf = __reduce_add_sync(full, covf);
        if (lane == 0 && ovf) atomicAdd(&counters->pairOverflow, ovf);
        if (lane == 0 && covf) atomicAdd(&counters->cellOverflow, covf);
        __syncthreads();
        for (int b = 0; b < kPerWarp; ++b) {
            const int local = warp * kPerWarp + b;
            const int i = tile * kWarpPairTile + local;
            if (i >= n) break;
            const int self = (int)vals[i];
            const uint32_t base = tile_excl + offs[local];
            const int c = cnts[local];
            for (int k = lane; k < c; k += 32) {
                const uint32_t o = base + (uint32_t)k;
                if (o < (uint32_t)g.maxPairs) pairs[o] = make_int2(self, pbuf[local * g.maxPairsPerBody + k]);
            }
        }
        __syncthreads();
    }
}

GridParams grid_params(const b3World_t* w) {
    GridParams g;
    g.invCell = w->invCell;
    g.dimX = w->cfg.gridDims[0];
    g.dimY = w->cfg.gridDims[1];
    g.dimZ = w->cfg.gridDims[2];
    g.cellBits = w->cellBits;
    g.maxBodiesPerCell = w->cfg.maxBodiesPerCell;
    g.maxPairsPerBody = w->cfg.maxPairsPerBody;
    g.maxPairs = w->cfg.maxPairs;
    g.numSmall = w->numSmall;
    return g;
}

}  // namespace

namespace b3 {

int launch_aabb_hash(b3World_t* w, cudaStream_t st) {
    const int n = (int)w->bodies.size();
    if (n == 0) return B3_OK;
    const GridParams g = grid_params(w);
    const float3 gdt = make_float3(w->sim.gravity.x * w->sim.dt, w->sim.gravity.y * w->sim.dt,
                                   w->sim.gravity.z * w->sim.dt);
    k_aabb_hash<<<(n + kAabbThreads - 1) / kAabbThreads, kAabbThreads, 0, st>>>(
        w->bodiesDev(), w->d.localAabb, g, gdt, w->d.smallSlot, w->d.aabbMin, w->d.aabbMax,
        w->d.keys, w->d.vals, 1);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int launch_sort_and_cells(b3World_t* w, cudaStream_t st) {
    if (w->sap) return launch_sap_sort(w, st);
    const int ns = w->numSmall;
    if (ns == 0) return B3_OK;
    bool alt = false;
    B3_TRY(radix_sort_pairs(w->d.keys, w->d.vals, w->d.keysAlt, w->d.valsAlt,
                            w->d.scalars + S_NUM_SMALL, ns, w->keyBits, w->d.sortScratch,
                            w->d.sortScratchBytes, w->d.scalars + S_ERR, st, &alt,
                            w->ctx->numSMs));
    if (alt) {
        B3_CUDA(cudaMemcpyAsync(w->d.keys, w->d.keysAlt, sizeof(uint32_t) * ns,
                                cudaMemcpyDeviceToDevice, st));
        B3_CUDA(cudaMemcpyAsync(w->d.vals, w->d.valsAlt, sizeof(uint32_t) * ns,
                                cudaMemcpyDeviceToDevice, st));
    }
    k_cell_start<<<(ns + 255) / 256, 256, 0, st>>>(w->d.keys, ns, w->d.scalars + S_STAMP,
                                                  w->d.cellTable);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

int launch_find_pairs(b3World_t* w, cudaStream_t st) {
    if (w->sap) return launch_sap_pairs(w, st);
    const int ns = w->numSmall;
    // numPairs = 0, tile counter = 0, status cleared
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_NUM_PAIRS, 0, sizeof(int32_t), st));
    B3_CUDA(cudaMemsetAsync(w->d.scalars + S_TILE, 0, sizeof(int32_t), st));
    if (ns == 0) return B3_OK;
    const bool warp = w->pairSearchMode == 1;
    const int tileBodies = warp ? kWarpPairTile : kPairTile;
    const int threads = warp ? kWarpPairThreads : kPairTile;
    const int tiles = (ns + tileBodies - 1) / tileBodies;
    B3_CUDA(cudaMemsetAsync(w->d.scanScratch, 0, sizeof(unsigned long long) * tiles, st));
    const GridParams g = grid_params(w);
    const size_t smem = (size_t)tileBodies * w->cfg.maxPairsPerBody * sizeof(int);
    const void* fn = warp ? (const void*)k_find_pairs_warp : (const void*)k_find_pairs;
    // opt in to the per-body pair buffers above 48 KB (128 KB at the
    // largest cap, 256 pairs per body in 128-body tiles)
    static size_t optIn[2] = {0, 0};
    if (smem > 48 * 1024 && smem > optIn[warp]) {
        B3_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        optIn[warp] = smem;
    }
    int occ = 1;
    B3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem));
    occ = occ < 1 ? 1 : occ;
    const int grid = std::min(tiles, w->ctx->numSMs * occ);
    if (warp)
        k_find_pairs_warp<<<grid, threads, smem, st>>>(
            w->d.keys, w->d.vals, w->d.aabbMin, w->d.aabbMax, w->d.cellTable, w->d.scalars + S_STAMP,
            w->d.largeStart, w->d.largeList, g, w->d.pairs, w->d.scalars + S_NUM_PAIRS,
            (unsigned long long*)w->d.scanScratch, w->d.scalars + S_TILE, w->d.counters,
            w->d.scalars + S_ERR);
    else
        k_find_pairs<<<grid, threads, smem, st>>>(
            w->d.keys, w->d.vals, w->d.aabbMin, w->d.aabbMax, w->d.cellTable, w->d.scalars + S_STAMP,
            w->d.largeStart, w->d.largeList, g, w->d.pairs, w->d.scalars + S_NUM_PAIRS,
            (unsigned long long*)w->d.scanScratch, w->d.scalars + S_TILE, w->d.counters,
            w->d.scalars + S_ERR);
    B3_CHECK_LAUNCH();
    return B3_OK;
}

}  // namespace b3
