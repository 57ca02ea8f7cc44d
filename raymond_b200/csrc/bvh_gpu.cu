// Device BVH builder: the compressed 8-wide BVH of device/traverse.cuh built
// on the GPU, in place of the host's binned-SAH build.
//
// The reference used Metal's closed acceleration-structure builder
// (ShapeBuilder.swift:7-94,302-319; EntityBuilder.swift:148-165); its
// algorithm is unknown, so this is a new design:
//
//  1. Triangle boxes and the centroid bounds (one pass).
//  2. 63-bit Morton codes of the centroids (21 bits per axis), sorted with
//     the triangle indices by an LSD radix sort of 8-bit digits: per pass a
//     tile histogram, an exclusive scan of the (digit, tile) counts and a
//     stable scatter that ranks a tile's keys warp by warp with match.any.
//  3. A binary tree by parallel locally-ordered clustering (Meister and
//     Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
//     Hierarchy Construction", TVCG 2018): clusters in Morton order, each
//     finds the neighbour within 16 positions whose union box has the
//     smallest surface area; mutual nearest neighbours merge; the survivors
//     are compacted by a scan, and the loop repeats until one cluster is
//     left.  Equal costs are ordered by a symmetric hash of the pair, so
//     regular geometry (grids of equal triangles) still merges in parallel;
//     an iteration that merges fewer than 1/16 of the clusters is replaced
//     by merging Morton neighbours pairwise, which bounds the iteration count.
//  4. The SAH-optimal collapse into 8-wide nodes, as the host builder makes
//     it (Ylitie, Karras and Laine 2017, section 3.1): bottom up, one launch
//     per clustering iteration (a node's children were made in earlier
//     iterations), every binary node gets the least surface-area cost of its
//     subtree as at most 1..8 slots of its parent (a leaf of at most 3
//     triangles, an inner node, or a spread over several slots) and the
//     choices that reach it.  Then level by level from the root, each node
//     collects its slots from those choices, places the children in octant
//     slots and quantises their boxes; scans of the children and leaf
//     triangles per node place the next level's nodes and the triangles.  A
//     tree the optimal collapse would make deeper than the traversal stack is
//     collapsed again greedily (open the inner child of largest area until a
//     node has 8 children).
//
// Every kernel's indexes are bounded by its element count; the host loop
// reads one 8-byte total per clustering iteration and per tree level.
#include "bvh_gpu.h"

#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bvh_build.h"

namespace rmd {
namespace {

constexpr int kRadius = 16;          // clustering search window (each side), by default
constexpr int kMaxRadius = 64;
constexpr uint32_t kLeafTris = 3;    // subtrees of at most this many triangles are leaves
constexpr uint32_t kMaxWideLevels = 32;  // the traversal kernels' stack holds one group per level
constexpr int kScanItems = 4;        // per thread
constexpr int kScanThreads = 1024;
constexpr uint32_t kScanTile = kScanItems * kScanThreads;  // 4096
constexpr int kSortThreads = 256;    // 8 warps
constexpr int kSortRounds = 16;      // 32 keys per warp per round
constexpr uint32_t kSortTile = kSortThreads * kSortRounds;  // 4096 keys

// -------------------------------------------------------------------- scan
__device__ __forceinline__ uint2 operator+(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ uint2 operator-(uint2 a, uint2 b) { return make_uint2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ uint32_t shflUp(uint32_t v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ uint2 shflUp(uint2 v, int d) {
    return make_uint2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}

// Inclusive scan of one value per thread over a block of kScanThreads;
// `total` = the block's sum.
template <class T>
__device__ T blockInclusiveScan(T v, T &total) {
    __shared__ T warpSums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T u = shflUp(inc, d);
        if (lane >= d) inc = inc + u;
    }
    if (lane == 31) warpSums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T wi = warpSums[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T u = shflUp(wi, d);
            if (lane >= d) wi = wi + u;
        }
        warpSums[lane] = wi;
    }
    __syncthreads();
    total = warpSums[kScanThreads / 32 - 1];
    if (warp > 0) inc = inc + warpSums[warp - 1];
    __syncthreads();
    return inc;
}

// Exclusive scan of kScanItems consecutive values per thread, in place in v;
// returns the block's sum.
template <class T>
__device__ T blockExclusiveScanItems(T (&v)[kScanItems]) {
    T sum = v[0];
#pragma unroll
    for (int k = 1; k < kScanItems; k++) sum = sum + v[k];
    T total;
    T run = blockInclusiveScan(sum, total) - sum;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const T x = v[k];
        v[k] = run;
        run = run + x;
    }
    return total;
}

// tile-wise exclusive scan of in into out; partials[b] = tile b's sum
template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const T *in, T *out, uint32_t m, T *partials) {
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    T v[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) v[k] = base + k < m ? in[base + k] : T{};
    const T total = blockExclusiveScanItems(v);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < m) out[base + k] = v[k];
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// in-place exclusive scan of at most kScanTile partials by one block; *total = their sum
template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_partials(T *partials, uint32_t m, T *total) {
    const uint32_t base = threadIdx.x * kScanItems;
    T v[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) v[k] = base + k < m ? partials[base + k] : T{};
    const T all = blockExclusiveScanItems(v);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < m) partials[base + k] = v[k];
    if (threadIdx.x == 0) *total = all;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_add(T *out, uint32_t m, const T *partials) {
    const uint32_t base = blockIdx.x * kScanTile;
    const T p = partials[blockIdx.x];
    for (uint32_t k = threadIdx.x; k < kScanTile; k += kScanThreads)
        if (base + k < m) out[base + k] = out[base + k] + p;
}

// ------------------------------------------------------------- primitives
__device__ __forceinline__ uint32_t orderedBits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedFloat(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ float3 load3(const float *p, uint32_t i) {
    return make_float3(p[3 * (size_t)i], p[3 * (size_t)i + 1], p[3 * (size_t)i + 2]);
}

// triangle boxes (lo.w = 1: the leaf's triangle count) and the centroid bounds
__global__ void k_bvh_prims(const float *v0, const float *v1, const float *v2, uint32_t n, float4 *lo, float4 *hi,
                            uint32_t *centroidBounds) {
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float3 a = load3(v0, i), b = load3(v1, i), c = load3(v2, i);
        const float3 l = make_float3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)));
        const float3 h = make_float3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)));
        lo[i] = make_float4(l.x, l.y, l.z, __uint_as_float(1u));
        hi[i] = make_float4(h.x, h.y, h.z, 0.0f);
        const float cc[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
        for (int k = 0; k < 3; k++) {
            cmin[k] = fminf(cmin[k], cc[k]);
            cmax[k] = fmaxf(cmax[k], cc[k]);
        }
    }
    for (int k = 0; k < 3; k++) {
        for (int d = 16; d > 0; d >>= 1) {
            cmin[k] = fminf(cmin[k], __shfl_xor_sync(0xffffffffu, cmin[k], d));
            cmax[k] = fmaxf(cmax[k], __shfl_xor_sync(0xffffffffu, cmax[k], d));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) {
            atomicMin(&centroidBounds[k], orderedBits(cmin[k]));
            atomicMax(&centroidBounds[3 + k], orderedBits(cmax[k]));
        }
}

// 21 bits spread to every third bit of 63
__device__ __forceinline__ uint64_t spread21(uint32_t x) {
    uint64_t v = x & 0x1fffffu;
    v = (v | (v << 32)) & 0x001f00000000ffffull;
    v = (v | (v << 16)) & 0x001f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_bvh_morton(const float4 *lo, const float4 *hi, uint32_t n, const uint32_t *centroidBounds,
                             uint64_t *keys, uint32_t *vals) {
    float cmin[3], scale[3];
    for (int k = 0; k < 3; k++) {
        cmin[k] = orderedFloat(centroidBounds[k]);
        const float ext = orderedFloat(centroidBounds[3 + k]) - cmin[k];
        scale[k] = ext > 0.0f ? 2097152.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 l = lo[i], h = hi[i];
        const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
        uint32_t q[3];
        for (int k = 0; k < 3; k++) {
            const float t = (c[k] - cmin[k]) * scale[k];
            q[k] = t <= 0.0f ? 0u : (t >= 2097151.0f ? 2097151u : (uint32_t)t);
        }
        keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
        vals[i] = i;
    }
}

// ------------------------------------------------------------- radix sort
// counts[d * tiles + tile] = keys of the tile whose digit is d
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint64_t *keys, uint32_t n, int shift,
                                                              uint32_t *counts, uint32_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (uint32_t k = threadIdx.x; k < kSortTile; k += kSortThreads) {
        const uint32_t i = base + k;
        if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: warp w ranks its 512 keys (16 rounds of 32, in
// order) by digit with match.any, the warps' digit counts are prefixed in
// shared memory, and offsets (the scanned counts) place the tile.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint64_t *keysIn, const uint32_t *valsIn,
                                                                 uint64_t *keysOut, uint32_t *valsOut, uint32_t n,
                                                                 int shift, const uint32_t *offsets, uint32_t tiles) {
    __shared__ uint32_t wh[kSortThreads / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = 0; w < kSortThreads / 32; w++) wh[w][threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t chunk = blockIdx.x * kSortTile + (uint32_t)warp * (32u * kSortRounds);
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t key[kSortRounds];
    uint32_t val[kSortRounds], dig[kSortRounds], rank[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; r++) {
        const uint32_t i = chunk + (uint32_t)r * 32u + (uint32_t)lane;
        const bool valid = i < n;
        key[r] = valid ? keysIn[i] : 0ull;
        val[r] = valid ? valsIn[i] : 0u;
        const uint32_t d = valid ? ((uint32_t)(key[r] >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = valid ? wh[warp][d] : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wh[warp][d] += (uint32_t)__popc(peers);
        __syncwarp();
        dig[r] = d;
        rank[r] = before + (uint32_t)__popc(peers & lt);
    }
    __syncthreads();
    {  // exclusive prefix over the warps, per digit
        uint32_t run = 0u;
        for (int w = 0; w < kSortThreads / 32; w++) {
            const uint32_t c = wh[w][threadIdx.x];
            wh[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; r++) {
        if (dig[r] < 256u) {
            const uint32_t pos = offsets[dig[r] * tiles + blockIdx.x] + wh[warp][dig[r]] + rank[r];
            keysOut[pos] = key[r];
            valsOut[pos] = val[r];
        }
    }
}

// -------------------------------------------------------------- clustering
__device__ __forceinline__ float unionArea(float4 al, float4 ah, float4 bl, float4 bh) {
    const float ex = fmaxf(ah.x, bh.x) - fminf(al.x, bl.x);
    const float ey = fmaxf(ah.y, bh.y) - fminf(al.y, bl.y);
    const float ez = fmaxf(ah.z, bh.z) - fminf(al.z, bl.z);
    return ex * ey + ey * ez + ez * ex;  // half the surface area
}

// symmetric tie order of the pair (i, j)
__device__ __forceinline__ uint32_t pairHash(uint32_t i, uint32_t j) {
    uint32_t a = min(i, j), b = max(i, j);
    uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}

// leaves: node k = sorted triangle k
__global__ void k_bvh_leaves(const uint32_t *sortedTri, uint32_t n, const float4 *triLo, const float4 *triHi,
                             float4 *nodeLo, float4 *nodeHi, int2 *nodeChild, uint32_t *cl, float4 *clLo,
                             float4 *clHi) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t t = sortedTri[k];
        const float4 l = triLo[t], h = triHi[t];
        nodeLo[k] = l;
        nodeHi[k] = h;
        nodeChild[k] = make_int2(-1, (int)t);
        cl[k] = k;
        clLo[k] = l;
        clHi[k] = h;
    }
}

// nearest neighbour of each cluster within kRadius positions
constexpr int kNnThreads = 256;
__global__ void __launch_bounds__(kNnThreads) k_ploc_nn(const float4 *clLo, const float4 *clHi, uint32_t n,
                                                         int radius, uint32_t *nn) {
    __shared__ float4 sLo[kNnThreads + 2 * kMaxRadius], sHi[kNnThreads + 2 * kMaxRadius];
    const int64_t base = (int64_t)blockIdx.x * kNnThreads;
    for (int k = threadIdx.x; k < kNnThreads + 2 * radius; k += kNnThreads) {
        const int64_t j = base - radius + k;
        if (j >= 0 && j < (int64_t)n) {
            sLo[k] = clLo[j];
            sHi[k] = clHi[j];
        }
    }
    __syncthreads();
    const int64_t i = base + threadIdx.x;
    if (i >= (int64_t)n) return;
    const float4 al = sLo[threadIdx.x + radius], ah = sHi[threadIdx.x + radius];
    uint64_t best = ~0ull;
    uint32_t bestJ = 0u;
    for (int d = -radius; d <= radius; d++) {
        const int64_t j = i + d;
        if (d == 0 || j < 0 || j >= (int64_t)n) continue;
        const float c = unionArea(al, ah, sLo[threadIdx.x + radius + d], sHi[threadIdx.x + radius + d]);
        // cost >= 0, so its bits order like the float; the hash orders ties
        const uint64_t key = ((uint64_t)__float_as_uint(fmaxf(c, 0.0f)) << 32) | pairHash((uint32_t)i, (uint32_t)j);
        if (key < best) {
            best = key;
            bestJ = (uint32_t)j;
        }
    }
    nn[i] = bestJ;
}

// per cluster: (survives, leads a merge).  pairwise: merge Morton neighbours
// (2k, 2k + 1) instead of mutual nearest neighbours.
__global__ void k_ploc_flags(uint32_t *nn, uint32_t n, int pairwise, uint2 *flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        bool leader, follower;
        if (pairwise) {
            leader = (i & 1u) == 0u && i + 1u < n;
            follower = (i & 1u) == 1u;
            if (leader) nn[i] = i + 1u;
        } else {
            const uint32_t j = nn[i];
            const bool mutual = nn[j] == i;
            leader = mutual && i < j;
            follower = mutual && i > j;
        }
        flags[i] = make_uint2(follower ? 0u : 1u, leader ? 1u : 0u);
    }
}

// survivors to their scanned positions; leaders create the merged node
__global__ void k_ploc_compact(const uint32_t *cl, const float4 *clLo, const float4 *clHi, const uint32_t *nn,
                               const uint2 *flags, const uint2 *pos, uint32_t n, uint32_t nodeBase, uint32_t *clOut,
                               float4 *clLoOut, float4 *clHiOut, float4 *nodeLo, float4 *nodeHi, int2 *nodeChild) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 f = flags[i];
        if (!f.x) continue;
        const uint32_t p = pos[i].x;
        if (f.y) {
            const uint32_t j = nn[i];
            const float4 al = clLo[i], ah = clHi[i], bl = clLo[j], bh = clHi[j];
            const uint32_t count = __float_as_uint(al.w) + __float_as_uint(bl.w);
            const float4 l = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), __uint_as_float(count));
            const float4 h = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
            const uint32_t id = nodeBase + pos[i].y;
            nodeLo[id] = l;
            nodeHi[id] = h;
            nodeChild[id] = make_int2((int)cl[i], (int)cl[j]);
            clOut[p] = id;
            clLoOut[p] = l;
            clHiOut[p] = h;
        } else {
            clOut[p] = cl[i];
            clLoOut[p] = clLo[i];
            clHiOut[p] = clHi[i];
        }
    }
}

// ------------------------------------------------------- optimal collapse
// cost[8 i + s - 1]: the least cost of node i's subtree given as at most s
// slots of its parent (leaf slot: area * triangles; inner node: area + its
// subtree as 8 slots); choice[8 i]: 1 if i as one slot is a leaf; choice[8 i +
// s - 1], s > 1: 0 if s - 1 slots do as well, else the left child's slots;
// split[i]: the left child's slots when i is an inner node.  Ties favour
// more slots (a shallower tree).  The host builder's recurrence.
__device__ __forceinline__ float boxArea(float4 l, float4 h) {
    const float ex = h.x - l.x, ey = h.y - l.y, ez = h.z - l.z;
    if (ex < 0.0f) return 0.0f;
    return 2.0f * (ex * ey + ey * ez + ez * ex);
}

__global__ void k_dp_leaves(const float4 *lo, const float4 *hi, uint32_t n, float *cost, uint8_t *choice) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float leaf = boxArea(lo[i], hi[i]);  // one triangle
        for (int k = 0; k < 8; k++) {
            cost[8 * (size_t)i + k] = leaf;
            choice[8 * (size_t)i + k] = k == 0 ? 1 : 0;
        }
    }
}

__global__ void k_dp_nodes(const float4 *lo, const float4 *hi, const int2 *child, uint32_t base, uint32_t count,
                           float *cost, uint8_t *choice, uint8_t *split) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const size_t i = (size_t)base + j;
        const int2 ch = child[i];
        const float4 l = lo[i], h = hi[i];
        const uint32_t tris = __float_as_uint(l.w);
        const float area = boxArea(l, h);
        const float leaf = tris <= kLeafTris ? area * (float)tris : FLT_MAX;
        float cl[8], cr[8];
        for (int k = 0; k < 8; k++) {
            cl[k] = cost[8 * (size_t)ch.x + k];
            cr[k] = cost[8 * (size_t)ch.y + k];
        }
        float dist[9];
        uint8_t distK[9];
        for (int s = 2; s <= 8; s++) {
            dist[s] = FLT_MAX;
            distK[s] = 1;
            for (int k = 1; k < s; k++) {
                const float v = cl[k - 1] + cr[s - k - 1];
                if (v < dist[s]) {
                    dist[s] = v;
                    distK[s] = (uint8_t)k;
                }
            }
        }
        const float inner = area + dist[8];
        split[i] = distK[8];
        float c = fminf(leaf, inner);
        cost[8 * i] = c;
        choice[8 * i] = tris <= kLeafTris && leaf <= inner ? 1 : 0;
        for (int s = 2; s <= 8; s++) {
            if (dist[s] <= c) {
                c = dist[s];
                choice[8 * i + s - 1] = distK[s];
            } else {
                choice[8 * i + s - 1] = 0;
            }
            cost[8 * i + s - 1] = c;
        }
    }
}

// ---------------------------------------------------------------- collapse
struct Tree {
    const float4 *lo, *hi;
    const int2 *child;
    const uint8_t *choice, *split;  // the optimal collapse's choices; null: the greedy collapse
    __device__ uint32_t count(int i) const { return __float_as_uint(lo[i].w); }
    __device__ bool leaf(int i) const { return child[i].x < 0 || count(i) <= kLeafTris; }
    // whether binary node i, as one slot of its parent, is a leaf
    __device__ bool leafSlot(int i) const { return choice ? choice[8 * (size_t)i] == 1 : leaf(i); }
    __device__ float area(int i) const {
        const float4 l = lo[i], h = hi[i];
        const float ex = h.x - l.x, ey = h.y - l.y, ez = h.z - l.z;
        if (ex < 0.0f) return 0.0f;
        return 2.0f * (ex * ey + ey * ez + ez * ex);
    }
};

// Children of one 8-wide node by slot (-1: empty) and its (inner children,
// leaf triangles); the same choices as the host's greedy collapse.
__global__ void k_collapse_plan(Tree t, const uint2 *entries, uint32_t m, int *slots, uint2 *counts) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const int root = (int)entries[e].x;
        int kids[8];
        int nk = 0;
        if (entries[e].y == 0u && t.count(root) <= kLeafTris) {
            kids[nk++] = root;  // the whole scene is one leaf
        } else if (t.choice) {
            // the slots of the optimal collapse: (subtree, slots it may take), left child first
            int stNode[16], stSlots[16];
            int top = 0;
            const int k0 = t.split[root];
            stNode[top] = t.child[root].y, stSlots[top++] = 8 - k0;
            stNode[top] = t.child[root].x, stSlots[top++] = k0;
            while (top > 0 && nk < 8) {
                const int x = stNode[--top];
                int sl = stSlots[top];
                const bool binLeaf = t.child[x].x < 0;
                while (sl > 1 && !binLeaf && t.choice[8 * (size_t)x + sl - 1] == 0) sl--;
                if (sl == 1 || binLeaf) {
                    kids[nk++] = x;
                } else if (top + 2 <= 16) {
                    const int k = t.choice[8 * (size_t)x + sl - 1];
                    stNode[top] = t.child[x].y, stSlots[top++] = sl - k;
                    stNode[top] = t.child[x].x, stSlots[top++] = k;
                }
            }
        } else {
            kids[nk++] = t.child[root].x;
            kids[nk++] = t.child[root].y;
        }
        while (!t.choice && nk < 8) {
            int best = -1;
            float bestArea = -1.0f;
            for (int i = 0; i < nk; i++)
                if (!t.leaf(kids[i])) {
                    const float a = t.area(kids[i]);
                    if (a > bestArea) {
                        bestArea = a;
                        best = i;
                    }
                }
            if (best < 0) break;
            const int k = kids[best];
            kids[best] = t.child[k].x;
            kids[nk++] = t.child[k].y;
        }
        float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = 0; i < nk; i++) {
            const float4 l = t.lo[kids[i]], h = t.hi[kids[i]];
            nlo[0] = fminf(nlo[0], l.x); nlo[1] = fminf(nlo[1], l.y); nlo[2] = fminf(nlo[2], l.z);
            nhi[0] = fmaxf(nhi[0], h.x); nhi[1] = fmaxf(nhi[1], h.y); nhi[2] = fmaxf(nhi[2], h.z);
        }
        float centre[3];
        for (int k = 0; k < 3; k++) centre[k] = 0.5f * (nlo[k] + nhi[k]);
        float score[8][8];
        for (int i = 0; i < nk; i++) {
            const float4 l = t.lo[kids[i]], h = t.hi[kids[i]];
            const float off[3] = {0.5f * (l.x + h.x) - centre[0], 0.5f * (l.y + h.y) - centre[1],
                                  0.5f * (l.z + h.z) - centre[2]};
            for (int sl = 0; sl < 8; sl++) {
                float v = 0.0f;
                for (int k = 0; k < 3; k++) v += ((sl >> k) & 1) ? off[k] : -off[k];
                score[i][sl] = v;
            }
        }
        int slotKid[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        bool kidDone[8] = {false, false, false, false, false, false, false, false};
        for (int round = 0; round < nk; round++) {
            int bi = -1, bs = -1;
            float bv = -FLT_MAX;
            for (int i = 0; i < nk; i++) {
                if (kidDone[i]) continue;
                for (int sl = 0; sl < 8; sl++)
                    if (slotKid[sl] < 0 && score[i][sl] > bv) {
                        bv = score[i][sl];
                        bi = i;
                        bs = sl;
                    }
            }
            if (bi < 0) break;  // scores are finite for finite boxes; guards non-finite input
            kidDone[bi] = true;
            slotKid[bs] = bi;
        }
        uint32_t inner = 0u, tris = 0u;
        for (int sl = 0; sl < 8; sl++) {
            const int node = slotKid[sl] >= 0 ? kids[slotKid[sl]] : -1;
            slots[8 * (size_t)e + sl] = node;
            if (node < 0) continue;
            if (t.leafSlot(node)) tris += t.count(node);
            else inner++;
        }
        counts[e] = make_uint2(inner, tris);
    }
}

// quantised child bounds, conservative in float (the host's rule)
__device__ void quantise(const float *nlo, const float *nhi, const float4 *klo, const float4 *khi, const bool *used,
                         rmdhost::GpuWideNode &w) {
    for (int k = 0; k < 3; k++) {
        const float lo = nlo[k], extent = nhi[k] - nlo[k];
        int e = -100;
        if (extent > 0.0f) {
            int ex;
            frexpf(extent / 255.0f, &ex);
            e = ex;
            while (lo + 255.0f * ldexpf(1.0f, e) < nhi[k]) e++;
        }
        e = max(-126, min(127, e));
        const float scale = ldexpf(1.0f, e);
        w.origin[k] = lo;
        w.exponent[k] = (uint8_t)(e + 127);
        for (int c = 0; c < 8; c++) {
            if (!used[c]) {
                w.qlo[k][c] = 255;
                w.qhi[k][c] = 0;
                continue;
            }
            const float cl = k == 0 ? klo[c].x : (k == 1 ? klo[c].y : klo[c].z);
            const float ch = k == 0 ? khi[c].x : (k == 1 ? khi[c].y : khi[c].z);
            int ql = (int)floorf((cl - lo) / scale);
            int qh = (int)ceilf((ch - lo) / scale);
            ql = max(0, min(255, ql));
            qh = max(0, min(255, qh));
            while (ql > 0 && lo + (float)ql * scale > cl) ql--;
            while (qh < 255 && lo + (float)qh * scale < ch) qh++;
            w.qlo[k][c] = (uint8_t)ql;
            w.qhi[k][c] = (uint8_t)qh;
        }
    }
}

// Writes the level's nodes, their leaf triangles and the next level's entries.
__global__ void k_collapse_emit(Tree t, const uint2 *entries, uint32_t m, const int *slots, const uint2 *offsets,
                                uint32_t nodeBase, uint32_t triBase, const float *v0, const float *v1, const float *v2,
                                const uint32_t *inst, const uint32_t *prim, rmdhost::GpuWideNode *nodes,
                                float4 *tris, uint2 *next) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        int kid[8];
        bool used[8];
        float4 klo[8], khi[8];
        float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int sl = 0; sl < 8; sl++) {
            kid[sl] = slots[8 * (size_t)e + sl];
            used[sl] = kid[sl] >= 0;
            if (!used[sl]) continue;
            klo[sl] = t.lo[kid[sl]];
            khi[sl] = t.hi[kid[sl]];
            nlo[0] = fminf(nlo[0], klo[sl].x); nlo[1] = fminf(nlo[1], klo[sl].y); nlo[2] = fminf(nlo[2], klo[sl].z);
            nhi[0] = fmaxf(nhi[0], khi[sl].x); nhi[1] = fmaxf(nhi[1], khi[sl].y); nhi[2] = fmaxf(nhi[2], khi[sl].z);
        }
        rmdhost::GpuWideNode w;
        memset(&w, 0, sizeof(w));
        quantise(nlo, nhi, klo, khi, used, w);
        const uint2 off = offsets[e];
        w.childBase = nodeBase + off.x;
        w.triBase = triBase + off.y;
        uint32_t innerAt = 0u, triAt = 0u;
        for (int sl = 0; sl < 8; sl++) {
            if (!used[sl]) continue;
            const int node = kid[sl];
            if (!t.leafSlot(node)) {
                w.imask |= (uint8_t)(1u << sl);
                next[off.x + innerAt] = make_uint2((uint32_t)node, w.childBase + innerAt);
                innerAt++;
                continue;
            }
            const uint32_t c = t.count(node);
            w.meta[sl] = (uint8_t)((((1u << c) - 1u) << 5) | triAt);
            // the leaf's triangles, depth first (at most kLeafTris, so a short stack)
            int stack[8];
            int sp = 0;
            stack[sp++] = node;
            while (sp > 0) {
                const int x = stack[--sp];
                const int2 ch = t.child[x];
                if (ch.x < 0) {
                    const uint32_t tri = (uint32_t)ch.y;
                    float4 *o = &tris[3 * ((size_t)w.triBase + triAt)];
                    const float3 a = load3(v0, tri), b = load3(v1, tri), cc = load3(v2, tri);
                    o[0] = make_float4(a.x, a.y, a.z, __uint_as_float(inst[tri]));
                    o[1] = make_float4(b.x, b.y, b.z, __uint_as_float(prim[tri]));
                    o[2] = make_float4(cc.x, cc.y, cc.z, 0.0f);
                    triAt++;
                } else if (sp + 2 <= 8) {
                    stack[sp++] = ch.y;
                    stack[sp++] = ch.x;
                }
            }
        }
        nodes[entries[e].y] = w;
    }
}

// --------------------------------------------------------------- host side
struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T *&p, size_t count) {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, std::max<size_t>(1, count) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        p = static_cast<T *>(q);
        return e;
    }
};

#define BVH_TRY(x)                               \
    do {                                         \
        const cudaError_t e_ = (x);              \
        if (e_ != cudaSuccess) return e_;        \
    } while (0)

int gridFor(uint32_t n, int threads) { return (int)std::max<uint32_t>(1, std::min<uint32_t>((n + threads - 1) / threads, 148u * 16u)); }

template <class T>
cudaError_t exclusiveScan(const T *in, T *out, uint32_t m, T *partials, T *total, cudaStream_t s) {
    const uint32_t tiles = std::max<uint32_t>(1, (m + kScanTile - 1) / kScanTile);
    if (tiles > kScanTile) return cudaErrorInvalidValue;
    k_scan_tiles<T><<<tiles, kScanThreads, 0, s>>>(in, out, m, partials);
    k_scan_partials<T><<<1, kScanThreads, 0, s>>>(partials, tiles, total);
    k_scan_add<T><<<tiles, kScanThreads, 0, s>>>(out, m, partials);
    return cudaGetLastError();
}

template <class T>
cudaError_t readTotal(const T *d, T &h, cudaStream_t s) {
    BVH_TRY(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
    return cudaStreamSynchronize(s);
}

}  // namespace
}  // namespace rmd

namespace rmdhost {

using namespace rmd;

cudaError_t buildWideBvhGpu(const float *v0, const float *v1, const float *v2, const uint32_t *inst,
                            const uint32_t *prim, uint32_t n, cudaStream_t s, GpuBvhResult &out) {
    out = GpuBvhResult();
    if (n == 0) return cudaSuccess;  // no nodes: everything misses
    if (n > kGpuBvhMaxTriangles) {
        out.error = "the device BVH builder takes at most 2^24 triangles";
        return cudaErrorInvalidValue;
    }
    Scratch S;
    float4 *triLo, *triHi, *nodeLo, *nodeHi, *clLo[2], *clHi[2];
    int2 *nodeChild;
    uint64_t *keys[2];
    uint32_t *vals[2], *centroidBounds, *counts, *offsets, *countPartials, *countTotal, *cl[2], *nn;
    uint2 *flags, *pos, *pairPartials, *pairTotal;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t nodes2 = 2 * (size_t)n;
    BVH_TRY(S.alloc(triLo, n));
    BVH_TRY(S.alloc(triHi, n));
    BVH_TRY(S.alloc(nodeLo, nodes2));
    BVH_TRY(S.alloc(nodeHi, nodes2));
    BVH_TRY(S.alloc(nodeChild, nodes2));
    for (int b = 0; b < 2; b++) {
        BVH_TRY(S.alloc(keys[b], n));
        BVH_TRY(S.alloc(vals[b], n));
        BVH_TRY(S.alloc(cl[b], n));
        BVH_TRY(S.alloc(clLo[b], n));
        BVH_TRY(S.alloc(clHi[b], n));
    }
    BVH_TRY(S.alloc(centroidBounds, 6));
    BVH_TRY(S.alloc(counts, 256 * (size_t)tiles));
    BVH_TRY(S.alloc(offsets, 256 * (size_t)tiles));
    BVH_TRY(S.alloc(countPartials, kScanTile));
    BVH_TRY(S.alloc(countTotal, 1));
    BVH_TRY(S.alloc(nn, n));
    BVH_TRY(S.alloc(flags, n));
    BVH_TRY(S.alloc(pos, n));
    BVH_TRY(S.alloc(pairPartials, kScanTile));
    BVH_TRY(S.alloc(pairTotal, 1));

    // 1. boxes and centroid bounds
    const uint32_t initBounds[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    BVH_TRY(cudaMemcpyAsync(centroidBounds, initBounds, sizeof(initBounds), cudaMemcpyHostToDevice, s));
    k_bvh_prims<<<gridFor(n, 256), 256, 0, s>>>(v0, v1, v2, n, triLo, triHi, centroidBounds);
    // 2. Morton codes, sorted with the triangle indices (8 passes of 8 bits)
    k_bvh_morton<<<gridFor(n, 256), 256, 0, s>>>(triLo, triHi, n, centroidBounds, keys[0], vals[0]);
    BVH_TRY(cudaGetLastError());
    int cur = 0;
    for (int shift = 0; shift < 64; shift += 8) {
        k_radix_hist<<<tiles, kSortThreads, 0, s>>>(keys[cur], n, shift, counts, tiles);
        BVH_TRY(exclusiveScan<uint32_t>(counts, offsets, 256u * tiles, countPartials, countTotal, s));
        k_radix_scatter<<<tiles, kSortThreads, 0, s>>>(keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], n, shift,
                                                      offsets, tiles);
        BVH_TRY(cudaGetLastError());
        cur ^= 1;
    }
    // 3. clustering: leaves are nodes 0..n-1 (sorted order), merges n..2n-2
    k_bvh_leaves<<<gridFor(n, 256), 256, 0, s>>>(vals[cur], n, triLo, triHi, nodeLo, nodeHi, nodeChild, cl[0],
                                                 clLo[0], clHi[0]);
    BVH_TRY(cudaGetLastError());
    // search radius: RMD_BVH_RADIUS overrides the default (1..64)
    int radius = kRadius;
    if (const char *env = std::getenv("RMD_BVH_RADIUS")) radius = std::max(1, std::min(kMaxRadius, std::atoi(env)));
    uint32_t clusters = n, nodeBase = n;
    std::vector<std::pair<uint32_t, uint32_t>> made;  // (first node, count) of each clustering iteration
    int c = 0;
    while (clusters > 1) {
        if (++out.clusterIterations > 4096) {
            out.error = "device BVH clustering did not converge";
            return cudaErrorInvalidValue;
        }
        k_ploc_nn<<<(clusters + kNnThreads - 1) / kNnThreads, kNnThreads, 0, s>>>(clLo[c], clHi[c], clusters, radius,
                                                                                  nn);
        k_ploc_flags<<<gridFor(clusters, 256), 256, 0, s>>>(nn, clusters, 0, flags);
        BVH_TRY(exclusiveScan<uint2>(flags, pos, clusters, pairPartials, pairTotal, s));
        uint2 total;
        BVH_TRY(readTotal(pairTotal, total, s));
        if (total.y < std::max<uint32_t>(1u, clusters / 16u)) {  // too few mutual pairs: merge neighbours pairwise
            k_ploc_flags<<<gridFor(clusters, 256), 256, 0, s>>>(nn, clusters, 1, flags);
            BVH_TRY(exclusiveScan<uint2>(flags, pos, clusters, pairPartials, pairTotal, s));
            BVH_TRY(readTotal(pairTotal, total, s));
        }
        k_ploc_compact<<<gridFor(clusters, 256), 256, 0, s>>>(cl[c], clLo[c], clHi[c], nn, flags, pos, clusters,
                                                               nodeBase, cl[c ^ 1], clLo[c ^ 1], clHi[c ^ 1], nodeLo,
                                                               nodeHi, nodeChild);
        BVH_TRY(cudaGetLastError());
        made.emplace_back(nodeBase, total.y);
        nodeBase += total.y;
        clusters = total.x;
        c ^= 1;
    }
    uint32_t root = 0;
    BVH_TRY(cudaMemcpyAsync(&root, cl[c], sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    BVH_TRY(cudaStreamSynchronize(s));

    // 4. collapse, level by level; at most n wide nodes (each has >= 2 triangles below it or is the root)
    GpuWideNode *wide;
    float4 *tris;
    uint2 *entries[2];
    int *slots;
    uint2 *plan, *planPos;
    BVH_TRY(cudaMalloc(&out.tris, (size_t)n * 3 * sizeof(float4)));
    tris = static_cast<float4 *>(out.tris);
    BVH_TRY(cudaMalloc(&out.nodes, (size_t)n * sizeof(GpuWideNode)));
    wide = static_cast<GpuWideNode *>(out.nodes);
    BVH_TRY(S.alloc(entries[0], n));
    BVH_TRY(S.alloc(entries[1], n));
    BVH_TRY(S.alloc(slots, 8 * (size_t)n));
    BVH_TRY(S.alloc(plan, n));
    BVH_TRY(S.alloc(planPos, n));
    // the optimal collapse's costs and choices, bottom up
    float *dpCost;
    uint8_t *dpChoice, *dpSplit;
    BVH_TRY(S.alloc(dpCost, 8 * nodes2));
    BVH_TRY(S.alloc(dpChoice, 8 * nodes2));
    BVH_TRY(S.alloc(dpSplit, nodes2));
    k_dp_leaves<<<gridFor(n, 256), 256, 0, s>>>(nodeLo, nodeHi, n, dpCost, dpChoice);
    for (const auto &r : made)
        if (r.second > 0)
            k_dp_nodes<<<gridFor(r.second, 128), 128, 0, s>>>(nodeLo, nodeHi, nodeChild, r.first, r.second, dpCost,
                                                               dpChoice, dpSplit);
    BVH_TRY(cudaGetLastError());
    const uint2 first = make_uint2(root, 0u);
    Tree t{nodeLo, nodeHi, nodeChild, dpChoice, dpSplit};
    uint32_t level = 0, width = 0, wideCount = 0, triCount = 0;
    int e = 0;
    for (bool restart = true; restart;) {  // the optimal collapse, or the greedy one if that is too deep
        restart = false;
        BVH_TRY(cudaMemcpyAsync(entries[0], &first, sizeof(first), cudaMemcpyHostToDevice, s));
        level = 0, width = 1, wideCount = 1, triCount = 0, e = 0;
    while (width > 0) {
        if (++level > kMaxWideLevels) {
            if (t.choice) {
                t.choice = t.split = nullptr;
                restart = true;
                break;
            }
            out.error = "device BVH deeper than the traversal stack (32 levels)";
            return cudaErrorInvalidValue;
        }
        k_collapse_plan<<<gridFor(width, 128), 128, 0, s>>>(t, entries[e], width, slots, plan);
        BVH_TRY(exclusiveScan<uint2>(plan, planPos, width, pairPartials, pairTotal, s));
        k_collapse_emit<<<gridFor(width, 128), 128, 0, s>>>(t, entries[e], width, slots, planPos, wideCount, triCount,
                                                            v0, v1, v2, inst, prim, wide, tris, entries[e ^ 1]);
        BVH_TRY(cudaGetLastError());
        uint2 total;
        BVH_TRY(readTotal(pairTotal, total, s));
        wideCount += total.x;
        triCount += total.y;
        width = total.x;
        e ^= 1;
        if (wideCount > n + 1) {
            out.error = "device BVH collapse produced more nodes than triangles";
            return cudaErrorInvalidValue;
        }
    }
    }
    if (triCount != n) {
        out.error = "device BVH collapse placed " + std::to_string(triCount) + " of " + std::to_string(n) +
                    " triangles";
        return cudaErrorInvalidValue;
    }
    out.nodeCount = wideCount;
    out.levels = level;
    return cudaStreamSynchronize(s);
}

}  // namespace rmdhost
