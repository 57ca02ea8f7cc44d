// Host BVH builder for the traversal kernels (device/traverse.cuh).
//
// The reference used Metal's closed acceleration-structure builder: one
// primitive structure per shape plus an instance structure
// (ShapeBuilder.swift:7-94,302-319; EntityBuilder.swift:148-165).  Here all
// instances are flattened into one binary BVH over world-space triangles,
// built with binned SAH (32 bins per axis) and OpenMP tasks for subtrees.
// Leaves hold 1..8 triangles; depth is capped so the 64-entry traversal stack
// cannot overflow.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace rmdhost {

namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float *p) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    void grow(const Box &b) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    float area() const {
        float e0 = hi[0] - lo[0], e1 = hi[1] - lo[1], e2 = hi[2] - lo[2];
        if (e0 < 0) return 0;
        return 2.0f * (e0 * e1 + e1 * e2 + e2 * e0);
    }
};

struct Prim {
    Box box;
    float c[3];
    uint32_t idx;
};

constexpr int kBins = 32;
constexpr int kMaxLeaf = 8;
constexpr int kMaxDepth = 56;

struct Builder {
    std::vector<Prim> prims;
    std::vector<GpuBvhNode> nodes;
    std::atomic<uint32_t> nodeCount{0};

    static void rangeBounds(const Prim *p, size_t n, Box &box, Box &cbox) {
        for (size_t i = 0; i < n; i++) {
            box.grow(p[i].box);
            cbox.grow(p[i].c);
        }
    }

    // chooses a split of [b, e); returns mid (== b when a leaf is better)
    size_t split(size_t b, size_t e, const Box &box, const Box &cbox, int depth) {
        const size_t n = e - b;
        if (n <= 1) return b;
        int bestAxis = -1, bestBin = 0;
        float bestCost = FLT_MAX;
        for (int axis = 0; axis < 3; axis++) {
            const float lo = cbox.lo[axis], hi = cbox.hi[axis];
            if (!(hi > lo)) continue;
            Box bins[kBins];
            uint32_t cnt[kBins] = {};
            const float scale = kBins / (hi - lo);
            for (size_t i = b; i < e; i++) {
                int k = std::min(kBins - 1, (int)((prims[i].c[axis] - lo) * scale));
                bins[k].grow(prims[i].box);
                cnt[k]++;
            }
            float rArea[kBins];
            uint32_t rCnt[kBins];
            Box acc;
            uint32_t c = 0;
            for (int k = kBins - 1; k > 0; k--) {
                acc.grow(bins[k]);
                c += cnt[k];
                rArea[k] = acc.area();
                rCnt[k] = c;
            }
            Box lacc;
            uint32_t lc = 0;
            for (int k = 0; k < kBins - 1; k++) {
                lacc.grow(bins[k]);
                lc += cnt[k];
                if (lc == 0 || rCnt[k + 1] == 0) continue;
                const float cost = lacc.area() * (float)lc + rArea[k + 1] * (float)rCnt[k + 1];
                if (cost < bestCost) {
                    bestCost = cost;
                    bestAxis = axis;
                    bestBin = k;
                }
            }
        }
        // SAH leaf test: traversal cost 1, intersection cost 1 per triangle
        const float leafCost = box.area() * (float)n;
        const bool forceSplit = n > (size_t)kMaxLeaf;
        if (!forceSplit && (bestAxis < 0 || bestCost + box.area() >= leafCost)) return b;
        size_t mid = b;
        if (bestAxis >= 0 && depth < kMaxDepth) {
            const float lo = cbox.lo[bestAxis];
            const float scale = kBins / (cbox.hi[bestAxis] - lo);
            Prim *it = std::partition(prims.data() + b, prims.data() + e, [&](const Prim &p) {
                return std::min(kBins - 1, (int)((p.c[bestAxis] - lo) * scale)) <= bestBin;
            });
            mid = (size_t)(it - prims.data());
        }
        if (mid == b || mid == e) {
            if (!forceSplit) return b;
            // no usable centroid split: split the list by its median centroid on the widest axis
            int axis = 0;
            float w = -1;
            for (int k = 0; k < 3; k++)
                if (cbox.hi[k] - cbox.lo[k] > w) {
                    w = cbox.hi[k] - cbox.lo[k];
                    axis = k;
                }
            mid = b + n / 2;
            std::nth_element(prims.data() + b, prims.data() + mid, prims.data() + e,
                             [axis](const Prim &x, const Prim &y) { return x.c[axis] < y.c[axis]; });
        }
        return mid;
    }

    static int leafLink(size_t first, size_t count) { return ~(int)(((uint32_t)first << 3) | (uint32_t)(count - 1)); }

    // builds the subtree of [b, e) whose bounds the parent already stored; returns its link
    int build(size_t b, size_t e, int depth) {
        Box box, cbox;
        rangeBounds(prims.data() + b, e - b, box, cbox);
        const size_t mid = split(b, e, box, cbox, depth);
        if (mid == b) return leafLink(b, e - b);
        const uint32_t id = nodeCount.fetch_add(1);
        fillNode(id, b, mid, e, depth);
        return (int)id;
    }

    void fillNode(uint32_t id, size_t b, size_t mid, size_t e, int depth) {
        Box lb, lc, rb, rc;
        rangeBounds(prims.data() + b, mid - b, lb, lc);
        rangeBounds(prims.data() + mid, e - mid, rb, rc);
        GpuBvhNode &node = nodes[id];
        node.c0xy[0] = lb.lo[0]; node.c0xy[1] = lb.hi[0]; node.c0xy[2] = lb.lo[1]; node.c0xy[3] = lb.hi[1];
        node.c1xy[0] = rb.lo[0]; node.c1xy[1] = rb.hi[0]; node.c1xy[2] = rb.lo[1]; node.c1xy[3] = rb.hi[1];
        node.cz[0] = lb.lo[2]; node.cz[1] = lb.hi[2]; node.cz[2] = rb.lo[2]; node.cz[3] = rb.hi[2];
        int l = 0, r = 0;
        const size_t big = 1 << 14;
        if (e - b > big) {
#pragma omp task shared(l) firstprivate(b, mid, depth)
            l = build(b, mid, depth + 1);
#pragma omp task shared(r) firstprivate(mid, e, depth)
            r = build(mid, e, depth + 1);
#pragma omp taskwait
        } else {
            l = build(b, mid, depth + 1);
            r = build(mid, e, depth + 1);
        }
        node.link[0] = l;
        node.link[1] = r;
        node.link[2] = node.link[3] = 0;
    }
};

}  // namespace

void buildBvh(const std::vector<float> &v0, const std::vector<float> &v1, const std::vector<float> &v2,
              const std::vector<uint32_t> &instance, const std::vector<uint32_t> &prim, GpuBvh &out) {
    const size_t n = instance.size();
    Builder B;
    B.prims.resize(n);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) {
        Prim &p = B.prims[i];
        p.box = Box();
        p.box.grow(&v0[3 * i]);
        p.box.grow(&v1[3 * i]);
        p.box.grow(&v2[3 * i]);
        for (int k = 0; k < 3; k++) p.c[k] = 0.5f * (p.box.lo[k] + p.box.hi[k]);
        p.idx = (uint32_t)i;
    }
    B.nodes.resize(std::max<size_t>(1, 2 * n));
    B.nodeCount = 1;  // node 0 is the root
    if (n == 0) {
        // no triangles: no nodes; the traversal kernels treat a null node array as "everything misses"
        out.nodes.clear();
        out.tris.clear();
        return;
    } else {
        Box box, cbox;
        Builder::rangeBounds(B.prims.data(), n, box, cbox);
        size_t mid = B.split(0, n, box, cbox, 0);
        if (mid == 0) {
            // the whole scene is one leaf: both children of the root are that leaf
            GpuBvhNode &root = B.nodes[0];
            root.c0xy[0] = box.lo[0]; root.c0xy[1] = box.hi[0]; root.c0xy[2] = box.lo[1]; root.c0xy[3] = box.hi[1];
            root.cz[0] = box.lo[2]; root.cz[1] = box.hi[2];
            for (int k = 0; k < 4; k++) root.c1xy[k] = root.c0xy[k];
            root.cz[2] = box.lo[2]; root.cz[3] = box.hi[2];
            root.link[0] = root.link[1] = Builder::leafLink(0, n);
            root.link[2] = root.link[3] = 0;
        } else {
#pragma omp parallel
#pragma omp single
            B.fillNode(0, 0, mid, n, 0);
        }
    }
    const uint32_t numNodes = B.nodeCount.load();
    out.nodes.assign(B.nodes.begin(), B.nodes.begin() + numNodes);
    out.tris.resize(12 * n);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) {
        const uint32_t s = B.prims[i].idx;
        float *t = &out.tris[12 * i];
        std::memcpy(t + 0, &v0[3 * s], 12);
        std::memcpy(t + 4, &v1[3 * s], 12);
        std::memcpy(t + 8, &v2[3 * s], 12);
        std::memcpy(t + 3, &instance[s], 4);
        std::memcpy(t + 7, &prim[s], 4);
        t[11] = 0.0f;
    }
}

}  // namespace rmdhost
