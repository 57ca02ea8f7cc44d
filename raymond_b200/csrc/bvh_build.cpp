// Host BVH builder for the traversal kernels (device/traverse.cuh).
//
// The reference used Metal's closed acceleration-structure builder: one
// primitive structure per shape plus an instance structure
// (ShapeBuilder.swift:7-94,302-319; EntityBuilder.swift:148-165).  Here all
// instances are flattened into one binary BVH over world-space triangles,
// built with binned SAH (32 bins per axis) and OpenMP tasks for subtrees as a
// binary tree with leaves of 1..3 triangles, then collapsed into the
// compressed 8-wide form (80-byte nodes) the traversal kernels walk.
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
constexpr int kMaxLeaf = 3;
constexpr int kMaxDepth = 56;
constexpr uint32_t kMaxWideDepth = 32;  // levels the traversal stack holds (TRAVERSAL_STACK)

// binary node with its own bounds, the input of the 8-wide collapse
struct BinNode {
    Box box;
    int child[2];           // -1 for a leaf
    uint32_t first, count;  // the subtree's triangles: [first, first + count) of Builder::prims
    bool leaf() const { return child[0] < 0; }
};

struct Builder {
    std::vector<Prim> prims;
    std::vector<BinNode> bin;
    std::atomic<uint32_t> nodeCount{0};
    size_t maxLeaf = kMaxLeaf;

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
        const bool forceSplit = n > maxLeaf;
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

    // binary tree with node bounds over [b, e); returns the node index
    int buildBin(size_t b, size_t e, int depth) {
        Box box, cbox;
        rangeBounds(prims.data() + b, e - b, box, cbox);
        const uint32_t id = nodeCount.fetch_add(1);
        bin[id].box = box;
        const size_t mid = split(b, e, box, cbox, depth);
        if (mid == b) {
            bin[id].child[0] = bin[id].child[1] = -1;
            bin[id].first = (uint32_t)b;
            bin[id].count = (uint32_t)(e - b);
            return (int)id;
        }
        int l = 0, r = 0;
        if (e - b > (size_t)(1 << 14)) {
#pragma omp task shared(l) firstprivate(b, mid, depth)
            l = buildBin(b, mid, depth + 1);
#pragma omp task shared(r) firstprivate(mid, e, depth)
            r = buildBin(mid, e, depth + 1);
#pragma omp taskwait
        } else {
            l = buildBin(b, mid, depth + 1);
            r = buildBin(mid, e, depth + 1);
        }
        bin[id].child[0] = l;
        bin[id].child[1] = r;
        bin[id].first = (uint32_t)b;
        bin[id].count = (uint32_t)(e - b);
        return (int)id;
    }

};

// Collapses the binary tree into 8-wide nodes (depth first).  Any subtree of
// at most 3 triangles may be a leaf (its triangles are consecutive), so a
// node holds at most 24 triangles.  The default collapse is SAH-optimal: a
// dynamic programme over the binary tree (Ylitie, Karras and Laine 2017,
// section 3.1) chooses, for every subtree, whether it becomes a leaf, an
// inner node, or is spread over several slots of its parent, with the cost
// model of the binary build (1 per node visit, 1 per triangle test, each
// weighted by surface area).  Against opening the largest child greedily it
// fills nodes with 6 children instead of 4.5 and takes 8 % off closest-hit
// traversal in the glossy room (3 % in the spheres-and-terrain frame).  The
// greedy collapse (open the inner child of largest surface area while the
// node has fewer than 8) stays as the fallback for a tree the optimal
// collapse would make deeper than the traversal stack.  Children go to the
// slot whose octant direction best matches their offset from the node centre,
// so a ray visits them roughly front to back by taking slot ^ (ray octant) in
// increasing order.
struct WideCollapse {
    const std::vector<BinNode> &bin;
    const std::vector<Prim> &prims;
    bool optimal = true;
    std::vector<GpuWideNode> nodes;
    std::vector<uint32_t> triOrder;  // output triangle -> index into prims
    uint32_t depth = 0;              // levels of the emitted tree

    static constexpr uint32_t kLeafTris = 3;
    bool isLeaf(int i) const { return bin[i].leaf() || bin[i].count <= kLeafTris; }

    // cost[8 n + i - 1]: the least cost of the subtree of n given as at most i
    // slots of its parent (a leaf slot costs area * count, an inner node area
    // + its subtree as 8 slots).  choice[8 n]: 1 if n as one slot is a leaf;
    // choice[8 n + i - 1], i > 1: 0 if i - 1 slots do as well, else the slots
    // of the left child.  innerSplit[n]: the left child's slots when n is an
    // inner node.  Ties favour more slots (a shallower tree).
    std::vector<float> cost;
    std::vector<uint8_t> choice;
    std::vector<uint8_t> innerSplit;
    static constexpr float kNodeCost = 1.0f, kTriCost = 1.0f;

    void solve(int n) {
        const BinNode &b = bin[n];
        float *c = &cost[8 * (size_t)n];
        uint8_t *ch = &choice[8 * (size_t)n];
        const float area = b.box.area();
        const float leaf = b.count <= kLeafTris ? area * kTriCost * (float)b.count : FLT_MAX;
        if (b.leaf()) {
            for (int i = 0; i < 8; i++) {
                c[i] = leaf;
                ch[i] = i == 0 ? 1 : 0;
            }
            return;
        }
        const int l = b.child[0], r = b.child[1];
        if (b.count > (1u << 14)) {
#pragma omp task firstprivate(l)
            solve(l);
#pragma omp task firstprivate(r)
            solve(r);
#pragma omp taskwait
        } else {
            solve(l);
            solve(r);
        }
        const float *cl = &cost[8 * (size_t)l], *cr = &cost[8 * (size_t)r];
        float dist[9];
        uint8_t distK[9];
        for (int i = 2; i <= 8; i++) {
            dist[i] = FLT_MAX;
            distK[i] = 1;
            for (int k = 1; k < i; k++) {
                const float v = cl[k - 1] + cr[i - k - 1];
                if (v < dist[i]) {
                    dist[i] = v;
                    distK[i] = (uint8_t)k;
                }
            }
        }
        const float inner = area * kNodeCost + dist[8];
        innerSplit[n] = distK[8];
        c[0] = std::min(leaf, inner);
        ch[0] = b.count <= kLeafTris && leaf <= inner ? 1 : 0;
        for (int i = 2; i <= 8; i++) {
            if (dist[i] <= c[i - 2]) {
                c[i - 1] = dist[i];
                ch[i - 1] = distK[i];
            } else {
                c[i - 1] = c[i - 2];
                ch[i - 1] = 0;
            }
        }
    }

    // the slots the subtree of n takes when it may take `slots`
    void collect(int n, int slots, int *kids, int &nk) const {
        while (slots > 1 && !bin[n].leaf() && choice[8 * (size_t)n + slots - 1] == 0) slots--;
        if (slots == 1 || bin[n].leaf()) {
            kids[nk++] = n;
            return;
        }
        const int k = choice[8 * (size_t)n + slots - 1];
        collect(bin[n].child[0], k, kids, nk);
        collect(bin[n].child[1], slots - k, kids, nk);
    }

    void solveAll(int root, size_t count) {
        cost.assign(8 * count, 0.0f);
        choice.assign(8 * count, 0);
        innerSplit.assign(count, 1);
#pragma omp parallel
#pragma omp single
        solve(root);
    }
    bool isLeafSlot(int i) const { return optimal ? choice[8 * (size_t)i] == 1 : isLeaf(i); }

    // Quantised child bounds, conservative in float: origin + q * scale
    // encloses the child on every side.
    static void quantise(const Box &node, const Box *kids, const bool *used, GpuWideNode &w) {
        for (int k = 0; k < 3; k++) {
            const float lo = node.lo[k], extent = node.hi[k] - node.lo[k];
            int e = -100;
            if (extent > 0.0f) {
                int ex;
                std::frexp(extent / 255.0f, &ex);
                e = ex;
                while (node.lo[k] + 255.0f * std::ldexp(1.0f, e) < node.hi[k]) e++;
            }
            e = std::max(-126, std::min(127, e));
            const float scale = std::ldexp(1.0f, e);
            w.origin[k] = lo;
            w.exponent[k] = (uint8_t)(e + 127);
            for (int c = 0; c < 8; c++) {
                if (!used[c]) {  // empty slot: an inverted box
                    w.qlo[k][c] = 255;
                    w.qhi[k][c] = 0;
                    continue;
                }
                int ql = (int)std::floor((kids[c].lo[k] - lo) / scale);
                int qh = (int)std::ceil((kids[c].hi[k] - lo) / scale);
                ql = std::max(0, std::min(255, ql));
                qh = std::max(0, std::min(255, qh));
                while (ql > 0 && lo + (float)ql * scale > kids[c].lo[k]) ql--;
                while (qh < 255 && lo + (float)qh * scale < kids[c].hi[k]) qh++;
                w.qlo[k][c] = (uint8_t)ql;
                w.qhi[k][c] = (uint8_t)qh;
            }
        }
    }

    void emit(int binIdx, uint32_t wideIdx, uint32_t level) {
        depth = std::max(depth, level);
        int kids[8];
        int nk = 0;
        const BinNode &root = bin[binIdx];
        if (wideIdx == 0 && root.count <= kLeafTris) {
            kids[nk++] = binIdx;  // the whole scene is one leaf
        } else if (optimal) {
            const int k = innerSplit[binIdx];
            collect(root.child[0], k, kids, nk);
            collect(root.child[1], 8 - k, kids, nk);
        } else {
            kids[nk++] = root.child[0];
            kids[nk++] = root.child[1];
            while (nk < 8) {
                int best = -1;
                float bestArea = -1.0f;
                for (int i = 0; i < nk; i++) {
                    const BinNode &c = bin[kids[i]];
                    if (!isLeaf(kids[i]) && c.box.area() > bestArea) {
                        bestArea = c.box.area();
                        best = i;
                    }
                }
                if (best < 0) break;
                const int k = kids[best];
                kids[best] = bin[k].child[0];
                kids[nk++] = bin[k].child[1];
            }
        }
        // slots: bit k of a slot means "on the high side of axis k"
        Box nodeBox;
        for (int i = 0; i < nk; i++) nodeBox.grow(bin[kids[i]].box);
        float centre[3];
        for (int k = 0; k < 3; k++) centre[k] = 0.5f * (nodeBox.lo[k] + nodeBox.hi[k]);
        float score[8][8];
        for (int i = 0; i < nk; i++) {
            const Box &b = bin[kids[i]].box;
            for (int sl = 0; sl < 8; sl++) {
                float v = 0.0f;
                for (int k = 0; k < 3; k++) {
                    const float off = 0.5f * (b.lo[k] + b.hi[k]) - centre[k];
                    v += ((sl >> k) & 1) ? off : -off;
                }
                score[i][sl] = v;
            }
        }
        int slotKid[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        bool kidDone[8] = {};
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
            kidDone[bi] = true;
            slotKid[bs] = bi;
        }
        GpuWideNode w;
        std::memset(&w, 0, sizeof(w));
        Box boxes[8];
        bool used[8];
        int numInner = 0;
        for (int sl = 0; sl < 8; sl++) {
            used[sl] = slotKid[sl] >= 0;
            if (used[sl]) {
                boxes[sl] = bin[kids[slotKid[sl]]].box;
                if (!isLeafSlot(kids[slotKid[sl]])) numInner++;
            }
        }
        quantise(nodeBox, boxes, used, w);
        w.childBase = (uint32_t)nodes.size();
        nodes.resize(nodes.size() + numInner);
        w.triBase = (uint32_t)triOrder.size();
        int innerBin[8];
        int ni = 0;
        for (int sl = 0; sl < 8; sl++) {
            if (!used[sl]) continue;
            const BinNode &c = bin[kids[slotKid[sl]]];
            if (!isLeafSlot(kids[slotKid[sl]])) {
                w.imask |= (uint8_t)(1u << sl);
                innerBin[ni++] = kids[slotKid[sl]];
            } else {
                const uint32_t offset = (uint32_t)triOrder.size() - w.triBase;
                w.meta[sl] = (uint8_t)((((1u << c.count) - 1u) << 5) | offset);
                for (uint32_t t = 0; t < c.count; t++) triOrder.push_back(c.first + t);
            }
        }
        nodes[wideIdx] = w;
        for (int i = 0; i < ni; i++) emit(innerBin[i], w.childBase + (uint32_t)i, level + 1);
    }
};

}  // namespace

void buildWideBvh(const std::vector<float> &v0, const std::vector<float> &v1, const std::vector<float> &v2,
                  const std::vector<uint32_t> &instance, const std::vector<uint32_t> &prim, GpuWideBvh &out) {
    const size_t n = instance.size();
    out.nodes.clear();
    out.tris.clear();
    if (n == 0) return;  // no nodes: the traversal kernels treat a null node array as "everything misses"
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
    B.bin.resize(2 * n);
    B.nodeCount = 0;
    int root = 0;
#pragma omp parallel
#pragma omp single
    root = B.buildBin(0, n, 0);
    WideCollapse W{B.bin, B.prims};
    W.solveAll(root, B.nodeCount.load());
    W.nodes.resize(1);
    W.triOrder.reserve(n);
    W.emit(root, 0, 1);
    if (W.depth > kMaxWideDepth) {  // deeper than the traversal stack: the greedy collapse instead
        W.optimal = false;
        W.depth = 0;
        W.nodes.assign(1, GpuWideNode{});
        W.triOrder.clear();
        W.emit(root, 0, 1);
    }
    out.nodes = std::move(W.nodes);
    out.tris.resize(12 * n);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; i++) {
        const uint32_t s = B.prims[W.triOrder[i]].idx;
        float *t = &out.tris[12 * i];
        std::memcpy(t + 0, &v0[3 * s], 12);
        std::memcpy(t + 4, &v1[3 * s], 12);
        std::memcpy(t + 8, &v2[3 * s], 12);
        std::memcpy(t + 3, &instance[s], 4);
        std::memcpy(t + 7, &prim[s], 4);
        t[11] = 0.0f;
    }
}

double wideBvhSahCost(const GpuWideNode *nodes, size_t count, uint32_t &levels) {
    levels = 0;
    if (count == 0) return 0.0;
    auto slotBox = [](const GpuWideNode &w, int c, double lo[3], double hi[3]) {
        for (int k = 0; k < 3; k++) {
            const double scale = std::ldexp(1.0, (int)w.exponent[k] - 127);
            lo[k] = (double)w.origin[k] + w.qlo[k][c] * scale;
            hi[k] = (double)w.origin[k] + w.qhi[k][c] * scale;
        }
    };
    auto area = [](const double lo[3], const double hi[3]) {
        const double e0 = std::max(0.0, hi[0] - lo[0]), e1 = std::max(0.0, hi[1] - lo[1]),
                     e2 = std::max(0.0, hi[2] - lo[2]);
        return 2.0 * (e0 * e1 + e1 * e2 + e2 * e0);
    };
    // the root's area: the union of its slots
    double rlo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, rhi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int c = 0; c < 8; c++) {
        const bool used = (nodes[0].imask >> c & 1) || nodes[0].meta[c];
        if (!used) continue;
        double lo[3], hi[3];
        slotBox(nodes[0], c, lo, hi);
        for (int k = 0; k < 3; k++) {
            rlo[k] = std::min(rlo[k], lo[k]);
            rhi[k] = std::max(rhi[k], hi[k]);
        }
    }
    const double rootArea = std::max(area(rlo, rhi), 1e-30);
    double cost = 0.0;
    std::vector<std::pair<uint32_t, std::pair<double, uint32_t>>> stack{{0u, {rootArea, 1u}}};
    while (!stack.empty()) {
        const auto [idx, rest] = stack.back();
        const auto [nodeArea, depth] = rest;
        stack.pop_back();
        if (idx >= count) continue;
        levels = std::max(levels, depth);
        cost += nodeArea / rootArea;
        const GpuWideNode &w = nodes[idx];
        uint32_t inner = 0;
        for (int c = 0; c < 8; c++) {
            double lo[3], hi[3];
            slotBox(w, c, lo, hi);
            if (w.imask >> c & 1) {
                stack.push_back({w.childBase + inner++, {area(lo, hi), depth + 1}});
            } else if (w.meta[c]) {
                cost += area(lo, hi) / rootArea * (double)__builtin_popcount((unsigned)(w.meta[c] >> 5));
            }
        }
    }
    return cost;
}

}  // namespace rmdhost
