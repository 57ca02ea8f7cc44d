// Oracle (test infrastructure only): binned-SAH BVH + watertight triangle test.
#include "bvh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace orc {

WatertightRay::WatertightRay(float3 o, float3 d) : org(o) {
    // WBW 2013, section 3: kz = dimension with the largest |d|
    float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    kx = kz + 1 == 3 ? 0 : kz + 1;
    ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < 0.0f) std::swap(kx, ky);  // preserve winding
    Sx = d[kx] / d[kz];
    Sy = d[ky] / d[kz];
    Sz = 1.0f / d[kz];
}

bool intersectTriangle(const WatertightRay &r, float3 v0, float3 v1, float3 v2, float tmin, float tmax, float &t,
                       float &b0, float &b1) {
    const float3 A = v0 - r.org, B = v1 - r.org, C = v2 - r.org;
    const float Ax = A[r.kx] - r.Sx * A[r.kz];
    const float Ay = A[r.ky] - r.Sy * A[r.kz];
    const float Bx = B[r.kx] - r.Sx * B[r.kz];
    const float By = B[r.ky] - r.Sy * B[r.kz];
    const float Cx = C[r.kx] - r.Sx * C[r.kz];
    const float Cy = C[r.ky] - r.Sy * C[r.kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // fall back to double on the edges
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * A[r.kz];
    const float Bz = r.Sz * B[r.kz];
    const float Cz = r.Sz * C[r.kz];
    const float T = U * Az + V * Bz + W * Cz;
    const float rcpDet = 1.0f / det;
    t = T * rcpDet;
    if (!(t >= tmin && t <= tmax)) return false;
    b0 = U * rcpDet;
    b1 = V * rcpDet;
    return true;
}

namespace {
struct Aabb {
    float3 lo{FLT_MAX, FLT_MAX, FLT_MAX}, hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(float3 p) {
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    void grow(const Aabb &b) {
        lo = vmin(lo, b.lo);
        hi = vmax(hi, b.hi);
    }
    float area() const {
        float3 e = hi - lo;
        if (e.x < 0) return 0;
        return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
};
struct BuildPrim {
    Aabb box;
    float3 c;
    uint32_t idx;
};
}  // namespace

void Bvh::build(std::vector<Tri> tris) {
    const size_t n = tris.size();
    std::vector<BuildPrim> prims(n);
    for (size_t i = 0; i < n; i++) {
        prims[i].box.grow(tris[i].v0);
        prims[i].box.grow(tris[i].v1);
        prims[i].box.grow(tris[i].v2);
        prims[i].c = (prims[i].box.lo + prims[i].box.hi) * 0.5f;
        prims[i].idx = (uint32_t)i;
    }
    nodes_.clear();
    nodes_.reserve(2 * n + 1);
    nodes_.push_back({});
    struct Job {
        int node;
        size_t begin, end;
    };
    std::vector<Job> stack{{0, 0, n}};
    const int kBins = 16;
    while (!stack.empty()) {
        Job job = stack.back();
        stack.pop_back();
        Aabb box, cbox;
        for (size_t i = job.begin; i < job.end; i++) {
            box.grow(prims[i].box);
            cbox.grow(prims[i].c);
        }
        Node &node = nodes_[job.node];
        for (int k = 0; k < 3; k++) {
            node.bmin[k] = box.lo[k];
            node.bmax[k] = box.hi[k];
        }
        size_t count = job.end - job.begin;
        int bestAxis = -1;
        float bestCost = FLT_MAX;
        int bestSplit = 0;
        if (count > 2) {
            for (int axis = 0; axis < 3; axis++) {
                float lo = cbox.lo[axis], hi = cbox.hi[axis];
                if (!(hi > lo)) continue;
                Aabb bins[kBins];
                int cnt[kBins] = {};
                float scale = kBins / (hi - lo);
                for (size_t i = job.begin; i < job.end; i++) {
                    int b = std::min(kBins - 1, (int)((prims[i].c[axis] - lo) * scale));
                    bins[b].grow(prims[i].box);
                    cnt[b]++;
                }
                float rightArea[kBins];
                int rightCnt[kBins];
                Aabb acc;
                int c = 0;
                for (int b = kBins - 1; b > 0; b--) {
                    acc.grow(bins[b]);
                    c += cnt[b];
                    rightArea[b] = acc.area();
                    rightCnt[b] = c;
                }
                Aabb lacc;
                int lc = 0;
                for (int b = 0; b < kBins - 1; b++) {
                    lacc.grow(bins[b]);
                    lc += cnt[b];
                    if (lc == 0 || rightCnt[b + 1] == 0) continue;
                    float cost = lacc.area() * lc + rightArea[b + 1] * rightCnt[b + 1];
                    if (cost < bestCost) {
                        bestCost = cost;
                        bestAxis = axis;
                        bestSplit = b;
                    }
                }
            }
        }
        const float leafCost = box.area() * (float)count;
        if (count <= 4 && (bestAxis < 0 || bestCost >= leafCost)) bestAxis = -1;
        if (count <= 1) bestAxis = -1;
        size_t mid = 0;
        if (bestAxis >= 0) {
            float lo = cbox.lo[bestAxis], hi = cbox.hi[bestAxis];
            float scale = kBins / (hi - lo);
            auto it = std::partition(prims.begin() + job.begin, prims.begin() + job.end, [&](const BuildPrim &p) {
                int b = std::min(kBins - 1, (int)((p.c[bestAxis] - lo) * scale));
                return b <= bestSplit;
            });
            mid = (size_t)(it - prims.begin());
            if (mid == job.begin || mid == job.end) bestAxis = -1;
        } else if (count > 4) {
            // degenerate centroids: split in the middle of the list
            bestAxis = 0;
            mid = job.begin + count / 2;
        }
        if (bestAxis < 0) {
            node.first = (int32_t)job.begin;
            node.count = (int32_t)count;
            continue;
        }
        int left = (int)nodes_.size();
        nodes_.push_back({});
        nodes_.push_back({});
        nodes_[job.node].first = left;
        nodes_[job.node].count = 0;
        stack.push_back({left, job.begin, mid});
        stack.push_back({left + 1, mid, job.end});
    }
    tris_.resize(n);
    for (size_t i = 0; i < n; i++) tris_[i] = tris[prims[i].idx];
}

// The closest-hit search culls boxes against the best distance found so far.
// A box's rounded near plane can lie beyond the rounded distance of a
// triangle on that plane: by a few ulps of the distance, and, for a triangle
// whose vertices lie far from the ray origin compared with the hit, by a few
// ulps of those vertex offsets.  A box holding a hit closer than the best one
// (a face coplanar with another, a box standing on the floor traced from the
// floor) would then be culled and the result would depend on the visiting
// order.  The bound is therefore widened by 2e-6 of the distance plus 1e-5
// of the box's largest offset from the origin, which leaves the closest hit
// that of an exhaustive search over every box the ray enters.
static inline bool slab(const float *bmin, const float *bmax, float3 org, float3 inv, float tmin, float tmax,
                        float &tnear) {
    float reach = 0.0f;
    for (int k = 0; k < 3; k++) reach = std::max(reach, std::max(std::fabs(bmin[k] - org[k]), std::fabs(bmax[k] - org[k])));
    float t0 = tmin, t1 = tmax * 1.000002f + 1e-5f * reach;
    for (int k = 0; k < 3; k++) {
        float a = (bmin[k] - org[k]) * inv[k];
        float b = (bmax[k] - org[k]) * inv[k];
        if (a > b) std::swap(a, b);
        if (a != a) a = -INFINITY;  // 0 * inf
        if (b != b) b = INFINITY;
        t0 = std::max(t0, a);
        t1 = std::min(t1, b * 1.0000004f);
    }
    tnear = t0;
    return t0 <= t1;
}

bool Bvh::intersect(float3 org, float3 dir, float tmin, float tmax, HitRecord &hit, bool exhaustive) const {
    if (nodes_.empty() || tris_.empty()) return false;
    WatertightRay wr(org, dir);
    float3 inv(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    float best = tmax;
    while (sp) {
        const Node &n = nodes_[stack[--sp]];
        float tn;
        if (!slab(n.bmin, n.bmax, org, inv, tmin, exhaustive ? INFINITY : best, tn)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const Tri &tr = tris_[n.first + i];
                float t, b0, b1;
                // equal distances go to the lower (instance, primitive), so the
                // result does not depend on the tree's visiting order
                if (intersectTriangle(wr, tr.v0, tr.v1, tr.v2, tmin, best, t, b0, b1) &&
                    (t < best || !found || tr.instance < hit.instance ||
                     (tr.instance == hit.instance && tr.prim < hit.prim))) {
                    best = t;
                    found = true;
                    hit.t = t;
                    hit.instance = tr.instance;
                    hit.prim = tr.prim;
                    hit.b0 = b0;
                    hit.b1 = b1;
                }
            }
        } else {
            const Node &l = nodes_[n.first], &r = nodes_[n.first + 1];
            float tl, tr;
            const float bound = exhaustive ? INFINITY : best;
            bool hl = slab(l.bmin, l.bmax, org, inv, tmin, bound, tl);
            bool hr = slab(r.bmin, r.bmax, org, inv, tmin, bound, tr);
            if (hl && hr) {
                if (tl <= tr) {
                    stack[sp++] = n.first + 1;
                    stack[sp++] = n.first;
                } else {
                    stack[sp++] = n.first;
                    stack[sp++] = n.first + 1;
                }
            } else if (hl) {
                stack[sp++] = n.first;
            } else if (hr) {
                stack[sp++] = n.first + 1;
            }
        }
    }
    return found;
}

bool Bvh::occluded(float3 org, float3 dir, float tmin, float tmax) const {
    if (nodes_.empty() || tris_.empty()) return false;
    WatertightRay wr(org, dir);
    float3 inv(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node &n = nodes_[stack[--sp]];
        float tn;
        if (!slab(n.bmin, n.bmax, org, inv, tmin, tmax, tn)) continue;
        if (n.count > 0) {
            for (int i = 0; i < n.count; i++) {
                const Tri &tr = tris_[n.first + i];
                float t, b0, b1;
                if (intersectTriangle(wr, tr.v0, tr.v1, tr.v2, tmin, tmax, t, b0, b1)) return true;
            }
        } else {
            stack[sp++] = n.first;
            stack[sp++] = n.first + 1;
        }
    }
    return false;
}

}  // namespace orc
