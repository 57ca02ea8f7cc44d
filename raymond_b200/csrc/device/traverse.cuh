// BVH traversal replacing Apple's closed `intersector<triangle_data,
// instancing>` (raymond/device/kernels/shading/raytrace.metal:11-85).
//
// Layout (built on the host, see bvh.cpp):
//   BvhNode, 64 B: both children's boxes in their parent (x/y of child 0,
//   x/y of child 1, z of both) and the two child links.  A link >= 0 is an
//   inner node; a link < 0 is a leaf ~(first << 3 | (count - 1)) into the
//   triangle array.
//   Triangles in leaf order, 48 B: world-space v0, v1, v2 (float4 each);
//   v0.w carries the instance index, v1.w the primitive index within the
//   instance's shape.
//
// Ray/triangle test: Woop, Benthin, Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1) 2013, evaluated with explicitly rounded products
// (no FMA contraction) so that shared edges stay watertight.  Hits report the
// reference's conventions: distance along the unit direction, barycentrics
// as (weight of v0, weight of v1), distance -1 on a miss.
#pragma once
#include "rt_math.cuh"

namespace rmd {

struct BvhNode {
    float4 c0xy;  // lo.x, hi.x, lo.y, hi.y of child 0
    float4 c1xy;  // same for child 1
    float4 cz;    // lo.z, hi.z of child 0, lo.z, hi.z of child 1
    int4 link;    // child 0, child 1, unused, unused
};

constexpr int TRAVERSAL_STACK = 64;
constexpr int STACK_SENTINEL = 0x7fffffff;

struct WatertightRay {
    int kx, ky, kz;
    float Sx, Sy, Sz;
    float3 org;
};

RMD_HD WatertightRay makeWatertight(float3 o, float3 d) {
    WatertightRay r;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz + 1 == 3 ? 0 : r.kz + 1;
    r.ky = r.kx + 1 == 3 ? 0 : r.kx + 1;
    if (comp(d, r.kz) < 0.0f) {
        const int t = r.kx;
        r.kx = r.ky;
        r.ky = t;
    }
    const float dz = comp(d, r.kz);
    r.Sx = __fdiv_rn(comp(d, r.kx), dz);
    r.Sy = __fdiv_rn(comp(d, r.ky), dz);
    r.Sz = __frcp_rn(dz);
    r.org = o;
    return r;
}

// Returns true with t in [tmin, tmax]; b0/b1 the weights of v0/v1.
RMD_HD bool intersectTriangle(const WatertightRay &r, float3 v0, float3 v1, float3 v2, float tmin, float tmax,
                              float &t, float &b0, float &b1) {
    const float3 A = make_float3(__fsub_rn(v0.x, r.org.x), __fsub_rn(v0.y, r.org.y), __fsub_rn(v0.z, r.org.z));
    const float3 B = make_float3(__fsub_rn(v1.x, r.org.x), __fsub_rn(v1.y, r.org.y), __fsub_rn(v1.z, r.org.z));
    const float3 C = make_float3(__fsub_rn(v2.x, r.org.x), __fsub_rn(v2.y, r.org.y), __fsub_rn(v2.z, r.org.z));
    const float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    const float Ax = __fsub_rn(comp(A, r.kx), __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(comp(A, r.ky), __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(comp(B, r.kx), __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(comp(B, r.ky), __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(comp(C, r.kx), __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(comp(C, r.ky), __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {  // edge: redo in double (WBW section 3.1)
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float Az = __fmul_rn(r.Sz, Akz);
    const float Bz = __fmul_rn(r.Sz, Bkz);
    const float Cz = __fmul_rn(r.Sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float rcpDet = __frcp_rn(det);
    t = __fmul_rn(T, rcpDet);
    if (!(t >= tmin && t <= tmax)) return false;
    b0 = __fmul_rn(U, rcpDet);
    b1 = __fmul_rn(V, rcpDet);
    return true;
}

struct TraceRay {
    float3 org, idir, oid;  // origin, 1/direction, origin/direction
    WatertightRay wr;
};

RMD_HD TraceRay makeTraceRay(float3 o, float3 d) {
    TraceRay r;
    const float ooeps = 8.271806125530277e-25f;  // 2^-80
    r.org = o;
    r.idir = make_float3(1.0f / (fabsf(d.x) > ooeps ? d.x : copysignf(ooeps, d.x)),
                         1.0f / (fabsf(d.y) > ooeps ? d.y : copysignf(ooeps, d.y)),
                         1.0f / (fabsf(d.z) > ooeps ? d.z : copysignf(ooeps, d.z)));
    r.oid = o * r.idir;
    r.wr = makeWatertight(o, d);
    return r;
}

// Slab tests of both children; returns entry distances (or > tmax on a miss).
RMD_HD void boxes(const BvhNode &n, const TraceRay &r, float tmin, float tmax, float &t0, float &t1, bool &h0,
                  bool &h1) {
    const float c0lox = n.c0xy.x * r.idir.x - r.oid.x, c0hix = n.c0xy.y * r.idir.x - r.oid.x;
    const float c0loy = n.c0xy.z * r.idir.y - r.oid.y, c0hiy = n.c0xy.w * r.idir.y - r.oid.y;
    const float c0loz = n.cz.x * r.idir.z - r.oid.z, c0hiz = n.cz.y * r.idir.z - r.oid.z;
    const float c1lox = n.c1xy.x * r.idir.x - r.oid.x, c1hix = n.c1xy.y * r.idir.x - r.oid.x;
    const float c1loy = n.c1xy.z * r.idir.y - r.oid.y, c1hiy = n.c1xy.w * r.idir.y - r.oid.y;
    const float c1loz = n.cz.z * r.idir.z - r.oid.z, c1hiz = n.cz.w * r.idir.z - r.oid.z;
    const float c0min = fmaxf(fmaxf(fminf(c0lox, c0hix), fminf(c0loy, c0hiy)), fmaxf(fminf(c0loz, c0hiz), tmin));
    const float c0max = fminf(fminf(fmaxf(c0lox, c0hix), fmaxf(c0loy, c0hiy)), fminf(fmaxf(c0loz, c0hiz), tmax));
    const float c1min = fmaxf(fmaxf(fminf(c1lox, c1hix), fminf(c1loy, c1hiy)), fmaxf(fminf(c1loz, c1hiz), tmin));
    const float c1max = fminf(fminf(fmaxf(c1lox, c1hix), fmaxf(c1loy, c1hiy)), fminf(fmaxf(c1loz, c1hiz), tmax));
    // widen the far bound by a few ulps (Ize 2013) so FMA rounding never culls a hit
    h0 = c0min <= c0max * 1.0000004f;
    h1 = c1min <= c1max * 1.0000004f;
    t0 = c0min;
    t1 = c1min;
}

// Traversal state of one ray.
struct TraversalState {
    TraceRay r;
    float tmin, tmax;  // tmax shrinks to the closest hit found so far
    int node;          // next node (>= 0), leaf (< 0), or STACK_SENTINEL once finished
    int sp;
    int hitTri;        // closest (any-hit: first) triangle hit, -1 if none
    float b0, b1;
};
// The node stack is a separate local array, so the scalar state above stays in registers.
typedef int TraversalStack[TRAVERSAL_STACK];

RMD_HD void beginTraversal(TraversalState &s, TraversalStack &stack, const BvhNode *nodes, float3 o, float3 d,
                           float tmin, float tmax) {
    s.r = makeTraceRay(o, d);
    s.tmin = tmin;
    s.tmax = tmax;
    s.sp = 0;
    stack[s.sp++] = STACK_SENTINEL;
    s.node = nodes != nullptr ? 0 : STACK_SENTINEL;  // a scene without triangles misses everything
    s.hitTri = -1;
    s.b0 = s.b1 = 0.0f;
}

// Depth-first traversal, one node or one leaf per step, nearer child first;
// a leaf is intersected as soon as it is reached so the closest hit found so
// far culls the rest.  ANY: stop at the first hit (raytrace.metal:52-85);
// otherwise keep the closest (raytrace.metal:11-50).  (The while-while loop
// and dynamic ray fetch of Aila & Laine, HPG 2009, both measured slower here:
// warp-vote instructions inside the loop cost more than they recover.)
template <bool ANY>
RMD_HD void traverse(TraversalState &s, TraversalStack &stack, const BvhNode *__restrict__ nodes,
                     const float4 *__restrict__ tris, uint32_t *errors) {
    while (s.node != STACK_SENTINEL) {
        if (s.node >= 0) {
            const BvhNode *np = &nodes[s.node];
            const BvhNode n = {__ldg(&np->c0xy), __ldg(&np->c1xy), __ldg(&np->cz), __ldg(&np->link)};
            float t0, t1;
            bool h0, h1;
            boxes(n, s.r, s.tmin, s.tmax, t0, t1, h0, h1);
            if (h0 && h1) {
                int nearN = n.link.x, farN = n.link.y;
                if (t1 < t0) {
                    nearN = n.link.y;
                    farN = n.link.x;
                }
                if (s.sp < TRAVERSAL_STACK) stack[s.sp++] = farN;
                else atomicOr(errors, 2u);
                s.node = nearN;
            } else if (h0) {
                s.node = n.link.x;
            } else if (h1) {
                s.node = n.link.y;
            } else {
                s.node = stack[--s.sp];
            }
        } else {
            const int code = ~s.node;
            const int first = code >> 3, count = (code & 7) + 1;
            bool found = false;
            for (int i = 0; i < count; i++) {
                const int ti = first + i;
                const float4 a = __ldg(&tris[3 * ti + 0]);
                const float4 b = __ldg(&tris[3 * ti + 1]);
                const float4 c = __ldg(&tris[3 * ti + 2]);
                float t, b0, b1;
                if (intersectTriangle(s.r.wr, xyz(a), xyz(b), xyz(c), s.tmin, s.tmax, t, b0, b1)) {
                    s.hitTri = ti;
                    if (ANY) {
                        found = true;
                        break;
                    }
                    s.tmax = t;
                    s.b0 = b0;
                    s.b1 = b1;
                }
            }
            s.node = (ANY && found) ? STACK_SENTINEL : stack[--s.sp];
        }
    }
}

// Closest-hit record of a finished traversal: hit = (t, b0, b1, primitive
// bits), inst = instance; t = -1 and inst = ~0 on a miss.
RMD_HD bool closestHit(const TraversalState &s, const float4 *__restrict__ tris, float4 &hit, uint32_t &inst) {
    if (s.hitTri < 0) {
        hit = make_float4(-1.0f, 0.0f, 0.0f, 0.0f);
        inst = 0xffffffffu;
        return false;
    }
    const float4 a = __ldg(&tris[3 * s.hitTri + 0]);
    const float4 b = __ldg(&tris[3 * s.hitTri + 1]);
    hit = make_float4(s.tmax, s.b0, s.b1, b.w);
    inst = __float_as_uint(a.w);
    return true;
}

// Single-ray forms of the two queries (test hooks).
RMD_HD bool traceClosest(const BvhNode *__restrict__ nodes, const float4 *__restrict__ tris, float3 o, float3 d,
                         float tmin, float tmax, float4 &hit, uint32_t &inst, uint32_t *errors) {
    TraversalState s;
    TraversalStack stack;
    beginTraversal(s, stack, nodes, o, d, tmin, tmax);
    traverse<false>(s, stack, nodes, tris, errors);
    return closestHit(s, tris, hit, inst);
}
RMD_HD bool traceAny(const BvhNode *__restrict__ nodes, const float4 *__restrict__ tris, float3 o, float3 d,
                     float tmin, float tmax, uint32_t *errors) {
    TraversalState s;
    TraversalStack stack;
    beginTraversal(s, stack, nodes, o, d, tmin, tmax);
    traverse<true>(s, stack, nodes, tris, errors);
    return s.hitTri >= 0;
}

}  // namespace rmd
