// BVH traversal replacing Apple's closed `intersector<triangle_data,
// instancing>` (raymond/device/kernels/shading/raytrace.metal:11-85).
//
// Layout (built on the host, bvh_build.cpp): a compressed 8-wide BVH after
// Ylitie, Karras and Laine, "Efficient incoherent ray traversal on GPUs
// through compressed wide BVHs" (HPG 2017).  A node is 80 bytes: its origin
// and per-axis power-of-two scale, a mask of inner-node slots, the index of
// its first inner child (inner children are consecutive) and of its first
// triangle (leaf children's triangles are consecutive, at most 3 per leaf and
// 24 per node), one meta byte per leaf slot (unary triangle count << 5 |
// offset), and the child boxes quantised to 8 bits per plane.
//   Triangles in leaf order, three copies of each side by side (144 B):
//   copy k holds v0, v1, v2 (float4 each) with the coordinates rotated so
//   that axis k comes last, (v[k+1], v[k+2], v[k]); copy 2 is (x, y, z).
//   v0.w carries the instance index, v1.w the primitive index within the
//   instance's shape.  A ray reads the copy of its dominant axis, so the
//   watertight test needs no per-triangle selection of components.
//
// Ray/triangle test: Woop, Benthin, Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1) 2013, evaluated with explicitly rounded products
// (no FMA contraction) so that shared edges stay watertight.  Hits report the
// reference's conventions: distance along the unit direction, barycentrics
// as (weight of v0, weight of v1), distance -1 on a miss.
#pragma once
#include "rt_math.cuh"

namespace rmd {

struct WideNode {
    float4 originScale;  // origin.xyz; w bits: exponent x, y, z (bytes 0-2), inner-slot mask (byte 3)
    uint4 bases;         // first inner child, first triangle, meta bytes of slots 0-3, 4-7
    uint4 qloXY;         // quantised lower bounds: x slots 0-3, 4-7; y slots 0-3, 4-7
    uint4 qloZqhiX;      // lower z; upper x
    uint4 qhiYZ;         // upper y; upper z
};

constexpr int TRAVERSAL_STACK = 32;  // node groups; one per level of the 8-wide tree at most

constexpr int TRI_FLOAT4 = 9;  // float4 per triangle: three rotated copies of its three vertices

// The ray in the frame of the triangle copy it reads: kz is its dominant
// axis, kx = kz + 1 and ky = kz + 2 (mod 3).  WBW swap kx and ky when d[kz]
// is negative to keep the winding; that only negates U, V, W, the
// determinant and T, which leaves t and the barycentrics unchanged bit for
// bit (rounding is symmetric), so the rotation alone is used.
struct WatertightRay {
    int kz;
    float Sx, Sy, Sz;
    float3 org;  // (o[kx], o[ky], o[kz])
};

RMD_HD WatertightRay makeWatertight(float3 o, float3 d) {
    WatertightRay r;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    const int kx = r.kz + 1 == 3 ? 0 : r.kz + 1;
    const int ky = kx + 1 == 3 ? 0 : kx + 1;
    const float dz = comp(d, r.kz);
    r.Sx = __fdiv_rn(comp(d, kx), dz);
    r.Sy = __fdiv_rn(comp(d, ky), dz);
    r.Sz = __frcp_rn(dz);
    r.org = make_float3(comp(o, kx), comp(o, ky), comp(o, r.kz));
    return r;
}

// Returns true with t in [tmin, tmax]; b0/b1 the weights of v0/v1.  The
// vertices are the ray's copy: (v[kx], v[ky], v[kz]).
RMD_HD bool intersectTriangle(const WatertightRay &r, float3 v0, float3 v1, float3 v2, float tmin, float tmax,
                              float &t, float &b0, float &b1) {
    const float3 A = make_float3(__fsub_rn(v0.x, r.org.x), __fsub_rn(v0.y, r.org.y), __fsub_rn(v0.z, r.org.z));
    const float3 B = make_float3(__fsub_rn(v1.x, r.org.x), __fsub_rn(v1.y, r.org.y), __fsub_rn(v1.z, r.org.z));
    const float3 C = make_float3(__fsub_rn(v2.x, r.org.x), __fsub_rn(v2.y, r.org.y), __fsub_rn(v2.z, r.org.z));
    const float Akz = A.z, Bkz = B.z, Ckz = C.z;
    const float Ax = __fsub_rn(A.x, __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(A.y, __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(B.x, __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(B.y, __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(C.x, __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(C.y, __fmul_rn(r.Sy, Ckz));
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

// Byte q = byte i of w as the float 256 + q / 128, exactly: one byte permute
// puts q in the mantissa of 256.  A plane at q quanta from the node origin
// then lies at t = (256 + q / 128) * (128 a) + (b - 32768 a), one multiply-add
// per plane with no conversion of q.
RMD_HD float bytePlane(uint32_t w, uint32_t i) {
    return __uint_as_float(__byte_perm(w, 0x43800000u, 0x7604u | (i << 4)));
}

// Ray/box tests of a node's 8 children.  Returns the children the ray enters
// within [tmin, tmax]: inner children as bits 24 + (slot ^ octant) (so the
// lowest bit is the nearest child in the node's octant order), leaf
// children's triangles as bits (offset .. offset + count - 1).
RMD_HD uint32_t intersectChildren(const WideNode &n, const float3 idir, const float3 org, uint32_t octant,
                                  float tmin, float tmax) {
    const uint32_t ew = __float_as_uint(n.originScale.w);
    const float sx = __uint_as_float((ew & 0xffu) << 23);
    const float sy = __uint_as_float(((ew >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((ew >> 16) & 0xffu) << 23);
    const uint32_t imask = ew >> 24;
    const float ax = sx * idir.x, ay = sy * idir.y, az = sz * idir.z;  // one quantum in t: exact, powers of two
    const float bx = (n.originScale.x - org.x) * idir.x;
    const float by = (n.originScale.y - org.y) * idir.y;
    const float bz = (n.originScale.z - org.z) * idir.z;
    // origin - org and its product with the rounded 1/d each round once, an
    // absolute error of at most 2^-23 |b| in every plane distance, which a
    // relative widening cannot cover when the hit lies close to the origin
    // next to a far node origin; b +- w and b - 32768 a round once more each
    // (2^-24 |b| + 2^-9 a).  Near planes therefore move down and far planes
    // up by w = 4e-7 |b| + a / 128 (per axis, so an axis the ray runs
    // parallel to stays decided).  (128 a) * (256 + q / 128) is exact.
    const float wx = fmaf(4.0e-7f, fabsf(bx), 0.0078125f * fabsf(ax));
    const float wy = fmaf(4.0e-7f, fabsf(by), 0.0078125f * fabsf(ay));
    const float wz = fmaf(4.0e-7f, fabsf(bz), 0.0078125f * fabsf(az));
    const float bxN = fmaf(-32768.0f, ax, bx - wx), bxF = fmaf(-32768.0f, ax, bx + wx);
    const float byN = fmaf(-32768.0f, ay, by - wy), byF = fmaf(-32768.0f, ay, by + wy);
    const float bzN = fmaf(-32768.0f, az, bz - wz), bzF = fmaf(-32768.0f, az, bz + wz);
    const float Ax = 128.0f * ax, Ay = 128.0f * ay, Az = 128.0f * az;
    // per axis the near plane is the lower bound for a positive direction
    const uint2 loX = make_uint2(n.qloXY.x, n.qloXY.y), hiX = make_uint2(n.qloZqhiX.z, n.qloZqhiX.w);
    const uint2 loY = make_uint2(n.qloXY.z, n.qloXY.w), hiY = make_uint2(n.qhiYZ.x, n.qhiYZ.y);
    const uint2 loZ = make_uint2(n.qloZqhiX.x, n.qloZqhiX.y), hiZ = make_uint2(n.qhiYZ.z, n.qhiYZ.w);
    const bool nx = idir.x < 0.0f, ny = idir.y < 0.0f, nz = idir.z < 0.0f;
    const uint2 nearX = nx ? hiX : loX, farX = nx ? loX : hiX;
    const uint2 nearY = ny ? hiY : loY, farY = ny ? loY : hiY;
    const uint2 nearZ = nz ? hiZ : loZ, farZ = nz ? loZ : hiZ;
    uint32_t hits = 0;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const uint32_t nxw = half ? nearX.y : nearX.x, fxw = half ? farX.y : farX.x;
        const uint32_t nyw = half ? nearY.y : nearY.x, fyw = half ? farY.y : farY.x;
        const uint32_t nzw = half ? nearZ.y : nearZ.x, fzw = half ? farZ.y : farZ.x;
        const uint32_t metaw = half ? n.bases.w : n.bases.z;
#pragma unroll
        for (uint32_t i = 0; i < 4; i++) {
            const uint32_t slot = 4 * half + i;
            const float t0x = fmaf(bytePlane(nxw, i), Ax, bxN), t1x = fmaf(bytePlane(fxw, i), Ax, bxF);
            const float t0y = fmaf(bytePlane(nyw, i), Ay, byN), t1y = fmaf(bytePlane(fyw, i), Ay, byF);
            const float t0z = fmaf(bytePlane(nzw, i), Az, bzN), t1z = fmaf(bytePlane(fzw, i), Az, bzF);
            const float enter = fmaxf(fmaxf(t0x, t0y), fmaxf(t0z, tmin));
            const float leave = fminf(fminf(t1x, t1y), fminf(t1z, tmax));
            // widen the far bound by a few ulps (Ize 2013) so FMA rounding never culls a hit
            if (enter <= leave * 1.0000004f) {
                if ((imask >> slot) & 1u) {
                    hits |= 1u << (24u + (slot ^ octant));
                } else {
                    const uint32_t meta = (metaw >> (8 * i)) & 0xffu;
                    hits |= (meta >> 5) << (meta & 31u);
                }
            }
        }
    }
    return hits;
}

// Traversal state of one ray: `group` and the stack hold where the traversal
// stands (sp < 0 once finished).
struct TraversalState {
    TraceRay r;
    float tmin, tmax;  // tmax shrinks to the closest hit found so far
    float slack;       // absolute widening of tmax when boxes are culled against it
    int hitTri;        // closest (any-hit: first) triangle hit, -1 if none
    uint32_t hitInst, hitPrim;  // its instance and primitive (the tie-break key)
    float b0, b1;
    uint2 group;       // node group being visited
    int sp;            // stack depth, -1 when finished
};
// Node groups waiting to be visited: a separate local array, so the scalar
// state above stays in registers.
typedef uint2 TraversalStack[TRAVERSAL_STACK];

RMD_HD uint32_t rayOctant(float3 idir) {
    return (idir.x < 0.0f ? 1u : 0u) | (idir.y < 0.0f ? 2u : 0u) | (idir.z < 0.0f ? 4u : 0u);
}

RMD_HD void beginTraversal(TraversalState &s, const WideNode *nodes, float3 o, float3 d, float tmin, float tmax) {
    s.r = makeTraceRay(o, d);
    s.tmin = tmin;
    s.tmax = tmax;
    s.hitTri = -1;
    s.hitInst = s.hitPrim = 0xffffffffu;
    s.b0 = s.b1 = 0.0f;
    // A box's rounded near plane can lie beyond the rounded distance of a
    // triangle on that plane: by a few ulps of the distance, and, for a
    // triangle whose vertices lie far from the origin compared with the hit,
    // by a few ulps of those offsets.  Boxes are therefore culled against
    // tmax widened by 2e-6 of it plus 1e-5 of the scene's largest offset from
    // the origin (the root's quantisation frame), so a box holding a hit
    // closer than the best so far (a face coplanar with another, a box on the
    // floor traced from the floor) is never culled, and the closest hit is
    // that of an exhaustive search, whatever the tree.
    s.slack = 0.0f;
    if (nodes != nullptr) {
        const float4 os = __ldg(&nodes[0].originScale);
        const uint32_t ew = __float_as_uint(os.w);
        const float ex = 255.0f * __uint_as_float((ew & 0xffu) << 23);
        const float ey = 255.0f * __uint_as_float(((ew >> 8) & 0xffu) << 23);
        const float ez = 255.0f * __uint_as_float(((ew >> 16) & 0xffu) << 23);
        const float ox = os.x - o.x, oy = os.y - o.y, oz = os.z - o.z;
        const float reach = fmaxf(fmaxf(fmaxf(fabsf(ox), fabsf(ox + ex)), fmaxf(fabsf(oy), fabsf(oy + ey))),
                                  fmaxf(fabsf(oz), fabsf(oz + ez)));
        s.slack = 1e-5f * reach;
    }
    // a virtual parent whose only inner child, in slot 0, is the root
    s.group = make_uint2(0u, (1u << (24u + rayOctant(s.r.idir))) | 1u);
    s.sp = nodes != nullptr ? 0 : -1;  // a scene without triangles misses everything
}

// Depth-first traversal of the 8-wide BVH.  A node group (first inner child,
// bits 24..31: inner children still to visit in octant order, bits 0..7: the
// node's inner-slot mask) is visited nearest child first; the rest of the
// group waits on the stack.  The triangles a node's leaf children hit are
// intersected as soon as the node is visited, so the closest hit found so far
// culls what follows.  ANY: stop at the first hit (raytrace.metal:52-85);
// otherwise keep the closest (raytrace.metal:11-50).
//
// One call visits one node (and its triangles) and returns true once the
// traversal has finished, so a persistent warp can hand a finished lane a new
// ray between two steps.
template <bool ANY>
RMD_HD bool traverseStep(TraversalState &s, TraversalStack &stack, const WideNode *__restrict__ nodes,
                         const float4 *__restrict__ tris, uint32_t *errors) {
    if (s.sp < 0) return true;
    const float3 idir = s.r.idir, org = s.r.org;
    const uint32_t octant = rayOctant(idir);
    uint2 group = s.group;
    int sp = s.sp;
    if (group.y > 0x00ffffffu) {
        const uint32_t key = __ffs(group.y >> 24) - 1;
        group.y &= ~(1u << (24u + key));
        const uint32_t slot = key ^ octant;
        const uint32_t index = group.x + __popc(group.y & ((1u << slot) - 1u) & 0xffu);
        if (group.y > 0x00ffffffu) {
            if (sp < TRAVERSAL_STACK) stack[sp++] = group;
            else atomicOr(errors, 2u);
        }
        const WideNode *np = &nodes[index];
        const WideNode n = {__ldg(&np->originScale), __ldg(&np->bases), __ldg(&np->qloXY),
                            __ldg(&np->qloZqhiX), __ldg(&np->qhiYZ)};
        const uint32_t hits = intersectChildren(n, idir, org, octant, s.tmin, fmaf(s.tmax, 1.000002f, s.slack));
        group = make_uint2(n.bases.x, (hits & 0xff000000u) | (__float_as_uint(n.originScale.w) >> 24));
        uint32_t triHits = hits & 0x00ffffffu;
        while (triHits) {
            const int ti = (int)n.bases.y + __ffs(triHits) - 1;
            triHits &= triHits - 1u;
            const float4 *tv = &tris[TRI_FLOAT4 * (size_t)ti + 3 * s.r.wr.kz];  // the ray's copy
            const float4 a = __ldg(&tv[0]);
            const float4 b = __ldg(&tv[1]);
            const float4 c = __ldg(&tv[2]);
            float t, b0, b1;
            if (intersectTriangle(s.r.wr, xyz(a), xyz(b), xyz(c), s.tmin, s.tmax, t, b0, b1)) {
                if (ANY) {
                    s.hitTri = ti;
                    s.sp = -1;
                    return true;
                }
                // Equal distances (coplanar overlapping faces) go to the lower
                // (instance, primitive), whatever order the tree is visited in,
                // so every BVH of the scene reports the same closest hit.
                const uint32_t inst = __float_as_uint(a.w), prim = __float_as_uint(b.w);
                if (t < s.tmax || s.hitTri < 0 || inst < s.hitInst || (inst == s.hitInst && prim < s.hitPrim)) {
                    s.hitTri = ti;
                    s.hitInst = inst;
                    s.hitPrim = prim;
                    s.tmax = t;
                    s.b0 = b0;
                    s.b1 = b1;
                }
            }
        }
    }
    if (group.y <= 0x00ffffffu) {
        if (sp == 0) {
            s.sp = -1;
            return true;
        }
        group = stack[--sp];
    }
    s.group = group;
    s.sp = sp;
    return false;
}

// The whole traversal of one ray.
template <bool ANY>
RMD_HD void traverse(TraversalState &s, TraversalStack &stack, const WideNode *__restrict__ nodes,
                     const float4 *__restrict__ tris, uint32_t *errors) {
    while (!traverseStep<ANY>(s, stack, nodes, tris, errors)) {
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
    const float4 a = __ldg(&tris[TRI_FLOAT4 * (size_t)s.hitTri + 6]);  // copy 2: the instance and primitive
    const float4 b = __ldg(&tris[TRI_FLOAT4 * (size_t)s.hitTri + 7]);
    hit = make_float4(s.tmax, s.b0, s.b1, b.w);
    inst = __float_as_uint(a.w);
    return true;
}

// Single-ray forms of the two queries (test hooks).
RMD_HD bool traceClosest(const WideNode *__restrict__ nodes, const float4 *__restrict__ tris, float3 o, float3 d,
                         float tmin, float tmax, float4 &hit, uint32_t &inst, uint32_t *errors) {
    TraversalState s;
    TraversalStack stack;
    beginTraversal(s, nodes, o, d, tmin, tmax);
    traverse<false>(s, stack, nodes, tris, errors);
    return closestHit(s, tris, hit, inst);
}
RMD_HD bool traceAny(const WideNode *__restrict__ nodes, const float4 *__restrict__ tris, float3 o, float3 d,
                     float tmin, float tmax, uint32_t *errors) {
    TraversalState s;
    TraversalStack stack;
    beginTraversal(s, nodes, o, d, tmin, tmax);
    traverse<true>(s, stack, nodes, tris, errors);
    return s.hitTri >= 0;
}

}  // namespace rmd
