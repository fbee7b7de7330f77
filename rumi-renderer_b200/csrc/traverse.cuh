// Closest-hit and any-hit traversal over the 32-byte-node BVH.
//
// Primitive tests restate the reference's Shape::Intersect routines operation by
// operation with correctly rounded intrinsics (no FMA contraction), so accept/reject
// decisions and hit distances equal the reference's x86 float arithmetic:
//   Triangle::Intersect  src/Shape/triangle.cpp:41-118
//   Rect::Intersect      src/Shape/rect.cpp:51-122
//   Sphere::Intersect    src/Shape/sphere.cpp:51-132 (+ SolveQuadratic src/Kernel/clibrary.h:62-87)
// The running closest distance plays the role of Ray::_tmin (0 = nothing hit yet), with
// the same tie rule: an equal t replaces the previous hit.
//
// Traversal: both children of an interior node are adjacent (one 64-byte pair, four
// float4 loads); leaf children are intersected at once, interior children are visited
// near-first with the far one pushed.  The stack keeps its top STACK_SMEM entries in
// shared memory (one column per thread) and spills deeper entries to a local array.
#pragma once
#include <cfloat>
#include "scene.cuh"

#define RUMI_MAX_BVH_DEPTH 64

// 1: the default walk (trace_mode 0, ray queries, batches, per-thread rays) is the
// compressed eight-wide tree; 0: the binary (or, with RUMI_BVH_WIDE, four-wide) tree.
#ifndef RUMI_WALK8
#define RUMI_WALK8 0
#endif

struct HitRec {
    float t;      // 0 = miss
    int id;       // canonical primitive id, -1 = miss
    float u, v;   // triangle barycentrics (reference naming)
    int back;     // triangle determinant < 0
};

// ---------------------------------------------------------------- primitive tests
RUMI_D bool isect_triangle(float3 o, float3 d, float tmax, float tbest, float4 A, float4 B, float4 C, float &t_out,
                           float &u_out, float &v_out, int &back) {
    const float3 v0 = f4xyz(A), e1 = f4xyz(B), e2 = f4xyz(C);
    const float3 P = rn_cross(d, e2);
    const float det = rn_dot(P, e1);
    if (-1e-8f < det && det < 1e-8f) return false;
    const float inv_det = __frcp_rn(det);
    const float3 T = rn_sub(o, v0);
    const float u = __fmul_rn(rn_dot(P, T), inv_det);
    if (u < 0.0f || u > 1.0f) return false;
    const float3 Q = rn_cross(T, e1);
    const float v = __fmul_rn(rn_dot(Q, d), inv_det);
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
    const float t = __fmul_rn(rn_dot(Q, e2), inv_det);
    if (t < RUMI_EPS) return false;
    if (tbest > RUMI_EPS && t > tbest) return false;
    if (__fsub_rn(tmax, t) < RUMI_EPS) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    back = det < 0.0f;
    return true;
}

// Rect geometry derived exactly as the Rect constructor does (src/Shape/rect.cpp:12-20).
struct RectGeom {
    float3 n;
    float length, width, inv_area;
};
RUMI_D RectGeom rect_geom(float3 l, float3 w) {
    RectGeom g;
    g.n = normalize_ref(rn_cross(l, w));
    g.length = __fsqrt_rn(rn_dot(l, l));
    g.width = __fsqrt_rn(rn_dot(w, w));
    g.inv_area = __frcp_rn(__fmul_rn(g.length, g.width));
    return g;
}

RUMI_D bool isect_rect(float3 o, float3 d, float tmax, float tbest, float4 A, float4 B, float4 C, bool emissive,
                       float &t_out) {
    const float3 p = f4xyz(A), l = f4xyz(B), w = f4xyz(C);
    const RectGeom g = rect_geom(l, w);
    const float cost = rn_dot(d, g.n);
    if (cost == 0.0f) return false;
    const float t = __fdiv_rn(-rn_dot(rn_sub(o, p), g.n), cost);
    if (t < 0.0f) return false;
    if (t < RUMI_EPS) return false;
    if (__fsub_rn(tmax, t) < RUMI_EPS) return false;
    if (!emissive && (0.0f < cost && cost < 1.0f)) return false;  // one-sided unless emissive
    if (t > tbest && tbest > 0.0f) return false;
    const float3 ip = rn_madd(o, d, t);
    const float3 on = rn_sub(ip, p);
    const float il = __fmul_rn(rn_dot(on, l), __fmul_rn(g.inv_area, g.width));
    if (il < 0.0f || il > g.length) return false;
    const float iw = __fmul_rn(rn_dot(on, w), __fmul_rn(g.inv_area, g.length));
    if (iw < 0.0f || iw > g.width) return false;
    t_out = t;
    return true;
}

RUMI_D bool isect_sphere(float3 o, float3 d, float tmax, float tbest, float4 A, float4 B, bool in_object, bool ibl,
                         float &t_out) {
    const float3 c = f4xyz(A);
    const float r = B.x;
    const float3 roc = rn_sub(o, c);
    const float Bq = __fmul_rn(2.0f, rn_dot(d, roc));
    const float Cq = __fsub_rn(rn_dot(roc, roc), __fmul_rn(r, r));
    const float disc = __fsub_rn(__fmul_rn(Bq, Bq), __fmul_rn(4.0f, Cq));
    if (disc < 0.0f) return false;
    float t0, t1;
    if (disc == 0.0f) {
        t0 = t1 = __fmul_rn(-Bq, 0.5f);
    } else {
        const float sq = __fsqrt_rn(disc);
        t0 = __fmul_rn(__fsub_rn(-Bq, sq), 0.5f);
        t1 = __fmul_rn(__fadd_rn(-Bq, sq), 0.5f);
    }
    if (t0 < 0.0f && t1 < 0.0f) return false;
    if (in_object) {
        float tmp = t0; t0 = t1; t1 = tmp;
    }
    if (ibl && __fsqrt_rn(rn_dot(roc, roc)) < r) {  // inside an image-based light's sphere
        float tmp = t0; t0 = t1; t1 = tmp;
    }
    if (t0 < RUMI_EPS) return false;
    if (__fsub_rn(tmax, t0) < RUMI_EPS) return false;
    if (t0 > tbest && tbest > 0.0f) return false;
    t_out = t0;
    return true;
}

// ---------------------------------------------------------------------- node test
// Reciprocal direction for the node slabs.  A zero component would give an infinite
// reciprocal, (lo - o) * inf = NaN slab ends and -- since fminf/fmaxf drop NaNs -- no
// culling on that axis: an axis-aligned ray would visit most of the tree.  Zero (and
// tiny) components are replaced by 2^-80 with their sign, which keeps every slab finite
// and the test conservative (the ray drifts by < 1e-23 per unit length on that axis).
RUMI_D float safe_rcp(float x) {
    const float eps = 8.2718061e-25f;  // 2^-80
    return 1.0f / (fabsf(x) > eps ? x : copysignf(eps, x));
}
RUMI_D float3 safe_inv(float3 d) { return mk3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z)); }

RUMI_D bool slab(float4 a, float4 b, float3 inv, float3 oinv, float tlimit, float &tnear) {
    // t = lo * inv - o * inv; conservative for zero direction components (NaN lanes are
    // dropped by fminf/fmaxf).
    const float tx0 = fmaf(a.x, inv.x, -oinv.x), tx1 = fmaf(a.w, inv.x, -oinv.x);
    const float ty0 = fmaf(a.y, inv.y, -oinv.y), ty1 = fmaf(b.x, inv.y, -oinv.y);
    const float tz0 = fmaf(a.z, inv.z, -oinv.z), tz1 = fmaf(b.y, inv.z, -oinv.z);
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    tnear = tn;
    return tn <= tf && tf >= 0.0f && tn <= tlimit;
}

// Node culling limit from the best hit so far.  Primitives at exactly the best distance
// (coplanar neighbours meeting at an edge) are all reached whatever order the leaves are
// tested in: the limit sits a relative 2^-16 above the best distance, above the rounding
// of the slab distances, and leaf_isect gives a tie to the larger primitive id (the one an
// exhaustive scan in canonical order reports last).  The speculative walk tests leaves in
// an order that depends on the rays sharing the warp, so without this a tie could go
// either way from run to run.
RUMI_D float cull_limit(float best_t, float tmax) {
    return best_t > 0.0f ? fminf(fmaf(fmaxf(best_t, 1.0f), 1.52587890625e-05f, best_t), tmax) : tmax;
}

struct TraceStats {
    int nodes;   // node bytes fetched, in 16-byte units (a binary node is 2, an eight-wide node 5)
    int prims;   // primitives tested
};

// Intersects every primitive of one leaf (records prims[3*first ...]: the binary tree's
// leaf_prims or the eight-wide tree's prims8).  Returns true when ANYHIT and a hit was found.
template <bool ANYHIT, bool STATS>
RUMI_D bool leaf_isect_in(const DevScene &s, const float4 *__restrict__ prims, int first, int count, float3 o,
                          float3 d, float tmax, bool in_object, HitRec &h, TraceStats &st) {
    if (first < 0 || count > s.n_prims - first) return false;  // malformed leaf guard
    for (int i = first; i < first + count; ++i) {
        const float4 A = __ldg(&prims[3 * i + 0]);
        const float4 B = __ldg(&prims[3 * i + 1]);
        const float4 C = __ldg(&prims[3 * i + 2]);
        if (STATS) st.prims++;
        const int tag = __float_as_int(B.w);
        const int kind = tag & 0xff;
        float t, u = 0.0f, v = 0.0f;
        int back = 0;
        bool ok;
        if (kind == PRIM_TRI)
            ok = isect_triangle(o, d, tmax, h.t, A, B, C, t, u, v, back);
        else if (kind == PRIM_RECT)
            ok = isect_rect(o, d, tmax, h.t, A, B, C, (tag & PRIM_FLAG_EMISSIVE) != 0, t);
        else
            ok = isect_sphere(o, d, tmax, h.t, A, B, in_object && !ANYHIT, (tag & PRIM_FLAG_IBL) != 0, t);
        if (ok && t == h.t && __float_as_int(A.w) < h.id) ok = false;  // a tie: the larger id stays
        if (ok) {
            h.t = t;
            h.id = __float_as_int(A.w);
            h.u = u;
            h.v = v;
            h.back = back;
        }
    }
    return ANYHIT && h.t > 0.0f;
}

template <bool ANYHIT, bool STATS>
RUMI_D bool leaf_isect(const DevScene &s, int first, int count, float3 o, float3 d, float tmax, bool in_object,
                       HitRec &h, TraceStats &st) {
    return leaf_isect_in<ANYHIT, STATS>(s, s.leaf_prims, first, count, o, d, tmax, in_object, h, st);
}

// Closest-hit (ANYHIT=false) or occlusion (ANYHIT=true) query over the binary tree.
// smem_stack: this thread's first shared-memory stack slot; consecutive slots are
// `stride` ints apart.
template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D HitRec trace_ray_bin(const DevScene &s, float3 o, float3 d, float tmax, bool in_object, int *smem_stack,
                            int stride, TraceStats &st) {
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) return h;  // bvh.cpp:161-162
    const float3 inv = safe_inv(d);
    const float3 oinv = mk3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    int spill[RUMI_MAX_BVH_DEPTH - STACK_SMEM > 0 ? RUMI_MAX_BVH_DEPTH - STACK_SMEM : 1];
    int sp = 0;

    // root
    {
        const float4 *rp = reinterpret_cast<const float4 *>(s.nodes);
        const float4 a = __ldg(rp), b = __ldg(rp + 1);
        if (STATS) st.nodes += 2;
        float tn;
        if (!slab(a, b, inv, oinv, tmax, tn)) return h;
        const int first = __float_as_int(b.z), count = __float_as_int(b.w);
        if (count > 0) {
            leaf_isect<ANYHIT, STATS>(s, first, count, o, d, tmax, in_object, h, st);
            return h;
        }
        // fall through with the root's children pair
        int cur = first;
        if ((unsigned)cur >= (unsigned)(s.n_nodes - 1)) return h;
        // every node pair is visited at most once per ray, so the bound is never reached
        // by a well-formed tree; it keeps a malformed one from looping
        for (int guard = 0; guard < s.n_nodes; ++guard) {
            const float4 *np = reinterpret_cast<const float4 *>(s.nodes + cur);
            const float4 a0 = __ldg(np + 0), b0 = __ldg(np + 1), a1 = __ldg(np + 2), b1 = __ldg(np + 3);
            if (STATS) st.nodes += 4;
            const float lim = cull_limit(h.t, tmax);
            float tn0, tn1;
            bool h0 = slab(a0, b0, inv, oinv, lim, tn0);
            bool h1 = slab(a1, b1, inv, oinv, lim, tn1);
            const int f0 = __float_as_int(b0.z), c0 = __float_as_int(b0.w);
            const int f1 = __float_as_int(b1.z), c1 = __float_as_int(b1.w);
            // leaves: nearest first
            const bool l0 = h0 && c0 > 0, l1 = h1 && c1 > 0;
            if (l0 || l1) {
                int fa = f0, ca = c0, fb = f1, cb = c1;
                float tnb = tn1;
                bool la = l0, lb = l1;
                if (l0 && l1 && tn1 < tn0) {
                    fa = f1; ca = c1; fb = f0; cb = c0; tnb = tn0;
                }
                if (!la) {  // only child 1 is a leaf
                    fa = f1; ca = c1; la = true; lb = false;
                }
                if (leaf_isect<ANYHIT, STATS>(s, fa, ca, o, d, tmax, in_object, h, st)) return h;
                if (lb && (h.t <= 0.0f || tnb <= h.t))
                    if (leaf_isect<ANYHIT, STATS>(s, fb, cb, o, d, tmax, in_object, h, st)) return h;
            }
            const bool i0 = h0 && c0 == 0 && (h.t <= 0.0f || tn0 <= h.t);
            const bool i1 = h1 && c1 == 0 && (h.t <= 0.0f || tn1 <= h.t);
            int next;
            if (i0 && i1) {
                const bool swap01 = tn1 < tn0;
                const int near_ = swap01 ? f1 : f0, far_ = swap01 ? f0 : f1;
                if (sp < STACK_SMEM)
                    smem_stack[sp * stride] = far_;
                else if (sp < RUMI_MAX_BVH_DEPTH)
                    spill[sp - STACK_SMEM] = far_;
                if (sp < RUMI_MAX_BVH_DEPTH) ++sp;  // the build caps depth at 63, so this always holds
                next = near_;
            } else if (i0) {
                next = f0;
            } else if (i1) {
                next = f1;
            } else {
                if (sp == 0) break;
                --sp;
                next = sp < STACK_SMEM ? smem_stack[sp * stride] : spill[sp - STACK_SMEM];
            }
            if ((unsigned)next >= (unsigned)(s.n_nodes - 1)) break;  // malformed tree guard
            cur = next;
        }
    }
    return h;
}

// ------------------------------------------------------------ four-wide traversal
// Stack entries: at most three pushes per four-wide level.
#define RUMI_STACK4 (3 * RUMI_MAX_BVH_DEPTH)

RUMI_D bool slab_s(float lx, float ly, float lz, float hx, float hy, float hz, float3 inv, float3 oinv, float tlimit,
                   float &tnear) {
    const float tx0 = fmaf(lx, inv.x, -oinv.x), tx1 = fmaf(hx, inv.x, -oinv.x);
    const float ty0 = fmaf(ly, inv.y, -oinv.y), ty1 = fmaf(hy, inv.y, -oinv.y);
    const float tz0 = fmaf(lz, inv.z, -oinv.z), tz1 = fmaf(hz, inv.z, -oinv.z);
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    tnear = tn;
    return tn <= tf && tf >= 0.0f && tn <= tlimit;
}

RUMI_D int sel4(int4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

#define RUMI_CSWAP(ka, sa, kb, sb)                  \
    if (kb < ka) {                                  \
        const float tk_ = ka; ka = kb; kb = tk_;    \
        const int ts_ = sa; sa = sb; sb = ts_;      \
    }

// The same query over the four-wide tree: a node's four child boxes are tested together
// and visited nearest first (leaves intersected at once, interior children: the nearest
// next, the others pushed farthest first).
template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D HitRec trace_ray_wide(const DevScene &s, float3 o, float3 d, float tmax, bool in_object, int *smem_stack,
                             int stride, TraceStats &st) {
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) return h;  // bvh.cpp:161-162
    if (s.n_nodes4 <= 0) return h;
    const float3 inv = safe_inv(d);
    const float3 oinv = mk3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
    int spill[RUMI_STACK4 - STACK_SMEM > 0 ? RUMI_STACK4 - STACK_SMEM : 1];
    int sp = 0;
    int cur = 0;
    // every node is visited at most once per ray, so the bound is never reached by a
    // well-formed tree; it keeps a malformed one from looping
    for (int guard = 0; guard < s.n_nodes4; ++guard) {
        const float4 *np = reinterpret_cast<const float4 *>(s.nodes4 + cur);
        const float4 lx = __ldg(np + 0), hx = __ldg(np + 1), ly = __ldg(np + 2), hy = __ldg(np + 3);
        const float4 lz = __ldg(np + 4), hz = __ldg(np + 5);
        const int4 ch = __ldg(reinterpret_cast<const int4 *>(np + 6));
        const int4 cn = __ldg(reinterpret_cast<const int4 *>(np + 7));
        if (STATS) st.nodes += 8;  // counted in 16-byte units
        const float lim = cull_limit(h.t, tmax);
        float k0, k1, k2, k3;
        if (!(cn.x >= 0 && slab_s(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, inv, oinv, lim, k0))) k0 = FLT_MAX;
        if (!(cn.y >= 0 && slab_s(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, inv, oinv, lim, k1))) k1 = FLT_MAX;
        if (!(cn.z >= 0 && slab_s(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, inv, oinv, lim, k2))) k2 = FLT_MAX;
        if (!(cn.w >= 0 && slab_s(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, inv, oinv, lim, k3))) k3 = FLT_MAX;
        int s0 = 0, s1 = 1, s2 = 2, s3 = 3;
        if (!ANYHIT) {  // near-first order; occlusion queries take any order
            RUMI_CSWAP(k0, s0, k1, s1);
            RUMI_CSWAP(k2, s2, k3, s3);
            RUMI_CSWAP(k0, s0, k2, s2);
            RUMI_CSWAP(k1, s1, k3, s3);
            RUMI_CSWAP(k1, s1, k2, s2);
        }
        // split the hit children (in that order) into leaves and interior nodes
        int lf0 = 0, lf1 = 0, lf2 = 0, lf3 = 0, lc0 = 0, lc1 = 0, lc2 = 0, lc3 = 0, nl = 0;
        float lk0 = 0.0f, lk1 = 0.0f, lk2 = 0.0f, lk3 = 0.0f;
        int c0 = -1, c1 = -1, c2 = -1, c3 = -1, ni = 0;
        float ck0 = 0.0f, ck1 = 0.0f, ck2 = 0.0f, ck3 = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float kj = j == 0 ? k0 : (j == 1 ? k1 : (j == 2 ? k2 : k3));
            const int sj = j == 0 ? s0 : (j == 1 ? s1 : (j == 2 ? s2 : s3));
            if (kj == FLT_MAX) continue;
            const int child = sel4(ch, sj), count = sel4(cn, sj);
            if (count > 0) {
                if (nl == 0) { lf0 = child; lc0 = count; lk0 = kj; }
                else if (nl == 1) { lf1 = child; lc1 = count; lk1 = kj; }
                else if (nl == 2) { lf2 = child; lc2 = count; lk2 = kj; }
                else { lf3 = child; lc3 = count; lk3 = kj; }
                ++nl;
            } else {
                if (ni == 0) { c0 = child; ck0 = kj; }
                else if (ni == 1) { c1 = child; ck1 = kj; }
                else if (ni == 2) { c2 = child; ck2 = kj; }
                else { c3 = child; ck3 = kj; }
                ++ni;
            }
        }
        // leaves now, nearest first (one copy of the primitive loop)
#pragma unroll 1
        for (int q = 0; q < nl; ++q) {
            const float lk = q == 0 ? lk0 : (q == 1 ? lk1 : (q == 2 ? lk2 : lk3));
            if (!ANYHIT && h.t > 0.0f && lk > h.t) break;
            const int lf = q == 0 ? lf0 : (q == 1 ? lf1 : (q == 2 ? lf2 : lf3));
            const int lc = q == 0 ? lc0 : (q == 1 ? lc1 : (q == 2 ? lc2 : lc3));
            if (leaf_isect<ANYHIT, STATS>(s, lf, lc, o, d, tmax, in_object, h, st)) return h;
        }
        // interior children beyond the closest hit so far are culled
        if (!ANYHIT && h.t > 0.0f) {
            if (ni > 3 && ck3 > h.t) ni = 3;
            if (ni > 2 && ck2 > h.t) ni = 2;
            if (ni > 1 && ck1 > h.t) ni = 1;
            if (ni > 0 && ck0 > h.t) ni = 0;
        }
        int next;
        if (ni == 0) {
            if (sp == 0) break;
            --sp;
            next = sp < STACK_SMEM ? smem_stack[sp * stride] : spill[sp - STACK_SMEM];
        } else {
            next = c0;
            // push the others farthest first, so the nearest of them is popped first
            for (int k = ni - 1; k >= 1; --k) {
                const int c = k == 3 ? c3 : (k == 2 ? c2 : c1);
                if (sp < STACK_SMEM)
                    smem_stack[sp * stride] = c;
                else if (sp < RUMI_STACK4)
                    spill[sp - STACK_SMEM] = c;
                if (sp < RUMI_STACK4) ++sp;  // three per level of a depth-limited tree: always holds
            }
        }
        if ((unsigned)next >= (unsigned)s.n_nodes4) break;  // malformed tree guard
        cur = next;
    }
    return h;
}

template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D HitRec trace_ray_w8(const DevScene &s, float3 o, float3 d, float tmax, bool in_object, int *smem_stack,
                           int stride, TraceStats &st);

template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D HitRec trace_ray(const DevScene &s, float3 o, float3 d, float tmax, bool in_object, int *smem_stack,
                        int stride, TraceStats &st) {
#if RUMI_WALK8
    return trace_ray_w8<ANYHIT, STACK_SMEM, STATS>(s, o, d, tmax, in_object, smem_stack, stride, st);
#elif RUMI_BVH_WIDE
    return trace_ray_wide<ANYHIT, STACK_SMEM, STATS>(s, o, d, tmax, in_object, smem_stack, stride, st);
#else
    return trace_ray_bin<ANYHIT, STACK_SMEM, STATS>(s, o, d, tmax, in_object, smem_stack, stride, st);
#endif
}

// ------------------------------------------------------------ resumable form
// The same traversal split into single node-pair steps, so a warp can refill a lane with
// a new ray as soon as that lane's ray finishes (dynamic fetch) instead of waiting for
// the slowest of its 32 rays.  cur: next node pair, -1: pop the stack, -2: finished.
struct TravState {
    float3 o, d, inv, oinv;
    float tmax;
    int cur, sp, steps;
    bool in_obj;
    HitRec h;
};

template <bool ANYHIT, bool STATS>
RUMI_D void trav_begin(const DevScene &s, TravState &T, float3 o, float3 d, float tmax, bool in_obj,
                       TraceStats &st) {
    T.o = o;
    T.d = d;
    T.tmax = tmax;
    T.in_obj = in_obj;
    T.sp = 0;
    T.steps = 0;
    T.h.t = 0.0f;
    T.h.id = -1;
    T.h.u = T.h.v = 0.0f;
    T.h.back = 0;
    T.cur = -2;
    if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) return;  // bvh.cpp:161-162
    T.inv = safe_inv(d);
    T.oinv = mk3(o.x * T.inv.x, o.y * T.inv.y, o.z * T.inv.z);
    const float4 *rp = reinterpret_cast<const float4 *>(s.nodes);
    const float4 a = __ldg(rp), b = __ldg(rp + 1);
    if (STATS) st.nodes += 2;
    float tn;
    if (!slab(a, b, T.inv, T.oinv, tmax, tn)) return;
    const int first = __float_as_int(b.z), count = __float_as_int(b.w);
    if (count > 0) {
        leaf_isect<ANYHIT, STATS>(s, first, count, o, d, tmax, in_obj, T.h, st);
        return;
    }
    if ((unsigned)first >= (unsigned)(s.n_nodes - 1)) return;
    T.cur = first;
}

template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D void trav_step(const DevScene &s, TravState &T, int *smem_stack, int stride, int *spill, TraceStats &st) {
    if (T.cur == -1) {
        if (T.sp == 0) {
            T.cur = -2;
            return;
        }
        --T.sp;
        T.cur = T.sp < STACK_SMEM ? smem_stack[T.sp * stride] : spill[T.sp - STACK_SMEM];
    }
    if ((unsigned)T.cur >= (unsigned)(s.n_nodes - 1) || ++T.steps > s.n_nodes) {  // malformed tree guard
        T.cur = -2;
        return;
    }
    const float4 *np = reinterpret_cast<const float4 *>(s.nodes + T.cur);
    const float4 a0 = __ldg(np + 0), b0 = __ldg(np + 1), a1 = __ldg(np + 2), b1 = __ldg(np + 3);
    if (STATS) st.nodes += 4;
    const float lim = cull_limit(T.h.t, T.tmax);
    float tn0, tn1;
    const bool h0 = slab(a0, b0, T.inv, T.oinv, lim, tn0);
    const bool h1 = slab(a1, b1, T.inv, T.oinv, lim, tn1);
    const int f0 = __float_as_int(b0.z), c0 = __float_as_int(b0.w);
    const int f1 = __float_as_int(b1.z), c1 = __float_as_int(b1.w);
    const bool l0 = h0 && c0 > 0, l1 = h1 && c1 > 0;
    if (l0 || l1) {
        int fa = f0, ca = c0, fb = f1, cb = c1;
        float tnb = tn1;
        bool lb = l1;
        if (l0 && l1 && tn1 < tn0) {
            fa = f1; ca = c1; fb = f0; cb = c0; tnb = tn0;
        }
        if (!l0) {
            fa = f1; ca = c1; lb = false;
        }
        if (leaf_isect<ANYHIT, STATS>(s, fa, ca, T.o, T.d, T.tmax, T.in_obj, T.h, st)) {
            T.cur = -2;
            return;
        }
        if (lb && (T.h.t <= 0.0f || tnb <= T.h.t))
            if (leaf_isect<ANYHIT, STATS>(s, fb, cb, T.o, T.d, T.tmax, T.in_obj, T.h, st)) {
                T.cur = -2;
                return;
            }
    }
    const bool i0 = h0 && c0 == 0 && (T.h.t <= 0.0f || tn0 <= T.h.t);
    const bool i1 = h1 && c1 == 0 && (T.h.t <= 0.0f || tn1 <= T.h.t);
    if (i0 && i1) {
        const bool swap01 = tn1 < tn0;
        const int near_ = swap01 ? f1 : f0, far_ = swap01 ? f0 : f1;
        if (T.sp < STACK_SMEM)
            smem_stack[T.sp * stride] = far_;
        else if (T.sp < RUMI_MAX_BVH_DEPTH)
            spill[T.sp - STACK_SMEM] = far_;
        if (T.sp < RUMI_MAX_BVH_DEPTH) ++T.sp;
        T.cur = near_;
    } else if (i0) {
        T.cur = f0;
    } else if (i1) {
        T.cur = f1;
    } else {
        T.cur = -1;
    }
}

// Step with postponed leaves: leaves reached by this node pair are recorded in the
// state (at most the pair's two children) instead of being intersected, so a warp can
// intersect the leaves of all its lanes together ("while-while" traversal).
struct PendingLeaves {
    int f0, c0, f1, c1;
    float tn1;
    int n;
};

template <int STACK_SMEM, bool STATS>
RUMI_D void trav_step_postpone(const DevScene &s, TravState &T, PendingLeaves &pl, int *smem_stack, int stride,
                               int *spill, TraceStats &st) {
    if (T.cur == -1) {
        if (T.sp == 0) {
            T.cur = -2;
            return;
        }
        --T.sp;
        T.cur = T.sp < STACK_SMEM ? smem_stack[T.sp * stride] : spill[T.sp - STACK_SMEM];
    }
    if ((unsigned)T.cur >= (unsigned)(s.n_nodes - 1) || ++T.steps > s.n_nodes) {
        T.cur = -2;
        return;
    }
    const float4 *np = reinterpret_cast<const float4 *>(s.nodes + T.cur);
    const float4 a0 = __ldg(np + 0), b0 = __ldg(np + 1), a1 = __ldg(np + 2), b1 = __ldg(np + 3);
    if (STATS) st.nodes += 4;
    const float lim = cull_limit(T.h.t, T.tmax);
    float tn0, tn1;
    const bool h0 = slab(a0, b0, T.inv, T.oinv, lim, tn0);
    const bool h1 = slab(a1, b1, T.inv, T.oinv, lim, tn1);
    const int f0 = __float_as_int(b0.z), c0 = __float_as_int(b0.w);
    const int f1 = __float_as_int(b1.z), c1 = __float_as_int(b1.w);
    const bool l0 = h0 && c0 > 0, l1 = h1 && c1 > 0;
    pl.n = 0;
    if (l0 && l1) {
        const bool sw = tn1 < tn0;
        pl.f0 = sw ? f1 : f0; pl.c0 = sw ? c1 : c0;
        pl.f1 = sw ? f0 : f1; pl.c1 = sw ? c0 : c1;
        pl.tn1 = sw ? tn0 : tn1;
        pl.n = 2;
    } else if (l0) {
        pl.f0 = f0; pl.c0 = c0; pl.n = 1;
    } else if (l1) {
        pl.f0 = f1; pl.c0 = c1; pl.n = 1;
    }
    const bool i0 = h0 && c0 == 0 && (T.h.t <= 0.0f || tn0 <= T.h.t);
    const bool i1 = h1 && c1 == 0 && (T.h.t <= 0.0f || tn1 <= T.h.t);
    if (i0 && i1) {
        const bool swap01 = tn1 < tn0;
        const int near_ = swap01 ? f1 : f0, far_ = swap01 ? f0 : f1;
        if (T.sp < STACK_SMEM)
            smem_stack[T.sp * stride] = far_;
        else if (T.sp < RUMI_MAX_BVH_DEPTH)
            spill[T.sp - STACK_SMEM] = far_;
        if (T.sp < RUMI_MAX_BVH_DEPTH) ++T.sp;
        T.cur = near_;
    } else if (i0) {
        T.cur = f0;
    } else if (i1) {
        T.cur = f1;
    } else {
        T.cur = -1;
    }
}

// Intersects the postponed leaves; returns true when ANYHIT found a hit.
template <bool ANYHIT, bool STATS>
RUMI_D bool run_pending(const DevScene &s, TravState &T, PendingLeaves &pl, TraceStats &st) {
    bool found = false;
    if (pl.n > 0) found = leaf_isect<ANYHIT, STATS>(s, pl.f0, pl.c0, T.o, T.d, T.tmax, T.in_obj, T.h, st);
    if (!found && pl.n > 1 && (T.h.t <= 0.0f || pl.tn1 <= T.h.t))
        found = leaf_isect<ANYHIT, STATS>(s, pl.f1, pl.c1, T.o, T.d, T.tmax, T.in_obj, T.h, st);
    pl.n = 0;
    return found;
}

// Speculative while-while traversal with per-lane refill (Aila & Laine, "Understanding
// the efficiency of ray traversal on GPUs", HPG 2009; Aila, Laine & Karras 2012): each
// lane walks interior node pairs until it holds a postponed leaf, and keeps walking
// (speculatively) until every lane of the warp holds one; then the warp intersects the
// postponed leaves together.  Rounds repeat until a lane's ray is finished, and finished
// lanes are refilled from the queue in warp-aggregated batches.
//   cur >= 0: a node pair to test; cur < 0, != WW_DONE: the leaf node -(cur + 1);
//   WW_DONE: the stack is empty.
#define WW_DONE (-0x7fffffff - 1)

// scene_of(i): the scene ray i is traced in (one scene, or per ray in a multi-scene batch).
template <bool ANYHIT, int STACK_SMEM, bool STATS, typename SceneOf, typename Fetch, typename Finish>
RUMI_D void traverse_queue_ww(SceneOf scene_of, int n, int *counter, int refill_min, int *smem_stack, int stride,
                              Fetch fetch, Finish finish, TraceStats &st) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int spill[RUMI_MAX_BVH_DEPTH - STACK_SMEM > 0 ? RUMI_MAX_BVH_DEPTH - STACK_SMEM : 1];
    const DevScene *sp_scene = scene_of(-1);
    const float4 *nodes = reinterpret_cast<const float4 *>(sp_scene->nodes);
    float3 o = mk3(0, 0, 0), d = mk3(0, 0, 0), inv = mk3(0, 0, 0), oinv = mk3(0, 0, 0);
    float tmax = 0.0f;
    bool in_obj = false;
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    int ray = -1, cur = WW_DONE, sp = 0, lf_first = 0, lf_count = 0, steps = 0;
    bool exhausted = false;
    auto pop = [&]() -> int {
        if (sp == 0) return WW_DONE;
        --sp;
        return sp < STACK_SMEM ? smem_stack[sp * stride] : spill[sp - STACK_SMEM];
    };
    auto push = [&](int v) {
        if (sp < STACK_SMEM)
            smem_stack[sp * stride] = v;
        else if (sp < RUMI_MAX_BVH_DEPTH)
            spill[sp - STACK_SMEM] = v;
        if (sp < RUMI_MAX_BVH_DEPTH) ++sp;  // the build caps depth at 63: always holds
    };
    // leaf node -> pending leaf range (a range check keeps a malformed tree harmless)
    auto take_leaf = [&](int node) {
        if ((unsigned)node >= (unsigned)sp_scene->n_nodes) {
            lf_count = 0;
            return;
        }
        const float4 b = __ldg(nodes + 2 * node + 1);
        lf_first = __float_as_int(b.z);
        lf_count = __float_as_int(b.w);
    };
    for (;;) {
        // finished rays -> results; idle lanes -> new rays
        if (ray >= 0 && cur == WW_DONE && lf_count == 0) {
            finish(ray, h);
            ray = -1;
        }
        const unsigned idle = __ballot_sync(0xffffffffu, ray < 0);
        if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
            int base = 0;
            const int leader = __ffs(idle) - 1;
            if (lane == leader) base = atomicAdd(counter, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= n) exhausted = true;
            if (ray < 0) {
                const int r = base + __popc(idle & lt);
                if (r < n) {
                    ray = r;
                    fetch(r, o, d, tmax, in_obj);
                    sp_scene = scene_of(r);
                    nodes = reinterpret_cast<const float4 *>(sp_scene->nodes);
                    h.t = 0.0f;
                    h.id = -1;
                    h.u = h.v = 0.0f;
                    h.back = 0;
                    sp = 0;
                    steps = 0;
                    cur = WW_DONE;
                    lf_count = 0;
                    if (!(d.x == 0.0f && d.y == 0.0f && d.z == 0.0f)) {  // bvh.cpp:161-162
                        inv = safe_inv(d);
                        oinv = mk3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
                        const float4 a = __ldg(nodes), b = __ldg(nodes + 1);
                        if (STATS) st.nodes += 2;
                        float tn;
                        if (slab(a, b, inv, oinv, tmax, tn)) {
                            const int first = __float_as_int(b.z), count = __float_as_int(b.w);
                            if (count > 0) {
                                lf_first = first;
                                lf_count = count;
                            } else if ((unsigned)first < (unsigned)(sp_scene->n_nodes - 1)) {
                                cur = first;
                            }
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, ray >= 0) == 0) break;
        // interior node pairs, speculatively past the first leaf
        while (cur >= 0) {
            if ((unsigned)cur >= (unsigned)(sp_scene->n_nodes - 1) || ++steps > sp_scene->n_nodes) {  // malformed tree guard
                cur = WW_DONE;
                lf_count = 0;
                break;
            }
            const float4 a0 = __ldg(nodes + 2 * cur), b0 = __ldg(nodes + 2 * cur + 1);
            const float4 a1 = __ldg(nodes + 2 * cur + 2), b1 = __ldg(nodes + 2 * cur + 3);
            if (STATS) st.nodes += 4;
            const float lim = cull_limit(h.t, tmax);
            float tn0, tn1;
            const bool h0 = slab(a0, b0, inv, oinv, lim, tn0);
            const bool h1 = slab(a1, b1, inv, oinv, lim, tn1);
            const int c0 = __float_as_int(b0.w), c1 = __float_as_int(b1.w);
            const bool v0 = h0 && c0 >= 0, v1 = h1 && c1 >= 0;
            const int e0 = c0 > 0 ? -(cur + 1) : __float_as_int(b0.z);
            const int e1 = c1 > 0 ? -(cur + 2) : __float_as_int(b1.z);
            if (v0 && v1) {
                const bool sw = tn1 < tn0;
                cur = sw ? e1 : e0;
                push(sw ? e0 : e1);
            } else if (v0) {
                cur = e0;
            } else if (v1) {
                cur = e1;
            } else {
                cur = pop();
            }
            if (cur < 0 && cur != WW_DONE && lf_count == 0) {  // postpone the leaf, keep walking
                take_leaf(-cur - 1);
                cur = pop();
            }
            if (!__any_sync(__activemask(), lf_count == 0 && cur >= 0)) break;
        }
        // the postponed leaves, then any leaf the walk stopped at
        while (lf_count > 0) {
            if (leaf_isect<ANYHIT, STATS>(*sp_scene, lf_first, lf_count, o, d, tmax, in_obj, h, st)) {
                cur = WW_DONE;
                lf_count = 0;
                break;
            }
            lf_count = 0;
            if (cur < 0 && cur != WW_DONE) {
                take_leaf(-cur - 1);
                cur = pop();
            }
        }
    }
}

// The same speculative while-while walk over the four-wide tree (nodes4): an interior
// step tests a node's four child boxes, continues with the nearest hit child and pushes
// the others farthest first; leaf children are stack entries -(1 + 4 * node + slot).
template <bool ANYHIT, int STACK_SMEM, bool STATS, typename SceneOf, typename Fetch, typename Finish>
RUMI_D void traverse_queue_ww4(SceneOf scene_of, int n, int *counter, int refill_min, int *smem_stack, int stride,
                               Fetch fetch, Finish finish, TraceStats &st) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int spill[RUMI_STACK4 - STACK_SMEM > 0 ? RUMI_STACK4 - STACK_SMEM : 1];
    const DevScene *sp_scene = scene_of(-1);
    const float4 *nodes = reinterpret_cast<const float4 *>(sp_scene->nodes4);
    float3 o = mk3(0, 0, 0), d = mk3(0, 0, 0), inv = mk3(0, 0, 0), oinv = mk3(0, 0, 0);
    float tmax = 0.0f;
    bool in_obj = false;
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    int ray = -1, cur = WW_DONE, sp = 0, lf_first = 0, lf_count = 0, steps = 0;
    bool exhausted = false;
    auto pop = [&]() -> int {
        if (sp == 0) return WW_DONE;
        --sp;
        return sp < STACK_SMEM ? smem_stack[sp * stride] : spill[sp - STACK_SMEM];
    };
    auto push = [&](int v) {
        if (sp < STACK_SMEM)
            smem_stack[sp * stride] = v;
        else if (sp < RUMI_STACK4)
            spill[sp - STACK_SMEM] = v;
        if (sp < RUMI_STACK4) ++sp;  // three per level of a depth-limited tree: always holds
    };
    auto take_leaf = [&](int ref) {
        const int k = -ref - 1, node = k >> 2, slot = k & 3;
        if ((unsigned)node >= (unsigned)sp_scene->n_nodes4) {
            lf_count = 0;
            return;
        }
        const int4 ch = __ldg(reinterpret_cast<const int4 *>(nodes + 8 * node + 6));
        const int4 cn = __ldg(reinterpret_cast<const int4 *>(nodes + 8 * node + 7));
        lf_first = sel4(ch, slot);
        lf_count = sel4(cn, slot);
    };
    for (;;) {
        if (ray >= 0 && cur == WW_DONE && lf_count == 0) {
            finish(ray, h);
            ray = -1;
        }
        const unsigned idle = __ballot_sync(0xffffffffu, ray < 0);
        if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
            int base = 0;
            const int leader = __ffs(idle) - 1;
            if (lane == leader) base = atomicAdd(counter, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= n) exhausted = true;
            if (ray < 0) {
                const int r = base + __popc(idle & lt);
                if (r < n) {
                    ray = r;
                    fetch(r, o, d, tmax, in_obj);
                    sp_scene = scene_of(r);
                    nodes = reinterpret_cast<const float4 *>(sp_scene->nodes4);
                    h.t = 0.0f;
                    h.id = -1;
                    h.u = h.v = 0.0f;
                    h.back = 0;
                    sp = 0;
                    steps = 0;
                    lf_count = 0;
                    cur = WW_DONE;
                    if (!(d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) && sp_scene->n_nodes4 > 0) {  // bvh.cpp:161-162
                        inv = safe_inv(d);
                        oinv = mk3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
                        cur = 0;
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, ray >= 0) == 0) break;
        while (cur >= 0) {
            if ((unsigned)cur >= (unsigned)sp_scene->n_nodes4 || ++steps > sp_scene->n_nodes4) {  // malformed tree guard
                cur = WW_DONE;
                lf_count = 0;
                break;
            }
            const float4 *np = nodes + 8 * cur;
            const float4 lx = __ldg(np + 0), hx = __ldg(np + 1), ly = __ldg(np + 2), hy = __ldg(np + 3);
            const float4 lz = __ldg(np + 4), hz = __ldg(np + 5);
            const int4 ch = __ldg(reinterpret_cast<const int4 *>(np + 6));
            const int4 cn = __ldg(reinterpret_cast<const int4 *>(np + 7));
            if (STATS) st.nodes += 8;  // counted in 16-byte units
            const float lim = cull_limit(h.t, tmax);
            float k0, k1, k2, k3;
            if (!(cn.x >= 0 && slab_s(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, inv, oinv, lim, k0))) k0 = FLT_MAX;
            if (!(cn.y >= 0 && slab_s(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, inv, oinv, lim, k1))) k1 = FLT_MAX;
            if (!(cn.z >= 0 && slab_s(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, inv, oinv, lim, k2))) k2 = FLT_MAX;
            if (!(cn.w >= 0 && slab_s(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, inv, oinv, lim, k3))) k3 = FLT_MAX;
            int s0 = 0, s1 = 1, s2 = 2, s3 = 3;
            if (!ANYHIT) {
                RUMI_CSWAP(k0, s0, k1, s1);
                RUMI_CSWAP(k2, s2, k3, s3);
                RUMI_CSWAP(k0, s0, k2, s2);
                RUMI_CSWAP(k1, s1, k3, s3);
                RUMI_CSWAP(k1, s1, k2, s2);
            }
            // entries of the hit children in order: node index or leaf reference
            auto entry = [&](int slot) {
                return sel4(cn, slot) > 0 ? -(1 + 4 * cur + slot) : sel4(ch, slot);
            };
            const int e0 = entry(s0), e1 = entry(s1), e2 = entry(s2), e3 = entry(s3);
            const int nh = (k0 != FLT_MAX) + (k1 != FLT_MAX) + (k2 != FLT_MAX) + (k3 != FLT_MAX);
            if (!ANYHIT) {
                // sorted: the hit children are the first nh
                if (nh > 3) push(e3);
                if (nh > 2) push(e2);
                if (nh > 1) push(e1);
                cur = nh > 0 ? e0 : pop();
            } else {
                int next = WW_DONE;
                if (k3 != FLT_MAX) next = e3;
                if (k2 != FLT_MAX) { if (next != WW_DONE) push(next); next = e2; }
                if (k1 != FLT_MAX) { if (next != WW_DONE) push(next); next = e1; }
                if (k0 != FLT_MAX) { if (next != WW_DONE) push(next); next = e0; }
                cur = next != WW_DONE ? next : pop();
            }
            if (cur < 0 && cur != WW_DONE && lf_count == 0) {  // postpone the leaf, keep walking
                take_leaf(cur);
                cur = pop();
            }
            if (!__any_sync(__activemask(), lf_count == 0 && cur >= 0)) break;
        }
        while (lf_count > 0) {
            if (leaf_isect<ANYHIT, STATS>(*sp_scene, lf_first, lf_count, o, d, tmax, in_obj, h, st)) {
                cur = WW_DONE;
                lf_count = 0;
                break;
            }
            lf_count = 0;
            if (cur < 0 && cur != WW_DONE) {
                take_leaf(cur);
                cur = pop();
            }
        }
    }
}

// ------------------------------------------------ compressed eight-wide traversal
// Walk over nodes8 (Bvh8Node, scene.cuh).  A node visit loads its 80 bytes and tests the
// eight quantised child boxes at once; the hit children form a group (node, hit slots in
// visiting order) that is taken apart one child at a time: an interior child is visited
// next (the rest of the group is pushed as one 32-bit stack entry, node << 8 | slots), a
// leaf child becomes the lane's postponed leaf.  Children are visited in the octant order
// the build arranged (slot k ^ oct for the k-th visit), so nothing is sorted.

// Depth of the eight-wide tree <= the binary tree's (63): one stack entry per level.
#define RUMI_STACK8 64

// Ray constants of the node test.
struct Ray8 {
    float3 inv, oinv;  // safe reciprocal direction and origin * inv
    unsigned int oct;  // bit a set when direction component a is negative
};

RUMI_D Ray8 make_ray8(float3 o, float3 d) {
    Ray8 r;
    r.inv = safe_inv(d);
    r.oinv = mk3(o.x * r.inv.x, o.y * r.inv.y, o.z * r.inv.z);
    // the sign bits of the reciprocal, which the slabs are computed with: a -0.0 component
    // has a negative reciprocal (-2^80) although it does not compare below zero, and its
    // near plane is the high one
    r.oct = (__float_as_uint(r.inv.x) >> 31) | ((__float_as_uint(r.inv.y) >> 31) << 1) |
            ((__float_as_uint(r.inv.z) >> 31) << 2);
    return r;
}

// Byte b of w as a float, exactly: the bits of 2^23 + byte, minus 2^23.
RUMI_D float q8(unsigned int w, int b) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + (unsigned)b)) - 8388608.0f;
}

// Slot bits (bit k = slot k) -> visiting order (bit k ^ oct).
RUMI_D unsigned int oct_order(unsigned int m, unsigned int oct) {
    if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
    return m;
}

// Bit k set where byte k of (lo, hi) is non-zero.
RUMI_D unsigned int nonzero_bytes(unsigned int lo, unsigned int hi) {
    const unsigned int a = __vcmpne4(lo, 0u) & 0x08040201u, b = __vcmpne4(hi, 0u) & 0x80402010u;
    return (a | b) * 0x01010101u >> 24;
}

// What taking a child from a node needs: the node's first two float4.
struct Group8 {
    unsigned int imask;
    int child_base, prim_base;
    unsigned int cnt_lo, cnt_hi;
};

RUMI_D Group8 group_of(float4 a, float4 b) {
    Group8 g;
    g.imask = __float_as_uint(a.x) >> 24;
    g.child_base = __float_as_int(a.y);
    g.prim_base = __float_as_int(a.z);
    g.cnt_lo = __float_as_uint(b.z);
    g.cnt_hi = __float_as_uint(b.w);
    return g;
}

// Tests node n's children; returns the hit slots in visiting order and the node's group.
template <bool STATS>
RUMI_D unsigned int visit8(const float4 *__restrict__ nodes, int n, const Ray8 &r, float lim, Group8 &g,
                           TraceStats &st) {
    const float4 *np = nodes + 5 * n;
    const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), d = __ldg(np + 3), e = __ldg(np + 4);
    if (STATS) st.nodes += 5;
    g = group_of(a, b);
    const unsigned int meta = __float_as_uint(a.x);
    // the quantum 2^e per axis straight from its biased exponent; the grid's map to ray t
    const float ax = __uint_as_float((meta & 0xFFu) << 23) * r.inv.x;
    const float ay = __uint_as_float(((meta >> 8) & 0xFFu) << 23) * r.inv.y;
    const float az = __uint_as_float(((meta >> 16) & 0xFFu) << 23) * r.inv.z;
    const float bx = fmaf(a.w, r.inv.x, -r.oinv.x);
    const float by = fmaf(b.x, r.inv.y, -r.oinv.y);
    const float bz = fmaf(b.y, r.inv.z, -r.oinv.z);
    // near / far planes by the direction's signs
    const bool sx = r.oct & 1u, sy = r.oct & 2u, sz = r.oct & 4u;
    const unsigned int lx0 = __float_as_uint(c.x), lx1 = __float_as_uint(c.y);
    const unsigned int ly0 = __float_as_uint(c.z), ly1 = __float_as_uint(c.w);
    const unsigned int lz0 = __float_as_uint(d.x), lz1 = __float_as_uint(d.y);
    const unsigned int hx0 = __float_as_uint(d.z), hx1 = __float_as_uint(d.w);
    const unsigned int hy0 = __float_as_uint(e.x), hy1 = __float_as_uint(e.y);
    const unsigned int hz0 = __float_as_uint(e.z), hz1 = __float_as_uint(e.w);
    const unsigned int nx[2] = {sx ? hx0 : lx0, sx ? hx1 : lx1}, fx[2] = {sx ? lx0 : hx0, sx ? lx1 : hx1};
    const unsigned int ny[2] = {sy ? hy0 : ly0, sy ? hy1 : ly1}, fy[2] = {sy ? ly0 : hy0, sy ? ly1 : hy1};
    const unsigned int nz[2] = {sz ? hz0 : lz0, sz ? hz1 : lz1}, fz[2] = {sz ? lz0 : hz0, sz ? lz1 : hz1};
    unsigned int hits = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int w = k >> 2, bb = k & 3;
        const float tnx = fmaf(q8(nx[w], bb), ax, bx), tfx = fmaf(q8(fx[w], bb), ax, bx);
        const float tny = fmaf(q8(ny[w], bb), ay, by), tfy = fmaf(q8(fy[w], bb), ay, by);
        const float tnz = fmaf(q8(nz[w], bb), az, bz), tfz = fmaf(q8(fz[w], bb), az, bz);
        const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
        const float tf = fminf(fminf(tfx, tfy), fminf(tfz, lim));
        hits |= (tn <= tf ? 1u : 0u) << k;
    }
    hits &= g.imask | nonzero_bytes(g.cnt_lo, g.cnt_hi);  // empty slots never hit
    return oct_order(hits, r.oct);
}

// Primitive range of leaf slot k of a group: prim_base + the counts of slots 0..k-1.
RUMI_D void leaf_of(const Group8 &g, int k, int &first, int &count) {
    const unsigned long long cnt = ((unsigned long long)g.cnt_hi << 32) | g.cnt_lo;
    const unsigned long long below = cnt & ((1ull << (8 * k)) - 1ull);
    // bytes -> four 16-bit pair sums (each <= 510) -> their total in the top 16 bits
    const unsigned long long s16 = (below & 0x00FF00FF00FF00FFull) + ((below >> 8) & 0x00FF00FF00FF00FFull);
    first = g.prim_base + (int)((s16 * 0x0001000100010001ull) >> 48);
    count = (int)((cnt >> (8 * k)) & 0xFFull);
}

// Speculative while-while walk with per-lane refill (as traverse_queue_ww) over nodes8.
template <bool ANYHIT, int STACK_SMEM, bool STATS, typename SceneOf, typename Fetch, typename Finish>
RUMI_D void traverse_queue_ww8(SceneOf scene_of, int n, int *counter, int refill_min, int *smem_stack, int stride,
                               Fetch fetch, Finish finish, TraceStats &st) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    unsigned int spill[RUMI_STACK8 - STACK_SMEM > 0 ? RUMI_STACK8 - STACK_SMEM : 1];
    const DevScene *sp_scene = scene_of(-1);
    const float4 *nodes = reinterpret_cast<const float4 *>(sp_scene->nodes8);
    const float4 *prims = sp_scene->prims8;
    float3 o = mk3(0, 0, 0), d = mk3(0, 0, 0);
    Ray8 r;
    r.inv = r.oinv = mk3(0, 0, 0);
    r.oct = 0;
    float tmax = 0.0f;
    bool in_obj = false;
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    Group8 g;
    g.imask = 0;
    g.child_base = g.prim_base = 0;
    g.cnt_lo = g.cnt_hi = 0;
    int ray = -1, gnode = 0, sp = 0, lf_first = 0, lf_count = 0, steps = 0;
    unsigned int ghits = 0;
    bool exhausted = false;
    auto push = [&](unsigned int v) {
        if (sp < STACK_SMEM)
            smem_stack[sp * stride] = (int)v;
        else if (sp < RUMI_STACK8)
            spill[sp - STACK_SMEM] = v;
        if (sp < RUMI_STACK8) ++sp;  // one entry per level of a depth-limited tree: always holds
    };
    // the next group from the stack (its node's first two float4 give the group's decode)
    auto pop = [&]() {
        --sp;
        const unsigned int v = sp < STACK_SMEM ? (unsigned int)smem_stack[sp * stride] : spill[sp - STACK_SMEM];
        gnode = (int)(v >> 8);
        ghits = v & 0xFFu;
        if ((unsigned)gnode >= (unsigned)sp_scene->n_nodes8) {  // malformed stack entry guard
            ghits = 0;
            sp = 0;
            return;
        }
        const float4 *np = nodes + 5 * gnode;
        g = group_of(__ldg(np), __ldg(np + 1));
        if (STATS) st.nodes += 2;
    };
    for (;;) {
        // finished rays -> results; idle lanes -> new rays
        if (ray >= 0 && ghits == 0 && sp == 0 && lf_count == 0) {
            finish(ray, h);
            ray = -1;
        }
        const unsigned idle = __ballot_sync(0xffffffffu, ray < 0);
        if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
            int base = 0;
            const int leader = __ffs(idle) - 1;
            if (lane == leader) base = atomicAdd(counter, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= n) exhausted = true;
            if (ray < 0) {
                const int rr = base + __popc(idle & lt);
                if (rr < n) {
                    ray = rr;
                    fetch(rr, o, d, tmax, in_obj);
                    sp_scene = scene_of(rr);
                    nodes = reinterpret_cast<const float4 *>(sp_scene->nodes8);
                    prims = sp_scene->prims8;
                    h.t = 0.0f;
                    h.id = -1;
                    h.u = h.v = 0.0f;
                    h.back = 0;
                    sp = 0;
                    steps = 0;
                    lf_count = 0;
                    ghits = 0;
                    if (!(d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) && sp_scene->n_nodes8 > 0) {  // bvh.cpp:161-162
                        r = make_ray8(o, d);
                        gnode = 0;
                        ghits = visit8<STATS>(nodes, 0, r, tmax, g, st);
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, ray >= 0) == 0) break;
        // interior steps, speculatively past the first postponed leaf; a lane stops when it
        // meets a second leaf (kept in its group) or runs out of work
        bool blocked = false;
        while (ray >= 0 && !blocked && (ghits != 0 || sp != 0)) {
            if (ghits == 0) pop();
            if (ghits != 0) {
                const int kslot = (__ffs(ghits) - 1) ^ (int)r.oct;
                if ((g.imask >> kslot) & 1u) {
                    ghits &= ghits - 1u;
                    const int child = g.child_base + __popc(g.imask & ((1u << kslot) - 1u));
                    if ((unsigned)child >= (unsigned)sp_scene->n_nodes8 || ++steps > sp_scene->n_nodes8) {
                        ghits = 0;  // malformed tree guard
                        sp = 0;
                    } else {
                        if (ghits != 0) push(((unsigned int)gnode << 8) | ghits);
                        gnode = child;
                        ghits = visit8<STATS>(nodes, child, r, cull_limit(h.t, tmax), g, st);
                    }
                } else if (lf_count == 0) {
                    ghits &= ghits - 1u;
                    leaf_of(g, kslot, lf_first, lf_count);
                } else {
                    blocked = true;
                }
            }
            if (!__any_sync(__activemask(), lf_count == 0 && (ghits != 0 || sp != 0))) break;
        }
        // the postponed leaf, then the leaf the walk stopped at
        if (ray >= 0 && lf_count > 0) {
            for (int rep = 0; rep < 2 && lf_count > 0; ++rep) {
                const bool any =
                    leaf_isect_in<ANYHIT, STATS>(*sp_scene, prims, lf_first, lf_count, o, d, tmax, in_obj, h, st);
                lf_count = 0;
                if (any) {
                    ghits = 0;
                    sp = 0;
                    break;
                }
                if (ghits != 0) {
                    const int kslot = (__ffs(ghits) - 1) ^ (int)r.oct;
                    if (!((g.imask >> kslot) & 1u)) {
                        ghits &= ghits - 1u;
                        leaf_of(g, kslot, lf_first, lf_count);
                    }
                }
            }
        }
    }
}

// One ray to completion over nodes8 (the per-thread form, for integrators that trace one
// ray at a time).  smem_stack: this thread's first shared-memory stack slot.
template <bool ANYHIT, int STACK_SMEM, bool STATS>
RUMI_D HitRec trace_ray_w8(const DevScene &s, float3 o, float3 d, float tmax, bool in_object, int *smem_stack,
                           int stride, TraceStats &st) {
    HitRec h;
    h.t = 0.0f;
    h.id = -1;
    h.u = h.v = 0.0f;
    h.back = 0;
    if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) return h;  // bvh.cpp:161-162
    if (s.n_nodes8 <= 0) return h;
    const float4 *nodes = reinterpret_cast<const float4 *>(s.nodes8);
    unsigned int spill[RUMI_STACK8 - STACK_SMEM > 0 ? RUMI_STACK8 - STACK_SMEM : 1];
    const Ray8 r = make_ray8(o, d);
    Group8 g;
    int gnode = 0, sp = 0;
    unsigned int ghits = visit8<STATS>(nodes, 0, r, tmax, g, st);
    // every node is visited at most once per ray: the bound only stops a malformed tree
    for (int guard = 0; guard <= s.n_nodes8;) {
        if (ghits == 0) {
            if (sp == 0) break;
            --sp;
            const unsigned int v = sp < STACK_SMEM ? (unsigned int)smem_stack[sp * stride] : spill[sp - STACK_SMEM];
            gnode = (int)(v >> 8);
            ghits = v & 0xFFu;
            if ((unsigned)gnode >= (unsigned)s.n_nodes8) break;  // malformed stack entry guard
            const float4 *np = nodes + 5 * gnode;
            g = group_of(__ldg(np), __ldg(np + 1));
            if (STATS) st.nodes += 2;
        }
        const int kslot = (__ffs(ghits) - 1) ^ (int)r.oct;
        ghits &= ghits - 1u;
        if ((g.imask >> kslot) & 1u) {
            const int child = g.child_base + __popc(g.imask & ((1u << kslot) - 1u));
            if ((unsigned)child >= (unsigned)s.n_nodes8) break;  // malformed tree guard
            ++guard;
            if (ghits != 0) {
                const unsigned int v = ((unsigned int)gnode << 8) | ghits;
                if (sp < STACK_SMEM)
                    smem_stack[sp * stride] = (int)v;
                else if (sp < RUMI_STACK8)
                    spill[sp - STACK_SMEM] = v;
                if (sp < RUMI_STACK8) ++sp;
            }
            gnode = child;
            ghits = visit8<STATS>(nodes, child, r, cull_limit(h.t, tmax), g, st);
        } else {
            int first, count;
            leaf_of(g, kslot, first, count);
            if (leaf_isect_in<ANYHIT, STATS>(s, s.prims8, first, count, o, d, tmax, in_object, h, st)) return h;
        }
    }
    return h;
}

// The default walk: the compressed eight-wide tree (RUMI_WALK8), else the binary or the
// four-wide tree by RUMI_BVH_WIDE.
template <bool ANYHIT, int STACK_SMEM, bool STATS, typename SceneOf, typename Fetch, typename Finish>
RUMI_D void traverse_queue_walk(SceneOf scene_of, int n, int *counter, int refill_min, int *smem_stack, int stride,
                                Fetch fetch, Finish finish, TraceStats &st) {
#if RUMI_WALK8
    traverse_queue_ww8<ANYHIT, STACK_SMEM, STATS>(scene_of, n, counter, refill_min, smem_stack, stride, fetch, finish,
                                                  st);
#elif RUMI_BVH_WIDE
    traverse_queue_ww4<ANYHIT, STACK_SMEM, STATS>(scene_of, n, counter, refill_min, smem_stack, stride, fetch, finish,
                                                  st);
#else
    traverse_queue_ww<ANYHIT, STACK_SMEM, STATS>(scene_of, n, counter, refill_min, smem_stack, stride, fetch, finish,
                                                 st);
#endif
}

// Persistent queue traversal shared by every ray kernel.
//   MODE 0: a warp takes 32 rays and traces each to completion.
//   MODE 1: per-lane refill; every iteration advances each ray by one node pair.
//   MODE 2: per-lane refill; interior node pairs until every busy lane holds postponed
//           leaves, then the warp intersects those leaves together.
//   MODE 3: speculative while-while with per-lane refill (traverse_queue_ww).
//   MODE 4: the same walk over the compressed eight-wide tree (traverse_queue_ww8).
// fetch(i, o, d, tmax, in_obj) loads ray i; finish(i, hit) consumes its result.
template <int MODE, bool ANYHIT, int STACK_SMEM, bool STATS, typename Fetch, typename Finish>
RUMI_D void traverse_queue(const DevScene &s, int n, int *counter, int refill_min, int *smem_stack, int stride,
                           Fetch fetch, Finish finish, TraceStats &st) {
#ifdef RUMI_HOST_BUILD
    // Host build of the kernels (CPU tests under sanitizers): one emulated thread takes
    // the queue's rays one after another through the per-ray walk; the warp-cooperative
    // schemes above have no single-thread form.
    (void)refill_min;
    for (;;) {
        const int i = atomicAdd(counter, 1);
        if (i >= n) return;
        float3 o, d;
        float tmax;
        bool in_obj;
        fetch(i, o, d, tmax, in_obj);
        finish(i, trace_ray<ANYHIT, STACK_SMEM, STATS>(s, o, d, tmax, in_obj, smem_stack, stride, st));
    }
#endif
    const int lane = threadIdx.x & 31;
    int spill[RUMI_MAX_BVH_DEPTH - STACK_SMEM > 0 ? RUMI_MAX_BVH_DEPTH - STACK_SMEM : 1];
    if (MODE == 3) {
#if RUMI_BVH_WIDE
        traverse_queue_ww4<ANYHIT, STACK_SMEM, STATS>([&](int) { return &s; }, n, counter, refill_min, smem_stack,
                                                      stride, fetch, finish, st);
#else
        traverse_queue_ww<ANYHIT, STACK_SMEM, STATS>([&](int) { return &s; }, n, counter, refill_min, smem_stack,
                                                     stride, fetch, finish, st);
#endif
        return;
    }
    if (MODE == 4) {
        traverse_queue_ww8<ANYHIT, STACK_SMEM, STATS>([&](int) { return &s; }, n, counter, refill_min, smem_stack,
                                                      stride, fetch, finish, st);
        return;
    }
    if (MODE == 0) {
        for (;;) {
            int base = 0;
            if (lane == 0) base = atomicAdd(counter, 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= n) break;
            const int i = base + lane;
            if (i < n) {
                float3 o, d;
                float tmax;
                bool in_obj;
                fetch(i, o, d, tmax, in_obj);
                const HitRec h = trace_ray<ANYHIT, STACK_SMEM, STATS>(s, o, d, tmax, in_obj, smem_stack, stride, st);
                finish(i, h);
            }
        }
        return;
    }
    const unsigned lt = (1u << lane) - 1u;
    TravState T;
    PendingLeaves pl;
    pl.n = 0;
    int ray = -1;
    bool exhausted = false;
    for (int outer = 0;; ++outer) {
        const unsigned idle = __ballot_sync(0xffffffffu, ray < 0);
        if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
            int base = 0;
            const int leader = __ffs(idle) - 1;
            if (lane == leader) base = atomicAdd(counter, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(idle) >= n) exhausted = true;
            if (ray < 0) {
                const int r = base + __popc(idle & lt);
                if (r < n) {
                    ray = r;
                    float3 o, d;
                    float tmax;
                    bool in_obj;
                    fetch(r, o, d, tmax, in_obj);
                    trav_begin<ANYHIT, STATS>(s, T, o, d, tmax, in_obj, st);
                    pl.n = 0;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, ray >= 0) == 0) break;
        if (MODE == 1) {
            if (ray >= 0 && T.cur != -2) trav_step<ANYHIT, STACK_SMEM, STATS>(s, T, smem_stack, stride, spill, st);
        } else {
            for (int it = 0; it < 4 * RUMI_MAX_BVH_DEPTH; ++it) {
                const bool want = ray >= 0 && pl.n == 0 && T.cur != -2;
                if (__ballot_sync(0xffffffffu, want) == 0) break;
                if (want) trav_step_postpone<STACK_SMEM, STATS>(s, T, pl, smem_stack, stride, spill, st);
            }
            if (ray >= 0 && pl.n > 0)
                if (run_pending<ANYHIT, STATS>(s, T, pl, st)) T.cur = -2;
        }
        if (ray >= 0 && T.cur == -2 && pl.n == 0) {
            finish(ray, T.h);
            ray = -1;
        }
    }
}
