// lucid_kernels.cuh — ray/primitive intersection and BVH traversal (device).
//
// Triangle and native-light intersection reproduce the reference's float
// sequences (geometry/intersection.hpp:58-396) so accepted hits and their
// (t, u, v) are identical to the CPU renderer.  BVH box tests are
// conservative instead of exact: boxes are padded and the far distance is
// widened by 2^-20, so the BVH never culls a triangle the exact triangle test
// accepts (the reference's own per-mesh slab test, intersection.hpp:257-302,
// can miss grazing hits; this traversal cannot).
#pragma once

#include "lucid_device.cuh"

namespace lucid {

// Möller–Trumbore (intersection.hpp:335-396) on a triangle stored as
// (v0, e1 = v1 - v0, e2 = v2 - v0); identical operation order, so accepted
// hits and their (t, u, v) equal the reference's bit for bit.
//
// The three IEEE divisions are deferred behind a conservative prefilter on
// the undivided numerators: with D = |det| and s = sign(det), a triangle is
// rejected early only when s*num lies outside the accepted interval by a
// relative margin of 2^-20 (or 2^-18 for u + v), far above the few-ulp
// rounding of the quotients.  Every triangle the prefilter passes is then
// decided by the exact divided test, so the result is unchanged.
LD bool isect_tri(V3 o, V3 d, V3 v0, V3 e1, V3 e2, float tmin, float tmax, float& t, float& u, float& v) {
    V3 pvec = cross(d, e2);
    float det = dot(e1, pvec);
    const float eps = 1e-6f * 1e-6f;
    if (det > -eps && det < eps) return false;
    V3 tvec = o - v0;
    float un = dot(tvec, pvec);
    float D = fabsf(det);
    float sg = det < 0.0f ? -1.0f : 1.0f;
    float a = un * sg;
    const float lo = -D * 9.5367431640625e-07f;            // -D * 2^-20 (exact)
    if (a < lo || a > D * 1.00000095367431640625f) return false;
    V3 qvec = cross(tvec, e1);
    float vn = dot(d, qvec);
    float b = vn * sg;
    if (b < lo || a + b > D * 1.000003814697265625f) return false;   // 1 + 2^-18
    float tn = dot(e2, qvec);
    float c = tn * sg;
    if (c > D * tmax * 1.00000095367431640625f) return false;
    if (c < D * tmin * 0.99999904632568359375f + lo) return false;
    float uu = un / det;
    if (uu < 0.0f || uu > 1.0f) return false;
    float vv = vn / det;
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    float tt = tn / det;
    if (tt >= tmin && tt <= tmax) { t = tt; u = uu; v = vv; return true; }
    return false;
}

struct HitRec {
    float t, u, v;
    int prim;
};

LD void load_tri(const float4* tris, int k, V3& v0, V3& e1, V3& e2, int& prim) {
    float4 a = __ldg(&tris[3 * k]);
    float4 b = __ldg(&tris[3 * k + 1]);
    float4 c = __ldg(&tris[3 * k + 2]);
    v0 = f3(a); e1 = f3(b); e2 = f3(c);
    prim = __float_as_int(a.w);
}

// Closest-hit tie rule: on equal t the larger global prim id wins.  Global
// ids are mesh-major, so across meshes this is the reference's "later mesh
// wins" (bvh.hpp:167-174 passes the running t as an inclusive bound).
LD void test_leaf_closest(const float4* tris, int code, V3 o, V3 d, float tmin, HitRec& h) {
    int w = ~code;
    int start = w >> 3, count = (w & 7) + 1;
    for (int k = start; k < start + count; ++k) {
        V3 v0, e1, e2;
        int prim;
        load_tri(tris, k, v0, e1, e2, prim);
        float t, u, v;
        if (isect_tri(o, d, v0, e1, e2, tmin, h.t, t, u, v)) {
            if (t < h.t || prim > h.prim) { h.t = t; h.u = u; h.v = v; h.prim = prim; }
        }
    }
}
LD bool test_leaf_any(const float4* tris, int code, V3 o, V3 d, float tmin, float tmax) {
    int w = ~code;
    int start = w >> 3, count = (w & 7) + 1;
    for (int k = start; k < start + count; ++k) {
        V3 v0, e1, e2;
        int prim;
        load_tri(tris, k, v0, e1, e2, prim);
        float t, u, v;
        if (isect_tri(o, d, v0, e1, e2, tmin, tmax, t, u, v)) return true;
    }
    return false;
}

// Conservative slab test of one box; returns entry distance in tn.
LD bool box_hit(float4 bmin, float4 bmax, V3 o, V3 inv, float tmin, float tfar_lim, float& tn) {
    float tx0 = (bmin.x - o.x) * inv.x, tx1 = (bmax.x - o.x) * inv.x;
    float ty0 = (bmin.y - o.y) * inv.y, ty1 = (bmax.y - o.y) * inv.y;
    float tz0 = (bmin.z - o.z) * inv.z, tz1 = (bmax.z - o.z) * inv.z;
    float t0 = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float t1 = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tfar_lim));
    tn = t0;
    return t0 <= t1 * 1.00000095367431640625f;   // widen by 2^-20
}

// Brute-force closest / any over a short triangle list (same tie rule).
LD void list_closest(const float4* tris, int count, V3 o, V3 d, float tmin, HitRec& h) {
    for (int k = 0; k < count; ++k) {
        V3 v0, e1, e2;
        int prim;
        load_tri(tris, k, v0, e1, e2, prim);
        float t, u, v;
        if (isect_tri(o, d, v0, e1, e2, tmin, h.t, t, u, v)) {
            if (t < h.t || prim > h.prim) { h.t = t; h.u = u; h.v = v; h.prim = prim; }
        }
    }
}
LD bool list_any(const float4* tris, int count, V3 o, V3 d, float tmin, float tmax) {
    for (int k = 0; k < count; ++k) {
        V3 v0, e1, e2;
        int prim;
        load_tri(tris, k, v0, e1, e2, prim);
        float t, u, v;
        if (isect_tri(o, d, v0, e1, e2, tmin, tmax, t, u, v)) return true;
    }
    return false;
}

// FMA slab test for rays whose origin lies inside the scene bounds (every
// secondary and shadow ray): t = b*inv - o*inv with one fused rounding.  Its
// absolute error, about 5 * max|coordinate| * 2^-24 in distance units, is
// 16x below the 2^-20 * max|coordinate| padding of every BVH box, so the
// test stays conservative.  Camera rays, whose origin can be far outside the
// scene, use box_hit above.
LD bool box_hit_fma(float4 bmin, float4 bmax, V3 ooi, V3 inv, float tmin, float tfar_lim, float& tn) {
    float tx0 = __fmaf_rn(bmin.x, inv.x, ooi.x), tx1 = __fmaf_rn(bmax.x, inv.x, ooi.x);
    float ty0 = __fmaf_rn(bmin.y, inv.y, ooi.y), ty1 = __fmaf_rn(bmax.y, inv.y, ooi.y);
    float tz0 = __fmaf_rn(bmin.z, inv.z, ooi.z), tz1 = __fmaf_rn(bmax.z, inv.z, ooi.z);
    float t0 = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float t1 = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tfar_lim));
    tn = t0;
    return t0 <= t1 * 1.00000095367431640625f;
}

// Traversal stack: a 4-wide node pushes at most three children, so a tree of
// depth D needs at most 3 (D - 1) entries; a binary node pushes at most one,
// so D - 1.  The host checks both bounds.
//
// Closest-hit queries traverse the binary tree and any-hit queries its 4-wide
// collapse: on the 1M-triangle scene the 4-wide tree made shadow rays 17 %
// faster and closest-hit rays 6 % slower than the binary tree.
constexpr int kStack = 96;

// One 4-wide node: its children's boxes tested against a ray.  `fma_form`
// selects the FMA slab form (origins inside the scene) or the subtraction
// form (camera rays); either is conservative (see box_hit / box_hit_fma).
struct Node4 {
    float4 x0, x1, y0, y1, z0, z1;
    int4 c;
};
LD void load_node4(const DevNode4* nodes, int i, Node4& q) {
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    q.x0 = __ldg(p); q.x1 = __ldg(p + 1); q.y0 = __ldg(p + 2); q.y1 = __ldg(p + 3);
    q.z0 = __ldg(p + 4); q.z1 = __ldg(p + 5);
    q.c = __ldg(reinterpret_cast<const int4*>(p + 6));
}
LD float lane4(const float4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
LD int lane4(const int4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

template <bool FMA>
LD bool child_hit(const Node4& q, int k, V3 o, V3 ooi, V3 inv, float tmin, float tfar, float& tn) {
    float4 lo = make_float4(lane4(q.x0, k), lane4(q.y0, k), lane4(q.z0, k), 0.0f);
    float4 hi = make_float4(lane4(q.x1, k), lane4(q.y1, k), lane4(q.z1, k), 0.0f);
    bool h = FMA ? box_hit_fma(lo, hi, ooi, inv, tmin, tfar, tn) : box_hit(lo, hi, o, inv, tmin, tfar, tn);
    return h && lane4(q.c, k) != kEmptyChild;
}

// Four (distance, code) pairs sorted by distance (misses carry +inf).
struct Hits4 {
    float t[4];
    int c[4];
    int n;
};
LD void cswap(Hits4& h, int i, int j) {
    if (h.t[j] < h.t[i]) {
        float t = h.t[i]; h.t[i] = h.t[j]; h.t[j] = t;
        int c = h.c[i]; h.c[i] = h.c[j]; h.c[j] = c;
    }
}
LD void sort4(Hits4& h) {
    cswap(h, 0, 1); cswap(h, 2, 3); cswap(h, 0, 2); cswap(h, 1, 3); cswap(h, 1, 2);
}
template <bool FMA>
LD void node_hits(const Node4& q, V3 o, V3 ooi, V3 inv, float tmin, float tfar, Hits4& h) {
    const float kInf = __int_as_float(0x7f800000);
    h.n = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float tn;
        bool hit = child_hit<FMA>(q, k, o, ooi, inv, tmin, tfar, tn);
        h.t[k] = hit ? tn : kInf;
        h.c[k] = lane4(q.c, k);
        h.n += hit ? 1 : 0;
    }
    sort4(h);
}

// Closest hit over the BVH (non-boundary triangles) in [tmin, h.t].
// Returns false when the traversal stack overflowed (a hit may be missed).
// FMA: the origin lies within the scene's coordinate bound (DevScene::
// coord_bound), so the FMA slab form is conservative (box_hit_fma).
template <bool FMA = false>
LD bool bvh_closest(const DevScene& sc, V3 o, V3 d, float tmin, HitRec& h) {
    if (sc.num_big_tris) list_closest(sc.big_tris, sc.num_big_tris, o, d, tmin, h);
    if (sc.num_bvh_tris == 0) return true;
    if (sc.root2 < 0) { test_leaf_closest(sc.bvh_tris, sc.root2, o, d, tmin, h); return true; }
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const V3 ooi = v3(-o.x * inv.x, -o.y * inv.y, -o.z * inv.z);
    int stack[kStack];
    int sp = 0;
    int node = sc.root2;
    bool ok = true;
    while (true) {
        const DevNode* n = sc.nodes2 + node;
        float4 a = __ldg(&n->lmin_lc), b = __ldg(&n->lmax_rc), c = __ldg(&n->rmin), e = __ldg(&n->rmax);
        int cl = __float_as_int(a.w), cr = __float_as_int(b.w);
        float tl, tr;
        bool hl = FMA ? box_hit_fma(a, b, ooi, inv, tmin, h.t, tl) : box_hit(a, b, o, inv, tmin, h.t, tl);
        bool hr = FMA ? box_hit_fma(c, e, ooi, inv, tmin, h.t, tr) : box_hit(c, e, o, inv, tmin, h.t, tr);
        if (hl && cl < 0) { test_leaf_closest(sc.bvh_tris, cl, o, d, tmin, h); hl = false; }
        if (hr && cr < 0) { test_leaf_closest(sc.bvh_tris, cr, o, d, tmin, h); hr = false; }
        if (hl && hr) {
            int nearc = (tl <= tr) ? cl : cr, farc = (tl <= tr) ? cr : cl;
            if (sp < kStack) stack[sp++] = farc; else ok = false;
            node = nearc;
        } else if (hl) {
            node = cl;
        } else if (hr) {
            node = cr;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return ok;
}

// Any hit over the BVH in [tmin, tmax]; overflow reported through ok.
LD bool bvh_any(const DevScene& sc, V3 o, V3 d, float tmin, float tmax, bool& ok) {
    if (sc.num_big_tris && list_any(sc.big_tris, sc.num_big_tris, o, d, tmin, tmax)) return true;
    if (sc.num_bvh_tris == 0) return false;
    if (sc.root < 0) return test_leaf_any(sc.bvh_tris, sc.root, o, d, tmin, tmax);
    V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    int stack[kStack];
    int sp = 0;
    int node = sc.root;
    for (;;) {
        if (node < 0) {
            if (test_leaf_any(sc.bvh_tris, node, o, d, tmin, tmax)) return true;
        } else {
            Node4 q;
            load_node4(sc.nodes, node, q);
            Hits4 hh;
            node_hits<false>(q, o, o, inv, tmin, tmax, hh);
            if (hh.n > 0) {
#pragma unroll
                for (int k = 3; k >= 1; --k)
                    if (hh.n > k) {
                        if (sp < kStack) stack[sp++] = hh.c[k]; else ok = false;
                    }
                node = hh.c[0];
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return false;
}

// ---- resumable while-while traversal for the persistent kernels ----
// Aila & Laine ("Understanding the efficiency of ray traversal on GPUs",
// HPG 2009): each lane descends internal nodes until it has found a leaf,
// postponing the leaf; the warp leaves the descent loop once every lane holds
// a leaf (or is done), then all lanes test their leaves together.  The stack
// keeps each entry's entry distance so closest-hit queries skip entries that
// a nearer hit has made unreachable.  A lane runs a bounded number of
// descend/test rounds between work refills.
struct Trav {
    V3 o, d, inv, ooi;   // ooi = -o * inv
    float tmin;
    HitRec h;        // closest: running best; any: h.t is the fixed limit
    int node;        // next entry (internal node index or leaf code), or kTravDone
    int leaf;        // postponed leaf code, 0 when none
    int sp;
    bool any_hit;
};
constexpr int kTravDone = 0x7fffffff;

template <bool ANY>
LD void trav_begin(Trav& s, const DevScene& sc, V3 o, V3 d, float tmin, float tmax) {
    s.o = o; s.d = d;
    s.inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    s.ooi = v3(-o.x * s.inv.x, -o.y * s.inv.y, -o.z * s.inv.z);
    s.tmin = tmin;
    s.h.t = tmax; s.h.u = 0.0f; s.h.v = 0.0f; s.h.prim = -1;
    s.sp = 0;
    s.leaf = 0;
    s.any_hit = false;
    s.node = kTravDone;
    if (sc.num_big_tris) {
        if (ANY) {
            if (list_any(sc.big_tris, sc.num_big_tris, o, d, tmin, tmax)) { s.any_hit = true; return; }
        } else {
            list_closest(sc.big_tris, sc.num_big_tris, o, d, tmin, s.h);
        }
    }
    if (sc.num_bvh_tris == 0) return;
    s.node = ANY ? sc.root : sc.root2;   // a leaf code when the whole BVH is one leaf
}

LD int trav_pop(Trav& s, const int* stack, const float* stack_t) {
    while (s.sp > 0) {
        --s.sp;
        if (stack_t[s.sp] <= s.h.t * 1.00000095367431640625f) return stack[s.sp];
    }
    return kTravDone;
}

// Any-hit stepping for shadow rays: leaves are tested as soon as they are
// reached (an occluder found early ends the ray), one node or leaf per step.
LD bool trav_run_any(Trav& s, int* stack, const DevScene& sc, bool& ok, int steps) {
    for (int k = 0; k < steps; ++k) {
        if (s.node == kTravDone) return true;
        if (s.node < 0) {
            if (test_leaf_any(sc.bvh_tris, s.node, s.o, s.d, s.tmin, s.h.t)) {
                s.any_hit = true;
                s.node = kTravDone;
                return true;
            }
        } else {
            Node4 q;
            load_node4(sc.nodes, s.node, q);
            Hits4 hh;
            node_hits<true>(q, s.o, s.ooi, s.inv, s.tmin, s.h.t, hh);
            if (hh.n > 0) {
#pragma unroll
                for (int j = 3; j >= 1; --j)
                    if (hh.n > j) {
                        if (s.sp < kStack) stack[s.sp++] = hh.c[j]; else ok = false;
                    }
                s.node = hh.c[0];
                continue;
            }
        }
        if (s.sp == 0) {
            s.node = kTravDone;
            return true;
        }
        s.node = stack[--s.sp];
    }
    return false;
}

// Runs up to `rounds` descend/test rounds; returns true when finished.
template <bool ANY>
LD bool trav_run(Trav& s, int* stack, float* stack_t, const DevScene& sc, bool& ok, int rounds) {
    static_assert(!ANY, "any-hit rays use trav_run_any over the 4-wide tree");
    for (int r = 0; r < rounds; ++r) {
        // descend until this lane holds a leaf (speculatively with its warp)
        while (s.node != kTravDone && s.leaf == 0) {
            if (s.node < 0) {                      // a leaf reached by popping
                s.leaf = s.node;
                s.node = trav_pop(s, stack, stack_t);
                break;
            }
            const DevNode* n = sc.nodes2 + s.node;
            float4 a = __ldg(&n->lmin_lc), b = __ldg(&n->lmax_rc), c = __ldg(&n->rmin), e = __ldg(&n->rmax);
            int cl = __float_as_int(a.w), cr = __float_as_int(b.w);
            float tl, tr;
            bool hl = box_hit_fma(a, b, s.ooi, s.inv, s.tmin, s.h.t, tl);
            bool hr = box_hit_fma(c, e, s.ooi, s.inv, s.tmin, s.h.t, tr);
            if (hl && hr) {
                bool lfirst = tl <= tr;
                if (s.sp < kStack) {
                    stack[s.sp] = lfirst ? cr : cl;
                    stack_t[s.sp] = lfirst ? tr : tl;
                    ++s.sp;
                } else {
                    ok = false;
                }
                s.node = lfirst ? cl : cr;
            } else if (hl) {
                s.node = cl;
            } else if (hr) {
                s.node = cr;
            } else {
                s.node = trav_pop(s, stack, stack_t);
            }
            if (s.node != kTravDone && s.node < 0) {   // postpone the leaf, keep descending
                s.leaf = s.node;
                s.node = trav_pop(s, stack, stack_t);
            }
            if (!__any_sync(__activemask(), s.leaf == 0 && s.node != kTravDone)) break;
        }
        if (s.leaf != 0) {
            if (ANY) {
                if (test_leaf_any(sc.bvh_tris, s.leaf, s.o, s.d, s.tmin, s.h.t)) {
                    s.any_hit = true;
                    s.node = kTravDone;
                    s.leaf = 0;
                    return true;
                }
            } else {
                test_leaf_closest(sc.bvh_tris, s.leaf, s.o, s.d, s.tmin, s.h);
            }
            s.leaf = 0;
        }
        if (s.node == kTravDone) return true;
    }
    return false;
}

// Closest boundary-only triangle in [tmin, h.t] over the whole list, one
// triangle after another.
LD void boundary_closest_all(const DevScene& sc, V3 o, V3 d, float tmin, HitRec& h) {
    for (int k = 0; k < sc.num_bnd_tris; ++k) {
        V3 v0, e1, e2;
        int prim;
        load_tri(sc.bnd_tris, k, v0, e1, e2, prim);
        float t, u, v;
        if (isect_tri(o, d, v0, e1, e2, tmin, h.t, t, u, v)) {
            if (t < h.t || prim > h.prim) { h.t = t; h.u = u; h.v = v; h.prim = prim; }
        }
    }
}

// Closest boundary-only triangle in [tmin, h.t] by brute force (these are the
// few triangles of volume-domain cubes), one mesh's group at a time; with
// BOXES, behind the conservative test of the group's padded box (inv = the
// componentwise reciprocal of d).
template <bool BOXES>
LD void boundary_closest(const DevScene& sc, V3 o, V3 d, V3 inv, float tmin, HitRec& h) {
    for (int g = 0; g < sc.num_bnd_groups; ++g) {
        const float4 lo = __ldg(&sc.bnd_box[2 * g]), hi = __ldg(&sc.bnd_box[2 * g + 1]);
        float tn;
        if (BOXES && !box_hit(lo, hi, o, inv, tmin, h.t, tn)) continue;
        const int first = __float_as_int(lo.w), end = first + __float_as_int(hi.w);
        for (int k = first; k < end; ++k) {
            V3 v0, e1, e2;
            int prim;
            load_tri(sc.bnd_tris, k, v0, e1, e2, prim);
            float t, u, v;
            if (isect_tri(o, d, v0, e1, e2, tmin, h.t, t, u, v)) {
                if (t < h.t || prim > h.prim) { h.t = t; h.u = u; h.v = v; h.prim = prim; }
            }
        }
    }
}

// intersectScene over every triangle (geometry/bvh.hpp:155-177).
LD HitRec scene_closest(const DevScene& sc, V3 o, V3 d, float tmin, float tmax, bool& ok) {
    HitRec h;
    h.t = tmax; h.u = 0.0f; h.v = 0.0f; h.prim = -1;
    ok &= bvh_closest(sc, o, d, tmin, h);
    if (sc.num_bnd_tris) boundary_closest<true>(sc, o, d, v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z), tmin, h);
    return h;
}

// intersect_skipping_volume_boundaries (path_tracer.hpp:82-95): the closest
// non-boundary hit after skipping at most 8 boundary hits, each skip moving
// the search start 1 mm past the boundary.  The real-surface BVH query is
// reused while its hit stays beyond the advanced search start.
template <bool FMA = false>
LD HitRec closest_skip_boundaries(const DevScene& sc, V3 o, V3 d, float tmin, bool& ok) {
    HitRec real;
    real.t = 1e30f; real.u = 0.0f; real.v = 0.0f; real.prim = -1;
    ok &= bvh_closest<FMA>(sc, o, d, tmin, real);
    if (!sc.num_bnd_tris) return real;
    const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float search = tmin;
    HitRec none;
    none.t = 1e30f; none.u = 0.0f; none.v = 0.0f; none.prim = -1;
    for (int peek = 0; peek < 8; ++peek) {
        if (real.prim >= 0 && real.t < search) {
            real = none;
            ok &= bvh_closest<FMA>(sc, o, d, search, real);
        }
        HitRec b;
        b.t = (real.prim >= 0) ? real.t : 1e30f; b.u = 0.0f; b.v = 0.0f;
        b.prim = (real.prim >= 0) ? real.prim : -1;
        int real_prim = b.prim;
        boundary_closest<true>(sc, o, d, inv, search, b);
        if (b.prim < 0) return none;                 // no hit at all
        if (b.prim == real_prim) return real;        // the real surface is closest
        search = b.t + 1e-3f;                        // skip the boundary hit
    }
    return none;
}

// is_shadowed_skipping_volume_boundaries (path_tracer.hpp:103-119).
LD bool shadowed_skip_boundaries(const DevScene& sc, V3 o, V3 d, float tmax, bool& ok) {
    if (!sc.num_bnd_tris) {
        if (tmax <= 0.0f) return false;
        return bvh_any(sc, o, d, RAY_T_MIN, tmax, ok);
    }
    const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    V3 po = o;
    float off = 0.0f;
    for (int peek = 0; peek < 8; ++peek) {
        float rem = tmax - off;
        if (rem <= 0.0f) return false;
        HitRec b;
        b.t = rem; b.u = 0.0f; b.v = 0.0f; b.prim = -1;
        boundary_closest<true>(sc, po, d, inv, RAY_T_MIN, b);
        if (b.prim < 0) return bvh_any(sc, po, d, RAY_T_MIN, rem, ok);
        if (bvh_any(sc, po, d, RAY_T_MIN, b.t, ok)) return true;
        float skip = b.t + 1e-3f;
        off += skip;
        po = po + d * skip;
    }
    return false;
}

// ---- native-light shapes (intersection.hpp:58-236) ----
LD bool isect_sphere(V3 o, V3 d, V3 c, float radius, float& th) {
    V3 oc = o - c;
    float b = 2.0f * dot(oc, d);
    float cc = len2(oc) - radius * radius;
    float disc = b * b - 4.0f * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(smax(0.0f, disc));
    float t = (-b - sq) / 2.0f;
    if (t < RAY_T_MIN) {
        t = (-b + sq) / 2.0f;
        if (t < RAY_T_MIN) return false;
    }
    th = t;
    return true;
}
LD bool isect_planar(V3 o, V3 d, V3 c, V3 n, V3 right, V3 up, float& t, float& x, float& y) {
    float den = dot(d, n);
    if (fabsf(den) < 1e-6f) return false;
    float num = dot(c - o, n);
    t = num / den;
    if (t < RAY_T_MIN) return false;
    V3 lh = (o + d * t) - c;
    x = dot(lh, right);
    y = dot(lh, up);
    return true;
}

// intersectNativeLights (scene_lights.hpp:176-246): index into the native
// light list and distance of the closest light hit nearer than `bound`, or
// -1 (bound 1e30: every hit).  Each light is first tested against its
// bounding sphere (light_bsph): skipped when the ray's line passes farther
// than the radius from the centre, or when the whole sphere lies behind the
// ray or beyond the nearest hit so far.  Both rejections keep a relative
// margin of 1e-5 over the few-ulp rounding of the exact tests below (whose
// accepted points lie on the light, inside the sphere), so they only skip
// lights the exact test would reject.
LD int native_lights_closest(const DevScene& sc, V3 o, V3 d, float bound, float& t_out) {
    int best = -1;
    float bt = bound;
    for (int i = 0; i < sc.num_native; ++i) {
        const float4 bs = __ldg(&sc.light_bsph[i]);
        if (!(bs.w >= 0.0f)) continue;
        const V3 oc = v3(bs.x - o.x, bs.y - o.y, bs.z - o.z);
        const float tca = dot(oc, d), oc2 = dot(oc, oc), r = bs.w;
        if (oc2 - tca * tca > r * r + 1e-5f * oc2) continue;                  // the line misses the sphere
        const float slack = 1e-5f * (fabsf(tca) + r) + 1e-30f;
        if (tca + r < RAY_T_MIN - slack || tca - r > bt + slack) continue;   // behind the ray / beyond bt
        const DevLight& L = sc.lights[sc.native_start + i];
        int type = __float_as_int(L.pos_type.w);
        float t;
        if (type == LIGHT_POINT) {
            float radius = L.emission_radius.w;
            if (radius > MIN_LENGTH && isect_sphere(o, d, f3(L.pos_type), radius, t) && t < bt) { bt = t; best = i; }
        } else if (type == LIGHT_AREA) {
            int shape = __float_as_int(L.v0_shape.w);
            float x, y;
            V3 n = f3(L.normal_area);
            bool h = isect_planar(o, d, f3(L.pos_type), n, f3(L.right_sx), f3(L.up_sy), t, x, y);
            if (h) {
                if (shape == AREA_DISK || shape == AREA_ELLIPSE) {
                    float nx = x / (L.right_sx.w * 0.5f), ny = y / (L.up_sy.w * 0.5f);
                    h = !(nx * nx + ny * ny > 1.0f);
                } else {
                    float hx = L.right_sx.w * 0.5f, hy = L.up_sy.w * 0.5f;
                    h = !(x * x > hx * hx || y * y > hy * hy);
                }
            }
            if (h && t < bt && dot(n, d) < 0) { bt = t; best = i; }
        }
    }
    t_out = bt;
    return best;
}

}  // namespace lucid
