// lucid_oracle.hpp — CPU restatement of the Lucid renderer's progressive
// path-tracing hot path.  TEST INFRASTRUCTURE ONLY: this is the parity oracle
// and the timed CPU baseline ("port").  Nothing in the product links it.
//
// Every function follows the reference C++ core (paths relative to
// LucidRenderer/cpp_renderer/) with the same FP32 operation order.  The
// mp-units type layer of the reference (units/render_units.hpp) is compile-time
// only: all its units are SI-coherent with magnitude 1, so each typed
// operation is restated here as the plain float operation it compiles to.
//
// Two deliberate pins, both documented at their sites:
//   * RNG draws passed as call arguments are taken left to right (the
//     reference's pinned toolchain, Apple Clang, evaluates left to right;
//     g++ would evaluate right to left).
//   * Transcendentals: "faithful" mode calls libm like the reference;
//     "device" mode calls lucid_math.h, which the CUDA kernels also use, so
//     GPU and oracle can be compared bit for bit.
//   * Optional canonical tie rule: on exactly equal hit distances within one
//     mesh the larger triangle index wins (the reference's winner depends on
//     its BVH's nth_element partition order, which differs between standard
//     libraries).  Across meshes the reference already lets the later mesh
//     win, which equals "largest (mesh, tri)".
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../blender-lucid-renderer_b200/csrc/lucid_math.h"
#include "oracle_nodes.hpp"

namespace orc {

// ------------------------------------------------------------------ options
struct Options {
    bool device_math = true;      // lucid_math.h instead of libm
    bool canonical_ties = true;   // see header comment
    // Draws passed together as call arguments (sampleBSDF's three, sampleLight's
    // and hg_sample's two: path_tracer.hpp:533,503,683) taken right to left, the
    // order g++ gives the reference when it is built here; false = left to
    // right, the reference's own toolchain and the product.
    bool draw_rtl = false;
};
inline Options& opts() { static Options o; return o; }

inline float osin(float x) { return opts().device_math ? lucid_math::lm_sinf(x) : std::sin(x); }
inline float ocos(float x) { return opts().device_math ? lucid_math::lm_cosf(x) : std::cos(x); }
inline float oexp(float x) { return opts().device_math ? lucid_math::lm_expf(x) : std::exp(x); }
inline float olog(float x) { return opts().device_math ? lucid_math::lm_logf(x) : std::log(x); }
inline float opow5(float x) { return opts().device_math ? lucid_math::lm_pow5(x) : std::pow(x, 5.0f); }

// std::min / std::max / std::clamp semantics (NaN propagation included).
inline float smin(float a, float b) { return (b < a) ? b : a; }
inline float smax(float a, float b) { return (a < b) ? b : a; }
inline float smax3(float a, float b, float c) { float m = a; if (m < b) m = b; if (m < c) m = c; return m; }
inline float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

constexpr float kPI = 3.14159274101257324219f;         // std::numbers::pi_v<float>
constexpr float kINV_PI = 0.31830987334251403809f;     // std::numbers::inv_pi_v<float>
constexpr float kTWO_PI = 2.0f * kPI;                  // 2.0f * GGX_PI (exact)
constexpr float kDirEps = 1e-6f;
constexpr float kDirEps2 = kDirEps * kDirEps;          // render_units.hpp:480-481
constexpr float kAreaEps = kDirEps * kDirEps;          // area_epsilon()
constexpr float MIN_PDF = 1e-6f;
constexpr float MIN_AREA = 1e-6f;
constexpr float MIN_LENGTH = 1e-6f;
constexpr float RAY_T_MIN = 1e-4f;                     // intersection.hpp:24
constexpr float RAY_T_MAX = 1e30f;
constexpr float GGX_EPSILON = 1e-6f;
constexpr float MIN_ROUGHNESS = 0.01f;

// ------------------------------------------------------------------ vectors
// render_units.hpp:55-160 (Vec3f): componentwise ops, dot = (xx'+yy')+zz'.
struct V3 {
    float x = 0, y = 0, z = 0;
    V3() = default;
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
    V3 operator+(V3 o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(V3 o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator-() const { return {-x, -y, -z}; }
    V3 operator*(float s) const { return {x * s, y * s, z * s}; }
    V3 operator/(float s) const { return {x / s, y / s, z / s}; }
    float len2() const { return x * x + y * y + z * z; }
    float len() const { return std::sqrt(len2()); }
};
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalize(V3 v) { float l = v.len(); if (l > 0.0f) return v / l; return v; }

// make_direction (render_units.hpp:485-494): nullopt below 1e-6 length.
inline bool make_dir(V3 v, V3& out) {
    float l2 = v.len2();
    if (l2 < kDirEps2) return false;
    out = v / std::sqrt(l2);
    return true;
}
inline V3 make_dir_or(V3 v, V3 fb = V3(0, 0, 1)) { V3 d; return make_dir(v, d) ? d : fb; }
inline V3 make_normal_or(V3 v, V3 fb = V3(0, 1, 0)) { V3 d; return make_dir(v, d) ? d : fb; }
// normalize_with_length (render_units.hpp:721-725)
inline void nwl(V3 v, V3& dir, float& len) { len = v.len(); dir = v / len; }

// reflect / refract (render_units.hpp:836-858)
inline V3 reflect(V3 i, V3 n) {
    float cos_i = dot(i, n);
    V3 r = i - n * (2.0f * cos_i);
    return make_dir_or(r);
}
inline bool refract(V3 i, V3 n, float eta, V3& out) {
    float cos_i = -dot(i, n);
    float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
    if (sin2_t > 1.0f) return false;
    float cos_t = std::sqrt(1.0f - sin2_t);
    V3 r = i * eta + n * (eta * cos_i - cos_t);
    return make_dir(r, out);
}

struct RGB {
    float r = 0, g = 0, b = 0;
    RGB() = default;
    RGB(float a, float bb, float c) : r(a), g(bb), b(c) {}
    RGB operator+(RGB o) const { return {r + o.r, g + o.g, b + o.b}; }
    RGB operator*(float s) const { return {r * s, g * s, b * s}; }
};
// Hadamard products: the reference writes {rad.r * t.r, ...}; IEEE
// multiplication is commutative so the operand order does not matter.
inline RGB mul(RGB a, RGB b) { return {a.r * b.r, a.g * b.g, a.b * b.b}; }
inline float luminance(RGB c) { return 0.2126f * c.r + 0.7152f * c.g + 0.0722f * c.b; }
inline bool is_emissive(RGB e) { return luminance(e) > 1e-6f; }
inline bool rgb_valid(RGB c) {
    return !std::isnan(c.r) && !std::isnan(c.g) && !std::isnan(c.b) &&
           !std::isinf(c.r) && !std::isinf(c.g) && !std::isinf(c.b);
}

// ------------------------------------------------------------------ RNG
// math/random.hpp:24-120
struct Rng {
    uint64_t state = 0x853c49e6748fea9bULL, inc = 0xda3e39cb94b95bdbULL;
};
inline uint32_t murmur3_finalize(uint32_t h) {
    h ^= h >> 16; h *= 0x85ebca6bU; h ^= h >> 13; h *= 0xc2b2ae35U; h ^= h >> 16; return h;
}
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
inline uint32_t jenkins_hash(uint32_t a) {
    a = (a + 0x7ed55d16) + (a << 12);
    a = (a ^ 0xc761c23c) ^ (a >> 19);
    a = (a + 0x165667b1) + (a << 5);
    a = (a + 0xd3a2646c) ^ (a << 9);
    a = (a + 0xfd7046c5) + (a << 3);
    a = (a ^ 0xb55a4f09) ^ (a >> 16);
    return a;
}
inline void seed_xyz(Rng& s, uint32_t x, uint32_t y, uint32_t sidx) {
    uint32_t h1 = jenkins_hash(x + 1);
    uint32_t h2 = jenkins_hash(y + 1 + h1);
    uint32_t h3 = jenkins_hash(sidx + 1 + h2);
    uint64_t seed1 = ((uint64_t)murmur3_finalize(h1 ^ h3) << 32) | murmur3_finalize(h2);
    uint64_t seed2 = ((uint64_t)murmur3_finalize(h2 ^ h1) << 32) | murmur3_finalize(h3);
    uint64_t stream = splitmix64(seed1);
    uint64_t initseq = splitmix64(seed2);
    s.inc = (stream << 1u) | 1u;
    s.state = 0;
    s.state = s.state * 6364136223846793005ULL + s.inc;
    s.state += initseq;
    s.state = s.state * 6364136223846793005ULL + s.inc;
    for (int i = 0; i < 8; i++) s.state = s.state * 6364136223846793005ULL + s.inc;
}
inline uint32_t pcg32(Rng& s) {
    uint64_t old = s.state;
    s.state = old * 6364136223846793005ULL + s.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}
inline float randf(Rng& s) { return std::ldexp((float)(pcg32(s) >> 9), -23); }
// Two / three draws that the reference passes as arguments of one call.
inline void draw2(Rng& s, float& u1, float& u2) {
    if (opts().draw_rtl) { u2 = randf(s); u1 = randf(s); }
    else { u1 = randf(s); u2 = randf(s); }
}
inline void draw3(Rng& s, float& u1, float& u2, float& u3) {
    if (opts().draw_rtl) { u3 = randf(s); u2 = randf(s); u1 = randf(s); }
    else { u1 = randf(s); u2 = randf(s); u3 = randf(s); }
}

// ------------------------------------------------------------------ scene
// core/material.hpp, core/scene.hpp, light/light.hpp
struct Volume {
    RGB color{1, 1, 1}, absorption{0, 0, 0};
    float density = 0, anisotropy = 0;
    std::vector<float> grid;
    int dims[3] = {0, 0, 0};
    float wmin[3] = {0, 0, 0}, wmax[3] = {0, 0, 0};
    float grid_max = 0;
    bool present() const { return density > 0.0f || has_grid(); }
    bool has_grid() const { return !grid.empty() && dims[0] > 0 && dims[1] > 0 && dims[2] > 0; }
};
struct Material {
    RGB albedo{0.8f, 0.8f, 0.8f};
    float metallic = 0, roughness = 0.5f;
    RGB emission{0, 0, 0};
    float transmission = 0, ior = 1.45f;
    bool use_nodes = false;       // "use_nodes" and a valid node tree (pybind_renderer.hpp:1381-1384)
    NodeTree tree;
    Volume volume;
    bool volume_boundary_only = false;
};
inline RGB mat_emission(const Material& m, V2 uv) {   // getEmission (path_tracer.hpp:67-72)
    if (!m.use_nodes) return m.emission;
    C3 e = node_emission(m.tree, uv);
    return RGB(e.r, e.g, e.b);
}
struct Tri {
    int i0 = 0, i1 = 0, i2 = 0;
    V3 face_n{0, 1, 0};
    V3 n0{0, 1, 0}, n1{0, 1, 0}, n2{0, 1, 0};
    V3 centroid;
    bool smooth = false;
    V2 uv0, uv1, uv2;             // "triangle_uvs" (pybind_renderer.hpp:1296-1336)
    bool has_uv = false;
};
struct BNode { V3 bmin, bmax; int left = -1, right = -1, tri_start = 0, tri_count = 0; };
struct Mesh {
    std::vector<V3> verts;
    std::vector<Tri> tris;
    Material mat;
    std::vector<BNode> nodes;
    std::vector<int> tri_idx;
    V3 bmin{1e30f, 1e30f, 1e30f}, bmax{-1e30f, -1e30f, -1e30f};
};
enum class LightType { EMISSIVE_MESH, POINT, SUN, SPOT, AREA };
enum class AreaShape { SQUARE, RECTANGLE, DISK, ELLIPSE };
struct Light {
    LightType type = LightType::EMISSIVE_MESH;
    V3 position{0, 0, 0};
    V3 normal{0, 0, 1};
    RGB emission{0, 0, 0};
    float area = 0;
    int mesh = -1, tri = -1;
    V3 v0, v1, v2;
    float energy = 1, radius = 0, spot_angle = 0, spot_blend = 0;
    V3 right{1, 0, 0}, up{0, 1, 0};
    float size_x = 1, size_y = 1;
    AreaShape shape = AreaShape::SQUARE;
};
struct Camera {
    V3 pos{0, 0, 0}, dir{0, 0, 1}, up{0, 1, 0}, right{1, 0, 0}, forward{0, 0, 1};
    float fov = 60.0f * (kPI / 180.0f);
    float aspect = 1.0f;
};
struct Scene {
    std::vector<Mesh> meshes;
    std::vector<Light> native;
    RGB env_color{0.05f, 0.05f, 0.05f};
    float env_strength = 1.0f;
};

// ------------------------------------------------------------------ BVH build
// core/scene.hpp:65-152 (median split on the longest axis, leaf <= 4).
inline int bvh_build_rec(Mesh& m, int start, int end) {
    int idx = (int)m.nodes.size();
    m.nodes.push_back(BNode());
    V3 bmin(1e30f, 1e30f, 1e30f), bmax(-1e30f, -1e30f, -1e30f);
    for (int i = start; i < end; ++i) {
        const Tri& t = m.tris[m.tri_idx[i]];
        for (int v = 0; v < 3; ++v) {
            const V3& p = m.verts[v == 0 ? t.i0 : (v == 1 ? t.i1 : t.i2)];
            bmin = V3(smin(bmin.x, p.x), smin(bmin.y, p.y), smin(bmin.z, p.z));
            bmax = V3(smax(bmax.x, p.x), smax(bmax.y, p.y), smax(bmax.z, p.z));
        }
    }
    m.nodes[idx].bmin = bmin;
    m.nodes[idx].bmax = bmax;
    int count = end - start;
    if (count <= 4) {
        m.nodes[idx].tri_start = start;
        m.nodes[idx].tri_count = count;
        return idx;
    }
    V3 ext = bmax - bmin;
    int axis = 0;
    if (ext.y > ext.x) axis = 1;
    if (ext.z > (axis == 0 ? ext.x : ext.y)) axis = 2;
    int mid = (start + end) / 2;
    std::nth_element(m.tri_idx.begin() + start, m.tri_idx.begin() + mid, m.tri_idx.begin() + end,
                     [&](int a, int b) {
                         const V3& ca = m.tris[a].centroid;
                         const V3& cb = m.tris[b].centroid;
                         float pa = axis == 0 ? ca.x : (axis == 1 ? ca.y : ca.z);
                         float pb = axis == 0 ? cb.x : (axis == 1 ? cb.y : cb.z);
                         return pa < pb;
                     });
    int l = bvh_build_rec(m, start, mid);
    int r = bvh_build_rec(m, mid, end);
    m.nodes[idx].left = l;
    m.nodes[idx].right = r;
    return idx;
}

// core/scene.hpp:191-227 finalizeMeshBounds (bounds, 1 mm padding, face
// normals, BVH build).
inline void finalize_mesh(Mesh& m) {
    for (const V3& v : m.verts) {
        m.bmin = V3(smin(m.bmin.x, v.x), smin(m.bmin.y, v.y), smin(m.bmin.z, v.z));
        m.bmax = V3(smax(m.bmax.x, v.x), smax(m.bmax.y, v.y), smax(m.bmax.z, v.z));
    }
    const float eps = 0.001f;
    V3 ext = m.bmax - m.bmin;
    if (ext.x < eps) { m.bmin = m.bmin - V3(1, 0, 0) * eps; m.bmax = m.bmax + V3(1, 0, 0) * eps; }
    if (ext.y < eps) { m.bmin = m.bmin - V3(0, 1, 0) * eps; m.bmax = m.bmax + V3(0, 1, 0) * eps; }
    if (ext.z < eps) { m.bmin = m.bmin - V3(0, 0, 1) * eps; m.bmax = m.bmax + V3(0, 0, 1) * eps; }
    for (Tri& t : m.tris) {
        V3 e1 = m.verts[t.i1] - m.verts[t.i0];
        V3 e2 = m.verts[t.i2] - m.verts[t.i0];
        V3 n;
        if (make_dir(cross(e1, e2), n)) t.face_n = n;
    }
    if (m.tris.empty()) return;
    m.tri_idx.resize(m.tris.size());
    for (size_t i = 0; i < m.tris.size(); ++i) {
        m.tri_idx[i] = (int)i;
        Tri& t = m.tris[i];
        const V3& a = m.verts[t.i0];
        const V3& b = m.verts[t.i1];
        const V3& c = m.verts[t.i2];
        V3 ab = b - a, ac = c - a;
        t.centroid = a + (ab + ac) / 3.0f;
    }
    m.nodes.reserve(2 * m.tris.size());
    bvh_build_rec(m, 0, (int)m.tris.size());
}

// ------------------------------------------------------------------ intersection
// geometry/intersection.hpp
struct Ray { V3 o, d; V3 at(float t) const { return o + d * t; } };

inline V3 inv_dir(V3 d) {   // intersection.hpp:412-419
    return V3(std::fabs(d.x) > 1e-8f ? 1.0f / d.x : 0.0f,
              std::fabs(d.y) > 1e-8f ? 1.0f / d.y : 0.0f,
              std::fabs(d.z) > 1e-8f ? 1.0f / d.z : 0.0f);
}

inline bool axis_slab(float dc, float ic, float dmin, float dmax, float& tmin, float& tmax) {
    if (std::fabs(dc) < 1e-8f) {
        bool outP = (dmin > 0.0f && dmax > 0.0f);
        bool outN = (dmin < 0.0f && dmax < 0.0f);
        return !(outP || outN);
    }
    float t1 = dmin * ic, t2 = dmax * ic;
    float amin = smin(t1, t2), amax = smax(t1, t2);
    tmin = smax(tmin, amin);
    tmax = smin(tmax, amax);
    return tmax >= tmin;
}
// intersection.hpp:257-302
inline bool isect_aabb(const Ray& r, V3 inv, V3 bmin, V3 bmax) {
    V3 tmn = bmin - r.o, tmx = bmax - r.o;
    float tmin = RAY_T_MIN * 0.0f, tmax = RAY_T_MAX;
    if (!axis_slab(r.d.x, inv.x, tmn.x, tmx.x, tmin, tmax)) return false;
    if (!axis_slab(r.d.y, inv.y, tmn.y, tmx.y, tmin, tmax)) return false;
    if (!axis_slab(r.d.z, inv.z, tmn.z, tmx.z, tmin, tmax)) return false;
    return tmax >= smax(tmin, 0.0f);
}
// intersection.hpp:335-396 (Möller–Trumbore)
inline bool isect_tri(const Ray& r, V3 v0, V3 v1, V3 v2, float& u, float& v, float& t,
                      float tMin, float tMax) {
    V3 e1 = v1 - v0, e2 = v2 - v0;
    V3 pvec = cross(r.d, e2);
    float det = dot(e1, pvec);
    if (det > -kAreaEps && det < kAreaEps) return false;
    V3 tvec = r.o - v0;
    float un = dot(tvec, pvec);
    float uu = un / det;
    if (uu < 0.0f || uu > 1.0f) return false;
    V3 qvec = cross(tvec, e1);
    float vn = dot(r.d, qvec);
    float vv = vn / det;
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    float tn = dot(e2, qvec);
    float tt = tn / det;
    if (tt >= tMin && tt <= tMax) { u = uu; v = vv; t = tt; return true; }
    return false;
}

struct Hit {
    bool hit = false;
    float t = 1e30f;
    V3 point{0, 0, 0};
    V3 normal{0, 1, 0};
    const Material* mat = nullptr;
    int mesh = -1, tri = -1;
    V2 uv;                        // (0, 0) when the hit triangle has no UVs
};

// geometry/bvh.hpp:34-142
inline void traverse(const Mesh& m, const Ray& r, V3 inv, Hit& res, int mi, float tMin, float tMax) {
    float cur = smin(tMax, res.t);
    if (m.nodes.empty()) return;   // meshes without triangles have no BVH
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        int ni = stack[--sp];
        const BNode& n = m.nodes[ni];
        if (!isect_aabb(r, inv, n.bmin, n.bmax)) continue;
        if (n.tri_count > 0) {
            for (int i = 0; i < n.tri_count; ++i) {
                int ti = m.tri_idx[n.tri_start + i];
                const Tri& tr = m.tris[ti];
                float u, v, t;
                if (!isect_tri(r, m.verts[tr.i0], m.verts[tr.i1], m.verts[tr.i2], u, v, t, tMin, cur)) continue;
                if (opts().canonical_ties && res.hit && t == res.t && res.mesh == mi && res.tri > ti) continue;
                cur = t;
                res.t = t;
                res.point = r.at(t);
                float w = 1.0f - u - v;
                if (tr.smooth) {
                    V3 ni3 = tr.n0 * w + tr.n1 * u + tr.n2 * v;
                    res.normal = make_normal_or(ni3, tr.face_n);
                } else {
                    res.normal = tr.face_n;
                }
                res.hit = true;
                res.mat = &m.mat;
                res.mesh = mi;
                res.tri = ti;
                // bvh.hpp:67-72 (the closest triangle's own UVs; the reference
                // leaves an earlier candidate's uv in place when it has none)
                res.uv = tr.has_uv ? V2{tr.uv0.x * w + tr.uv1.x * u + tr.uv2.x * v, tr.uv0.y * w + tr.uv1.y * u + tr.uv2.y * v}
                                   : V2{};
            }
        } else {
            if (sp < 62) {
                if (n.right >= 0) stack[sp++] = n.right;
                if (n.left >= 0) stack[sp++] = n.left;
            }
        }
    }
}

// geometry/bvh.hpp:155-177
inline Hit intersect_scene(const Scene& s, const Ray& r, float tMin = RAY_T_MIN, float tMax = RAY_T_MAX) {
    Hit res;
    res.t = tMax;
    res.point = V3(0, 0, 0);
    res.normal = V3(0, 1, 0);
    res.hit = false;
    V3 inv = inv_dir(r.d);
    for (size_t mi = 0; mi < s.meshes.size(); ++mi) {
        const Mesh& m = s.meshes[mi];
        if (!isect_aabb(r, inv, m.bmin, m.bmax)) continue;
        traverse(m, r, inv, res, (int)mi, tMin, res.t);
    }
    return res;
}

// intersection.hpp:58-236 (native-light shapes)
inline bool isect_sphere(const Ray& r, V3 c, float radius, float& tHit, V3& n) {
    V3 oc = r.o - c;
    float b = 2.0f * dot(oc, r.d);
    float cc = oc.len2() - radius * radius;
    float disc = b * b - 4.0f * cc;
    if (disc < 0.0f) return false;
    float sq = std::sqrt(smax(0.0f, disc));
    float t = (-b - sq) / 2.0f;
    if (t < RAY_T_MIN) {
        t = (-b + sq) / 2.0f;
        if (t < RAY_T_MIN) return false;
    }
    tHit = t;
    V3 hp = r.o + r.d * t;
    n = normalize(hp - c);
    return true;
}
inline bool isect_planar(const Ray& r, V3 c, V3 n, V3 right, V3 up, float& t, V3& hp, float& x, float& y) {
    float denom = dot(r.d, n);
    if (std::fabs(denom) < 1e-6f) return false;
    V3 cp = c - r.o;
    float num = dot(cp, n);
    t = num / denom;
    if (t < RAY_T_MIN) return false;
    hp = r.o + r.d * t;
    V3 lh = hp - c;
    x = dot(lh, right);
    y = dot(lh, up);
    return true;
}
inline bool isect_rect(const Ray& r, V3 c, V3 n, V3 right, V3 up, float sx, float sy, float& tHit, V3& hp) {
    float t, x, y; V3 p;
    if (!isect_planar(r, c, n, right, up, t, p, x, y)) return false;
    float hx = sx * 0.5f, hy = sy * 0.5f;
    if (x * x > hx * hx || y * y > hy * hy) return false;
    tHit = t; hp = p;
    return true;
}
inline bool isect_ellipse(const Ray& r, V3 c, V3 n, V3 right, V3 up, float rx, float ry, float& tHit, V3& hp) {
    float t, x, y; V3 p;
    if (!isect_planar(r, c, n, right, up, t, p, x, y)) return false;
    float nx = x / rx, ny = y / ry;
    if (nx * nx + ny * ny > 1.0f) return false;
    tHit = t; hp = p;
    return true;
}

struct LightHit { bool hit = false; float t = 1e30f; V3 point, normal{0, 0, 1}; RGB emission; int index = -1; };

// light/scene_lights.hpp:176-246
inline LightHit intersect_native(const Scene& s, const Ray& r, int depth) {
    LightHit res;
    if (depth == 0) return res;
    for (size_t i = 0; i < s.native.size(); ++i) {
        const Light& L = s.native[i];
        float t; V3 hp, n;
        if (L.type == LightType::POINT) {
            if (L.radius > MIN_LENGTH && isect_sphere(r, L.position, L.radius, t, n) && t < res.t) {
                res.hit = true; res.t = t; res.point = r.at(t); res.normal = n;
                res.emission = L.emission; res.index = (int)i;
            }
        } else if (L.type == LightType::AREA) {
            bool h;
            if (L.shape == AreaShape::DISK || L.shape == AreaShape::ELLIPSE)
                h = isect_ellipse(r, L.position, L.normal, L.right, L.up, L.size_x * 0.5f, L.size_y * 0.5f, t, hp);
            else
                h = isect_rect(r, L.position, L.normal, L.right, L.up, L.size_x, L.size_y, t, hp);
            if (h && t < res.t) {
                float facing = dot(L.normal, r.d);
                if (facing < 0) {
                    res.hit = true; res.t = t; res.point = hp; res.normal = L.normal;
                    res.emission = L.emission; res.index = (int)i;
                }
            }
        }
    }
    return res;
}

// ------------------------------------------------------------------ lights
// light/scene_lights.hpp:56-164
struct SceneLights {
    std::vector<Light> lights;
    std::vector<float> cdf;
    float total = 0;
    int native_start = 0;
    // prim -> light index, replacing the linear findLightIndex scan
    // (path_tracer.hpp:414-422); a lookup returns the same first match.
    std::vector<std::vector<int>> tri_light;
};
inline float area_ratio(float num, float den) { return (den < MIN_AREA) ? 0.0f : num / den; }
inline float tri_area(V3 v0, V3 v1, V3 v2) { return cross(v1 - v0, v2 - v0).len() * 0.5f; }

inline SceneLights build_lights(const Scene& s) {
    SceneLights sl;
    sl.total = 0;
    sl.tri_light.resize(s.meshes.size());
    for (size_t mi = 0; mi < s.meshes.size(); ++mi) {
        const Mesh& m = s.meshes[mi];
        sl.tri_light[mi].assign(m.tris.size(), -1);
        RGB e = mat_emission(m.mat, V2{});   // scene_lights.hpp:64-69: node emission at uv (0, 0)
        if (!is_emissive(e)) continue;
        for (size_t ti = 0; ti < m.tris.size(); ++ti) {
            const Tri& t = m.tris[ti];
            Light L;
            L.v0 = m.verts[t.i0]; L.v1 = m.verts[t.i1]; L.v2 = m.verts[t.i2];
            L.normal = t.face_n;
            L.emission = e;
            L.area = tri_area(L.v0, L.v1, L.v2);
            L.mesh = (int)mi; L.tri = (int)ti;
            L.position = (L.v0 + L.v1 + L.v2) / 3.0f;
            if (L.area > MIN_AREA) {
                sl.tri_light[mi][ti] = (int)sl.lights.size();
                sl.lights.push_back(L);
                sl.total += L.area;
            }
        }
    }
    sl.native_start = (int)sl.lights.size();
    for (const Light& nl : s.native) {
        Light L = nl;
        if (L.area < MIN_AREA) L.area = 1.0f;
        sl.lights.push_back(L);
        sl.total += L.area;
    }
    sl.cdf.resize(sl.lights.size());
    float cum = 0;
    for (size_t i = 0; i < sl.lights.size(); ++i) {
        cum += sl.lights[i].area;
        sl.cdf[i] = area_ratio(cum, sl.total);
    }
    return sl;
}
inline int select_light(const SceneLights& sl, float u, float& prob) {
    if (sl.lights.empty()) { prob = 0; return -1; }
    int idx = (int)(std::lower_bound(sl.cdf.begin(), sl.cdf.end(), u) - sl.cdf.begin());
    idx = std::min(idx, (int)sl.lights.size() - 1);
    prob = area_ratio(sl.lights[idx].area, sl.total);
    return idx;
}
inline float light_pick_pdf(const SceneLights& sl, int i) {
    if (i < 0 || i >= (int)sl.lights.size()) return 0.0f;
    return area_ratio(sl.lights[i].area, sl.total);
}

// render_units.hpp:1393-1448
inline float inv_sq(float d) { if (d < MIN_LENGTH) return 0.0f; float d2 = d * d; return 1.0f / d2; }
inline float pdfw_from_area(float dist, float area, float c) {
    if (area < MIN_AREA || c < 1e-6f) return 0.0f;
    float d2 = dist * dist;
    return (d2 / area) / c;
}
inline float mis_power(float pf, float pg) {
    float f2 = pf * pf, g2 = pg * pg;
    return f2 / (f2 + g2 + 1e-10f);
}

struct LightSample { V3 pos, normal{0, 0, 1}; RGB emission; float pdf = 0, dist = 0; V3 dir{0, 0, 1}; };

// light/light.hpp:146-170
inline V3 sample_tri_point(V3 v0, V3 v1, V3 v2, float u1, float u2) {
    float su1 = std::sqrt(u1);
    float b0 = 1.0f - su1;
    float b1 = u2 * su1;
    float b2 = 1.0f - b0 - b1;
    V3 d1, d2; float l1, l2;
    nwl(v1 - v0, d1, l1);
    nwl(v2 - v0, d2, l2);
    return v0 + d1 * (l1 * b1) + d2 * (l2 * b2);
}

// light/light.hpp:187-335
inline LightSample sample_light(const Light& L, V3 sp, float u1, float u2) {
    LightSample s;
    s.emission = L.emission;
    switch (L.type) {
        case LightType::POINT: {
            if (L.radius > MIN_LENGTH) {
                float z = 1.0f - 2.0f * u1;
                float r = std::sqrt(smax(0.0f, 1.0f - z * z));
                float phi = kTWO_PI * u2;
                V3 od(r * ocos(phi), r * osin(phi), z);
                s.pos = L.position + od * L.radius;
                s.normal = od;
            } else {
                s.pos = L.position;
                s.normal = V3(0, 1, 0);
            }
            nwl(s.pos - sp, s.dir, s.dist);
            if (L.radius < MIN_LENGTH) {
                s.emission = L.emission * inv_sq(s.dist);
                s.pdf = 1.0f;
            } else {
                float cl = dot(s.normal, -s.dir);
                s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, L.area, cl);
            }
            break;
        }
        case LightType::SUN: {
            s.dir = -L.normal;
            s.pos = sp + s.dir * 1000000.0f;
            s.normal = L.normal;
            s.dist = 1000000.0f;
            s.pdf = 1.0f;
            break;
        }
        case LightType::SPOT: {
            s.pos = L.position;
            s.normal = L.normal;
            nwl(s.pos - sp, s.dir, s.dist);
            s.emission = L.emission * inv_sq(s.dist);
            float ca = dot(L.normal, -s.dir);
            float cc = ocos(L.spot_angle * 0.5f);
            if (ca < cc) {
                s.emission = RGB(0, 0, 0);
            } else if (L.spot_blend > 0.0f) {
                float t = (ca - cc) / (1.0f - cc);
                float fo = smin(1.0f, t / L.spot_blend);
                s.emission = s.emission * fo;
            }
            s.pdf = 1.0f;
            break;
        }
        case LightType::AREA: {
            float lx, ly;
            if (L.shape == AreaShape::DISK || L.shape == AreaShape::ELLIPSE) {
                float rs = std::sqrt(u1);
                float th = kTWO_PI * u2;
                lx = L.size_x * 0.5f * rs * ocos(th);
                ly = L.size_y * 0.5f * rs * osin(th);
            } else {
                lx = L.size_x * (u1 - 0.5f);
                ly = L.size_y * (u2 - 0.5f);
            }
            s.pos = L.position + L.right * lx + L.up * ly;
            s.normal = L.normal;
            nwl(s.pos - sp, s.dir, s.dist);
            float cl = dot(s.normal, -s.dir);
            s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, L.area, cl);
            break;
        }
        case LightType::EMISSIVE_MESH:
        default: {
            s.pos = sample_tri_point(L.v0, L.v1, L.v2, u1, u2);
            s.normal = L.normal;
            nwl(s.pos - sp, s.dir, s.dist);
            float cl = std::fabs(dot(s.normal, -s.dir));
            s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, L.area, cl);
            break;
        }
    }
    return s;
}
// light/light.hpp:344-358
inline float pdf_light(const Light& L, V3 sp, V3 lp, V3 ln) {
    V3 d; float dist;
    nwl(lp - sp, d, dist);
    float cl = std::fabs(dot(ln, -d));
    if (cl < 1e-6f || L.area < MIN_AREA) return 0.0f;
    return pdfw_from_area(dist, L.area, cl);
}

// ------------------------------------------------------------------ BSDF
// bsdf/ggx.hpp
inline float safe_sqrt(float x) { return std::sqrt(smax(0.0f, x)); }
inline void onb(V3 n, V3& t, V3& b) {
    if (n.z < -0.9999f) { t = V3(0, -1, 0); b = V3(-1, 0, 0); return; }
    float a = 1.0f / (1.0f + n.z);
    float bb = -n.x * n.y * a;
    t = make_dir_or(V3(1.0f - n.x * n.x * a, bb, -n.x));
    b = make_dir_or(V3(bb, 1.0f - n.y * n.y * a, -n.y));
}
inline V3 local_to_world(V3 l, V3 n, V3 t, V3 b) {
    return make_dir_or(V3(t.x * l.x + b.x * l.y + n.x * l.z,
                          t.y * l.x + b.y * l.y + n.y * l.z,
                          t.z * l.x + b.z * l.y + n.z * l.z));
}
inline V3 world_to_local(V3 w, V3 n, V3 t, V3 b) { return make_dir_or(V3(dot(w, t), dot(w, b), dot(w, n))); }
inline float ggxD(float NdotH, float r) {
    float alpha = r * r, a2 = alpha * alpha;
    float nh2 = NdotH * NdotH;
    float den = nh2 * (a2 - 1.0f) + 1.0f;
    return a2 * kINV_PI / (den * den + GGX_EPSILON);
}
inline float ggxG1(float NdotV, float r) {
    float alpha = r * r, a2 = alpha * alpha;
    return 2.0f * NdotV / (NdotV + safe_sqrt(a2 + (1.0f - a2) * NdotV * NdotV));
}
inline float ggxG2(float NdotL, float NdotV, float r) {
    if (NdotL <= 0.0f || NdotV <= 0.0f) return 0.0f;
    float alpha = r * r, a2 = alpha * alpha;
    float lL = safe_sqrt(a2 + (1.0f - a2) * NdotL * NdotL);
    float lV = safe_sqrt(a2 + (1.0f - a2) * NdotV * NdotV);
    float den = NdotV * lL + NdotL * lV;
    if (den < GGX_EPSILON) return 0.0f;
    return 2.0f * NdotL * NdotV / den;
}
inline V3 sample_vndf(V3 wo, float rough, float u1, float u2, V3 n, V3 t, V3 b) {
    V3 wl = world_to_local(wo, n, t, b);
    float alpha = rough * rough;
    V3 ws = make_dir_or(V3(wl.x * alpha, wl.y * alpha, wl.z));
    V3 t1;
    if (ws.z < 0.9999f) {
        V3 c;
        t1 = make_dir(cross(V3(0, 0, 1), ws), c) ? c : V3(1, 0, 0);
    } else {
        t1 = V3(1, 0, 0);
    }
    V3 t2;
    if (!make_dir(cross(ws, t1), t2)) t2 = V3(0, 1, 0);
    float r = std::sqrt(u1);
    float phi = kTWO_PI * u2;
    float p1 = r * ocos(phi);
    float p2 = r * osin(phi);
    float s = 0.5f * (1.0f + ws.z);
    p2 = (1.0f - s) * std::sqrt(1.0f - p1 * p1) + s * p2;
    V3 h = t1 * p1 + t2 * p2 + ws * std::sqrt(smax(0.0f, 1.0f - p1 * p1 - p2 * p2));
    h = V3(h.x * alpha, h.y * alpha, smax(0.0f, h.z));
    V3 hl = make_dir_or(h);
    return local_to_world(hl, n, t, b);
}
inline float pdf_vndf(V3 wo, V3 h, float rough, V3 n) {
    float NdotH = dot(n, h), VdotH = dot(wo, h), NdotV = dot(n, wo);
    if (NdotH <= 0.0f || VdotH <= 0.0f || NdotV <= 0.0f) return 0.0f;
    float D = ggxD(NdotH, rough), G1 = ggxG1(NdotV, rough);
    return D * G1 / (4.0f * NdotV);
}
inline V3 sample_cos_hemi(float u1, float u2, V3 n) {
    float r = std::sqrt(u1);
    float th = kTWO_PI * u2;
    float x = r * ocos(th), y = r * osin(th);
    float z = std::sqrt(smax(0.0f, 1.0f - u1));
    V3 t, b;
    onb(n, t, b);
    return local_to_world(V3(x, y, z), n, t, b);
}
inline float pdf_cos_hemi(float NdotL) { return smax(0.0f, NdotL) * kINV_PI; }

// bsdf/fresnel.hpp
inline RGB schlick_rgb(float c, RGB f0) {
    float f = opow5(1.0f - c);
    return RGB(f0.r + (1.0f - f0.r) * f, f0.g + (1.0f - f0.g) * f, f0.b + (1.0f - f0.b) * f);
}
inline float fresnel_dielectric(float ci, float eta) {
    ci = sclamp(std::fabs(ci), 0.0f, 1.0f);
    float si2 = 1.0f - ci * ci;
    float st2 = eta * eta * si2;
    if (st2 >= 1.0f) return 1.0f;
    float ct = std::sqrt(smax(0.0f, 1.0f - st2));
    float eci = eta * ci, ect = eta * ct;
    float rs = (eci - ct) / (eci + ct + 1e-6f);
    float rp = (ci - ect) / (ci + ect + 1e-6f);
    return 0.5f * (rs * rs + rp * rp);
}

// bsdf/bsdf.hpp
struct MatParams { RGB albedo{0.8f, 0.8f, 0.8f}; float metallic = 0, roughness = 0.5f, transmission = 0, ior = 1.45f; };
enum BsdfKind { KIND_EVAL = 0, KIND_PRECOMP = 1 };
enum SampleType { ST_DIFFUSE = 0, ST_SPECULAR = 1, ST_TRANSMISSION = 2 };
struct BsdfSample {
    V3 wi{0, 0, 1};
    int kind = KIND_EVAL;
    RGB f;              // EvaluatedBSDF::f   or PrecomputedWeight::weight
    float pdf = 0;      // EvaluatedBSDF::pdf
    int type = ST_DIFFUSE;
    bool valid() const { return kind == KIND_PRECOMP ? true : pdf > MIN_PDF; }
};
inline MatParams mat_params(const Material& m, V2 uv) {   // path_tracer.hpp:45-64
    MatParams p;
    p.albedo = m.albedo; p.metallic = m.metallic; p.roughness = m.roughness;
    p.transmission = m.transmission; p.ior = m.ior;
    if (m.use_nodes) {
        C3 a = node_albedo(m.tree, uv);
        p.albedo = RGB(a.r, a.g, a.b);
        p.metallic = node_scalar(m.tree, "Metallic", nullptr, 0.0f);
        p.roughness = node_scalar(m.tree, "Roughness", nullptr, 0.5f);
        p.transmission = node_scalar(m.tree, "Transmission", "Transmission Weight", 0.0f);
        p.ior = node_scalar(m.tree, "IOR", nullptr, 1.45f);
    }
    p.roughness = smax(p.roughness, MIN_ROUGHNESS);
    return p;
}
inline RGB bsdf_weight(RGB f, float c, float pdf) {   // render_units.hpp:1413-1420 (+ 1073)
    if (pdf < MIN_PDF) return RGB(0, 0, 0);
    RGB base = (pdf < MIN_PDF) ? RGB(0, 0, 0) : RGB(f.r / pdf, f.g / pdf, f.b / pdf);
    return RGB(base.r * c, base.g * c, base.b * c);
}
inline RGB eval_specular(const MatParams& m, V3 wo, V3 wi, V3 n, float NdotL, float NdotV) {
    if (NdotL <= 0.0f || NdotV <= 0.0f) return RGB(0, 0, 0);
    V3 h = make_dir_or(wo + wi);
    float NdotH = smax(dot(n, h), 0.0f);
    float VdotH = smax(dot(wo, h), 0.0f);
    float r = smax(m.roughness, MIN_ROUGHNESS);
    float D = ggxD(NdotH, r);
    float alpha = r * r, a2 = alpha * alpha;
    float lL = safe_sqrt(a2 + (1.0f - a2) * NdotL * NdotL);
    float lV = safe_sqrt(a2 + (1.0f - a2) * NdotV * NdotV);
    float g2d = 0.5f / (NdotV * lL + NdotL * lV + GGX_EPSILON);
    RGB f0(m.albedo.r * m.metallic + 0.04f * (1.0f - m.metallic),
           m.albedo.g * m.metallic + 0.04f * (1.0f - m.metallic),
           m.albedo.b * m.metallic + 0.04f * (1.0f - m.metallic));
    RGB F = schlick_rgb(VdotH, f0);
    float spec = D * g2d;
    return RGB(spec * F.r, spec * F.g, spec * F.b);
}
inline RGB eval_bsdf(const MatParams& m, V3 wo, V3 wi, V3 n) {
    float NdotL = dot(n, wi), NdotV = dot(n, wo);
    if (NdotL <= 0.0f || NdotV <= 0.0f) return RGB(0, 0, 0);
    RGB spec = eval_specular(m, wo, wi, n, NdotL, NdotV);
    V3 h = make_dir_or(wo + wi);
    float VdotH = smax(dot(wo, h), 0.0f);
    RGB F = schlick_rgb(VdotH, RGB(0.04f, 0.04f, 0.04f));
    RGB diff(m.albedo.r * kINV_PI, m.albedo.g * kINV_PI, m.albedo.b * kINV_PI);
    RGB kd((1.0f - F.r) * (1.0f - m.metallic), (1.0f - F.g) * (1.0f - m.metallic), (1.0f - F.b) * (1.0f - m.metallic));
    diff = mul(diff, kd);
    return diff + spec;
}
inline float spec_prob(const MatParams& m) {
    if (m.metallic > 0.99f) return 1.0f;
    float sp = 0.5f * (1.0f + m.metallic) * (1.0f - m.roughness * 0.5f);
    return sclamp(sp, 0.1f, 0.9f);
}
// bsdf/bsdf.hpp:198-345; u4 is the extra randf() drawn inside the glass branch
// (bsdf.hpp:221), only when the branch is taken.
inline BsdfSample sample_bsdf(const MatParams& m, V3 wo, V3 n, float u1, float u2, float u3, Rng& rng) {
    BsdfSample s;
    float rough = smax(m.roughness, MIN_ROUGHNESS);
    if (m.transmission > 0.0f && u3 < m.transmission) {
        float won = dot(wo, n);
        bool front = won > 0.0f;
        V3 fn = front ? n : -n;
        float eta = front ? (1.0f / m.ior) : m.ior;
        V3 t, b;
        onb(fn, t, b);
        V3 h = sample_vndf(wo, rough, u1, u2, fn, t, b);
        float ci = std::fabs(dot(wo, h));
        float F = fresnel_dielectric(ci, eta);
        V3 inc = -wo;
        float u4 = randf(rng);
        V3 refr;
        bool reflect_branch = (u4 < F) || !refract(inc, h, eta, refr);
        if (reflect_branch) {
            s.wi = reflect(inc, h);
            float NdotL = dot(fn, s.wi), NdotV = dot(fn, wo);
            if (NdotL <= 0.0f || NdotV <= 0.0f) { s.kind = KIND_EVAL; s.f = RGB(0, 0, 0); s.pdf = 0; return s; }
            float G2 = ggxG2(NdotL, NdotV, rough), G1 = ggxG1(NdotV, rough);
            float w = G2 / (G1 + GGX_EPSILON);
            s.kind = KIND_PRECOMP; s.f = RGB(w, w, w); s.type = ST_SPECULAR;
        } else {
            s.wi = refr;
            float NdotL = std::fabs(dot(s.wi, fn)), NdotV = std::fabs(dot(wo, fn));
            float G2 = ggxG2(NdotL, NdotV, rough), G1 = ggxG1(NdotV, rough);
            float w = G2 / (G1 + GGX_EPSILON);
            s.kind = KIND_PRECOMP; s.f = RGB(w, w, w); s.type = ST_TRANSMISSION;
        }
        return s;
    }
    float sp = spec_prob(m);
    V3 t, b;
    onb(n, t, b);
    if (u1 < sp) {
        V3 h = sample_vndf(wo, rough, u1 / sp, u2, n, t, b);
        s.wi = reflect(-wo, h);
        float NdotL = dot(n, s.wi);
        if (NdotL <= 0.0f) { s.kind = KIND_EVAL; s.f = RGB(0, 0, 0); s.pdf = 0; return s; }
        RGB f = eval_bsdf(m, wo, s.wi, n);
        float ps = pdf_vndf(wo, h, rough, n);
        float pd = pdf_cos_hemi(NdotL);
        float pdf = (sp * ps + (1.0f - sp) * pd) * (1.0f - m.transmission);
        if (rough < 0.05f && m.metallic > 0.5f) {
            s.kind = KIND_PRECOMP; s.f = bsdf_weight(f, NdotL, pdf);
        } else {
            s.kind = KIND_EVAL; s.f = f; s.pdf = pdf;
        }
        s.type = ST_SPECULAR;
    } else {
        float u1a = (u1 - sp) / (1.0f - sp);
        s.wi = sample_cos_hemi(u1a, u2, n);
        float NdotL = dot(n, s.wi);
        if (NdotL <= 0.0f) { s.kind = KIND_EVAL; s.f = RGB(0, 0, 0); s.pdf = 0; return s; }
        RGB f = eval_bsdf(m, wo, s.wi, n);
        V3 h = make_dir_or(wo + s.wi);
        float ps = pdf_vndf(wo, h, rough, n);
        float pd = pdf_cos_hemi(NdotL);
        float pdf = (sp * ps + (1.0f - sp) * pd) * (1.0f - m.transmission);
        s.kind = KIND_EVAL; s.f = f; s.pdf = pdf;
        s.type = ST_DIFFUSE;
    }
    return s;
}
inline float pdf_bsdf(const MatParams& m, V3 wo, V3 wi, V3 n) {   // bsdf.hpp:352-375
    float NdotL = dot(n, wi);
    if (NdotL <= 0.0f) return 0.0f;
    float sp = spec_prob(m);
    float rough = smax(m.roughness, MIN_ROUGHNESS);
    V3 h = make_dir_or(wo + wi);
    float ps = pdf_vndf(wo, h, rough, n);
    float pd = pdf_cos_hemi(NdotL);
    return (sp * ps + (1.0f - sp) * pd) * (1.0f - m.transmission);
}
// bsdf.hpp:92-113
inline bool throughput_update(const BsdfSample& s, V3 sn, RGB& w) {
    if (s.kind == KIND_PRECOMP) { w = s.f; return true; }
    float c = std::fabs(dot(sn, s.wi));
    if (c <= 1e-6f || s.pdf < MIN_PDF) return false;
    w = bsdf_weight(s.f, c, s.pdf);
    return true;
}
inline float next_mis_pdf(const BsdfSample& s) { return s.kind == KIND_EVAL ? s.pdf : 0.0f; }

// ------------------------------------------------------------------ volumes
// volume/phase.hpp
constexpr float HG_INV_4PI = 1.0f / (4.0f * kPI);
inline float hg_eval(float g, float c) {
    float gg = g * g;
    float den = 1.0f + gg - 2.0f * g * c;
    float d = smax(den, 1e-8f);
    return HG_INV_4PI * (1.0f - gg) / (d * std::sqrt(d));
}
inline V3 hg_sample(float g, V3 wo, float u1, float u2, float& pdf) {
    float ct;
    if (std::fabs(g) < 1e-3f) {
        ct = 1.0f - 2.0f * u1;
    } else {
        float gg = g * g;
        float sqr = (1.0f - gg) / (1.0f - g + 2.0f * g * u1);
        ct = (1.0f + gg - sqr * sqr) / (2.0f * g);
        ct = sclamp(ct, -1.0f, 1.0f);
    }
    float st = std::sqrt(smax(0.0f, 1.0f - ct * ct));
    float phi = kTWO_PI * u2;
    V3 t, b;
    onb(wo, t, b);
    V3 l(st * ocos(phi), st * osin(phi), ct);
    V3 wi(t.x * l.x + b.x * l.y + wo.x * l.z, t.y * l.x + b.y * l.y + wo.y * l.z,
          t.z * l.x + b.z * l.y + wo.z * l.z);
    pdf = hg_eval(g, ct);
    return wi;
}
// volume/transmittance.hpp:35-59
inline bool ray_aabb_segment(const Ray& r, float tmax, const float* bmn, const float* bmx, float& te, float& tx) {
    float t0 = 0.0f, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        float ro = a == 0 ? r.o.x : a == 1 ? r.o.y : r.o.z;
        float rd = a == 0 ? r.d.x : a == 1 ? r.d.y : r.d.z;
        if (std::fabs(rd) < 1e-12f) {
            if (ro < bmn[a] || ro > bmx[a]) return false;
            continue;
        }
        float inv = 1.0f / rd;
        float ta = (bmn[a] - ro) * inv, tb = (bmx[a] - ro) * inv;
        if (ta > tb) std::swap(ta, tb);
        if (ta > t0) t0 = ta;
        if (tb < t1) t1 = tb;
        if (t0 > t1) return false;
    }
    te = smax(0.0f, t0);
    tx = t1;
    return tx > te;
}
// volume/transmittance.hpp:298-352
inline float grid_trilinear(const Volume& v, float wx, float wy, float wz) {
    float u = (wx - v.wmin[0]) / smax(1e-12f, v.wmax[0] - v.wmin[0]);
    float vv = (wy - v.wmin[1]) / smax(1e-12f, v.wmax[1] - v.wmin[1]);
    float w = (wz - v.wmin[2]) / smax(1e-12f, v.wmax[2] - v.wmin[2]);
    if (u < 0.0f || u > 1.0f || vv < 0.0f || vv > 1.0f || w < 0.0f || w > 1.0f) return 0.0f;
    int nx = v.dims[0], ny = v.dims[1], nz = v.dims[2];
    float fx = u * (float)nx - 0.5f, fy = vv * (float)ny - 0.5f, fz = w * (float)nz - 0.5f;
    if (fx < 0.0f || fx > (float)(nx - 1) || fy < 0.0f || fy > (float)(ny - 1) || fz < 0.0f || fz > (float)(nz - 1))
        return 0.0f;
    int ix = std::clamp((int)fx, 0, nx - 2), iy = std::clamp((int)fy, 0, ny - 2), iz = std::clamp((int)fz, 0, nz - 2);
    float tx = fx - (float)ix, ty = fy - (float)iy, tz = fz - (float)iz;
    auto at = [&](int i, int j, int k) {
        return v.grid[(size_t)i + (size_t)nx * (size_t)j + (size_t)nx * (size_t)ny * (size_t)k];
    };
    float c00 = at(ix, iy, iz) * (1.0f - tx) + at(ix + 1, iy, iz) * tx;
    float c10 = at(ix, iy + 1, iz) * (1.0f - tx) + at(ix + 1, iy + 1, iz) * tx;
    float c01 = at(ix, iy, iz + 1) * (1.0f - tx) + at(ix + 1, iy, iz + 1) * tx;
    float c11 = at(ix, iy + 1, iz + 1) * (1.0f - tx) + at(ix + 1, iy + 1, iz + 1) * tx;
    float c0 = c00 * (1.0f - ty) + c10 * ty;
    float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}
inline int vol_nsteps(const Volume& v, float seg, float& step) {
    float extent = smax3(v.wmax[0] - v.wmin[0], v.wmax[1] - v.wmin[1], v.wmax[2] - v.wmin[2]);
    int md = std::max({v.dims[0], v.dims[1], v.dims[2]});
    float voxel = extent / (float)std::max(1, md);
    step = smax(1e-4f, voxel * 0.5f);
    return std::min(2048, (int)(seg / step) + 1);
}
// volume/transmittance.hpp:77-128 (absorption only, Stage A)
inline RGB absorption_transmittance(const Scene& s, const Ray& r, float tmax) {
    float tr = 0, tg = 0, tb = 0;
    for (const Mesh& m : s.meshes) {
        const Volume& v = m.mat.volume;
        if (!v.present() || !v.has_grid()) continue;
        float ti = 0, to = 0;
        if (!ray_aabb_segment(r, tmax, v.wmin, v.wmax, ti, to)) continue;
        float seg = to - ti;
        if (seg <= 0.0f) continue;
        float step;
        int ns = vol_nsteps(v, seg, step);
        for (int i = 0; i < ns; ++i) {
            float t = ti + ((float)i + 0.5f) * step;
            if (t > to) break;
            float d = grid_trilinear(v, r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t);
            if (d <= 0.0f) continue;
            float sa = v.density * d * step;
            tr += sa * (1.0f - v.color.r);
            tg += sa * (1.0f - v.color.g);
            tb += sa * (1.0f - v.color.b);
        }
    }
    return RGB(oexp(-tr), oexp(-tg), oexp(-tb));
}
// volume/transmittance.hpp:145-209
inline RGB extinction_transmittance(const Scene& s, const Ray& r, float tmax) {
    float tr = 0, tg = 0, tb = 0;
    for (const Mesh& m : s.meshes) {
        const Volume& v = m.mat.volume;
        if (!v.present() || !v.has_grid()) continue;
        float ti = 0, to = 0;
        if (!ray_aabb_segment(r, tmax, v.wmin, v.wmax, ti, to)) continue;
        float seg = to - ti;
        if (seg <= 0.0f) continue;
        float step;
        int ns = vol_nsteps(v, seg, step);
        float er = 1.0f + v.absorption.r, eg = 1.0f + v.absorption.g, eb = 1.0f + v.absorption.b;
        for (int i = 0; i < ns; ++i) {
            float t = ti + ((float)i + 0.5f) * step;
            if (t > to) break;
            float d = grid_trilinear(v, r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t);
            if (d <= 0.0f) continue;
            float base = v.density * d * step;
            tr += base * er;
            tg += base * eg;
            tb += base * eb;
        }
    }
    return RGB(oexp(-tr), oexp(-tg), oexp(-tb));
}
// volume/transmittance.hpp:220-288 (delta tracking)
struct ScatterEvent { bool happened = false; float t = 0; const Volume* vol = nullptr; };
inline ScatterEvent sample_volume_distance(const Scene& s, const Ray& r, float tmax, Rng& rng) {
    ScatterEvent out;
    float best = tmax;
    for (const Mesh& m : s.meshes) {
        const Volume& v = m.mat.volume;
        if (!v.present() || !v.has_grid()) continue;
        if (v.density <= 0.0f || v.grid_max <= 0.0f) continue;
        float ti = 0, to = 0;
        if (!ray_aabb_segment(r, tmax, v.wmin, v.wmax, ti, to)) continue;
        if (ti >= best) continue;
        float se = smin(to, best);
        if (se <= ti) continue;
        float em = smax3(1.0f + v.absorption.r, 1.0f + v.absorption.g, 1.0f + v.absorption.b);
        float smx = v.density * v.grid_max * em;
        if (smx <= 0.0f) continue;
        float t = ti;
        bool sc = false;
        for (int it = 0; it < 4096; ++it) {
            float us = smax(1e-12f, 1.0f - randf(rng));
            t += -olog(us) / smx;
            if (t >= se) break;
            float d = grid_trilinear(v, r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t);
            float st = v.density * d * em;
            if (randf(rng) * smx < st) { sc = true; break; }
        }
        if (sc && t < best) { best = t; out.happened = true; out.t = t; out.vol = &v; }
    }
    return out;
}

// ------------------------------------------------------------------ integrators
// Per-sample parity record.  hash = FNV-1a 64 over 32-bit event words:
// per bounce [hit mesh, hit tri, native light idx] (-1 when absent), in
// volume_mis also [scatter flag], and for every NEE shadow test
// [0x5EED0000 | occluded].
struct SampleRec {
    float rgb[3] = {0, 0, 0};
    int32_t primary_mesh = -1, primary_tri = -1;
    uint32_t bounces = 0;
    uint32_t nee_tests = 0, nee_occluded = 0;
    uint64_t hash = 1469598103934665603ULL;
};
inline void hpush(SampleRec* r, uint32_t w) {
    if (!r) return;
    for (int i = 0; i < 4; ++i) { r->hash ^= (w >> (8 * i)) & 0xffu; r->hash *= 1099511628211ULL; }
}

// path_tracer.hpp:82-95
inline void intersect_skip_boundaries(const Scene& s, const Ray& r, float tMin, int depth, Hit& hit, LightHit& lh) {
    hit.hit = false;
    float sm = tMin;
    for (int peek = 0; peek < 8; ++peek) {
        Hit h = intersect_scene(s, r, sm);
        if (!h.hit) break;
        if (!h.mat->volume_boundary_only) { hit = h; break; }
        sm = h.t + 1e-3f;
    }
    lh = intersect_native(s, r, depth);
}
// path_tracer.hpp:103-119
inline bool shadowed_skip_boundaries(const Scene& s, const Ray& r, float tmax) {
    Ray probe = r;
    float off = 0.0f;
    for (int peek = 0; peek < 8; ++peek) {
        float rem = tmax - off;
        if (rem <= 0.0f) return false;
        Hit h = intersect_scene(s, probe, RAY_T_MIN, rem);
        if (!h.hit) return false;
        if (!h.mat->volume_boundary_only) return true;
        float skip = h.t + 1e-3f;
        off += skip;
        probe = Ray{probe.at(skip), probe.d};
    }
    return false;
}

enum class Algo { SIMPLE, NEE, MIS, VOLUME_SIMPLE, VOLUME_MIS };

// One integrator body covering traceSimple (128-198), traceVolumeSimple
// (209-282), traceNEE (292-397), traceMIS (406-570) and traceVolumeMIS
// (586-835); the branches select exactly the statements each variant has.
inline RGB trace(const Scene& s, const SceneLights& sl, const Ray& ray, int max_depth, Algo algo, Rng& rng,
                 SampleRec* rec) {
    const bool nee = algo == Algo::NEE || algo == Algo::MIS || algo == Algo::VOLUME_MIS;
    const bool mis = algo == Algo::MIS || algo == Algo::VOLUME_MIS;
    RGB result(0, 0, 0), T(1, 1, 1);
    Ray cur = ray;
    float last_pdf = 0.0f;
    float tMin = 0.0f;
    for (int depth = 0; depth < max_depth; ++depth) {
        Hit hit; LightHit lh;
        intersect_skip_boundaries(s, cur, tMin, depth, hit, lh);
        if (rec) {
            rec->bounces++;
            if (depth == 0) { rec->primary_mesh = hit.hit ? hit.mesh : -1; rec->primary_tri = hit.hit ? hit.tri : -1; }
            hpush(rec, (uint32_t)(hit.hit ? hit.mesh : -1));
            hpush(rec, (uint32_t)(hit.hit ? hit.tri : -1));
            // the native light hit that takes effect: nearer than the surface
            // hit (the light branch below and the CUDA trace kernel's bound)
            hpush(rec, (uint32_t)(lh.hit && (!hit.hit || lh.t < hit.t) ? lh.index : -1));
        }
        if (algo == Algo::VOLUME_SIMPLE) {
            float ts = 1e6f;
            if (hit.hit) ts = smin(ts, hit.t);
            if (lh.hit) ts = smin(ts, lh.t);
            RGB Ts = absorption_transmittance(s, cur, ts);
            T = mul(T, Ts);
        }
        if (algo == Algo::VOLUME_MIS) {
            float ts = 1e6f;
            if (hit.hit) ts = smin(ts, hit.t);
            if (lh.hit) ts = smin(ts, lh.t);
            ScatterEvent vs = sample_volume_distance(s, cur, ts, rng);
            hpush(rec, vs.happened && vs.vol ? 1u : 0u);
            if (vs.happened && vs.vol) {
                const Volume& v = *vs.vol;
                float ar = v.color.r / (1.0f + v.absorption.r);
                float ag = v.color.g / (1.0f + v.absorption.g);
                float ab = v.color.b / (1.0f + v.absorption.b);
                T = mul(T, RGB(ar, ag, ab));
                V3 x = cur.at(vs.t);
                V3 wo = -cur.d;
                float g = v.anisotropy;
                if (!sl.lights.empty()) {
                    float usel = randf(rng);
                    float lsp;
                    int li = select_light(sl, usel, lsp);
                    if (li >= 0 && lsp > 1e-6f) {
                        float u1, u2; draw2(rng, u1, u2);
                        LightSample ls = sample_light(sl.lights[li], x, u1, u2);
                        if (ls.pdf > MIN_PDF) {
                            Ray sr{x, ls.dir};
                            bool occ = shadowed_skip_boundaries(s, sr, ls.dist);
                            if (rec) { rec->nee_tests++; rec->nee_occluded += occ; hpush(rec, 0x5EED0000u | (uint32_t)occ); }
                            if (!occ) {
                                RGB Tsh = extinction_transmittance(s, sr, ls.dist);
                                float ct = dot(wo, ls.dir);
                                float pe = hg_eval(g, ct);
                                float pp = hg_eval(g, ct);
                                float pl = ls.pdf * lsp;
                                float mw = mis_power(pl, pp);
                                RGB pw = bsdf_weight(RGB(pe, pe, pe), 1.0f, pl);
                                RGB c = mul(pw * mw, mul(Tsh, ls.emission));
                                result = result + mul(T, c);
                            }
                        }
                    }
                }
                float u1, u2; draw2(rng, u1, u2);
                float ppdf;
                V3 wi = hg_sample(g, wo, u1, u2, ppdf);
                last_pdf = ppdf;
                cur = Ray{x, wi};
                tMin = RAY_T_MIN;
                if (depth >= 3) {
                    float mt = smax3(T.r, T.g, T.b);
                    float rr = smin(mt, 0.95f);
                    if (randf(rng) > rr) break;
                    T = T * (1.0f / rr);
                }
                if (!rgb_valid(T)) break;
                continue;
            }
        }
        if (lh.hit && (!hit.hit || lh.t < hit.t)) {
            if (mis) {
                float lpdf = 0.0f;
                if (!sl.lights.empty() && lh.index >= 0) {
                    int sli = sl.native_start + lh.index;
                    if (!(sli >= 0 && sli < (int)sl.lights.size())) sli = -1;
                    if (sli >= 0) {
                        float sp = light_pick_pdf(sl, sli);
                        if (sp > 0.0f) lpdf = pdf_light(sl.lights[sli], cur.o, lh.point, lh.normal) * sp;
                    }
                }
                float mw = (last_pdf > MIN_PDF && lpdf > MIN_PDF) ? mis_power(last_pdf, lpdf) : 1.0f;
                result = result + mul(T, lh.emission) * mw;
            } else {
                result = result + mul(T, lh.emission);
            }
            break;
        }
        if (!hit.hit) {
            RGB env = s.env_color * s.env_strength;
            result = result + mul(T, env);
            break;
        }
        MatParams m = mat_params(*hit.mat, hit.uv);
        RGB emission = mat_emission(*hit.mat, hit.uv);
        V3 n = hit.normal;
        V3 wo = -cur.d;
        bool front = dot(wo, n) > 0;
        V3 sn = n;
        if (m.transmission < 0.5f && !front) sn = -n;
        bool has_em = is_emissive(emission);
        if (!nee) {
            result = result + mul(T, emission);
        } else if (!mis) {
            if (has_em && depth == 0) result = result + mul(T, emission);
        } else if (has_em) {
            float mw = 1.0f;
            if (!sl.lights.empty() && last_pdf > MIN_PDF) {
                int li = sl.tri_light[hit.mesh][hit.tri];
                if (li >= 0) {
                    float sp = light_pick_pdf(sl, li);
                    if (sp > 0.0f) {
                        float lpdf = pdf_light(sl.lights[li], cur.o, hit.point, hit.normal) * sp;
                        if (lpdf > MIN_PDF) mw = mis_power(last_pdf, lpdf);
                    }
                }
            }
            result = result + mul(T, emission) * mw;
        }
        bool transmissive = m.transmission > 0.5f;
        if (nee && !sl.lights.empty() && !has_em && !transmissive) {
            float usel = randf(rng);
            float lsp;
            int li = select_light(sl, usel, lsp);
            if (li >= 0 && lsp > 1e-6f) {
                float u1, u2; draw2(rng, u1, u2);
                LightSample ls = sample_light(sl.lights[li], hit.point, u1, u2);
                if (ls.pdf > MIN_PDF) {
                    float NdotL = dot(sn, ls.dir);
                    if (NdotL > 1e-6f) {
                        Ray sr{hit.point, ls.dir};
                        bool occ = shadowed_skip_boundaries(s, sr, ls.dist);
                        if (rec) { rec->nee_tests++; rec->nee_occluded += occ; hpush(rec, 0x5EED0000u | (uint32_t)occ); }
                        if (!occ) {
                            if (algo == Algo::VOLUME_MIS) {
                                RGB Tsh = extinction_transmittance(s, sr, ls.dist);
                                RGB f = eval_bsdf(m, wo, ls.dir, sn);
                                float pl = ls.pdf * lsp;
                                float pb = pdf_bsdf(m, wo, ls.dir, sn);
                                float mw = mis_power(pl, pb);
                                RGB bw = bsdf_weight(f, NdotL, pl);
                                RGB c = mul(bw * mw, mul(Tsh, ls.emission));
                                result = result + mul(T, c);
                            } else if (mis) {
                                RGB f = eval_bsdf(m, wo, ls.dir, sn);
                                float pl = ls.pdf * lsp;
                                float pb = pdf_bsdf(m, wo, ls.dir, sn);
                                float mw = mis_power(pl, pb);
                                RGB bw = bsdf_weight(f, NdotL, pl);
                                RGB c = mul(bw * mw, ls.emission);
                                result = result + mul(T, c);
                            } else {
                                RGB f = eval_bsdf(m, wo, ls.dir, sn);
                                float pl = ls.pdf * lsp;
                                RGB bw = bsdf_weight(f, NdotL, pl);
                                RGB c = mul(bw, ls.emission);
                                result = result + mul(T, c);
                            }
                        }
                    }
                }
            }
        }
        V3 smp_n = (m.transmission > 0.5f) ? n : sn;
        float u1, u2, u3;
        draw3(rng, u1, u2, u3);   // left-to-right pin (right to left when draw_rtl)
        BsdfSample bs = sample_bsdf(m, wo, smp_n, u1, u2, u3, rng);
        if (!bs.valid()) break;
        RGB w;
        if (!throughput_update(bs, smp_n, w)) break;
        T = mul(T, w);
        if (mis) last_pdf = next_mis_pdf(bs);
        if (depth >= 3) {
            float mt = smax3(T.r, T.g, T.b);
            float rr = smin(mt, 0.95f);
            if (randf(rng) > rr) break;
            T = T * (1.0f / rr);
        }
        if (!rgb_valid(T)) break;
        cur = Ray{hit.point, bs.wi};
        tMin = RAY_T_MIN;
    }
    return result;
}

// ------------------------------------------------------------------ tile renderer
// pybind_renderer.hpp:131-160 set_camera
inline void set_camera(Camera& c, float px, float py, float pz, float dx, float dy, float dz, float ux, float uy,
                       float uz, float fov_deg) {
    c.pos = V3(px, py, pz);
    V3 dir = make_dir_or(V3(dx, dy, dz), V3(0, 0, -1));
    c.dir = dir;
    V3 up = make_dir_or(V3(ux, uy, uz), V3(0, 1, 0));
    c.fov = fov_deg * (kPI / 180.0f);
    V3 fwd = dir;
    V3 right = make_dir_or(cross(fwd, up), V3(1, 0, 0));
    V3 upc = make_dir_or(cross(right, fwd), V3(0, 1, 0));
    c.forward = fwd; c.right = right; c.up = upc;
}

inline Algo algo_from_string(const std::string& a) {
    if (a == "simple") return Algo::SIMPLE;
    if (a == "mis") return Algo::MIS;
    if (a == "volume_simple") return Algo::VOLUME_SIMPLE;
    if (a == "volume_mis") return Algo::VOLUME_MIS;
    return Algo::NEE;
}

// Primary ray for (global_x, global_y) — pybind_renderer.hpp:253-265.
inline V3 primary_dir(const Camera& c, float ndc_x, float ndc_y, float scale) {
    V3 v(c.forward.x + c.right.x * (ndc_x * scale) + c.up.x * (ndc_y * scale),
         c.forward.y + c.right.y * (ndc_x * scale) + c.up.y * (ndc_y * scale),
         c.forward.z + c.right.z * (ndc_x * scale) + c.up.z * (ndc_y * scale));
    return make_dir_or(v, c.forward);
}

// The per-pixel body of render_tile (pybind_renderer.hpp:245-344) without the
// exposure/clamp/Y-flip, returning the radiance sum over the call's samples.
inline RGB render_pixel(const Scene& s, const SceneLights& sl, const Camera& cam, int gx, int gy, int full_w,
                        int full_h, int samples, int sample_offset, int max_depth, Algo algo, float scale,
                        SampleRec* recs, double* acc64 = nullptr) {
    float ndc_x = (2.0f * ((float)gx + 0.5f) / (float)full_w - 1.0f) * cam.aspect;
    float ndc_y = 1.0f - 2.0f * ((float)gy + 0.5f) / (float)full_h;
    V3 wd = primary_dir(cam, ndc_x, ndc_y, scale);
    RGB rad(0, 0, 0);
    for (int si = 0; si < samples; ++si) {
        Rng rng;
        seed_xyz(rng, (uint32_t)gx, (uint32_t)gy, (uint32_t)(sample_offset + si));
        Ray r{cam.pos, wd};
        if (samples > 1) {
            float jx = (randf(rng) - 0.5f) / (float)full_w;
            float jy = (randf(rng) - 0.5f) / (float)full_h;
            r.d = primary_dir(cam, ndc_x + jx, ndc_y + jy, scale);
        }
        SampleRec* rec = recs ? &recs[si] : nullptr;
        if (rec) *rec = SampleRec();
        RGB sr = trace(s, sl, r, max_depth, algo, rng, rec);
        if (rec) { rec->rgb[0] = sr.r; rec->rgb[1] = sr.g; rec->rgb[2] = sr.b; }
        rad = rad + sr;
        if (acc64) { acc64[0] += (double)sr.r; acc64[1] += (double)sr.g; acc64[2] += (double)sr.b; }
    }
    return rad;
}

// render_debug's primary-hit passes (renderer.hpp:59-93).
inline RGB debug_pass(const Scene& s, const Ray& r, int mode) {
    Hit h = intersect_scene(s, r, 0.0f, RAY_T_MAX);
    // render_debug maps the normal pass to 0..1 after traceNormal, so a miss
    // (black) comes out grey (pybind_renderer.hpp:412-415)
    if (!h.hit) return mode == 0 ? RGB(0, 0, 0) * 0.5f + RGB(0.5f, 0.5f, 0.5f) : RGB(0, 0, 0);
    if (mode == 0) return RGB(h.normal.x, h.normal.y, h.normal.z) * 0.5f + RGB(0.5f, 0.5f, 0.5f);
    if (mode == 1) {
        if (!h.mat->use_nodes) return h.mat->albedo;
        C3 a = node_albedo(h.mat->tree, h.uv);
        return RGB(a.r, a.g, a.b);
    }
    return mat_emission(*h.mat, h.uv);   // apply_camera_sensitivity with the default sensitivity 1
}

}  // namespace orc
