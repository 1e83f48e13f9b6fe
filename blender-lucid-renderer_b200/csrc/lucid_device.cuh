// lucid_device.cuh — device-side data layout and per-path math of the B200
// wavefront path tracer.
//
// The shading, light-sampling, volume and RNG functions here reproduce the
// float operation sequence of the reference CPU integrators
// (LucidRenderer/cpp_renderer/include/{bsdf,light,volume,math}/*.hpp and
// integrator/path_tracer.hpp) so that a GPU path and the CPU path for the
// same (pixel, sample) agree bit for bit.  The translation unit is compiled
// with -fmad=false: no multiply-add is fused unless written as __fmaf_rn,
// which only the conservative BVH box test does.  Transcendentals come from
// lucid_math.h (shared with the CPU checker).
#pragma once

#include <stdint.h>

#include "lucid_math.h"
#include "lucid_types.h"

namespace lucid {

#define LD __device__ __forceinline__

// ---------------------------------------------------------------- vectors
struct V3 {
    float x, y, z;
};
LD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
LD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
LD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
LD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
LD V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
LD V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
LD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
LD float len2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
LD float len(V3 a) { return sqrtf(len2(a)); }
LD V3 f3(float4 a) { return v3(a.x, a.y, a.z); }

// std::min / std::max semantics (the reference's NaN behaviour included)
LD float smin(float a, float b) { return (b < a) ? b : a; }
LD float smax(float a, float b) { return (a < b) ? b : a; }
LD float smax3(float a, float b, float c) { float m = a; if (m < b) m = b; if (m < c) m = c; return m; }
LD float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

constexpr float kPI = 3.14159274101257324219f;
constexpr float kINV_PI = 0.31830987334251403809f;
constexpr float kTWO_PI = 2.0f * kPI;
constexpr float kDirEps2 = 1e-6f * 1e-6f;
constexpr float MIN_PDF = 1e-6f;
constexpr float MIN_AREA = 1e-6f;
constexpr float MIN_LENGTH = 1e-6f;
constexpr float RAY_T_MIN = 1e-4f;
constexpr float GGX_EPSILON = 1e-6f;
constexpr float MIN_ROUGHNESS = 0.01f;

// make_direction: fails below 1e-6 length (render_units.hpp:485-494)
LD bool make_dir(V3 v, V3& out) {
    float l2 = len2(v);
    if (l2 < kDirEps2) return false;
    out = v / sqrtf(l2);
    return true;
}
LD V3 make_dir_or(V3 v, V3 fb) { V3 d; return make_dir(v, d) ? d : fb; }
LD V3 make_dir_or(V3 v) { return make_dir_or(v, v3(0.f, 0.f, 1.f)); }
LD void nwl(V3 v, V3& d, float& l) { l = len(v); d = v / l; }
LD V3 normalize_nz(V3 v) { float l = len(v); if (l > 0.0f) return v / l; return v; }

LD V3 reflect(V3 i, V3 n) {
    float ci = dot(i, n);
    return make_dir_or(i - n * (2.0f * ci));
}
LD bool refract(V3 i, V3 n, float eta, V3& out) {
    float ci = -dot(i, n);
    float s2 = eta * eta * (1.0f - ci * ci);
    if (s2 > 1.0f) return false;
    float ct = sqrtf(1.0f - s2);
    return make_dir(i * eta + n * (eta * ci - ct), out);
}

struct RGB {
    float r, g, b;
};
LD RGB rgb(float r, float g, float b) { RGB c; c.r = r; c.g = g; c.b = b; return c; }
LD RGB operator+(RGB a, RGB b) { return rgb(a.r + b.r, a.g + b.g, a.b + b.b); }
LD RGB operator*(RGB a, float s) { return rgb(a.r * s, a.g * s, a.b * s); }
LD RGB mul(RGB a, RGB b) { return rgb(a.r * b.r, a.g * b.g, a.b * b.b); }
LD bool rgb_valid(RGB c) {
    return !isnan(c.r) && !isnan(c.g) && !isnan(c.b) && !isinf(c.r) && !isinf(c.g) && !isinf(c.b);
}
LD RGB c3(float4 a) { return rgb(a.x, a.y, a.z); }

// ---------------------------------------------------------------- RNG
// PCG32 stream seeded per (x, y, sample) — math/random.hpp:64-120.
struct Rng {
    uint64_t state, inc;
};
LD uint32_t murmur3_finalize(uint32_t h) {
    h ^= h >> 16; h *= 0x85ebca6bU; h ^= h >> 13; h *= 0xc2b2ae35U; h ^= h >> 16; return h;
}
LD uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
LD uint32_t jenkins_hash(uint32_t a) {
    a = (a + 0x7ed55d16) + (a << 12);
    a = (a ^ 0xc761c23c) ^ (a >> 19);
    a = (a + 0x165667b1) + (a << 5);
    a = (a + 0xd3a2646c) ^ (a << 9);
    a = (a + 0xfd7046c5) + (a << 3);
    a = (a ^ 0xb55a4f09) ^ (a >> 16);
    return a;
}
LD Rng seed_xyz(uint32_t x, uint32_t y, uint32_t s) {
    uint32_t h1 = jenkins_hash(x + 1);
    uint32_t h2 = jenkins_hash(y + 1 + h1);
    uint32_t h3 = jenkins_hash(s + 1 + h2);
    uint64_t seed1 = ((uint64_t)murmur3_finalize(h1 ^ h3) << 32) | murmur3_finalize(h2);
    uint64_t seed2 = ((uint64_t)murmur3_finalize(h2 ^ h1) << 32) | murmur3_finalize(h3);
    Rng r;
    r.inc = (splitmix64(seed1) << 1u) | 1u;
    uint64_t initseq = splitmix64(seed2);
    r.state = r.inc;                     // 0 * mult + inc
    r.state += initseq;
    r.state = r.state * 6364136223846793005ULL + r.inc;
#pragma unroll
    for (int i = 0; i < 8; i++) r.state = r.state * 6364136223846793005ULL + r.inc;
    return r;
}
LD uint32_t pcg32(Rng& s) {
    uint64_t old = s.state;
    s.state = old * 6364136223846793005ULL + s.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31));
}
// ldexpf(float(u >> 9), -23): exact scaling by 2^-23.
LD float randf(Rng& s) { return (float)(pcg32(s) >> 9) * 1.1920928955078125e-07f; }

// ---------------------------------------------------------------- BSDF
LD float safe_sqrt(float x) { return sqrtf(smax(0.0f, x)); }
LD void onb(V3 n, V3& t, V3& b) {
    if (n.z < -0.9999f) { t = v3(0.f, -1.f, 0.f); b = v3(-1.f, 0.f, 0.f); return; }
    float a = 1.0f / (1.0f + n.z);
    float bb = -n.x * n.y * a;
    t = make_dir_or(v3(1.0f - n.x * n.x * a, bb, -n.x));
    b = make_dir_or(v3(bb, 1.0f - n.y * n.y * a, -n.y));
}
LD V3 local_to_world(V3 l, V3 n, V3 t, V3 b) {
    return make_dir_or(v3(t.x * l.x + b.x * l.y + n.x * l.z, t.y * l.x + b.y * l.y + n.y * l.z,
                          t.z * l.x + b.z * l.y + n.z * l.z));
}
LD float ggxD(float nh, float r) {
    float al = r * r, a2 = al * al;
    float nh2 = nh * nh;
    float den = nh2 * (a2 - 1.0f) + 1.0f;
    return a2 * kINV_PI / (den * den + GGX_EPSILON);
}
LD float ggxG1(float nv, float r) {
    float al = r * r, a2 = al * al;
    return 2.0f * nv / (nv + safe_sqrt(a2 + (1.0f - a2) * nv * nv));
}
LD float ggxG2(float nl, float nv, float r) {
    if (nl <= 0.0f || nv <= 0.0f) return 0.0f;
    float al = r * r, a2 = al * al;
    float lL = safe_sqrt(a2 + (1.0f - a2) * nl * nl);
    float lV = safe_sqrt(a2 + (1.0f - a2) * nv * nv);
    float den = nv * lL + nl * lV;
    if (den < GGX_EPSILON) return 0.0f;
    return 2.0f * nl * nv / den;
}
// Heitz 2018 VNDF sampling as written in bsdf/ggx.hpp:130-170
LD V3 sample_vndf(V3 wo, float rough, float u1, float u2, V3 n, V3 t, V3 b) {
    V3 wl = make_dir_or(v3(dot(wo, t), dot(wo, b), dot(wo, n)));
    float al = rough * rough;
    V3 ws = make_dir_or(v3(wl.x * al, wl.y * al, wl.z));
    V3 t1;
    if (ws.z < 0.9999f) {
        V3 c;
        t1 = make_dir(cross(v3(0.f, 0.f, 1.f), ws), c) ? c : v3(1.f, 0.f, 0.f);
    } else {
        t1 = v3(1.f, 0.f, 0.f);
    }
    V3 t2;
    if (!make_dir(cross(ws, t1), t2)) t2 = v3(0.f, 1.f, 0.f);
    float r = sqrtf(u1);
    float phi = kTWO_PI * u2;
    float p1 = r * lucid_math::lm_cosf(phi);
    float p2 = r * lucid_math::lm_sinf(phi);
    float s = 0.5f * (1.0f + ws.z);
    p2 = (1.0f - s) * sqrtf(1.0f - p1 * p1) + s * p2;
    V3 h = t1 * p1 + t2 * p2 + ws * sqrtf(smax(0.0f, 1.0f - p1 * p1 - p2 * p2));
    h = v3(h.x * al, h.y * al, smax(0.0f, h.z));
    return local_to_world(make_dir_or(h), n, t, b);
}
LD float pdf_vndf(V3 wo, V3 h, float rough, V3 n) {
    float nh = dot(n, h), vh = dot(wo, h), nv = dot(n, wo);
    if (nh <= 0.0f || vh <= 0.0f || nv <= 0.0f) return 0.0f;
    float D = ggxD(nh, rough), G1 = ggxG1(nv, rough);
    return D * G1 / (4.0f * nv);
}
LD V3 sample_cos_hemi(float u1, float u2, V3 n) {
    float r = sqrtf(u1);
    float th = kTWO_PI * u2;
    float x = r * lucid_math::lm_cosf(th), y = r * lucid_math::lm_sinf(th);
    float z = sqrtf(smax(0.0f, 1.0f - u1));
    V3 t, b;
    onb(n, t, b);
    return local_to_world(v3(x, y, z), n, t, b);
}
LD float pdf_cos_hemi(float nl) { return smax(0.0f, nl) * kINV_PI; }
LD RGB schlick_rgb(float c, RGB f0) {
    float f = lucid_math::lm_pow5(1.0f - c);
    return rgb(f0.r + (1.0f - f0.r) * f, f0.g + (1.0f - f0.g) * f, f0.b + (1.0f - f0.b) * f);
}
LD float fresnel_dielectric(float ci, float eta) {
    ci = sclamp(fabsf(ci), 0.0f, 1.0f);
    float si2 = 1.0f - ci * ci;
    float st2 = eta * eta * si2;
    if (st2 >= 1.0f) return 1.0f;
    float ct = sqrtf(smax(0.0f, 1.0f - st2));
    float eci = eta * ci, ect = eta * ct;
    float rs = (eci - ct) / (eci + ct + 1e-6f);
    float rp = (ci - ect) / (ci + ect + 1e-6f);
    return 0.5f * (rs * rs + rp * rp);
}

struct Mat {
    RGB albedo;
    float metallic, roughness, transmission, ior;
};
LD RGB bsdf_weight(RGB f, float c, float pdf) {
    if (pdf < MIN_PDF) return rgb(0.f, 0.f, 0.f);
    return rgb((f.r / pdf) * c, (f.g / pdf) * c, (f.b / pdf) * c);
}
LD RGB eval_bsdf(const Mat& m, V3 wo, V3 wi, V3 n) {
    float nl = dot(n, wi), nv = dot(n, wo);
    if (nl <= 0.0f || nv <= 0.0f) return rgb(0.f, 0.f, 0.f);
    // evalSpecular (bsdf.hpp:132-160)
    V3 h = make_dir_or(wo + wi);
    float nh = smax(dot(n, h), 0.0f);
    float vh = smax(dot(wo, h), 0.0f);
    float r = smax(m.roughness, MIN_ROUGHNESS);
    float D = ggxD(nh, r);
    float al = r * r, a2 = al * al;
    float lL = safe_sqrt(a2 + (1.0f - a2) * nl * nl);
    float lV = safe_sqrt(a2 + (1.0f - a2) * nv * nv);
    float g2d = 0.5f / (nv * lL + nl * lV + GGX_EPSILON);
    float om = 1.0f - m.metallic;
    RGB f0 = rgb(m.albedo.r * m.metallic + 0.04f * om, m.albedo.g * m.metallic + 0.04f * om,
                 m.albedo.b * m.metallic + 0.04f * om);
    RGB F = schlick_rgb(vh, f0);
    float spec = D * g2d;
    RGB sp = rgb(spec * F.r, spec * F.g, spec * F.b);
    // evalBSDF (bsdf.hpp:166-190): the half vector is recomputed identically.
    RGB Fd = schlick_rgb(vh, rgb(0.04f, 0.04f, 0.04f));
    RGB diff = rgb(m.albedo.r * kINV_PI, m.albedo.g * kINV_PI, m.albedo.b * kINV_PI);
    RGB kd = rgb((1.0f - Fd.r) * om, (1.0f - Fd.g) * om, (1.0f - Fd.b) * om);
    return mul(diff, kd) + sp;
}
LD float spec_prob(const Mat& m) {
    if (m.metallic > 0.99f) return 1.0f;
    float sp = 0.5f * (1.0f + m.metallic) * (1.0f - m.roughness * 0.5f);
    return sclamp(sp, 0.1f, 0.9f);
}
LD float pdf_bsdf(const Mat& m, V3 wo, V3 wi, V3 n) {
    float nl = dot(n, wi);
    if (nl <= 0.0f) return 0.0f;
    float sp = spec_prob(m);
    float r = smax(m.roughness, MIN_ROUGHNESS);
    V3 h = make_dir_or(wo + wi);
    return (sp * pdf_vndf(wo, h, r, n) + (1.0f - sp) * pdf_cos_hemi(nl)) * (1.0f - m.transmission);
}

enum { BS_EVAL = 0, BS_PRECOMP = 1 };
struct BsdfSample {
    V3 wi;
    int kind;
    RGB f;      // f (evaluated) or the precomputed throughput weight
    float pdf;
    int type;   // 0 diffuse, 1 specular, 2 transmission
};
// sampleBSDF (bsdf.hpp:198-345).  The glass branch draws one extra uniform.
LD BsdfSample sample_bsdf(const Mat& m, V3 wo, V3 n, float u1, float u2, float u3, Rng& rng) {
    BsdfSample s;
    s.wi = v3(0.f, 0.f, 1.f);
    s.kind = BS_EVAL;
    s.f = rgb(0.f, 0.f, 0.f);
    s.pdf = 0.0f;
    s.type = 0;
    float rough = smax(m.roughness, MIN_ROUGHNESS);
    if (m.transmission > 0.0f && u3 < m.transmission) {
        bool front = dot(wo, n) > 0.0f;
        V3 fn = front ? n : -n;
        float eta = front ? (1.0f / m.ior) : m.ior;
        V3 t, b;
        onb(fn, t, b);
        V3 h = sample_vndf(wo, rough, u1, u2, fn, t, b);
        float F = fresnel_dielectric(fabsf(dot(wo, h)), eta);
        V3 inc = -wo;
        float u4 = randf(rng);
        V3 refr;
        bool refl = (u4 < F) || !refract(inc, h, eta, refr);
        if (refl) {
            s.wi = reflect(inc, h);
            float nl = dot(fn, s.wi), nv = dot(fn, wo);
            if (nl <= 0.0f || nv <= 0.0f) return s;
            float w = ggxG2(nl, nv, rough) / (ggxG1(nv, rough) + GGX_EPSILON);
            s.kind = BS_PRECOMP; s.f = rgb(w, w, w); s.type = 1;
        } else {
            s.wi = refr;
            float nl = fabsf(dot(s.wi, fn)), nv = fabsf(dot(wo, fn));
            float w = ggxG2(nl, nv, rough) / (ggxG1(nv, rough) + GGX_EPSILON);
            s.kind = BS_PRECOMP; s.f = rgb(w, w, w); s.type = 2;
        }
        return s;
    }
    float sp = spec_prob(m);
    V3 t, b;
    onb(n, t, b);
    if (u1 < sp) {
        V3 h = sample_vndf(wo, rough, u1 / sp, u2, n, t, b);
        s.wi = reflect(-wo, h);
        float nl = dot(n, s.wi);
        if (nl <= 0.0f) return s;
        RGB f = eval_bsdf(m, wo, s.wi, n);
        float pdf = (sp * pdf_vndf(wo, h, rough, n) + (1.0f - sp) * pdf_cos_hemi(nl)) * (1.0f - m.transmission);
        if (rough < 0.05f && m.metallic > 0.5f) {
            s.kind = BS_PRECOMP; s.f = bsdf_weight(f, nl, pdf);
        } else {
            s.kind = BS_EVAL; s.f = f; s.pdf = pdf;
        }
        s.type = 1;
    } else {
        float u1a = (u1 - sp) / (1.0f - sp);
        s.wi = sample_cos_hemi(u1a, u2, n);
        float nl = dot(n, s.wi);
        if (nl <= 0.0f) return s;
        RGB f = eval_bsdf(m, wo, s.wi, n);
        V3 h = make_dir_or(wo + s.wi);
        float pdf = (sp * pdf_vndf(wo, h, rough, n) + (1.0f - sp) * pdf_cos_hemi(nl)) * (1.0f - m.transmission);
        s.kind = BS_EVAL; s.f = f; s.pdf = pdf;
        s.type = 0;
    }
    return s;
}

// ---------------------------------------------------------------- lights
LD float inv_sq(float d) { if (d < MIN_LENGTH) return 0.0f; float d2 = d * d; return 1.0f / d2; }
LD float pdfw_from_area(float dist, float area, float c) {
    if (area < MIN_AREA || c < 1e-6f) return 0.0f;
    float d2 = dist * dist;
    return (d2 / area) / c;
}
LD float mis_power(float pf, float pg) {
    float f2 = pf * pf, g2 = pg * pg;
    return f2 / (f2 + g2 + 1e-10f);
}

struct LightSample {
    V3 pos, normal, dir;
    RGB emission;
    float pdf, dist;
};

// sampleLightTyped (light/light.hpp:187-335)
// Not inlined: the shading kernel samples lights at two call sites (volume
// scatter and surface NEE) and is limited by instruction fetch; one shared
// copy measured 3.6 % faster on the 1M-triangle frame.
static __device__ __noinline__ LightSample sample_light(const DevLight& L, V3 sp, float u1, float u2) {
    LightSample s;
    int type = __float_as_int(L.pos_type.w);
    s.emission = c3(L.emission_radius);
    s.normal = v3(0.f, 0.f, 1.f);
    s.pdf = 0.0f;
    s.dist = 0.0f;
    V3 lpos = f3(L.pos_type), lnorm = f3(L.normal_area);
    float area = L.normal_area.w, radius = L.emission_radius.w;
    if (type == LIGHT_POINT) {
        if (radius > MIN_LENGTH) {
            float z = 1.0f - 2.0f * u1;
            float r = sqrtf(smax(0.0f, 1.0f - z * z));
            float phi = kTWO_PI * u2;
            V3 od = v3(r * lucid_math::lm_cosf(phi), r * lucid_math::lm_sinf(phi), z);
            s.pos = lpos + od * radius;
            s.normal = od;
        } else {
            s.pos = lpos;
            s.normal = v3(0.f, 1.f, 0.f);
        }
        nwl(s.pos - sp, s.dir, s.dist);
        if (radius < MIN_LENGTH) {
            s.emission = s.emission * inv_sq(s.dist);
            s.pdf = 1.0f;
        } else {
            float cl = dot(s.normal, -s.dir);
            s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, area, cl);
        }
    } else if (type == LIGHT_SUN) {
        s.dir = -lnorm;
        s.pos = sp + s.dir * 1000000.0f;
        s.normal = lnorm;
        s.dist = 1000000.0f;
        s.pdf = 1.0f;
    } else if (type == LIGHT_SPOT) {
        s.pos = lpos;
        s.normal = lnorm;
        nwl(s.pos - sp, s.dir, s.dist);
        s.emission = s.emission * inv_sq(s.dist);
        float ca = dot(lnorm, -s.dir);
        float cc = L.v1_cosc.w;          // cos(spot_angle * 0.5) with lucid_math
        float blend = L.v2_blend.w;
        if (ca < cc) {
            s.emission = rgb(0.f, 0.f, 0.f);
        } else if (blend > 0.0f) {
            float t = (ca - cc) / (1.0f - cc);
            s.emission = s.emission * smin(1.0f, t / blend);
        }
        s.pdf = 1.0f;
    } else if (type == LIGHT_AREA) {
        int shape = __float_as_int(L.v0_shape.w);
        float sx = L.right_sx.w, sy = L.up_sy.w;
        float lx, ly;
        if (shape == AREA_DISK || shape == AREA_ELLIPSE) {
            float rs = sqrtf(u1);
            float th = kTWO_PI * u2;
            lx = sx * 0.5f * rs * lucid_math::lm_cosf(th);
            ly = sy * 0.5f * rs * lucid_math::lm_sinf(th);
        } else {
            lx = sx * (u1 - 0.5f);
            ly = sy * (u2 - 0.5f);
        }
        s.pos = lpos + f3(L.right_sx) * lx + f3(L.up_sy) * ly;
        s.normal = lnorm;
        nwl(s.pos - sp, s.dir, s.dist);
        float cl = dot(s.normal, -s.dir);
        s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, area, cl);
    } else {
        // emissive triangle: sampleTrianglePoint (light.hpp:146-170)
        V3 p0 = f3(L.v0_shape), p1 = f3(L.v1_cosc), p2 = f3(L.v2_blend);
        float su1 = sqrtf(u1);
        float b0 = 1.0f - su1;
        float b1 = u2 * su1;
        float b2 = 1.0f - b0 - b1;
        V3 d1, d2;
        float l1, l2;
        nwl(p1 - p0, d1, l1);
        nwl(p2 - p0, d2, l2);
        s.pos = p0 + d1 * (l1 * b1) + d2 * (l2 * b2);
        s.normal = lnorm;
        nwl(s.pos - sp, s.dir, s.dist);
        float cl = fabsf(dot(s.normal, -s.dir));
        s.pdf = (cl < 1e-6f) ? 0.0f : pdfw_from_area(s.dist, area, cl);
    }
    return s;
}
// pdfLightSampleTyped (light.hpp:344-358)
LD float pdf_light(float area, V3 sp, V3 lp, V3 ln) {
    V3 d;
    float dist;
    nwl(lp - sp, d, dist);
    float cl = fabsf(dot(ln, -d));
    if (cl < 1e-6f || area < MIN_AREA) return 0.0f;
    return pdfw_from_area(dist, area, cl);
}
LD float area_ratio(float num, float den) { return (den < MIN_AREA) ? 0.0f : num / den; }

// SceneLights::selectLight's index (scene_lights.hpp:130-144):
// min(std::lower_bound(cdf, u), n - 1).  The guide table narrows the binary
// search to the entries between two bucket boundaries; the result is the
// same index.  u is a multiple of 2^-23, so u * kLightGuide is exact.
LD int select_light(const DevScene& sc, float u) {
    int k = min((int)(u * (float)kLightGuide), kLightGuide - 1);
    int lo = __ldg(&sc.light_guide[k]), hi = __ldg(&sc.light_guide[k + 1]);
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&sc.light_cdf[mid]) < u) lo = mid + 1; else hi = mid;
    }
    return min(lo, sc.num_lights - 1);
}

// ---------------------------------------------------------------- volumes
constexpr float HG_INV_4PI = 1.0f / (4.0f * kPI);
LD float hg_eval(float g, float c) {
    float gg = g * g;
    float den = 1.0f + gg - 2.0f * g * c;
    float d = smax(den, 1e-8f);
    return HG_INV_4PI * (1.0f - gg) / (d * sqrtf(d));
}
LD V3 hg_sample(float g, V3 wo, float u1, float u2, float& pdf) {
    float ct;
    if (fabsf(g) < 1e-3f) {
        ct = 1.0f - 2.0f * u1;
    } else {
        float gg = g * g;
        float sqr = (1.0f - gg) / (1.0f - g + 2.0f * g * u1);
        ct = sclamp((1.0f + gg - sqr * sqr) / (2.0f * g), -1.0f, 1.0f);
    }
    float st = sqrtf(smax(0.0f, 1.0f - ct * ct));
    float phi = kTWO_PI * u2;
    V3 t, b;
    onb(wo, t, b);
    V3 l = v3(st * lucid_math::lm_cosf(phi), st * lucid_math::lm_sinf(phi), ct);
    pdf = hg_eval(g, ct);
    return v3(t.x * l.x + b.x * l.y + wo.x * l.z, t.y * l.x + b.y * l.y + wo.y * l.z,
              t.z * l.x + b.z * l.y + wo.z * l.z);
}
LD bool ray_aabb_segment(V3 o, V3 d, float tmax, const DevVolume& v, float& te, float& tx) {
    float t0 = 0.0f, t1 = tmax;
    const float* bmn = v.wmin;
    const float* bmx = v.wmax;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float ro = a == 0 ? o.x : a == 1 ? o.y : o.z;
        float rd = a == 0 ? d.x : a == 1 ? d.y : d.z;
        if (fabsf(rd) < 1e-12f) {
            if (ro < bmn[a] || ro > bmx[a]) return false;
            continue;
        }
        float inv = 1.0f / rd;
        float ta = (bmn[a] - ro) * inv, tb = (bmx[a] - ro) * inv;
        if (ta > tb) { float tt = ta; ta = tb; tb = tt; }
        if (ta > t0) t0 = ta;
        if (tb < t1) t1 = tb;
        if (t0 > t1) return false;
    }
    te = smax(0.0f, t0);
    tx = t1;
    return tx > te;
}
LD float grid_trilinear(const DevVolume& v, const float* grid, float wx, float wy, float wz) {
    float u = (wx - v.wmin[0]) / smax(1e-12f, v.wmax[0] - v.wmin[0]);
    float vv = (wy - v.wmin[1]) / smax(1e-12f, v.wmax[1] - v.wmin[1]);
    float w = (wz - v.wmin[2]) / smax(1e-12f, v.wmax[2] - v.wmin[2]);
    if (u < 0.0f || u > 1.0f || vv < 0.0f || vv > 1.0f || w < 0.0f || w > 1.0f) return 0.0f;
    int nx = v.dims[0], ny = v.dims[1], nz = v.dims[2];
    float fx = u * (float)nx - 0.5f, fy = vv * (float)ny - 0.5f, fz = w * (float)nz - 0.5f;
    if (fx < 0.0f || fx > (float)(nx - 1) || fy < 0.0f || fy > (float)(ny - 1) || fz < 0.0f || fz > (float)(nz - 1))
        return 0.0f;
    int ix = min(max((int)fx, 0), nx - 2), iy = min(max((int)fy, 0), ny - 2), iz = min(max((int)fz, 0), nz - 2);
    float tx = fx - (float)ix, ty = fy - (float)iy, tz = fz - (float)iz;
    const float* g = grid + v.grid_offset;
    size_t sx = 1, sy = (size_t)nx, sz = (size_t)nx * (size_t)ny;
    size_t base = (size_t)ix + sy * (size_t)iy + sz * (size_t)iz;
    float c000 = g[base], c100 = g[base + sx], c010 = g[base + sy], c110 = g[base + sx + sy];
    float c001 = g[base + sz], c101 = g[base + sx + sz], c011 = g[base + sy + sz], c111 = g[base + sx + sy + sz];
    float c00 = c000 * (1.0f - tx) + c100 * tx;
    float c10 = c010 * (1.0f - tx) + c110 * tx;
    float c01 = c001 * (1.0f - tx) + c101 * tx;
    float c11 = c011 * (1.0f - tx) + c111 * tx;
    float c0 = c00 * (1.0f - ty) + c10 * ty;
    float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}
LD int vol_nsteps(const DevVolume& v, float seg, float& step) {
    float extent = smax3(v.wmax[0] - v.wmin[0], v.wmax[1] - v.wmin[1], v.wmax[2] - v.wmin[2]);
    int md = max(max(v.dims[0], v.dims[1]), v.dims[2]);
    float voxel = extent / (float)max(1, md);
    step = smax(1e-4f, voxel * 0.5f);
    return min(2048, (int)(seg / step) + 1);
}
// transmittance_along_segment / extinction_transmittance_along_segment
// (volume/transmittance.hpp:77-209): extinction == false gives the Stage-A
// absorption-only variant.
LD RGB volume_transmittance(const DevScene& sc, V3 o, V3 d, float tmax, bool extinction) {
    float tr = 0.0f, tg = 0.0f, tb = 0.0f;
    for (int i = 0; i < sc.num_volumes; ++i) {
        const DevVolume& v = sc.volumes[i];
        float ti = 0.0f, to = 0.0f;
        if (!ray_aabb_segment(o, d, tmax, v, ti, to)) continue;
        float seg = to - ti;
        if (seg <= 0.0f) continue;
        float step;
        int ns = vol_nsteps(v, seg, step);
        float er, eg, eb;
        if (extinction) { er = 1.0f + v.absorption[0]; eg = 1.0f + v.absorption[1]; eb = 1.0f + v.absorption[2]; }
        else { er = 1.0f - v.color[0]; eg = 1.0f - v.color[1]; eb = 1.0f - v.color[2]; }
        for (int k = 0; k < ns; ++k) {
            float t = ti + ((float)k + 0.5f) * step;
            if (t > to) break;
            float dd = grid_trilinear(v, sc.grid, o.x + d.x * t, o.y + d.y * t, o.z + d.z * t);
            if (dd <= 0.0f) continue;
            float base = v.density * dd * step;
            tr += base * er;
            tg += base * eg;
            tb += base * eb;
        }
    }
    return rgb(lucid_math::lm_expf(-tr), lucid_math::lm_expf(-tg), lucid_math::lm_expf(-tb));
}
// sample_volume_distance (transmittance.hpp:220-288).  Returns the volume
// index that scattered, or -1.
LD int sample_volume_distance(const DevScene& sc, V3 o, V3 d, float tmax, Rng& rng, float& t_out) {
    int out = -1;
    float best = tmax;
    for (int i = 0; i < sc.num_volumes; ++i) {
        const DevVolume& v = sc.volumes[i];
        if (v.density <= 0.0f || v.grid_max <= 0.0f) continue;
        float ti = 0.0f, to = 0.0f;
        if (!ray_aabb_segment(o, d, tmax, v, ti, to)) continue;
        if (ti >= best) continue;
        float se = smin(to, best);
        if (se <= ti) continue;
        float em = smax3(1.0f + v.absorption[0], 1.0f + v.absorption[1], 1.0f + v.absorption[2]);
        float smx = v.density * v.grid_max * em;
        if (smx <= 0.0f) continue;
        float t = ti;
        bool scattered = false;
        for (int it = 0; it < 4096; ++it) {
            float us = smax(1e-12f, 1.0f - randf(rng));
            t += -lucid_math::lm_logf(us) / smx;
            if (t >= se) break;
            float dd = grid_trilinear(v, sc.grid, o.x + d.x * t, o.y + d.y * t, o.z + d.z * t);
            float st = v.density * dd * em;
            if (randf(rng) * smx < st) { scattered = true; break; }
        }
        if (scattered && t < best) { best = t; out = i; t_out = t; }
    }
    return out;
}

// ---------------------------------------------------------------- parity hash
LD uint64_t hpush(uint64_t h, uint32_t w) {
#pragma unroll
    for (int i = 0; i < 4; ++i) { h ^= (w >> (8 * i)) & 0xffu; h *= 1099511628211ULL; }
    return h;
}

}  // namespace lucid
