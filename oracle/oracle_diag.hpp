// oracle_diag.hpp — CPU restatement of the reference's path-diagnostics
// integrators and DiagnosticFilm.  TEST INFRASTRUCTURE ONLY.
//
//   trace{Simple,NEE,MIS}WithDiagnostics   integrator/path_tracer.hpp:880-1514
//   PathDiagnosticRecorder                  diagnostics/diagnostic_integrator.hpp:87-389
//   classify_bsdf / is_delta_bsdf           diagnostic_integrator.hpp:25-60
//   PathTrace::hash / coarse_type           diagnostics/path_types.hpp:321-372
//   PathStatistics / PathGroup              diagnostics/path_stats.hpp:63-232
//   PixelPathData<16,4>                     diagnostics/pixel_path_data.hpp:53-220
//   DiagnosticFilm::record_path             diagnostics/diagnostic_film.hpp:94-106
//
// The reference updates a film cell from several OpenMP threads at once when
// the subsample factor merges pixels of one micro-tile (a data race); this
// restatement fixes the order to the single-threaded loop order: micro-tiles
// row-major, pixels row-major inside a micro-tile, samples, records in path
// order.
#pragma once

#include <array>
#include <cmath>
#include <vector>

#include "lucid_oracle.hpp"

namespace orc {

enum DBsdf : uint8_t { B_DIFFUSE = 0, B_GLOSSY = 1, B_MIRROR = 2, B_GLASS = 3, B_EMISSION = 4, B_ENV = 5 };
enum DLight : uint8_t { L_UNKNOWN = 0, L_POINT = 1, L_AREA = 2, L_DIRECTIONAL = 3, L_SPOT = 4, L_ENV = 5, L_EMISSIVE = 6 };
enum DStrategy : uint8_t { S_BSDF = 0, S_NEE = 1, S_MIS_BSDF = 2, S_MIS_NEE = 3 };
constexpr int kMaxPathDepth = 16;

struct PVertex {
    int32_t object_id = -1;
    int16_t material_id = -1;
    uint8_t bsdf = B_DIFFUSE;
    uint8_t flags = 0;   // 1 delta, 2 light sampled
};

struct PTrace {
    PVertex v[kMaxPathDepth];
    V3 pos[kMaxPathDepth], nrm[kMaxPathDepth];
    size_t depth = 0;
    RGB contrib;
    uint8_t light_type = L_UNKNOWN;
    uint8_t strategy = S_BSDF;
    uint64_t hash() const {   // path_types.hpp:321-343
        uint64_t h = 14695981039346656037ULL;
        h ^= depth;
        h *= 1099511628211ULL;
        for (size_t i = 0; i < depth; ++i) {
            h ^= static_cast<uint64_t>(static_cast<int64_t>(v[i].object_id));
            h *= 1099511628211ULL;
            h ^= static_cast<uint64_t>(static_cast<int64_t>(v[i].material_id));
            h *= 1099511628211ULL;
            h ^= static_cast<uint64_t>(v[i].bsdf);
            h *= 1099511628211ULL;
            h ^= static_cast<uint64_t>(v[i].flags);
            h *= 1099511628211ULL;
        }
        return h;
    }
    uint8_t coarse_type() const {   // path_types.hpp:354-372
        uint8_t t = 0;
        for (size_t i = 0; i < depth; ++i) {
            if (v[i].flags & 2) t |= 1;
            if (v[i].flags & 1) t |= 2;
        }
        if (depth > 2) t |= 4;
        return t;
    }
};

inline uint8_t classify_bsdf(const MatParams& m) {
    if (m.transmission > 0.5f) return B_GLASS;
    if (m.roughness < 0.01f && m.metallic > 0.5f) return B_MIRROR;
    if (m.metallic > 0.5f || m.roughness < 0.5f) return B_GLOSSY;
    return B_DIFFUSE;
}
inline bool is_delta_bsdf(const MatParams& m) {
    if (m.transmission > 0.5f && m.roughness < 0.01f) return true;
    if (m.metallic > 0.5f && m.roughness < 0.01f) return true;
    return false;
}
// to_light_source_type (path_types.hpp): EMISSIVE_MESH/AREA -> Area, POINT,
// SUN -> Directional, SPOT.
inline uint8_t light_source_type(LightType t) {
    switch (t) {
        case LightType::EMISSIVE_MESH: return L_AREA;
        case LightType::POINT: return L_POINT;
        case LightType::SUN: return L_DIRECTIONAL;
        case LightType::SPOT: return L_SPOT;
        case LightType::AREA: return L_AREA;
    }
    return L_UNKNOWN;
}

struct Recorder {
    PTrace cur;
    std::vector<PTrace> completed;
    void begin() { cur = PTrace(); completed.clear(); }
    void vertex(int32_t obj, uint8_t type, bool delta, V3 p, V3 n) {   // record_vertex_with_geometry
        if (cur.depth >= (size_t)kMaxPathDepth) return;
        PVertex v;
        v.object_id = obj; v.material_id = 0; v.bsdf = type; v.flags = delta ? 1 : 0;
        cur.v[cur.depth] = v;
        cur.pos[cur.depth] = p;
        cur.nrm[cur.depth] = n;
        ++cur.depth;
    }
    // record_completed_path_with_geometry (diagnostic_integrator.hpp:349-389)
    void completed_path(uint8_t strategy, int32_t light_id, uint8_t ltype, RGB c, V3 lpos) {
        PTrace p = cur;
        if (p.depth < (size_t)kMaxPathDepth) {
            PVertex v;
            v.object_id = (ltype == L_ENV) ? -1 : -(light_id + 2);
            v.material_id = -1;
            v.bsdf = B_EMISSION;
            v.flags = 0;
            p.v[p.depth] = v;
            p.pos[p.depth] = lpos;
            p.nrm[p.depth] = V3(0, 0, 0);
            ++p.depth;
        }
        p.light_type = ltype;
        p.strategy = strategy;
        p.contrib = c;
        completed.push_back(p);
    }
};

enum class DiagAlgo { SIMPLE, NEE, MIS };

// ray_hit_position / env_hit_position (path_tracer.hpp:852-876)
inline V3 ray_hit_pos(const Ray& r, float t) { return V3(r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t); }
inline V3 env_pos(const Ray& r) { return V3(r.o.x + r.d.x * 1000.0f, r.o.y + r.d.y * 1000.0f, r.o.z + r.d.z * 1000.0f); }

inline RGB trace_diag(const Scene& s, const SceneLights& sl, const Ray& ray, int max_depth, DiagAlgo algo, Rng& rng,
                      Recorder& rec) {
    RGB result(0, 0, 0), T(1, 1, 1);
    Ray cur = ray;
    float last_pdf = 0.0f;
    float tMin = 0.0f;
    const bool mis = algo == DiagAlgo::MIS;
    for (int depth = 0; depth < max_depth; ++depth) {
        Hit hit = intersect_scene(s, cur, tMin);
        LightHit lh = intersect_native(s, cur, depth);
        if (lh.hit && (!hit.hit || lh.t < hit.t)) {
            if (algo != DiagAlgo::NEE || depth == 0) {
                uint8_t lt = L_UNKNOWN;
                if (lh.index >= 0 && lh.index < (int)s.native.size()) lt = light_source_type(s.native[lh.index].type);
                V3 lp = ray_hit_pos(cur, lh.t);
                float mw = 1.0f;
                if (mis) {
                    float lpdf = 0.0f;
                    if (!sl.lights.empty() && lh.index >= 0) {
                        int sli = sl.native_start + lh.index;
                        if (sli >= 0 && sli < (int)sl.lights.size()) {
                            float sp = light_pick_pdf(sl, sli);
                            if (sp > 0.0f) lpdf = pdf_light(sl.lights[sli], cur.o, lh.point, lh.normal) * sp;
                        }
                    }
                    mw = (last_pdf > MIN_PDF && lpdf > MIN_PDF) ? mis_power(last_pdf, lpdf) : 1.0f;
                }
                RGB pc = mis ? mul(T, lh.emission) * mw : mul(T, lh.emission);
                rec.completed_path(mis ? S_MIS_BSDF : S_BSDF, lh.index, lt, pc, lp);
                result = result + pc;
            }
            break;
        }
        if (!hit.hit) {
            if (algo != DiagAlgo::NEE || depth == 0) {
                RGB env = mul(T, s.env_color * s.env_strength);
                rec.completed_path(mis ? S_MIS_BSDF : S_BSDF, -1, L_ENV, env, env_pos(cur));
                result = result + env;
            }
            break;
        }
        MatParams m = mat_params(*hit.mat, hit.uv);
        RGB emission = mat_emission(*hit.mat, hit.uv);
        uint8_t bt = classify_bsdf(m);
        bool delta = is_delta_bsdf(m);
        bool has_em = is_emissive(emission);
        V3 n = hit.normal;
        V3 wo = -cur.d;
        bool front = dot(wo, n) > 0;
        V3 sn = n;
        if (m.transmission < 0.5f && !front) sn = -n;
        if (algo == DiagAlgo::SIMPLE) {
            if (has_em) {
                RGB ec = mul(T, emission);
                rec.completed_path(S_BSDF, hit.mesh, L_EMISSIVE, ec, hit.point);
                result = result + ec;
                break;
            }
            rec.vertex(hit.mesh, bt, delta, hit.point, hit.normal);
        } else {
            bool do_nee = false;
            if (has_em && (mis || depth == 0)) {
                float mw = 1.0f;
                if (mis && !sl.lights.empty() && last_pdf > MIN_PDF) {
                    int li = sl.tri_light[hit.mesh][hit.tri];
                    if (li >= 0) {
                        float sp = light_pick_pdf(sl, li);
                        if (sp > 0.0f) {
                            float lpdf = pdf_light(sl.lights[li], cur.o, hit.point, hit.normal) * sp;
                            if (lpdf > MIN_PDF) mw = mis_power(last_pdf, lpdf);
                        }
                    }
                }
                RGB ec = mis ? mul(T, emission) * mw : mul(T, emission);
                rec.completed_path(mis ? S_MIS_BSDF : S_BSDF, hit.mesh, L_EMISSIVE, ec, hit.point);
                result = result + ec;
            } else if (!has_em) {
                rec.vertex(hit.mesh, bt, delta, hit.point, hit.normal);
                do_nee = true;
            }
            bool transmissive = m.transmission > 0.5f;
            if (do_nee && !sl.lights.empty() && !transmissive) {
                float usel = randf(rng);
                float lsp;
                int li = select_light(sl, usel, lsp);
                if (li >= 0 && lsp > 1e-6f) {
                    const Light& L = sl.lights[li];
                    float u1, u2; draw2(rng, u1, u2);
                    LightSample ls = sample_light(L, hit.point, u1, u2);
                    if (ls.pdf > MIN_PDF) {
                        float NdotL = dot(sn, ls.dir);
                        if (NdotL > 1e-6f) {
                            Ray sr{hit.point, ls.dir};
                            Hit sh = intersect_scene(s, sr, RAY_T_MIN, ls.dist);
                            if (!sh.hit) {
                                RGB f = eval_bsdf(m, wo, ls.dir, sn);
                                float pl = ls.pdf * lsp;
                                RGB nr;
                                if (mis) {
                                    float pb = pdf_bsdf(m, wo, ls.dir, sn);
                                    float mw = mis_power(pl, pb);
                                    nr = mul(bsdf_weight(f, NdotL, pl) * mw, ls.emission);
                                } else {
                                    nr = mul(bsdf_weight(f, NdotL, pl), ls.emission);
                                }
                                RGB tot = mul(T, nr);
                                rec.completed_path(mis ? S_MIS_NEE : S_NEE, li - sl.native_start,
                                                   light_source_type(L.type), tot, ls.pos);
                                result = result + tot;
                            }
                        }
                    }
                }
            }
        }
        V3 smp_n = (m.transmission > 0.5f) ? n : sn;
        float u1, u2, u3;
        draw3(rng, u1, u2, u3);
        BsdfSample bs = sample_bsdf(m, wo, smp_n, u1, u2, u3, rng);
        if (!bs.valid()) break;
        RGB w;
        if (!throughput_update(bs, smp_n, w)) break;
        T = mul(T, w);
        if (mis) last_pdf = next_mis_pdf(bs);
        if (depth >= 3) {
            float rr = smin(smax3(T.r, T.g, T.b), 0.95f);
            if (randf(rng) > rr) break;
            T = T * (1.0f / rr);
        }
        if (!rgb_valid(T)) break;
        cur = Ray{hit.point, bs.wi};
        tMin = RAY_T_MIN;
    }
    return result;
}

// ---- film ---------------------------------------------------------------
struct PStats {   // path_stats.hpp:63-100
    uint32_t count = 0;
    RGB mean, m2, variance;
    void add(RGB v) {
        ++count;
        if (count == 1) { mean = v; m2 = RGB(); variance = RGB(); return; }
        RGB d(v.r - mean.r, v.g - mean.g, v.b - mean.b);
        mean.r += d.r / (float)count; mean.g += d.g / (float)count; mean.b += d.b / (float)count;
        RGB d2(v.r - mean.r, v.g - mean.g, v.b - mean.b);
        m2.r += d.r * d2.r; m2.g += d.g * d2.g; m2.b += d.b * d2.b;
        float nm1 = (float)(count - 1);
        variance.r = m2.r / nm1; variance.g = m2.g / nm1; variance.b = m2.b / nm1;
    }
    float total_variance() const { return variance.r + variance.g + variance.b; }
    float mean_luminance() const { return 0.2126f * mean.r + 0.7152f * mean.g + 0.0722f * mean.b; }
};
struct PGroup {   // path_stats.hpp:142-232
    uint64_t hash = 0;
    PStats stats;
    uint8_t depth = 0, coarse = 0, light_type = 0, strategy = 0;
    PVertex v[kMaxPathDepth];
    V3 pos[kMaxPathDepth], nrm[kMaxPathDepth];
    void init_from(const PTrace& t) {
        hash = t.hash();
        depth = (uint8_t)std::min(t.depth, (size_t)kMaxPathDepth);
        coarse = t.coarse_type();
        light_type = t.light_type;
        strategy = t.strategy;
        for (size_t i = 0; i < depth; ++i) { v[i] = t.v[i]; pos[i] = t.pos[i]; nrm[i] = t.nrm[i]; }
        stats = PStats();
        stats.add(t.contrib);
    }
};
struct PixelData {   // pixel_path_data.hpp: PixelPathData<16, 4>
    static constexpr int kGroups = 16, kOutliers = 4;
    PGroup groups[kGroups];
    PStats coarse[8];
    uint64_t outlier_hash[kOutliers] = {};
    RGB outlier_c[kOutliers];
    size_t num_groups = 0, num_outliers = 0, total = 0, overflow = 0;
    PStats total_stats;
    bool is_outlier(const PTrace& t) const {
        if (total < 10) return false;
        const float th = 3.0f;
        float sr = std::sqrt(total_stats.variance.r + 1e-10f), sg = std::sqrt(total_stats.variance.g + 1e-10f),
              sb = std::sqrt(total_stats.variance.b + 1e-10f);
        float dr = std::fabs(t.contrib.r - total_stats.mean.r), dg = std::fabs(t.contrib.g - total_stats.mean.g),
              db = std::fabs(t.contrib.b - total_stats.mean.b);
        return (dr > th * sr) || (dg > th * sg) || (db > th * sb);
    }
    void record(const PTrace& t) {
        ++total;
        total_stats.add(t.contrib);
        coarse[t.coarse_type()].add(t.contrib);
        if (is_outlier(t)) {
            size_t i = num_outliers % kOutliers;
            outlier_hash[i] = t.hash();
            outlier_c[i] = t.contrib;
            ++num_outliers;
        }
        uint64_t h = t.hash();
        for (size_t i = 0; i < num_groups; ++i)
            if (groups[i].hash == h) { groups[i].stats.add(t.contrib); return; }
        if (num_groups < (size_t)kGroups) { groups[num_groups++].init_from(t); return; }
        size_t mi = 0;
        float mv = groups[0].stats.total_variance();
        for (size_t i = 1; i < num_groups; ++i) {
            float var = groups[i].stats.total_variance();
            float adj = var * std::log2((float)(groups[i].stats.count + 1));
            float madj = mv * std::log2((float)(groups[mi].stats.count + 1));
            if (adj < madj) { mi = i; mv = var; }
        }
        ++overflow;
        groups[mi].init_from(t);
    }
};
struct DiagFilm {
    size_t w = 0, h = 0, sf = 2, sw = 0, shh = 0;
    std::vector<PixelData> px;
    size_t recorded = 0;
    void init(size_t width, size_t height, size_t subsample) {
        w = width; h = height; sf = subsample; sw = w / sf; shh = h / sf;
        px.assign(sw * shh, PixelData());
        recorded = 0;
    }
    void record(size_t x, size_t y, const PTrace& t) {
        size_t sx = x / sf, sy = y / sf;
        if (sx >= sw || sy >= shh) return;
        px[sy * sw + sx].record(t);
        ++recorded;
    }
    const PixelData* at(size_t x, size_t y) const {
        size_t sx = x / sf, sy = y / sf;
        if (sx >= sw || sy >= shh) return nullptr;
        return &px[sy * sw + sx];
    }
};

inline DiagAlgo diag_algo_from(Algo a) {
    // render_tile's diagnostics dispatch (pybind_renderer.hpp:300-309):
    // "simple", "mis", everything else -> NEE
    if (a == Algo::SIMPLE) return DiagAlgo::SIMPLE;
    if (a == Algo::MIS) return DiagAlgo::MIS;
    return DiagAlgo::NEE;
}

}  // namespace orc
