// lucid_diag.cpp — host DiagnosticFilm: ordered replay of the GPU's completed
// path records (see lucid_diag.h).  Compiled with -ffp-contract=off.
#include "lucid_diag.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <thread>

namespace lucid {

void DiagStats::add(const float* v) {   // path_stats.hpp:63-100
    ++count;
    if (count == 1) {
        for (int c = 0; c < 3; ++c) { mean[c] = v[c]; m2[c] = 0.0f; var[c] = 0.0f; }
        return;
    }
    float d[3], d2[3];
    for (int c = 0; c < 3; ++c) d[c] = v[c] - mean[c];
    for (int c = 0; c < 3; ++c) mean[c] += d[c] / (float)count;
    for (int c = 0; c < 3; ++c) d2[c] = v[c] - mean[c];
    for (int c = 0; c < 3; ++c) m2[c] += d[c] * d2[c];
    float nm1 = (float)(count - 1);
    for (int c = 0; c < 3; ++c) var[c] = m2[c] / nm1;
}

// PathTrace::hash (path_types.hpp:321-343): FNV-1a over the depth and every
// vertex's (object id, material id 0 or -1, BSDF class, flags), with the
// signed ids sign-extended to 64 bits.
uint64_t DiagFilm::hash(const DiagRecord& r) {
    // the diagnostic integrators record material 0 on surfaces and -1 on the
    // final light vertex, the only Emission vertex of their paths
    int16_t material[kDiagMaxDepth];
    for (int i = 0; i < kDiagMaxDepth; ++i) material[i] = r.bsdf[i] == 4 ? -1 : 0;
    return hash(r, material);
}

uint64_t DiagFilm::hash(const DiagRecord& r, const int16_t* material_ids) {
    uint64_t h = 14695981039346656037ULL;
    h ^= (uint64_t)r.depth;
    h *= 1099511628211ULL;
    for (int i = 0; i < r.depth; ++i) {
        const int16_t material = material_ids[i];
        h ^= (uint64_t)(int64_t)r.object_id[i];
        h *= 1099511628211ULL;
        h ^= (uint64_t)(int64_t)material;
        h *= 1099511628211ULL;
        h ^= (uint64_t)r.bsdf[i];
        h *= 1099511628211ULL;
        h ^= (uint64_t)r.flags[i];
        h *= 1099511628211ULL;
    }
    return h;
}

uint8_t DiagFilm::coarse_type(const DiagRecord& r) {   // path_types.hpp:354-372
    uint8_t t = 0;
    for (int i = 0; i < r.depth; ++i) {
        if (r.flags[i] & 2) t |= 1;
        if (r.flags[i] & 1) t |= 2;
    }
    if (r.depth > 2) t |= 4;
    return t;
}

// PixelPathData::record_path (pixel_path_data.hpp:53-89).
void DiagPixel::record(const DiagRecord& r, uint64_t h, uint8_t coarse_t) {
    ++total;
    total_stats.add(r.contrib);
    coarse[coarse_t].add(r.contrib);
    if (total >= 10) {   // is_outlier (:172-192)
        const float th = 3.0f;
        bool out = false;
        for (int c = 0; c < 3; ++c) {
            float sd = std::sqrt(total_stats.var[c] + 1e-10f);
            float dv = std::fabs(r.contrib[c] - total_stats.mean[c]);
            out = out || (dv > th * sd);
        }
        if (out) {
            size_t i = num_outliers % kOutliers;
            outlier_hash[i] = h;
            for (int c = 0; c < 3; ++c) outlier_c[i][c] = r.contrib[c];
            ++num_outliers;
        }
    }
    for (size_t i = 0; i < num_groups; ++i)
        if (ghash[i] == h) { groups[i].stats.add(r.contrib); return; }
    auto init_from = [&](DiagGroup& g) {   // PathGroup::init_from (path_stats.hpp:161-178)
        g.hash = h;
        g.depth = (uint8_t)std::min<int>(r.depth, kDiagMaxDepth);
        g.coarse = coarse_t;
        g.light_type = r.light_type;
        g.strategy = r.strategy;
        for (int k = 0; k < g.depth; ++k) {
            g.object_id[k] = r.object_id[k]; g.bsdf[k] = r.bsdf[k]; g.flags[k] = r.flags[k];
            for (int c = 0; c < 3; ++c) { g.pos[k][c] = r.pos[k][c]; g.nrm[k][c] = r.nrm[k][c]; }
        }
        g.stats = DiagStats();
        g.stats.add(r.contrib);
    };
    if (num_groups < (size_t)kGroups) {
        ghash[num_groups] = h;
        init_from(groups[num_groups++]);
        return;
    }
    // evict_and_add (:203-220)
    size_t mi = 0;
    float mv = groups[0].stats.total_variance();
    for (size_t i = 1; i < num_groups; ++i) {
        float var = groups[i].stats.total_variance();
        float adj = var * std::log2((float)(groups[i].stats.count + 1));
        float madj = mv * std::log2((float)(groups[mi].stats.count + 1));
        if (adj < madj) { mi = i; mv = var; }
    }
    ++overflow;
    ghash[mi] = h;
    init_from(groups[mi]);
}

// A film of the same cell count as the last one only resets the cells that
// recorded paths since (a 1080p film at subsample 2 holds 4 GB of cells).
void DiagFilm::init(int tile_w, int tile_h, int subsample) {
    w_ = tile_w; h_ = tile_h; sf_ = std::max(1, subsample);
    sw_ = w_ / sf_; sh_ = h_ / sf_;
    const size_t n = (size_t)sw_ * sh_;
    if (px_.size() == n && dirty_.size() == n) {
        clear();
    } else {
        px_.assign(n, DiagPixel());
        dirty_.assign(n, 0);
    }
    recorded_ = 0;
    valid_ = true;
}

void DiagFilm::clear() {
    if (dirty_.size() != px_.size()) {
        for (auto& p : px_) p = DiagPixel();
        dirty_.assign(px_.size(), 0);
    } else {
        for (size_t c = 0; c < px_.size(); ++c)
            if (dirty_[c]) { px_[c].reset(); dirty_[c] = 0; }
    }
    recorded_ = 0;
}

void DiagFilm::replay(const uint8_t* units, const uint32_t* index, size_t n, int tile_w, unsigned threads) {
    // the reference's single-threaded loop order: 8x8 micro-tiles row-major,
    // pixels row-major inside one, samples, records along the path.  Cells
    // are independent, so the records are bucketed by cell, each cell's
    // bucket is sorted by (order key, arrival index) -- unique, and the
    // arrival index keeps each thread's program order for ties -- and the
    // cells are replayed, all on the host's threads.
    if (n == 0 || px_.empty()) return;
    const int nmx = (tile_w + 7) / 8;
    const size_t ncell = px_.size();
    auto head = [&](size_t i) {
        return reinterpret_cast<const DiagRecHead*>(units + (size_t)index[i] * kDiagUnitBytes);
    };
    auto key = [&](const DiagRecHead& r) {
        int x = (int)(r.pixel % (uint32_t)tile_w), y = (int)(r.pixel / (uint32_t)tile_w);
        uint64_t order = (uint64_t)((y / 8) * nmx + x / 8) * 64u + (uint64_t)((y % 8) * 8 + (x % 8));
        return (order << 40) | ((uint64_t)r.sample << 16) | (uint64_t)r.seq;
    };
    auto cell_of = [&](const DiagRecHead& r) -> uint32_t {
        int x = (int)(r.pixel % (uint32_t)tile_w), y = (int)(r.pixel / (uint32_t)tile_w);
        int sx = x / sf_, sy = y / sf_;
        return (sx >= sw_ || sy >= sh_) ? (uint32_t)ncell : (uint32_t)((size_t)sy * sw_ + sx);
    };
    const unsigned hw = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<size_t>(hw, std::max<size_t>(1, n / 4096));
    auto parallel = [&](auto&& fn) {   // fn(t, i0, i1) over the records
        if (nt <= 1) { fn(0u, (size_t)0, n); return; }
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) th.emplace_back(fn, t, n * t / nt, n * (t + 1) / nt);
        for (auto& x : th) x.join();
    };
    // counting sort by cell (bucket order inside a cell does not matter: the
    // per-cell sort below fixes it); the scratch arrays are kept between
    // calls, since first-touch page faults on fresh ones cost as much as the
    // sort itself
    if (scr_count_.size() < ncell + 1) scr_count_.resize(ncell + 1);
    if (scr_start_.size() < ncell + 2) scr_start_.resize(ncell + 2);
    if (scr_cell_.size() < n) scr_cell_.resize(n);
    if (scr_order_.size() < n) scr_order_.resize(n);
    uint32_t* count = scr_count_.data();
    uint32_t* start = scr_start_.data();
    uint32_t* cell = scr_cell_.data();
    std::pair<uint64_t, uint32_t>* order = scr_order_.data();
    std::memset(count, 0, (ncell + 1) * sizeof(uint32_t));
    parallel([&](unsigned, size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; ++i) {
            cell[i] = cell_of(*head(i));
            __atomic_fetch_add(&count[cell[i]], 1u, __ATOMIC_RELAXED);
        }
    });
    start[0] = 0;
    for (size_t c = 0; c <= ncell; ++c) start[c + 1] = start[c] + count[c];
    for (size_t c = 0; c <= ncell; ++c) count[c] = start[c];
    parallel([&](unsigned, size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; ++i)
            order[__atomic_fetch_add(&count[cell[i]], 1u, __ATOMIC_RELAXED)] = {key(*head(i)), (uint32_t)i};
    });
    const size_t in_film = start[ncell];
    recorded_ += in_film;
    if (in_film == 0) return;
    if (dirty_.size() != ncell) dirty_.assign(ncell, 1);
    auto work = [&](size_t c0, size_t c1) {
        for (size_t c = c0; c < c1; ++c) {
            auto b = order + start[c], e = order + start[c + 1];
            if (b == e) continue;
            dirty_[c] = 1;
            if (e - b > 1) std::sort(b, e);
            DiagRecord r;
            for (auto it = b; it != e; ++it) {
                diag_expand(head(it->second), r);
                px_[c].record(r, hash(r), coarse_type(r));
            }
        }
    };
    if (nt <= 1) {
        work(0, ncell);
        return;
    }
    // split the cells so that each thread gets about the same number of
    // records (a band's records fill only the band's rows of cells)
    std::vector<size_t> cut(nt + 1, ncell);
    cut[0] = 0;
    for (unsigned t = 1; t < nt; ++t) {
        const uint32_t target = (uint32_t)(in_film * t / nt);
        cut[t] = (size_t)(std::upper_bound(start, start + ncell + 1, target) - start) - 1;
        cut[t] = std::max(cut[t], cut[t - 1]);
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        if (cut[t + 1] > cut[t]) th.emplace_back(work, cut[t], cut[t + 1]);
    for (auto& t : th) t.join();
}

void DiagFilm::record_path(long long x, long long y, const DiagRecord& r, const int16_t* material) {
    if (!valid_ || x < 0 || y < 0) return;
    const long long sx = x / sf_, sy = y / sf_;
    if (sx >= sw_ || sy >= sh_) return;
    const size_t c = (size_t)sy * sw_ + sx;
    px_[c].record(r, hash(r, material), coarse_type(r));
    if (c < dirty_.size()) dirty_[c] = 1;
    ++recorded_;
}

const DiagPixel* DiagFilm::at(int x, int y) const {
    if (!valid_ || x < 0 || y < 0) return nullptr;
    int sx = x / sf_, sy = y / sf_;
    if (sx >= sw_ || sy >= sh_) return nullptr;
    return &px_[(size_t)sy * sw_ + sx];
}
DiagPixel* DiagFilm::at_mut(int x, int y) { return const_cast<DiagPixel*>(at(x, y)); }

void DiagFilm::stats(LucidDiagStats* out) const {
    std::memset(out, 0, sizeof(*out));
    for (const auto& p : px_)
        if (p.total > 0) {
            ++out->active_pixels;
            out->total_samples += p.total;
            out->total_groups += p.num_groups;
            out->total_overflow += p.overflow;
        }
    out->paths_recorded = recorded_;
}

void DiagFilm::variance_map(float* out) const {
    for (int y = 0; y < h_; ++y)
        for (int x = 0; x < w_; ++x) {
            const DiagPixel* p = at(x, y);
            out[(size_t)y * w_ + x] = p ? p->total_stats.total_variance() : 0.0f;
        }
}

void DiagFilm::export_group(const DiagGroup& g, LucidDiagGroup* o) {
    std::memset(o, 0, sizeof(*o));
    o->hash = g.hash; o->count = g.stats.count; o->depth = g.depth; o->coarse_type = g.coarse;
    o->light_type = g.light_type; o->strategy = g.strategy;
    for (int c = 0; c < 3; ++c) { o->mean_rgb[c] = g.stats.mean[c]; o->variance_rgb[c] = g.stats.var[c]; }
    o->mean_luminance = g.stats.mean_luminance();
    o->total_variance = g.stats.total_variance();
    for (int k = 0; k < g.depth; ++k) {
        o->object_ids[k] = g.object_id[k]; o->bsdf[k] = g.bsdf[k]; o->flags[k] = g.flags[k];
        for (int c = 0; c < 3; ++c) { o->positions[k][c] = g.pos[k][c]; o->normals[k][c] = g.nrm[k][c]; }
    }
}

// get_pixel_diagnostic (pybind_renderer.hpp:1008-1102).
int DiagFilm::export_pixel(int x, int y, bool sort_by_mean, LucidDiagPixel* info, LucidDiagGroup* groups, int cap) {
    std::memset(info, 0, sizeof(*info));
    DiagPixel* p = at_mut(x, y);
    if (!p) return 0;
    if (sort_by_mean)
        std::sort(p->groups, p->groups + p->num_groups, [](const DiagGroup& a, const DiagGroup& b) {
            return a.stats.mean_luminance() > b.stats.mean_luminance();
        });
    else
        std::sort(p->groups, p->groups + p->num_groups, [](const DiagGroup& a, const DiagGroup& b) {
            return a.stats.total_variance() > b.stats.total_variance();
        });
    for (size_t i = 0; i < p->num_groups; ++i) p->ghash[i] = p->groups[i].hash;   // keep the lookup array in step
    info->valid = 1;
    info->sample_count = (uint32_t)p->total;
    info->group_count = (uint32_t)p->num_groups;
    info->outlier_count = (uint32_t)p->num_outliers;
    info->overflow_count = (uint32_t)p->overflow;
    info->variance = p->total_stats.total_variance();
    for (int c = 0; c < 3; ++c) info->mean_rgb[c] = p->total_stats.mean[c];
    int n = (int)std::min<size_t>(p->num_groups, (size_t)std::max(cap, 0));
    for (int i = 0; i < n; ++i) export_group(p->groups[i], groups + i);
    return n;
}

// top_groups_by_variance / top_groups_by_mean (diagnostic_film.hpp:160-222):
// cells in row-major order, groups in cell order, std::partial_sort.
int DiagFilm::export_top(int n, bool by_mean, LucidDiagGroup* groups, int32_t* xy, int cap) const {
    struct Ref { int x, y; const DiagGroup* g; };
    std::vector<Ref> all;
    for (int sy = 0; sy < sh_; ++sy)
        for (int sx = 0; sx < sw_; ++sx) {
            const DiagPixel& px = px_[(size_t)sy * sw_ + sx];
            for (size_t i = 0; i < px.num_groups; ++i)
                if (px.groups[i].stats.count >= (by_mean ? 1u : 2u)) all.push_back({sx * sf_, sy * sf_, &px.groups[i]});
        }
    size_t limit = std::min((size_t)std::max(n, 0), all.size());
    if (by_mean)
        std::partial_sort(all.begin(), all.begin() + limit, all.end(), [](const Ref& a, const Ref& b) {
            return a.g->stats.mean_luminance() > b.g->stats.mean_luminance();
        });
    else
        std::partial_sort(all.begin(), all.begin() + limit, all.end(), [](const Ref& a, const Ref& b) {
            return a.g->stats.total_variance() > b.g->stats.total_variance();
        });
    int m = (int)std::min(limit, (size_t)std::max(cap, 0));
    for (int i = 0; i < m; ++i) {
        export_group(*all[i].g, groups + i);
        if (xy) { xy[2 * i] = all[i].x; xy[2 * i + 1] = all[i].y; }
    }
    return m;
}

}  // namespace lucid

// ---- DiagnosticExporter (diagnostics/diagnostic_export.hpp:78-220) ----
namespace lucid {

namespace {
const char* coarse_name(int t) {   // coarse_type_name (path_stats.hpp:26-40)
    static const char* names[8] = {"Direct-NoDelta-BSDF",   "Direct-NoDelta-NEE",   "Direct-Delta-BSDF",
                                   "Direct-Delta-NEE",      "Indirect-NoDelta-BSDF", "Indirect-NoDelta-NEE",
                                   "Indirect-Delta-BSDF",   "Indirect-Delta-NEE"};
    return names[t & 7];
}
void copy_str(char* dst, size_t cap, const char* src) {
    std::strncpy(dst, src, cap - 1);
    dst[cap - 1] = 0;
}
}  // namespace

// get_coarse_stats: cells are read at film position (2 sx, 2 sy) for every
// sampled (sx, sy), as the reference does whatever the subsample factor; a
// cell's stats are merged with a sample-weighted mean and the largest
// variance.
void DiagFilm::coarse_export(LucidDiagCoarse* out) const {
    struct Agg {
        uint64_t count = 0;
        float mean[3] = {0, 0, 0}, var[3] = {0, 0, 0};
    } agg[8];
    for (int sy = 0; sy < sh_; ++sy)
        for (int sx = 0; sx < sw_; ++sx) {
            const DiagPixel* px = at(sx * 2, sy * 2);
            if (!px) continue;
            for (int t = 0; t < 8; ++t) {
                const DiagStats& cs = px->coarse[t];
                if (cs.count == 0) continue;
                agg[t].count += cs.count;
                const float w = (float)cs.count / (float)agg[t].count;
                for (int c = 0; c < 3; ++c) {
                    agg[t].mean[c] = agg[t].mean[c] * (1.0f - w) + cs.mean[c] * w;
                    agg[t].var[c] = std::max(agg[t].var[c], cs.var[c]);
                }
            }
        }
    for (int t = 0; t < 8; ++t) {
        LucidDiagCoarse& o = out[t];
        std::memset(&o, 0, sizeof(o));
        o.type_id = t;
        copy_str(o.name, sizeof(o.name), coarse_name(t));
        o.sample_count = agg[t].count;
        o.mean_luminance = 0.2126f * agg[t].mean[0] + 0.7152f * agg[t].mean[1] + 0.0722f * agg[t].mean[2];
        o.variance_luminance = 0.2126f * 0.2126f * agg[t].var[0] + 0.7152f * 0.7152f * agg[t].var[1] +
                               0.0722f * 0.0722f * agg[t].var[2];
        for (int c = 0; c < 3; ++c) { o.mean_rgb[c] = agg[t].mean[c]; o.variance_rgb[c] = agg[t].var[c]; }
    }
}

// generate_suggestions: patterns among the ten highest-variance groups, then
// the share of cells that overflowed their group capacity.
int DiagFilm::suggestions(LucidDiagSuggestion* out, int cap) const {
    struct S {
        const char *cat, *sev, *msg, *act;
    };
    std::vector<S> list;
    std::vector<LucidDiagGroup> top(10);
    const int n = export_top(10, false, top.data(), nullptr, 10);
    if (n == 0) return 0;
    size_t glossy = 0, diffuse = 0, indirect = 0;
    for (int i = 0; i < n; ++i) {
        bool has_glossy = false;
        const bool has_indirect = top[i].depth > 2;
        for (int v = 0; v < top[i].depth && v < kDiagMaxDepth; ++v)
            if (top[i].bsdf[v] == 1) has_glossy = true;   // BsdfType::Glossy
        if (has_glossy) ++glossy;
        if (has_indirect) ++indirect;
        if (!has_glossy && !has_indirect) ++diffuse;
    }
    if (glossy > 3)
        list.push_back({"Settings", "warning", "High variance detected in glossy reflections",
                        "Consider increasing samples or using adaptive sampling for glossy materials"});
    if (indirect > 3)
        list.push_back({"Algorithm", "info", "Significant variance from indirect illumination",
                        "MIS algorithm recommended; consider path guiding for complex scenes"});
    if (diffuse > 3)
        list.push_back({"Scene", "info", "High variance in diffuse lighting",
                        "Check for small or distant light sources; consider area lights"});
    LucidDiagStats st;
    stats(&st);
    if (st.total_samples > 0 && (double)st.total_overflow > (double)st.active_pixels * 0.1)
        list.push_back({"Settings", "warning", "Many path types exceeded tracking capacity",
                        "Consider using 'Detailed' preset for more accurate analysis"});
    for (int i = 0; i < (int)list.size() && i < cap; ++i) {
        copy_str(out[i].category, sizeof(out[i].category), list[i].cat);
        copy_str(out[i].severity, sizeof(out[i].severity), list[i].sev);
        copy_str(out[i].message, sizeof(out[i].message), list[i].msg);
        copy_str(out[i].action, sizeof(out[i].action), list[i].act);
    }
    return (int)list.size();
}

// export_binary: "PVAR", version 1, film and sampled sizes (uint32), the
// subsample factor and capacities (one byte each, one zero byte), then per
// cell in row order: group count (uint16), samples (uint32), mean rgb and
// total variance (float32), all little-endian and unpadded.
std::vector<uint8_t> DiagFilm::export_binary() const {
    std::vector<uint8_t> b;
    auto put = [&](const void* p, size_t n) {
        const uint8_t* q = static_cast<const uint8_t*>(p);
        b.insert(b.end(), q, q + n);
    };
    put("PVAR", 4);
    const uint32_t hdr[5] = {1u, (uint32_t)w_, (uint32_t)h_, (uint32_t)sw_, (uint32_t)sh_};
    put(hdr, sizeof(hdr));
    const uint8_t cfg[4] = {(uint8_t)sf_, (uint8_t)max_groups_, (uint8_t)max_outliers_, 0};
    put(cfg, 4);
    b.reserve(b.size() + px_.size() * 22);
    for (const DiagPixel& p : px_) {
        const uint16_t gc = (uint16_t)p.num_groups;
        const uint32_t ts = (uint32_t)p.total;
        const float v = p.total_stats.total_variance();
        put(&gc, 2);
        put(&ts, 4);
        put(p.total_stats.mean, 12);
        put(&v, 4);
    }
    return b;
}

std::string DiagFilm::metadata_json() const {
    return "{\n  \"width\": " + std::to_string(w_) + ",\n  \"height\": " + std::to_string(h_) +
           ",\n  \"sampled_width\": " + std::to_string(sw_) + ",\n  \"sampled_height\": " + std::to_string(sh_) +
           ",\n  \"subsample_factor\": " + std::to_string(sf_) + ",\n  \"max_groups\": " +
           std::to_string(max_groups_) + ",\n  \"max_outliers\": " + std::to_string(max_outliers_) +
           ",\n  \"total_samples\": " + std::to_string(recorded_) + "\n}\n";
}

}  // namespace lucid
