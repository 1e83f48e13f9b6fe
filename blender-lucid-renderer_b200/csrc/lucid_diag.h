// lucid_diag.h — DiagnosticFilm for the CUDA tracer (host side).
//
// The diagnostic kernels append one record per completed path (a path that
// reached a light, the environment or an emitter; diagnostic_integrator.hpp:
// 349-389) to a device buffer with warp-aggregated atomics.  After the render
// the records are sorted into the single-threaded order of the reference's
// tile loop (micro-tiles, pixels, samples, records along the path) and
// replayed into the per-pixel statistics below: Welford mean/variance,
// coarse-type stats, a 3-sigma outlier ring and up to 16 path groups per film
// cell keyed by the FNV-1a path hash, with the reference's log2-weighted
// variance eviction (diagnostics/pixel_path_data.hpp:53-220).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/lucid_cuda.h"

namespace lucid {

constexpr int kDiagMaxDepth = 16;

// One completed path as the kernels write it (512 B).
struct DiagRecord {
    uint32_t pixel;      // tile-local pixel index (y * tile_w + x)
    uint32_t sample;     // sample index within the call
    uint32_t seq;        // bounce at which the path completed
    uint8_t strategy, light_type, depth, pad;
    float contrib[3];
    int32_t object_id[kDiagMaxDepth];
    uint8_t bsdf[kDiagMaxDepth];
    uint8_t flags[kDiagMaxDepth];
    float pos[kDiagMaxDepth][3];
    float nrm[kDiagMaxDepth][3];
    uint32_t pad2;
};
static_assert(sizeof(DiagRecord) == 512, "DiagRecord layout");

// The compact form the diagnostic kernel writes: a 32-B head and one 32-B
// entry per vertex, in 16-B units, found through an index of unit offsets
// (a Cornell path of a few bounces takes 100-200 B instead of 512).  The
// replay expands each one into a DiagRecord.
struct DiagRecHead {
    uint32_t pixel, sample, seq;
    uint8_t strategy, light_type, depth, pad;
    float contrib[3];
    uint32_t pad2;
};
struct DiagRecVertex {
    int32_t object_id;
    uint8_t bsdf, flags, pad0, pad1;
    float pos[3];
    float nrm[3];
};
static_assert(sizeof(DiagRecHead) == 32 && sizeof(DiagRecVertex) == 32, "compact record layout");
constexpr size_t kDiagUnitBytes = 16;
inline unsigned diag_record_units(int depth) { return 2u + 2u * (unsigned)depth; }
inline void diag_expand(const DiagRecHead* h, DiagRecord& r) {
    r.pixel = h->pixel; r.sample = h->sample; r.seq = h->seq;
    r.strategy = h->strategy; r.light_type = h->light_type; r.depth = h->depth; r.pad = 0;
    r.contrib[0] = h->contrib[0]; r.contrib[1] = h->contrib[1]; r.contrib[2] = h->contrib[2];
    const DiagRecVertex* v = reinterpret_cast<const DiagRecVertex*>(h + 1);
    const int d = h->depth < kDiagMaxDepth ? h->depth : kDiagMaxDepth;
    for (int k = 0; k < d; ++k) {
        r.object_id[k] = v[k].object_id; r.bsdf[k] = v[k].bsdf; r.flags[k] = v[k].flags;
        for (int a = 0; a < 3; ++a) { r.pos[k][a] = v[k].pos[a]; r.nrm[k][a] = v[k].nrm[a]; }
    }
}

struct DiagStats {   // PathStatistics (path_stats.hpp:63-100)
    uint32_t count = 0;
    float mean[3] = {0, 0, 0}, m2[3] = {0, 0, 0}, var[3] = {0, 0, 0};
    void add(const float* v);
    float total_variance() const { return var[0] + var[1] + var[2]; }
    float mean_luminance() const { return 0.2126f * mean[0] + 0.7152f * mean[1] + 0.0722f * mean[2]; }
};

struct DiagGroup {   // PathGroup (path_stats.hpp:142-232)
    uint64_t hash = 0;
    DiagStats stats;
    uint8_t depth = 0, coarse = 0, light_type = 0, strategy = 0;
    int32_t object_id[kDiagMaxDepth] = {};
    uint8_t bsdf[kDiagMaxDepth] = {};
    uint8_t flags[kDiagMaxDepth] = {};
    float pos[kDiagMaxDepth][3] = {};
    float nrm[kDiagMaxDepth][3] = {};
};

struct DiagPixel {   // PixelPathData<16, 4>
    static constexpr int kGroups = 16, kOutliers = 4;
    // the groups' hashes side by side (the lookup of every recorded path
    // reads two cache lines instead of one per ~540-B group)
    uint64_t ghash[kGroups] = {};
    DiagGroup groups[kGroups];
    DiagStats coarse[8];
    uint64_t outlier_hash[kOutliers] = {};
    float outlier_c[kOutliers][3] = {};
    size_t num_groups = 0, num_outliers = 0, total = 0, overflow = 0;
    DiagStats total_stats;
    void record(const DiagRecord& r, uint64_t hash, uint8_t coarse_type);
    // Back to an empty cell: counters and statistics (group and outlier
    // entries past the counts are never read, so they are left as they are).
    void reset() {
        num_groups = num_outliers = total = overflow = 0;
        total_stats = DiagStats();
        for (auto& c : coarse) c = DiagStats();
    }
};

class DiagFilm {
public:
    void init(int tile_w, int tile_h, int subsample);
    void clear();
    void reset() { px_.clear(); dirty_.clear(); valid_ = false; w_ = h_ = sw_ = sh_ = 0; recorded_ = 0; }
    // Sorts the records (compact form: record i starts at unit index[i] of
    // `units`) into the reference's loop order and replays them.
    // threads: host threads to use (0: all).
    void replay(const uint8_t* units, const uint32_t* index, size_t n, int tile_w, unsigned threads = 0);
    // DiagnosticFilm::record_path (diagnostic_film.hpp:94-106): one path at
    // film pixel (x, y); out-of-range pixels are ignored.  material: the
    // vertices' material ids (the path hash includes them).
    void record_path(long long x, long long y, const DiagRecord& r, const int16_t* material);
    const DiagPixel* at(int x, int y) const;
    DiagPixel* at_mut(int x, int y);
    void stats(LucidDiagStats* out) const;
    void variance_map(float* out) const;   // tile_w * tile_h floats, cell variance per pixel
    // get_pixel_diagnostic's export: sorts the cell's groups in place.
    int export_pixel(int x, int y, bool sort_by_mean, LucidDiagPixel* info, LucidDiagGroup* groups, int cap);
    int export_top(int n, bool by_mean, LucidDiagGroup* groups, int32_t* xy, int cap) const;
    static void export_group(const DiagGroup& g, LucidDiagGroup* o);
    // DiagnosticExporter (diagnostic_export.hpp:78-220)
    void coarse_export(LucidDiagCoarse* out) const;   // 8 entries
    int suggestions(LucidDiagSuggestion* out, int cap) const;
    std::vector<uint8_t> export_binary() const;
    std::string metadata_json() const;
    void set_limits(int max_groups, int max_outliers) { max_groups_ = max_groups; max_outliers_ = max_outliers; }
    int width() const { return w_; }
    int height() const { return h_; }
    int sampled_width() const { return sw_; }
    int sampled_height() const { return sh_; }
    int subsample() const { return sf_; }
    size_t total_recorded() const { return recorded_; }
    bool valid() const { return valid_; }
    static uint64_t hash(const DiagRecord& r);
    // PathTrace::hash (path_types.hpp:321-343) with explicit material ids
    static uint64_t hash(const DiagRecord& r, const int16_t* material);
    static uint8_t coarse_type(const DiagRecord& r);

private:
    int w_ = 0, h_ = 0, sf_ = 2, sw_ = 0, sh_ = 0, max_groups_ = 16, max_outliers_ = 4;
    bool valid_ = false;
    size_t recorded_ = 0;
    std::vector<DiagPixel> px_;
    // replay scratch (counts per cell, bucket starts, each record's cell, the
    // (order key, record) pairs), kept between calls
    std::vector<uint32_t> scr_count_, scr_start_, scr_cell_;
    std::vector<std::pair<uint64_t, uint32_t>> scr_order_;
    std::vector<unsigned char> dirty_;   // cells that recorded a path since they were last reset
};

}  // namespace lucid
