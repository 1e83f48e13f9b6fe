// lucid_diag_capi.cpp — C ABI of standalone diagnostic films (host only).
//
// The reference module exports DiagnosticFilm, DiagnosticPathTracer,
// DiagnosticExporter, PathTrace and PathDiagnosticRecorder for callers that
// record paths themselves (src/pybind_module.cpp:433-539; the add-on's
// DiagnosticsManager, LucidRenderer/diagnostics.py:111-330).  A standalone
// film here is the same host DiagFilm the renderer replays its device records
// into (csrc/lucid_diag.cpp); a PathTrace becomes one DiagRecord plus its
// material ids.  No CUDA call is made.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/lucid_cuda.h"
#include "lucid_diag.h"

struct LucidDiagFilm {
    lucid::DiagFilm film;
    LucidDiagConfig cfg{};
    std::mutex mu;
};

namespace {

void to_record(const LucidPathTrace& t, lucid::DiagRecord& r, int16_t* material) {
    std::memset(&r, 0, sizeof(r));
    const int d = (int)std::min<uint32_t>(t.depth, (uint32_t)lucid::kDiagMaxDepth);
    r.depth = (uint8_t)d;
    r.strategy = t.strategy;
    r.light_type = t.light_type;
    for (int c = 0; c < 3; ++c) r.contrib[c] = t.contribution[c];
    for (int i = 0; i < lucid::kDiagMaxDepth; ++i) material[i] = 0;
    for (int i = 0; i < d; ++i) {
        r.object_id[i] = t.vertices[i].object_id;
        r.bsdf[i] = t.vertices[i].bsdf_type;
        r.flags[i] = t.vertices[i].flags;
        material[i] = t.vertices[i].material_id;
        for (int c = 0; c < 3; ++c) { r.pos[i][c] = t.positions[i][c]; r.nrm[i][c] = t.normals[i][c]; }
    }
}

}  // namespace

extern "C" {

int lucid_diag_film_create(long long width, long long height, const LucidDiagConfig* config, LucidDiagFilm** out) {
    if (!out) return LUCID_ERR_INVALID;
    *out = nullptr;
    LucidDiagConfig c{2, 16, 4, 16, 0.001f, 3.0f, 0};   // PathRecordingConfig::standard()
    if (config) c = *config;
    if (width < 0 || height < 0 || width > (1 << 20) || height > (1 << 20) || c.subsample_factor < 1)
        return LUCID_ERR_INVALID;
    LucidDiagFilm* f = new (std::nothrow) LucidDiagFilm();
    if (!f) return LUCID_ERR_OOM;
    try {
        f->cfg = c;
        f->film.init((int)width, (int)height, c.subsample_factor);
        f->film.set_limits(c.max_groups_per_pixel, c.max_outliers_per_pixel);
    } catch (const std::bad_alloc&) {
        delete f;
        return LUCID_ERR_OOM;
    }
    *out = f;
    return LUCID_OK;
}

void lucid_diag_film_destroy(LucidDiagFilm* film) { delete film; }

int lucid_diag_film_record_path(LucidDiagFilm* film, long long x, long long y, const LucidPathTrace* trace) {
    if (!film || !trace) return LUCID_ERR_INVALID;
    lucid::DiagRecord r;
    int16_t material[lucid::kDiagMaxDepth];
    to_record(*trace, r, material);
    std::lock_guard<std::mutex> lk(film->mu);
    film->film.record_path(x, y, r, material);
    return LUCID_OK;
}

int lucid_diag_film_clear(LucidDiagFilm* film) {
    if (!film) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    film->film.clear();
    return LUCID_OK;
}

int lucid_diag_film_info(LucidDiagFilm* film, long long* out5) {
    if (!film || !out5) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    out5[0] = film->film.width();
    out5[1] = film->film.height();
    out5[2] = film->film.sampled_width();
    out5[3] = film->film.sampled_height();
    out5[4] = (long long)film->film.total_recorded();
    return LUCID_OK;
}

int lucid_diag_film_stats(LucidDiagFilm* film, LucidDiagStats* out) {
    if (!film || !out) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    film->film.stats(out);
    return LUCID_OK;
}

int lucid_diag_film_pixel(LucidDiagFilm* film, long long x, long long y, int sort_by_mean, LucidDiagPixel* info,
                          LucidDiagGroup* groups, int cap) {
    if (!film || !info) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    std::memset(info, 0, sizeof(*info));
    if (x < 0 || y < 0 || x > (1 << 30) || y > (1 << 30)) return 0;
    return film->film.export_pixel((int)x, (int)y, sort_by_mean != 0, info, groups, groups ? cap : 0);
}

int lucid_diag_film_top_groups(LucidDiagFilm* film, int n, int by_mean, LucidDiagGroup* groups, int32_t* xy,
                               int cap) {
    if (!film) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    return film->film.export_top(n, by_mean != 0, groups, xy, groups ? cap : 0);
}

int lucid_diag_film_coarse_stats(LucidDiagFilm* film, LucidDiagCoarse* out) {
    if (!film || !out) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    film->film.coarse_export(out);
    return 8;
}

int lucid_diag_film_suggestions(LucidDiagFilm* film, LucidDiagSuggestion* out, int cap) {
    if (!film) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    return film->film.suggestions(out, out ? cap : 0);
}

long long lucid_diag_film_export_binary(LucidDiagFilm* film, uint8_t* out, size_t cap) {
    if (!film) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    const std::vector<uint8_t> b = film->film.export_binary();
    if (out) std::memcpy(out, b.data(), std::min(cap, b.size()));
    return (long long)b.size();
}

long long lucid_diag_film_metadata_json(LucidDiagFilm* film, char* out, size_t cap) {
    if (!film) return LUCID_ERR_INVALID;
    std::lock_guard<std::mutex> lk(film->mu);
    const std::string m = film->film.metadata_json();
    if (out && cap > 0) {
        const size_t n = std::min(cap - 1, m.size());
        std::memcpy(out, m.data(), n);
        out[n] = 0;
    }
    return (long long)m.size();
}

uint64_t lucid_path_trace_hash(const LucidPathTrace* trace) {
    if (!trace) return 0;
    lucid::DiagRecord r;
    int16_t material[lucid::kDiagMaxDepth];
    to_record(*trace, r, material);
    return lucid::DiagFilm::hash(r, material);
}

int lucid_path_trace_coarse_type(const LucidPathTrace* trace) {
    if (!trace) return LUCID_ERR_INVALID;
    lucid::DiagRecord r;
    int16_t material[lucid::kDiagMaxDepth];
    to_record(*trace, r, material);
    return lucid::DiagFilm::coarse_type(r);
}

}  // extern "C"
