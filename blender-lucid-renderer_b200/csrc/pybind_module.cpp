// pybind_module.cpp — the `lucidrenderer` Python module over the C ABI.
//
// Mirrors the reference module surface (LucidRenderer/cpp_renderer/src/
// pybind_module.cpp:38-543, PyRenderer in include/pybind_renderer.hpp) so the
// Blender add-on's callers (render_session.py, engine.py, viewport.py) work
// unchanged.  Every render entry point runs the CUDA wavefront tracer; there
// is no CPU path.  Render calls release the GIL, and cancel() may be called
// from another thread.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lucid_cuda.h"

namespace py = pybind11;

namespace {

// ---- diagnostics value types (diagnostics/path_stats_config.hpp,
// diagnostic_export.hpp:26-49, pybind_renderer.hpp:971-981) ----
struct PathRecordingConfig {
    int subsample_factor = 2, max_groups_per_pixel = 16, max_outliers_per_pixel = 4, max_depth = 16;
    float variance_threshold = 0.001f, outlier_threshold = 3.0f;
    static PathRecordingConfig minimal() { return {4, 8, 2, 8, 0.01f, 5.0f}; }
    static PathRecordingConfig standard() { return {}; }
    static PathRecordingConfig detailed() { return {1, 32, 8, 16, 0.0001f, 2.0f}; }
    // sampled pixels x (8 coarse stats + groups + outliers + 32 B) + 1 MiB
    size_t estimate_memory_bytes(size_t w, size_t h) const {
        size_t sf = (size_t)std::max(1, subsample_factor);
        size_t pixels = (w / sf) * (h / sf);
        size_t stats = 4 + 9 * sizeof(float);
        size_t group = 8 + stats + 16 * 8 + 2 * 16 * 12 + 4;
        size_t per_pixel = 8 * stats + (size_t)max_groups_per_pixel * group +
                           (size_t)max_outliers_per_pixel * (8 + 12) + 32;
        return pixels * per_pixel + 1024 * 1024;
    }
};

struct ExportedGroupInfo {
    size_t pixel_x = 0, pixel_y = 0;
    std::string signature, signature_heckbert;
    std::vector<int32_t> object_ids;
    std::string object_path;
    uint32_t sample_count = 0;
    float mean_luminance = 0.0f, variance_luminance = 0.0f;
    std::array<float, 3> mean_rgb{}, variance_rgb{};
    uint8_t depth = 0, coarse_type = 0;
    std::string coarse_type_name, strategy_name;
    std::vector<std::array<float, 3>> positions, normals;
};

enum class TopGroupSortBy { Variance, Mean };
// BsdfType and LightSourceType (diagnostics/path_types.hpp:28-120)
enum class BsdfType : uint8_t { Diffuse = 0, Glossy = 1, Mirror = 2, Glass = 3, Emission = 4, Environment = 5 };
enum class LightSourceType : uint8_t { Unknown = 0, Point = 1, Area = 2, Directional = 3, Spot = 4, Environment = 5,
                                       Emissive = 6 };

struct PixelDiagnosticInfo {
    bool valid = false;
    size_t sample_count = 0;
    float variance = 0.0f;
    size_t group_count = 0, outlier_count = 0;
    std::array<float, 3> mean_rgb{};
    std::vector<ExportedGroupInfo> top_groups;
};

struct GlobalDiagnosticStats {
    size_t total_samples = 0, active_pixels = 0, total_groups = 0, total_overflow = 0;
    float total_variance = 0.0f;
};

// ExportedCoarseStats and DiagnosticSuggestion (diagnostic_export.hpp:45-72).
struct ExportedCoarseStats {
    uint8_t type_id = 0;
    std::string name;
    size_t sample_count = 0;
    float mean_luminance = 0.0f, variance_luminance = 0.0f;
    std::array<float, 3> mean_rgb{}, variance_rgb{};
};
struct DiagnosticSuggestion {
    std::string category, severity, message, action;
};

// bsdf_type_short / bsdf_type_heckbert / light_source_heckbert
// (diagnostics/path_types.hpp:56-157), coarse_type_name (path_stats.hpp:26-40).
char bsdf_short(uint8_t t) { return t < 6 ? "DGMTLE"[t] : '?'; }
char bsdf_heckbert(uint8_t t) { return t < 6 ? "DSSSEE"[t] : '?'; }
const char* light_heckbert(uint8_t t) {
    switch (t) {
        case 1: case 3: case 4: return "LSD";
        case 2: return "LDD";
        case 5: return "LDE";
    }
    return "L??";
}
const char* coarse_name(uint8_t t) {
    static const char* n[8] = {"Direct-NoDelta-BSDF",   "Direct-NoDelta-NEE",   "Direct-Delta-BSDF",
                               "Direct-Delta-NEE",      "Indirect-NoDelta-BSDF", "Indirect-NoDelta-NEE",
                               "Indirect-Delta-BSDF",   "Indirect-Delta-NEE"};
    return n[t & 7];
}
const char* strategy_name(uint8_t s) {
    static const char* n[4] = {"BSDF", "NEE", "MIS_BSDF", "MIS_NEE"};
    return s < 4 ? n[s] : "Unknown";
}
std::string signature_of(const LucidDiagGroup& g) {
    std::string sig;
    for (int i = 0; i < g.depth; ++i) sig += bsdf_short(g.bsdf[i]);
    return sig;
}
std::string heckbert_of(const LucidDiagGroup& g) {   // PathGroup::signature_heckbert (path_stats.hpp:210-238)
    std::string sig = light_heckbert(g.light_type);
    int end = g.depth;
    while (end > 0 && (g.bsdf[end - 1] == 4 || g.bsdf[end - 1] == 5)) --end;
    if (end > 0) {
        sig += ' ';
        for (int i = 0; i < end; ++i) {
            sig += bsdf_heckbert(g.bsdf[i]);
            if (i + 1 < end) sig += ' ';
        }
    }
    return sig + " DSE";
}
float variance_luminance(const LucidDiagGroup& g) {   // PathStatistics::variance_luminance (path_stats.hpp:117-123)
    return 0.2126f * 0.2126f * g.variance_rgb[0] + 0.7152f * 0.7152f * g.variance_rgb[1] +
           0.0722f * 0.0722f * g.variance_rgb[2];
}

// The film an exporter reads: a renderer's (lucid_cuda_diag_*) or a
// standalone DiagnosticFilm (lucid_diag_film_*).
struct FilmRef {
    LucidCudaCtx* ctx = nullptr;
    LucidDiagFilm* film = nullptr;
    int stats(LucidDiagStats* s) const { return film ? lucid_diag_film_stats(film, s) : lucid_cuda_diag_stats(ctx, s); }
    int top(int n, int by_mean, LucidDiagGroup* g, int32_t* xy, int cap) const {
        return film ? lucid_diag_film_top_groups(film, n, by_mean, g, xy, cap)
                    : lucid_cuda_diag_top_groups(ctx, n, by_mean, g, xy, cap);
    }
    int coarse(LucidDiagCoarse* c) const { return film ? lucid_diag_film_coarse_stats(film, c) : lucid_cuda_diag_coarse_stats(ctx, c); }
    int suggestions(LucidDiagSuggestion* o, int cap) const {
        return film ? lucid_diag_film_suggestions(film, o, cap) : lucid_cuda_diag_suggestions(ctx, o, cap);
    }
    long long binary(uint8_t* o, size_t cap) const {
        return film ? lucid_diag_film_export_binary(film, o, cap) : lucid_cuda_diag_export_binary(ctx, o, cap);
    }
    long long metadata(char* o, size_t cap) const {
        return film ? lucid_diag_film_metadata_json(film, o, cap) : lucid_cuda_diag_metadata_json(ctx, o, cap);
    }
};

GlobalDiagnosticStats global_stats_of(const FilmRef& f) {   // DiagnosticFilm::global_stats (diagnostic_film.hpp:130-154)
    LucidDiagStats st{};
    GlobalDiagnosticStats out;
    if (f.stats(&st) != LUCID_OK) return out;
    out.total_samples = st.total_samples; out.active_pixels = st.active_pixels;
    out.total_groups = st.total_groups; out.total_overflow = st.total_overflow;
    return out;
}
// DiagnosticExporter::convert_refs (diagnostic_export.hpp:257-285)
std::vector<ExportedGroupInfo> top_groups_of(const FilmRef& f, size_t count, bool by_mean) {
    std::vector<LucidDiagGroup> g(std::max<size_t>(count, 1));
    std::vector<int32_t> xy(2 * g.size());
    int n = f.top((int)count, by_mean ? 1 : 0, g.data(), xy.data(), (int)g.size());
    std::vector<ExportedGroupInfo> out;
    for (int i = 0; i < n; ++i) {
        ExportedGroupInfo e;
        e.pixel_x = (size_t)xy[2 * i]; e.pixel_y = (size_t)xy[2 * i + 1];
        e.signature = signature_of(g[i]);
        e.sample_count = g[i].count;
        e.mean_luminance = g[i].mean_luminance;
        e.variance_luminance = variance_luminance(g[i]);
        for (int c = 0; c < 3; ++c) { e.mean_rgb[c] = g[i].mean_rgb[c]; e.variance_rgb[c] = g[i].variance_rgb[c]; }
        e.depth = g[i].depth; e.coarse_type = g[i].coarse_type;
        e.coarse_type_name = coarse_name(g[i].coarse_type);
        out.push_back(std::move(e));
    }
    return out;
}
// DiagnosticExporter queries (diagnostic_export.hpp:78-220)
std::vector<ExportedCoarseStats> coarse_stats_of(const FilmRef& f) {
    LucidDiagCoarse c[8];
    std::vector<ExportedCoarseStats> out;
    if (f.coarse(c) != 8) return out;
    for (int t = 0; t < 8; ++t) {
        ExportedCoarseStats e;
        e.type_id = (uint8_t)c[t].type_id; e.name = c[t].name; e.sample_count = (size_t)c[t].sample_count;
        e.mean_luminance = c[t].mean_luminance; e.variance_luminance = c[t].variance_luminance;
        for (int k = 0; k < 3; ++k) { e.mean_rgb[k] = c[t].mean_rgb[k]; e.variance_rgb[k] = c[t].variance_rgb[k]; }
        out.push_back(std::move(e));
    }
    return out;
}
std::vector<DiagnosticSuggestion> suggestions_of(const FilmRef& f) {
    LucidDiagSuggestion sg[8];
    int n = f.suggestions(sg, 8);
    std::vector<DiagnosticSuggestion> out;
    for (int i = 0; i < n && i < 8; ++i) out.push_back({sg[i].category, sg[i].severity, sg[i].message, sg[i].action});
    return out;
}
py::bytes binary_of(const FilmRef& f) {
    long long n = f.binary(nullptr, 0);
    if (n <= 0) return py::bytes("");
    std::string b((size_t)n, '\0');
    f.binary(reinterpret_cast<uint8_t*>(&b[0]), b.size());
    return py::bytes(b);
}
std::string metadata_of(const FilmRef& f) {
    long long n = f.metadata(nullptr, 0);
    if (n <= 0) return std::string();
    std::string m((size_t)n + 1, '\0');
    f.metadata(&m[0], m.size());
    m.resize((size_t)n);
    return m;
}

class Renderer {
public:
    Renderer() {
        const char* dev = std::getenv("LUCID_CUDA_DEVICE");
        int rc = lucid_cuda_create(dev ? std::atoi(dev) : 0, &ctx_);
        if (rc != LUCID_OK) throw std::runtime_error("lucid_cuda_create failed");
    }
    ~Renderer() { lucid_cuda_destroy(ctx_); }
    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;

    void cancel() { lucid_cuda_cancel(ctx_); }
    bool is_cancelled() { return lucid_cuda_is_cancelled(ctx_) == 1; }
    void reset_cancel() { lucid_cuda_reset_cancel(ctx_); }

    // load_scene_json (pybind_renderer.hpp:111-126): false + stderr on failure
    bool load_scene_json(const std::string& s) {
        int rc = lucid_cuda_load_scene_json(ctx_, s.data(), s.size());
        if (rc != LUCID_OK) {
            std::fprintf(stderr, "[lucidrenderer] Failed to load scene: %s\n", lucid_cuda_last_error(ctx_));
            scene_loaded_ = false;
            return false;
        }
        scene_loaded_ = true;
        int st[8];
        lucid_cuda_scene_stats(ctx_, st);
        mesh_count_ = st[0];
        return true;
    }
    void set_camera(float px, float py, float pz, float dx, float dy, float dz, float ux, float uy, float uz,
                    float fov) {
        lucid_cuda_set_camera(ctx_, px, py, pz, dx, dy, dz, ux, uy, uz, fov);
        camera_set_ = true;
        cam_pos_[0] = px; cam_pos_[1] = py; cam_pos_[2] = pz;
    }
    void set_algorithm(const std::string& a) {
        algorithm_ = a;
        lucid_cuda_set_algorithm(ctx_, a.c_str());
    }
    std::string get_algorithm() const { return algorithm_; }
    bool is_scene_loaded() const { return scene_loaded_; }
    bool is_camera_set() const { return camera_set_; }
    int get_mesh_count() const { return scene_loaded_ ? mesh_count_ : 0; }

    // Renders into `px` (tw * th * 4 floats; a zero image when the render
    // fails before its copy, the library's own guarantee); the
    // return-code handling of pybind_renderer.hpp:185-361 (no scene: a zero
    // buffer and a message; cancelled: the partial sum).
    void render_into(float* px, int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth) {
        LucidRenderParams p{tx, ty, tw, th, fw, fh, samples, offset, depth, 0};
        int rc = lucid_cuda_render(ctx_, &p, px, nullptr);
        if (rc != LUCID_ERR_NO_SCENE) { last_tile_w_ = tw; last_tile_h_ = th; }
        if (rc == LUCID_ERR_NO_SCENE) {
            // the reference returns a zero buffer (pybind_renderer.hpp:200-203)
            std::fprintf(stderr, "[lucidrenderer] Scene or camera not set\n");
            return;
        }
        if (rc == LUCID_ERR_CANCELLED) return;   // partial result, is_cancelled() stays true
        if (rc != LUCID_OK) throw std::runtime_error(std::string("render failed: ") + lucid_cuda_last_error(ctx_));
    }
    std::vector<float> render(int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth) {
        if (tw <= 0 || th <= 0) throw std::invalid_argument("tile size must be positive");
        std::vector<float> px((size_t)tw * th * 4, 0.0f);
        render_into(px.data(), tx, ty, tw, th, fw, fh, samples, offset, depth);
        return px;
    }
    std::vector<float> render_debug(int tx, int ty, int tw, int th, int fw, int fh, const std::string& mode) {
        if (tw <= 0 || th <= 0) throw std::invalid_argument("tile size must be positive");
        std::vector<float> px((size_t)tw * th * 4, 0.0f);
        int rc = lucid_cuda_render_debug(ctx_, tx, ty, tw, th, fw, fh, mode.c_str(), px.data());
        if (rc == LUCID_ERR_NO_SCENE) return px;
        if (rc != LUCID_OK) throw std::runtime_error(std::string("render_debug failed: ") + lucid_cuda_last_error(ctx_));
        return px;
    }

    // object names for diagnostics display (pybind_renderer.hpp:1141-1173)
    void set_object_names(const std::vector<std::string>& n) { names_ = n; }
    std::string get_object_name(int id) const {
        if (id < 0) return "Environment";
        if ((size_t)id < names_.size()) return names_[id];
        return "Object_" + std::to_string(id);
    }
    // object_path_string without a light type (pybind_renderer.hpp:1198-1268)
    std::string object_path_string(const std::vector<int32_t>& ids) const {
        if (ids.empty()) return "Camera";
        std::string path;
        size_t start = ids.size();
        int32_t last = ids[start - 1];
        if (last <= -2) { path = "Light(?)"; --start; }
        else if (last == -1) { path = "Environment(?)"; --start; }
        else path = "(terminated)";
        for (size_t i = start; i > 0; --i) path += " \xe2\x86\x92 " + get_object_name(ids[i - 1]);
        return path + " \xe2\x86\x92 Camera";
    }

    // object_path_string with the light type (pybind_renderer.hpp:1198-1268)
    std::string object_path_typed(const std::vector<int32_t>& ids, uint8_t light_type) const {
        if (ids.empty()) return "Camera";
        std::string path;
        size_t start = ids.size();
        int32_t last = ids[start - 1];
        if (light_type == 5) {
            path = "Environment";
            if (last == -1) --start;
        } else if (light_type == 6) {
            path = get_object_name(last);
            --start;
        } else if (light_type >= 1 && light_type <= 4) {
            static const char* names[5] = {"", "PointLight", "AreaLight", "SunLight", "SpotLight"};
            path = names[light_type];
            if (last <= -2) --start;
        } else if (last <= -2) { path = "Light(?)"; --start; }
        else if (last == -1) { path = "Environment(?)"; --start; }
        else path = "(terminated)";
        for (size_t i = start; i > 0; --i) path += " \xe2\x86\x92 " + get_object_name(ids[i - 1]);
        return path + " \xe2\x86\x92 Camera";
    }

    // ---- path diagnostics (pybind_renderer.hpp:893-1102) ----
    void enable_diagnostics(const PathRecordingConfig& c) {
        LucidDiagConfig cfg{c.subsample_factor, c.max_groups_per_pixel, c.max_outliers_per_pixel, c.max_depth,
                            c.variance_threshold, c.outlier_threshold, 0};
        if (lucid_cuda_diag_enable(ctx_, &cfg) != LUCID_OK)
            throw std::invalid_argument(std::string("enable_diagnostics: ") + lucid_cuda_last_error(ctx_));
        diag_cfg_ = c;
    }
    void disable_diagnostics() { lucid_cuda_diag_disable(ctx_); }
    bool is_diagnostics_enabled() { return lucid_cuda_diag_enabled(ctx_) == 1; }
    void clear_diagnostics() { lucid_cuda_diag_clear(ctx_); }
    GlobalDiagnosticStats get_diagnostic_stats() { return global_stats_of(FilmRef{ctx_, nullptr}); }
    size_t diag_paths_recorded() {
        LucidDiagStats st{};
        return lucid_cuda_diag_stats(ctx_, &st) == LUCID_OK ? (size_t)st.paths_recorded : 0;
    }
    std::vector<float> get_diagnostic_variance_map() {
        std::vector<float> v((size_t)last_tile_w_ * last_tile_h_);
        int n = v.empty() ? 0 : lucid_cuda_diag_variance_map(ctx_, v.data(), v.size());
        v.resize(n > 0 ? (size_t)n : 0);
        return v;
    }
    // DiagnosticFilm::metadata_json (diagnostic_film.hpp:230-243)
    std::string export_diagnostic_json() {
        if (lucid_cuda_diag_enabled(ctx_) != 1 || last_tile_w_ == 0) return "{}";
        int sf = std::max(1, diag_cfg_.subsample_factor);
        std::string j = "{\n";
        j += "  \"width\": " + std::to_string(last_tile_w_) + ",\n";
        j += "  \"height\": " + std::to_string(last_tile_h_) + ",\n";
        j += "  \"sampled_width\": " + std::to_string(last_tile_w_ / sf) + ",\n";
        j += "  \"sampled_height\": " + std::to_string(last_tile_h_ / sf) + ",\n";
        j += "  \"subsample_factor\": " + std::to_string(sf) + ",\n";
        j += "  \"max_groups\": " + std::to_string(diag_cfg_.max_groups_per_pixel) + ",\n";
        j += "  \"max_outliers\": " + std::to_string(diag_cfg_.max_outliers_per_pixel) + ",\n";
        j += "  \"total_samples\": " + std::to_string(diag_paths_recorded()) + "\n";
        j += "}\n";
        return j;
    }
    // DiagnosticExporter::convert_refs (diagnostic_export.hpp:257-285)
    std::vector<ExportedGroupInfo> get_top_variance_groups(size_t count) { return top_groups(count, false); }
    std::vector<ExportedGroupInfo> top_groups(size_t count, bool by_mean) {
        return top_groups_of(FilmRef{ctx_, nullptr}, count, by_mean);
    }
    FilmRef film_ref() { return FilmRef{ctx_, nullptr}; }
    // get_pixel_diagnostic (pybind_renderer.hpp:1008-1102)
    PixelDiagnosticInfo get_pixel_diagnostic(size_t x, size_t y, TopGroupSortBy sort_by) {
        PixelDiagnosticInfo info;
        LucidDiagPixel px{};
        std::vector<LucidDiagGroup> g(64);
        int n = lucid_cuda_diag_pixel(ctx_, (int)x, (int)y, sort_by == TopGroupSortBy::Mean, &px, g.data(), (int)g.size());
        if (n < 0 || !px.valid) return info;
        info.valid = true;
        info.sample_count = px.sample_count;
        info.variance = px.variance;
        info.group_count = px.group_count;
        info.outlier_count = px.outlier_count;
        for (int c = 0; c < 3; ++c) info.mean_rgb[c] = px.mean_rgb[c];
        for (int i = 0; i < n; ++i) {
            const LucidDiagGroup& gi = g[i];
            ExportedGroupInfo e;
            e.pixel_x = x; e.pixel_y = y;
            e.signature = signature_of(gi);
            e.signature_heckbert = heckbert_of(gi);
            e.object_ids.assign(gi.object_ids, gi.object_ids + gi.depth);
            e.sample_count = gi.count;
            e.mean_luminance = gi.mean_luminance;
            e.variance_luminance = gi.total_variance;
            for (int c = 0; c < 3; ++c) { e.mean_rgb[c] = gi.mean_rgb[c]; e.variance_rgb[c] = gi.variance_rgb[c]; }
            e.depth = gi.depth; e.coarse_type = gi.coarse_type;
            e.coarse_type_name = coarse_name(gi.coarse_type);
            e.strategy_name = strategy_name(gi.strategy);
            e.object_path = object_path_typed(e.object_ids, gi.light_type);
            e.positions.push_back({cam_pos_[0], cam_pos_[1], cam_pos_[2]});
            for (int k = 0; k < gi.depth; ++k) {
                e.positions.push_back({gi.positions[k][0], gi.positions[k][1], gi.positions[k][2]});
                e.normals.push_back({gi.normals[k][0], gi.normals[k][1], gi.normals[k][2]});
            }
            info.top_groups.push_back(std::move(e));
        }
        return info;
    }

    // async accumulator (pybind_renderer.hpp:689-856)
    void start_async(int w, int h, int depth) {
        int rc = lucid_cuda_async_start(ctx_, w, h, depth);
        if (rc == LUCID_OK) { async_w_ = w; async_h_ = h; }
        else if (rc != LUCID_ERR_NO_SCENE)
            std::fprintf(stderr, "[lucidrenderer] start_async failed: %s\n", lucid_cuda_last_error(ctx_));
    }
    std::pair<int, std::vector<float>> poll_async() {
        int n = 0;
        std::vector<float> px((size_t)async_w_ * async_h_ * 4);
        if (lucid_cuda_async_running(ctx_) != 1 && lucid_cuda_async_revision(ctx_) <= 0) return {0, {}};
        if (lucid_cuda_async_poll(ctx_, &n, px.data(), px.size()) != LUCID_OK || n == 0) return {0, {}};
        return {n, std::move(px)};
    }
    void reset_async(int w, int h, int depth) {
        if (lucid_cuda_async_reset(ctx_, w, h, depth) != LUCID_OK)
            std::fprintf(stderr, "[lucidrenderer] reset_async failed: %s\n", lucid_cuda_last_error(ctx_));
        else { async_w_ = w; async_h_ = h; }
    }
    void stop_async() { lucid_cuda_async_stop(ctx_); }
    bool async_running() { return lucid_cuda_async_running(ctx_) == 1; }
    int async_revision() { int r = lucid_cuda_async_revision(ctx_); return r < 0 ? 0 : r; }

    LucidCudaCtx* ctx() { return ctx_; }

private:
    LucidCudaCtx* ctx_ = nullptr;
    bool scene_loaded_ = false, camera_set_ = false;
    int mesh_count_ = 0;
    std::string algorithm_ = "nee";
    std::vector<std::string> names_;
    int async_w_ = 0, async_h_ = 0;
    float cam_pos_[3] = {0.0f, 0.0f, 0.0f};
    int last_tile_w_ = 0, last_tile_h_ = 0;
    PathRecordingConfig diag_cfg_;
};

std::string adapter_info() {
    LucidCudaCtx* c = nullptr;
    if (lucid_cuda_create(0, &c) != LUCID_OK) return "<unavailable>";
    char buf[256];
    std::string s = lucid_cuda_device_info(c, buf, sizeof(buf)) == LUCID_OK ? std::string(buf) : "<unavailable>";
    lucid_cuda_destroy(c);
    return s;
}

}  // namespace

// ---- standalone diagnostics (src/pybind_module.cpp:433-539) ----
// PathTrace (diagnostics/path_types.hpp:249-372)
struct PathTrace {
    LucidPathTrace t{};
    size_t depth() const { return t.depth; }
};

// PathDiagnosticRecorder (diagnostics/diagnostic_integrator.hpp:87-248):
// builds one PathTrace vertex by vertex.
class PathDiagnosticRecorder {
public:
    // begin_path: PathTrace::clear (path_types.hpp:272-278); the vertex
    // positions and normals are left as they were, as there
    void begin_path() {
        cur_.depth = 0;
        cur_.contribution[0] = cur_.contribution[1] = cur_.contribution[2] = 0.0f;
        cur_.light_type = 0;
        cur_.strategy = 0;
    }
    void record_vertex(int32_t object_id, int16_t material_id, uint8_t type, bool is_delta, bool is_light_sampled) {
        push(object_id, material_id, type, (uint8_t)((is_delta ? 1 : 0) | (is_light_sampled ? 2 : 0)));
    }
    void record_environment_hit() {
        if (push(-1, -1, 5, 0)) cur_.light_type = 5;
    }
    void record_light_hit(int32_t light_id, uint8_t light_source_type) {
        if (push(-(light_id + 2), -1, 4, 0)) cur_.light_type = light_source_type;
    }
    void record_emissive_hit(int32_t object_id, int16_t material_id) {
        if (push(object_id, material_id, 4, 0)) cur_.light_type = 6;
    }
    size_t current_depth() const { return cur_.depth; }
    PathTrace end_path(float r, float g, float b) {
        cur_.contribution[0] = r; cur_.contribution[1] = g; cur_.contribution[2] = b;
        PathTrace p;
        p.t = cur_;
        return p;
    }

private:
    bool push(int32_t obj, int16_t mat, uint8_t type, uint8_t flags) {
        if (cur_.depth >= 16) return false;
        LucidPathVertex& v = cur_.vertices[cur_.depth++];
        v.object_id = obj; v.material_id = mat; v.bsdf_type = type; v.flags = flags;
        return true;
    }
    LucidPathTrace cur_{};
};

// DiagnosticFilm (diagnostics/diagnostic_film.hpp:59-313) over a host film
// of the C ABI.
class DiagnosticFilm {
public:
    DiagnosticFilm(size_t width, size_t height, const PathRecordingConfig& c) : cfg_(c) {
        LucidDiagConfig cfg{c.subsample_factor, c.max_groups_per_pixel, c.max_outliers_per_pixel, c.max_depth,
                            c.variance_threshold, c.outlier_threshold, 0};
        if (lucid_diag_film_create((long long)width, (long long)height, &cfg, &f_) != LUCID_OK)
            throw std::invalid_argument("DiagnosticFilm: invalid size or subsample_factor");
    }
    ~DiagnosticFilm() { lucid_diag_film_destroy(f_); }
    DiagnosticFilm(const DiagnosticFilm&) = delete;
    DiagnosticFilm& operator=(const DiagnosticFilm&) = delete;
    size_t info(int k) const {
        long long v[5] = {0, 0, 0, 0, 0};
        lucid_diag_film_info(f_, v);
        return (size_t)v[k];
    }
    void record_path(size_t x, size_t y, const PathTrace& t) { lucid_diag_film_record_path(f_, (long long)x, (long long)y, &t.t); }
    void clear() { lucid_diag_film_clear(f_); }
    FilmRef ref() const { return FilmRef{nullptr, f_}; }

private:
    LucidDiagFilm* f_ = nullptr;
    PathRecordingConfig cfg_;
};

// DiagnosticPathTracer (diagnostic_integrator.hpp:408-463): a film plus an
// enabled flag and the subsampling test.
class DiagnosticPathTracer {
public:
    DiagnosticPathTracer(size_t w, size_t h, const PathRecordingConfig& c) : film_(w, h, c), cfg_(c) {}
    void set_enabled(bool e) { enabled_ = e; }
    bool is_enabled() const { return enabled_; }
    bool should_record(size_t x, size_t y) const {
        const size_t sf = (size_t)std::max(1, cfg_.subsample_factor);
        return enabled_ && x % sf == 0 && y % sf == 0;
    }
    void record_path(size_t x, size_t y, const PathTrace& t) {
        if (enabled_) film_.record_path(x, y, t);
    }
    void clear() { film_.clear(); }
    DiagnosticFilm& film() { return film_; }

private:
    DiagnosticFilm film_;
    PathRecordingConfig cfg_;
    bool enabled_ = true;
};

// DiagnosticExporter (diagnostic_export.hpp:78-285) over a DiagnosticFilm,
// as in the reference, or over a Renderer's film (an addition).
struct DiagnosticExporter {
    FilmRef f;
};

PYBIND11_MODULE(lucidrenderer, m) {
    m.doc() = "Lucid path tracer on NVIDIA B200 (sm_100a CUDA wavefront tracer)";
    py::class_<Renderer>(m, "Renderer")
        .def(py::init<>())
        .def("cancel", &Renderer::cancel, "Request cancellation; callable from another thread")
        .def("is_cancelled", &Renderer::is_cancelled)
        .def("reset_cancel", &Renderer::reset_cancel)
        .def("load_scene_json", &Renderer::load_scene_json, py::arg("json_str"), py::call_guard<py::gil_scoped_release>())
        .def("set_camera", &Renderer::set_camera, py::arg("pos_x"), py::arg("pos_y"), py::arg("pos_z"), py::arg("dir_x"),
             py::arg("dir_y"), py::arg("dir_z"), py::arg("up_x"), py::arg("up_y"), py::arg("up_z"), py::arg("fov_deg"))
        .def("set_algorithm", &Renderer::set_algorithm, py::arg("algorithm"))
        .def("set_object_names", &Renderer::set_object_names, py::arg("names"))
        .def("get_object_name", &Renderer::get_object_name, py::arg("object_id"))
        .def("object_path_string", &Renderer::object_path_string, py::arg("object_ids"))
        .def("render_tile", &Renderer::render, py::call_guard<py::gil_scoped_release>(), py::arg("tile_x"),
             py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"), py::arg("full_h"),
             py::arg("samples") = 1, py::arg("sample_offset") = 0, py::arg("max_depth") = 8,
             "Render a tile on the GPU; RGBA sum over the call's samples, Y-flipped")
        .def("render_tile_gpu", &Renderer::render, py::call_guard<py::gil_scoped_release>(), py::arg("tile_x"),
             py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"), py::arg("full_h"),
             py::arg("samples") = 1, py::arg("sample_offset") = 0, py::arg("max_depth") = 8)
        .def("render_tile_numpy",
             [](Renderer& self, int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth,
                py::object out) {
                 // the engine's film copy lands directly in the returned array
                 if (tw <= 0 || th <= 0) throw std::invalid_argument("tile size must be positive");
                 py::array_t<float, py::array::c_style> arr;
                 if (out.is_none()) {
                     arr = py::array_t<float, py::array::c_style>({th, tw, 4});
                 } else {
                     if (!py::isinstance<py::array_t<float>>(out))
                         throw std::invalid_argument("out must be a float32 numpy array");
                     arr = py::reinterpret_borrow<py::array_t<float, py::array::c_style>>(out);
                     if (!(arr.flags() & py::array::c_style) || !arr.writeable() ||
                         arr.size() != (py::ssize_t)tw * th * 4)
                         throw std::invalid_argument("out must be a writable C-contiguous float32 array of "
                                                     "tile_w * tile_h * 4 elements");
                 }
                 float* px = arr.mutable_data();   // every return path of the render writes it
                 {
                     py::gil_scoped_release release;
                     self.render_into(px, tx, ty, tw, th, fw, fh, samples, offset, depth);
                 }
                 return arr;
             },
             py::arg("tile_x"), py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"),
             py::arg("full_h"), py::arg("samples") = 1, py::arg("sample_offset") = 0, py::arg("max_depth") = 8,
             py::arg("out") = py::none(),
             "render_tile into a (tile_h, tile_w, 4) float32 array (or into `out`, reused between calls)")
        .def("render_debug", &Renderer::render_debug, py::call_guard<py::gil_scoped_release>(), py::arg("tile_x"),
             py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"), py::arg("full_h"),
             py::arg("mode"))
        .def("render_debug_gpu", &Renderer::render_debug, py::call_guard<py::gil_scoped_release>(), py::arg("tile_x"),
             py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"), py::arg("full_h"),
             py::arg("mode"))
        .def("render_start_async", &Renderer::start_async, py::call_guard<py::gil_scoped_release>(),
             py::arg("width"), py::arg("height"), py::arg("max_depth") = 8)
        .def("render_poll_async",
             [](Renderer& self) {
                 std::pair<int, std::vector<float>> r;
                 {
                     py::gil_scoped_release release;
                     r = self.poll_async();
                 }
                 py::array_t<float> arr(static_cast<py::ssize_t>(r.second.size()));
                 if (!r.second.empty()) std::memcpy(arr.mutable_data(), r.second.data(), r.second.size() * sizeof(float));
                 return py::make_tuple(r.first, arr);
             },
             "(samples, RGBA numpy): averaged over samples, Y-flipped; samples == 0 means no snapshot yet")
        .def("render_snapshot_revision_async", &Renderer::async_revision, py::call_guard<py::gil_scoped_release>())
        .def("render_stop_async", &Renderer::stop_async, py::call_guard<py::gil_scoped_release>())
        .def("render_reset_async", &Renderer::reset_async, py::call_guard<py::gil_scoped_release>(),
             py::arg("width"), py::arg("height"), py::arg("max_depth") = 8)
        .def("is_render_async_running", &Renderer::async_running, py::call_guard<py::gil_scoped_release>())
        .def("enable_diagnostics", &Renderer::enable_diagnostics, py::arg("config"),
             "Enable diagnostic path recording with given configuration")
        .def("disable_diagnostics", &Renderer::disable_diagnostics)
        .def("is_diagnostics_enabled", &Renderer::is_diagnostics_enabled)
        .def("clear_diagnostics", &Renderer::clear_diagnostics)
        .def("get_diagnostic_stats", &Renderer::get_diagnostic_stats)
        .def("get_diagnostic_variance_map",
             [](Renderer& self) {
                 std::vector<float> v = self.get_diagnostic_variance_map();
                 py::array_t<float> arr(static_cast<py::ssize_t>(v.size()));
                 if (!v.empty()) std::memcpy(arr.mutable_data(), v.data(), v.size() * sizeof(float));
                 return arr;
             },
             "Per-pixel variance as a 1D numpy array (width * height)")
        .def("export_diagnostic_json", &Renderer::export_diagnostic_json)
        .def("get_top_variance_groups", &Renderer::get_top_variance_groups, py::arg("count") = 10)
        .def("get_pixel_diagnostic",
             [](Renderer& self, size_t x, size_t y, const std::string& sort_by) {
                 return self.get_pixel_diagnostic(x, y, sort_by == "mean" ? TopGroupSortBy::Mean
                                                                          : TopGroupSortBy::Variance);
             },
             py::arg("x"), py::arg("y"), py::arg("sort_by") = "variance",
             "Diagnostic data of one pixel, groups sorted by 'variance' (default) or 'mean'")
        .def("is_scene_loaded", &Renderer::is_scene_loaded)
        .def("is_camera_set", &Renderer::is_camera_set)
        .def("get_algorithm", &Renderer::get_algorithm)
        .def("get_mesh_count", &Renderer::get_mesh_count)
        .def("__repr__", [](const Renderer& r) {
            return "<lucidrenderer.Renderer scene_loaded=" + std::string(r.is_scene_loaded() ? "True" : "False") +
                   " meshes=" + std::to_string(r.get_mesh_count()) + " algorithm='" + r.get_algorithm() + "'>";
        });
    py::class_<PathRecordingConfig>(m, "PathRecordingConfig")
        .def(py::init<>())
        .def_readwrite("subsample_factor", &PathRecordingConfig::subsample_factor)
        .def_readwrite("max_groups_per_pixel", &PathRecordingConfig::max_groups_per_pixel)
        .def_readwrite("max_outliers_per_pixel", &PathRecordingConfig::max_outliers_per_pixel)
        .def_readwrite("max_depth", &PathRecordingConfig::max_depth)
        .def_readwrite("variance_threshold", &PathRecordingConfig::variance_threshold)
        .def_readwrite("outlier_threshold", &PathRecordingConfig::outlier_threshold)
        .def_static("minimal", &PathRecordingConfig::minimal)
        .def_static("standard", &PathRecordingConfig::standard)
        .def_static("detailed", &PathRecordingConfig::detailed)
        .def("estimate_memory_bytes", &PathRecordingConfig::estimate_memory_bytes, py::arg("width"), py::arg("height"))
        .def("__repr__", [](const PathRecordingConfig& c) {
            return "<PathRecordingConfig subsample=" + std::to_string(c.subsample_factor) +
                   " max_groups=" + std::to_string(c.max_groups_per_pixel) + ">";
        });
    py::class_<ExportedGroupInfo>(m, "ExportedGroupInfo")
        .def(py::init<>())
        .def_readonly("pixel_x", &ExportedGroupInfo::pixel_x)
        .def_readonly("pixel_y", &ExportedGroupInfo::pixel_y)
        .def_readonly("signature", &ExportedGroupInfo::signature)
        .def_readonly("signature_heckbert", &ExportedGroupInfo::signature_heckbert)
        .def_readonly("object_ids", &ExportedGroupInfo::object_ids)
        .def_readonly("object_path", &ExportedGroupInfo::object_path)
        .def_readonly("sample_count", &ExportedGroupInfo::sample_count)
        .def_readonly("mean_luminance", &ExportedGroupInfo::mean_luminance)
        .def_readonly("variance_luminance", &ExportedGroupInfo::variance_luminance)
        .def_readonly("mean_rgb", &ExportedGroupInfo::mean_rgb)
        .def_readonly("variance_rgb", &ExportedGroupInfo::variance_rgb)
        .def_readonly("depth", &ExportedGroupInfo::depth)
        .def_readonly("coarse_type", &ExportedGroupInfo::coarse_type)
        .def_readonly("coarse_type_name", &ExportedGroupInfo::coarse_type_name)
        .def_readonly("strategy_name", &ExportedGroupInfo::strategy_name)
        .def_readonly("positions", &ExportedGroupInfo::positions, "camera first, then the path vertices")
        .def_readonly("normals", &ExportedGroupInfo::normals)
        .def("__repr__", [](const ExportedGroupInfo& g) {
            return "<ExportedGroupInfo signature='" + g.signature + "' heckbert='" + g.signature_heckbert + "'" +
                   " path='" + g.object_path + "'" + " strategy='" + g.strategy_name + "'" +
                   " mean=" + std::to_string(g.mean_luminance) + " var=" + std::to_string(g.variance_luminance) +
                   " positions=" + std::to_string(g.positions.size()) + ">";
        });
    py::enum_<TopGroupSortBy>(m, "TopGroupSortBy")
        .value("Variance", TopGroupSortBy::Variance)
        .value("Mean", TopGroupSortBy::Mean)
        .export_values();
    py::class_<PixelDiagnosticInfo>(m, "PixelDiagnosticInfo")
        .def(py::init<>())
        .def_readonly("valid", &PixelDiagnosticInfo::valid)
        .def_readonly("sample_count", &PixelDiagnosticInfo::sample_count)
        .def_readonly("variance", &PixelDiagnosticInfo::variance)
        .def_readonly("group_count", &PixelDiagnosticInfo::group_count)
        .def_readonly("outlier_count", &PixelDiagnosticInfo::outlier_count)
        .def_readonly("mean_rgb", &PixelDiagnosticInfo::mean_rgb)
        .def_readonly("top_groups", &PixelDiagnosticInfo::top_groups)
        .def("__repr__", [](const PixelDiagnosticInfo& p) {
            if (!p.valid) return std::string("<PixelDiagnosticInfo invalid>");
            return "<PixelDiagnosticInfo samples=" + std::to_string(p.sample_count) +
                   " variance=" + std::to_string(p.variance) + " groups=" + std::to_string(p.group_count) + ">";
        });
    py::class_<GlobalDiagnosticStats>(m, "GlobalDiagnosticStats")
        .def(py::init<>())
        .def_readonly("total_samples", &GlobalDiagnosticStats::total_samples)
        .def_readonly("active_pixels", &GlobalDiagnosticStats::active_pixels)
        .def_readonly("total_groups", &GlobalDiagnosticStats::total_groups)
        .def_readonly("total_overflow", &GlobalDiagnosticStats::total_overflow)
        .def_readonly("total_variance", &GlobalDiagnosticStats::total_variance);
    py::class_<ExportedCoarseStats>(m, "ExportedCoarseStats")
        .def(py::init<>())
        .def_readonly("type_id", &ExportedCoarseStats::type_id)
        .def_readonly("name", &ExportedCoarseStats::name)
        .def_readonly("sample_count", &ExportedCoarseStats::sample_count)
        .def_readonly("mean_luminance", &ExportedCoarseStats::mean_luminance)
        .def_readonly("variance_luminance", &ExportedCoarseStats::variance_luminance)
        .def_readonly("mean_rgb", &ExportedCoarseStats::mean_rgb)
        .def_readonly("variance_rgb", &ExportedCoarseStats::variance_rgb);
    py::class_<DiagnosticSuggestion>(m, "DiagnosticSuggestion")
        .def(py::init<>())
        .def_readonly("category", &DiagnosticSuggestion::category)
        .def_readonly("severity", &DiagnosticSuggestion::severity)
        .def_readonly("message", &DiagnosticSuggestion::message)
        .def_readonly("action", &DiagnosticSuggestion::action)
        .def("__repr__", [](const DiagnosticSuggestion& s) {
            return "<DiagnosticSuggestion [" + s.severity + "] " + s.category + ": " + s.message + ">";
        });
    // DiagnosticFilm / DiagnosticPathTracer / DiagnosticExporter / enums /
    // PathTrace / PathDiagnosticRecorder (src/pybind_module.cpp:433-539)
    py::class_<DiagnosticFilm>(m, "DiagnosticFilm")
        .def(py::init<size_t, size_t, const PathRecordingConfig&>(), py::arg("width"), py::arg("height"),
             py::arg("config"), "Create diagnostic film for given dimensions")
        .def("width", [](const DiagnosticFilm& f) { return f.info(0); })
        .def("height", [](const DiagnosticFilm& f) { return f.info(1); })
        .def("sampled_width", [](const DiagnosticFilm& f) { return f.info(2); })
        .def("sampled_height", [](const DiagnosticFilm& f) { return f.info(3); })
        .def("total_paths_recorded", [](const DiagnosticFilm& f) { return f.info(4); })
        .def("global_stats", [](const DiagnosticFilm& f) { return global_stats_of(f.ref()); })
        .def("metadata_json", [](const DiagnosticFilm& f) { return metadata_of(f.ref()); })
        .def("record_path", &DiagnosticFilm::record_path, py::arg("x"), py::arg("y"), py::arg("trace"),
             "Record a path trace at pixel (x, y)")
        .def("clear", &DiagnosticFilm::clear);
    py::class_<DiagnosticPathTracer>(m, "DiagnosticPathTracer")
        .def(py::init<size_t, size_t, const PathRecordingConfig&>(), py::arg("width"), py::arg("height"),
             py::arg("config"), "Create diagnostic path tracer")
        .def("is_enabled", &DiagnosticPathTracer::is_enabled)
        .def("set_enabled", &DiagnosticPathTracer::set_enabled)
        .def("film", &DiagnosticPathTracer::film, py::return_value_policy::reference_internal);
    py::class_<DiagnosticExporter>(m, "DiagnosticExporter")
        .def(py::init([](const DiagnosticFilm& f) { return DiagnosticExporter{f.ref()}; }), py::arg("film"),
             py::keep_alive<1, 2>(), "Create exporter for a diagnostic film")
        .def(py::init([](Renderer& r) { return DiagnosticExporter{r.film_ref()}; }), py::arg("renderer"),
             py::keep_alive<1, 2>(), "Create exporter for the film of a Renderer's last diagnostic render")
        .def("get_global_stats", [](const DiagnosticExporter& e) { return global_stats_of(e.f); })
        .def("get_top_variance_groups", [](const DiagnosticExporter& e, size_t n) { return top_groups_of(e.f, n, false); },
             py::arg("n") = 10)
        .def("get_top_mean_groups", [](const DiagnosticExporter& e, size_t n) { return top_groups_of(e.f, n, true); },
             py::arg("n") = 10)
        .def("get_coarse_stats", [](const DiagnosticExporter& e) { return coarse_stats_of(e.f); })
        .def("generate_suggestions", [](const DiagnosticExporter& e) { return suggestions_of(e.f); })
        .def("export_metadata_json", [](const DiagnosticExporter& e) { return metadata_of(e.f); })
        .def("export_binary", [](const DiagnosticExporter& e) { return binary_of(e.f); });
    py::enum_<BsdfType>(m, "BsdfType")
        .value("Diffuse", BsdfType::Diffuse)
        .value("Glossy", BsdfType::Glossy)
        .value("Mirror", BsdfType::Mirror)
        .value("Glass", BsdfType::Glass)
        .value("Emission", BsdfType::Emission)
        .value("Environment", BsdfType::Environment)
        .export_values();
    py::enum_<LightSourceType>(m, "LightSourceType")
        .value("Unknown", LightSourceType::Unknown)
        .value("Point", LightSourceType::Point)
        .value("Area", LightSourceType::Area)
        .value("Directional", LightSourceType::Directional)
        .value("Spot", LightSourceType::Spot)
        .value("Environment", LightSourceType::Environment)
        .value("Emissive", LightSourceType::Emissive)
        .export_values();
    py::class_<PathTrace>(m, "PathTrace")
        .def(py::init<>(), "Create empty path trace")
        .def_property_readonly("depth", &PathTrace::depth)
        .def("get_contribution", [](const PathTrace& p) {
            return std::array<float, 3>{p.t.contribution[0], p.t.contribution[1], p.t.contribution[2]};
        });
    py::class_<PathDiagnosticRecorder>(m, "PathDiagnosticRecorder")
        .def(py::init<>(), "Create a new path recorder")
        .def("begin_path", &PathDiagnosticRecorder::begin_path, "Start recording a new path")
        .def("record_vertex", [](PathDiagnosticRecorder& r, int32_t object_id, int16_t material_id, BsdfType t,
                                 bool is_delta, bool is_light_sampled) {
                 r.record_vertex(object_id, material_id, (uint8_t)t, is_delta, is_light_sampled);
             },
             py::arg("object_id"), py::arg("material_id"), py::arg("bsdf_type"), py::arg("is_delta"),
             py::arg("is_light_sampled"), "Record a surface interaction vertex")
        .def("record_environment_hit", &PathDiagnosticRecorder::record_environment_hit, "Record environment map hit")
        .def("record_light_hit", [](PathDiagnosticRecorder& r, int32_t light_id, LightSourceType t) {
                 r.record_light_hit(light_id, (uint8_t)t);
             },
             py::arg("light_id"), py::arg("light_source_type") = LightSourceType::Unknown,
             "Record light hit with optional light source type for Heckbert notation")
        .def("record_emissive_hit", &PathDiagnosticRecorder::record_emissive_hit, py::arg("object_id"),
             py::arg("material_id"), "Record emissive mesh hit")
        .def("current_depth", &PathDiagnosticRecorder::current_depth, "Get current path depth")
        .def("end_path", &PathDiagnosticRecorder::end_path, py::arg("r"), py::arg("g"), py::arg("b"),
             "Finalize path and return PathTrace")
        .def("end_path_lum", [](PathDiagnosticRecorder& r, float l) { return r.end_path(l, l, l); },
             py::arg("luminance"), "Finalize path with grayscale luminance");
    m.attr("__version__") = "1.0.0";
    m.attr("openmp_enabled") = false;
    m.attr("dawn_enabled") = false;
    m.attr("cuda_enabled") = true;
    m.def("gpu_adapter_info", &adapter_info, "Name and compute capability of the CUDA device in use");
}
