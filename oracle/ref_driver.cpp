// C ABI over the Lucid reference's own PyRenderer
// (LucidRenderer/cpp_renderer/include/pybind_renderer.hpp), compiled from the
// reference's unmodified headers and src/node_evaluator.cpp against the
// project-written mp-units API shim in ref_shim/.  TEST INFRASTRUCTURE: the
// pin of the oracle (tests/test_reference_pin.py) and the timed CPU baseline
// of bench.py --impl reference.  Nothing in the product links or loads it.
#include "pybind_renderer.hpp"

#include <cstdlib>
#include <cstring>

extern "C" {

void* ref_create() { return new PyRenderer(); }
void ref_destroy(void* r) { delete static_cast<PyRenderer*>(r); }

int ref_load_scene_json(void* r, const char* json) {
    return static_cast<PyRenderer*>(r)->load_scene_json(std::string(json)) ? 1 : 0;
}

void ref_set_camera(void* r, float px, float py, float pz, float dx, float dy, float dz, float ux, float uy, float uz,
                    float fov_deg) {
    static_cast<PyRenderer*>(r)->set_camera(px, py, pz, dx, dy, dz, ux, uy, uz, fov_deg);
}

void ref_set_algorithm(void* r, const char* name) { static_cast<PyRenderer*>(r)->set_algorithm(std::string(name)); }

// render_tile into out (tile_w * tile_h * 4 floats)
int ref_render_tile(void* r, int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth,
                    float* out) {
    std::vector<float> px = static_cast<PyRenderer*>(r)->render_tile(tx, ty, tw, th, fw, fh, samples, offset, depth);
    if (px.size() != (size_t)tw * th * 4) return -1;
    std::memcpy(out, px.data(), px.size() * sizeof(float));
    return 0;
}

int ref_render_debug(void* r, int tx, int ty, int tw, int th, int fw, int fh, const char* mode, float* out) {
    std::vector<float> px = static_cast<PyRenderer*>(r)->render_debug(tx, ty, tw, th, fw, fh, std::string(mode));
    if (px.size() != (size_t)tw * th * 4) return -1;
    std::memcpy(out, px.data(), px.size() * sizeof(float));
    return 0;
}

// ---- the reference's DiagnosticFilm / PathDiagnosticRecorder / DiagnosticExporter
// (diagnostics/*.hpp), driven vertex by vertex from the caller.
void* ref_film_create(long long w, long long h, int subsample, int max_groups, int max_outliers, int max_depth,
                      float variance_threshold, float outlier_threshold) {
    render::diagnostics::PathRecordingConfig c;
    c.subsample_factor = subsample;
    c.max_groups_per_pixel = max_groups;
    c.max_outliers_per_pixel = max_outliers;
    c.max_depth = max_depth;
    c.variance_threshold = variance_threshold;
    c.outlier_threshold = outlier_threshold;
    return new render::diagnostics::DiagnosticFilm((size_t)w, (size_t)h, c);
}
void ref_film_destroy(void* f) { delete static_cast<render::diagnostics::DiagnosticFilm*>(f); }
void ref_film_clear(void* f) { static_cast<render::diagnostics::DiagnosticFilm*>(f)->clear(); }

void* ref_recorder_create() { return new render::diagnostics::PathDiagnosticRecorder(); }
void ref_recorder_destroy(void* r) { delete static_cast<render::diagnostics::PathDiagnosticRecorder*>(r); }
void ref_recorder_begin(void* r) { static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->begin_path(); }
void ref_recorder_vertex(void* r, int obj, int mat, int type, int delta, int light_sampled) {
    static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->record_vertex(
        obj, (int16_t)mat, (render::diagnostics::BsdfType)type, delta != 0, light_sampled != 0);
}
void ref_recorder_environment(void* r) { static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->record_environment_hit(); }
void ref_recorder_light(void* r, int light_id, int type) {
    static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->record_light_hit(
        light_id, (render::diagnostics::LightSourceType)type);
}
void ref_recorder_emissive(void* r, int obj, int mat) {
    static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->record_emissive_hit(obj, (int16_t)mat);
}
// end_path(rgb) and DiagnosticFilm::record_path(x, y, trace); returns the trace's hash
unsigned long long ref_recorder_end_into(void* r, void* film, long long x, long long y, float cr, float cg, float cb) {
    render::diagnostics::PathTrace t =
        static_cast<render::diagnostics::PathDiagnosticRecorder*>(r)->end_path(render::RGB3f{cr, cg, cb});
    static_cast<render::diagnostics::DiagnosticFilm*>(film)->record_path((size_t)x, (size_t)y, t);
    return (unsigned long long)t.hash();
}

// Everything the exporter and the film report, as JSON (caller frees with ref_free).
char* ref_film_report(void* fp, int top_n, int subsample) {
    using namespace render::diagnostics;
    const DiagnosticFilm& f = *static_cast<DiagnosticFilm*>(fp);
    DiagnosticExporter e(f);
    nlohmann::json j;
    j["width"] = f.width(); j["height"] = f.height();
    j["sampled_width"] = f.sampled_width(); j["sampled_height"] = f.sampled_height();
    j["total_paths_recorded"] = f.total_paths_recorded();
    GlobalDiagnosticStats g = e.get_global_stats();
    j["global"] = nlohmann::json::array({g.total_samples, g.active_pixels, g.total_groups, g.total_overflow});
    auto groups = [](const std::vector<ExportedGroupInfo>& v) {
        nlohmann::json a = nlohmann::json::array();
        for (const auto& x : v)
            a.push_back({{"x", x.pixel_x}, {"y", x.pixel_y}, {"signature", x.signature}, {"count", x.sample_count},
                         {"mean_luminance", x.mean_luminance}, {"variance_luminance", x.variance_luminance},
                         {"mean_rgb", x.mean_rgb}, {"variance_rgb", x.variance_rgb}, {"depth", x.depth},
                         {"coarse_type", x.coarse_type}, {"coarse_type_name", x.coarse_type_name}});
        return a;
    };
    j["top_variance"] = groups(e.get_top_variance_groups((size_t)top_n));
    j["top_mean"] = groups(e.get_top_mean_groups((size_t)top_n));
    nlohmann::json cs = nlohmann::json::array();
    for (const auto& c : e.get_coarse_stats())
        cs.push_back({{"type_id", c.type_id}, {"name", c.name}, {"count", c.sample_count},
                      {"mean_luminance", c.mean_luminance}, {"variance_luminance", c.variance_luminance},
                      {"mean_rgb", c.mean_rgb}, {"variance_rgb", c.variance_rgb}});
    j["coarse"] = cs;
    nlohmann::json sg = nlohmann::json::array();
    for (const auto& x : e.generate_suggestions())
        sg.push_back({{"category", x.category}, {"severity", x.severity}, {"message", x.message}, {"action", x.action}});
    j["suggestions"] = sg;
    j["metadata_json"] = e.export_metadata_json();
    std::vector<uint8_t> b = e.export_binary();
    j["binary"] = b;
    nlohmann::json cells = nlohmann::json::array();
    for (size_t sy = 0; sy < f.sampled_height(); ++sy)
        for (size_t sx = 0; sx < f.sampled_width(); ++sx) {
            const auto* p = f.pixel_data(sx * (size_t)subsample, sy * (size_t)subsample);
            nlohmann::json hs = nlohmann::json::array();
            for (size_t k = 0; k < p->group_count(); ++k) {
                const PathGroup* pg = p->top_group(k);
                hs.push_back(nlohmann::json::array({std::to_string(pg->path_hash), pg->stats.count}));
            }
            cells.push_back(nlohmann::json::array({p->total_samples(), p->group_count(), p->overflow_count(), p->outlier_count(), hs}));
        }
    j["cells"] = cells;
    std::string out = j.dump();
    char* c = static_cast<char*>(std::malloc(out.size() + 1));
    std::memcpy(c, out.c_str(), out.size() + 1);
    return c;
}
void ref_free(char* p) { std::free(p); }

// ---- PyRenderer's own diagnostics (pybind_renderer.hpp:893-1102)
void ref_enable_diagnostics(void* r, int subsample, int max_groups, int max_outliers, int max_depth,
                            float variance_threshold, float outlier_threshold) {
    render::diagnostics::PathRecordingConfig c;
    c.subsample_factor = subsample;
    c.max_groups_per_pixel = max_groups;
    c.max_outliers_per_pixel = max_outliers;
    c.max_depth = max_depth;
    c.variance_threshold = variance_threshold;
    c.outlier_threshold = outlier_threshold;
    static_cast<PyRenderer*>(r)->enable_diagnostics(c);
}
void ref_disable_diagnostics(void* r) { static_cast<PyRenderer*>(r)->disable_diagnostics(); }

// get_diagnostic_stats, every pixel's get_pixel_diagnostic (by variance),
// get_top_variance_groups, export_diagnostic_json, as JSON.
char* ref_diag_report(void* rp, int tile_w, int tile_h, int top_n) {
    PyRenderer& r = *static_cast<PyRenderer*>(rp);
    nlohmann::json j;
    auto st = r.get_diagnostic_stats();
    j["stats"] = nlohmann::json::array({st.total_samples, st.active_pixels, st.total_groups, st.total_overflow});
    auto group = [](const render::diagnostics::ExportedGroupInfo& g) {
        return nlohmann::json{{"signature", g.signature}, {"heckbert", g.signature_heckbert},
                              {"object_ids", g.object_ids}, {"count", g.sample_count},
                              {"mean_luminance", g.mean_luminance}, {"variance_luminance", g.variance_luminance},
                              {"mean_rgb", g.mean_rgb}, {"variance_rgb", g.variance_rgb}, {"depth", g.depth},
                              {"coarse_type", g.coarse_type}, {"strategy", g.strategy_name},
                              {"object_path", g.object_path}, {"positions", g.positions}, {"normals", g.normals},
                              {"x", g.pixel_x}, {"y", g.pixel_y}};
    };
    nlohmann::json px = nlohmann::json::array();
    for (int y = 0; y < tile_h; ++y)
        for (int x = 0; x < tile_w; ++x) {
            auto info = r.get_pixel_diagnostic((size_t)x, (size_t)y);
            nlohmann::json gs = nlohmann::json::array();
            for (const auto& g : info.top_groups) gs.push_back(group(g));
            px.push_back({{"valid", info.valid}, {"samples", info.sample_count}, {"variance", info.variance},
                          {"groups", info.group_count}, {"outliers", info.outlier_count}, {"mean_rgb", info.mean_rgb},
                          {"top", gs}});
        }
    j["pixels"] = px;
    nlohmann::json tv = nlohmann::json::array();
    for (const auto& g : r.get_top_variance_groups((size_t)top_n)) tv.push_back(group(g));
    j["top_variance"] = tv;
    j["json"] = r.export_diagnostic_json();
    std::string out = j.dump();
    char* c = static_cast<char*>(std::malloc(out.size() + 1));
    std::memcpy(c, out.c_str(), out.size() + 1);
    return c;
}

// OpenMP threads of the reference's render loops (omp_set_num_threads).
void ref_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}

int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
