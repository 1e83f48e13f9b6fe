// C ABI over the Lucid reference's own PyRenderer
// (LucidRenderer/cpp_renderer/include/pybind_renderer.hpp), compiled from the
// reference's unmodified headers and src/node_evaluator.cpp against the
// project-written mp-units API shim in ref_shim/.  TEST INFRASTRUCTURE: the
// pin of the oracle (tests/test_reference_pin.py) and the timed CPU baseline
// of bench.py --impl reference.  Nothing in the product links or loads it.
#include "pybind_renderer.hpp"

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

int ref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
