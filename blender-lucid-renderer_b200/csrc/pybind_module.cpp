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

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lucid_cuda.h"

namespace py = pybind11;

namespace {

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
    }
    void set_algorithm(const std::string& a) {
        algorithm_ = a;
        lucid_cuda_set_algorithm(ctx_, a.c_str());
    }
    std::string get_algorithm() const { return algorithm_; }
    bool is_scene_loaded() const { return scene_loaded_; }
    bool is_camera_set() const { return camera_set_; }
    int get_mesh_count() const { return scene_loaded_ ? mesh_count_ : 0; }

    std::vector<float> render(int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth) {
        if (tw <= 0 || th <= 0) throw std::invalid_argument("tile size must be positive");
        std::vector<float> px((size_t)tw * th * 4, 0.0f);
        LucidRenderParams p{tx, ty, tw, th, fw, fh, samples, offset, depth, 0};
        int rc = lucid_cuda_render(ctx_, &p, px.data(), nullptr);
        if (rc == LUCID_ERR_NO_SCENE) {
            // the reference returns a zero buffer (pybind_renderer.hpp:200-203)
            std::fprintf(stderr, "[lucidrenderer] Scene or camera not set\n");
            return px;
        }
        if (rc == LUCID_ERR_CANCELLED) return px;   // partial result, is_cancelled() stays true
        if (rc != LUCID_OK) throw std::runtime_error(std::string("render failed: ") + lucid_cuda_last_error(ctx_));
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
             [](Renderer& self, int tx, int ty, int tw, int th, int fw, int fh, int samples, int offset, int depth) {
                 std::vector<float> px;
                 {
                     py::gil_scoped_release release;
                     px = self.render(tx, ty, tw, th, fw, fh, samples, offset, depth);
                 }
                 py::array_t<float> arr({th, tw, 4});
                 std::memcpy(arr.mutable_data(), px.data(), px.size() * sizeof(float));
                 return arr;
             },
             py::arg("tile_x"), py::arg("tile_y"), py::arg("tile_w"), py::arg("tile_h"), py::arg("full_w"),
             py::arg("full_h"), py::arg("samples") = 1, py::arg("sample_offset") = 0, py::arg("max_depth") = 8)
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
        .def("is_scene_loaded", &Renderer::is_scene_loaded)
        .def("is_camera_set", &Renderer::is_camera_set)
        .def("get_algorithm", &Renderer::get_algorithm)
        .def("get_mesh_count", &Renderer::get_mesh_count)
        .def("__repr__", [](const Renderer& r) {
            return "<lucidrenderer.Renderer scene_loaded=" + std::string(r.is_scene_loaded() ? "True" : "False") +
                   " meshes=" + std::to_string(r.get_mesh_count()) + " algorithm='" + r.get_algorithm() + "'>";
        });
    m.attr("__version__") = "1.0.0";
    m.attr("openmp_enabled") = false;
    m.attr("dawn_enabled") = false;
    m.attr("cuda_enabled") = true;
    m.def("gpu_adapter_info", &adapter_info, "Name and compute capability of the CUDA device in use");
}
