// lucid_oracle.cpp — JSON scene loading and a C API over the CPU oracle.
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).
//
// The loader restates PyRenderer::loadSceneFromJsonString
// (include/pybind_renderer.hpp:1258-1542) and parseNativeLights (:1544-1746):
// same JSON keys, same defaults, same float conversions (double arithmetic
// with M_PI where the reference uses it), same sidecar grid loading.
// Node-graph evaluation (src/node_evaluator.cpp) is not restated: materials
// use their plain fields; the node tree is parsed only to detect
// volume-boundary-only meshes (Material Output with an unlinked Surface).
#include "lucid_oracle.hpp"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <nlohmann/json.hpp>
#include <stdexcept>
#include <string>

#ifdef _OPENMP
#include <omp.h>
#endif

using json = nlohmann::json;

namespace orc {

// node_evaluator.cpp:82-163, reduced to what the loader needs: is the
// Material Output's Surface input linked?
static bool surface_socket_linked(const json& nt, bool& valid) {
    valid = false;
    if (!nt.contains("nodes") || !nt.is_object()) return true;
    const auto& nodes = nt["nodes"];
    std::map<std::pair<std::string, std::string>, bool> linked;
    if (nt.contains("links")) {
        for (const auto& l : nt["links"]) {
            std::string to_node = l["to_node"];
            std::string to_socket = l["to_socket"];
            linked[{to_node, to_socket}] = true;
        }
    }
    valid = !nodes.empty();
    if (!valid) return true;
    for (const auto& n : nodes) {
        if (n.value("type", "") != "ShaderNodeOutputMaterial") continue;
        std::string name = n.value("name", "");
        if (!n.contains("inputs")) return false;
        for (const auto& in : n["inputs"]) {
            if (in.value("name", "") == "Surface") return linked.count({name, "Surface"}) > 0;
        }
        return false;
    }
    return true;   // no output node: the reference keeps surface_socket_linked = true
}

static void parse_native_lights(const json& arr, Scene& sc) {
    const double PI = M_PI;
    const float EPS = 1e-6f;   // EPSILON = GGX_EPSILON (pbr.hpp:34)
    for (const auto& lj : arr) {
        Light L;
        std::string type = lj.value("type", "POINT");
        if (lj.contains("position"))
            L.position = V3(lj["position"][0].get<float>(), lj["position"][1].get<float>(), lj["position"][2].get<float>());
        if (lj.contains("direction"))
            L.normal = make_normal_or(V3(lj["direction"][0].get<float>(), lj["direction"][1].get<float>(),
                                         lj["direction"][2].get<float>()), V3(0, 0, -1));
        float cr = 1, cg = 1, cb = 1;
        if (lj.contains("color")) { cr = lj["color"][0].get<float>(); cg = lj["color"][1].get<float>(); cb = lj["color"][2].get<float>(); }
        float energy = lj.value("energy", 1.0f);
        L.energy = energy;
        if (type == "POINT") {
            L.type = LightType::POINT;
            float radius = lj.value("radius", 0.0f);
            L.radius = radius;
            float area = 4.0f * PI * radius * radius;
            if (area < EPS) area = 1.0f;
            L.area = area;
            if (radius > EPS) {
                L.emission = RGB((float)(cr * (energy / (PI * area))), (float)(cg * (energy / (PI * area))),
                                 (float)(cb * (energy / (PI * area))));
            } else {
                float factor = energy / (4.0f * PI);
                L.emission = RGB(cr * factor, cg * factor, cb * factor);
            }
        } else if (type == "SUN") {
            L.type = LightType::SUN;
            L.area = 1.0f;
            L.emission = RGB(cr * energy, cg * energy, cb * energy);
        } else if (type == "SPOT") {
            L.type = LightType::SPOT;
            float radius = lj.value("radius", 0.0f);
            L.radius = radius;
            float sa = lj.value("spot_size", static_cast<float>(M_PI / 4.0f));
            L.spot_angle = sa;
            L.spot_blend = lj.value("spot_blend", 0.0f);
            L.area = 1.0f;
            float half = sa * 0.5f;
            float solid = 2.0f * PI * (1.0f - std::cos(half));
            float factor = energy / solid;
            L.emission = RGB(cr * factor, cg * factor, cb * factor);
        } else if (type == "AREA") {
            L.type = LightType::AREA;
            float sx = lj.value("size", 1.0f);
            float sy = lj.value("size_y", sx);
            L.size_x = sx; L.size_y = sy;
            float area;
            std::string shape = lj.value("shape", "SQUARE");
            if (shape == "DISK") { L.shape = AreaShape::DISK; float r = sx * 0.5f; area = PI * r * r; }
            else if (shape == "ELLIPSE") { L.shape = AreaShape::ELLIPSE; float rx = sx * 0.5f, ry = sy * 0.5f; area = PI * rx * ry; }
            else if (shape == "RECTANGLE") { L.shape = AreaShape::RECTANGLE; area = sx * sy; }
            else { L.shape = AreaShape::SQUARE; area = sx * sy; }
            L.area = area;
            if (lj.contains("right"))
                L.right = make_dir_or(V3(lj["right"][0].get<float>(), lj["right"][1].get<float>(), lj["right"][2].get<float>()), V3(1, 0, 0));
            if (lj.contains("up"))
                L.up = make_dir_or(V3(lj["up"][0].get<float>(), lj["up"][1].get<float>(), lj["up"][2].get<float>()), V3(0, 1, 0));
            float factor = energy / (PI * area);
            L.emission = RGB(cr * factor, cg * factor, cb * factor);
        }
        L.mesh = -1; L.tri = -1;
        sc.native.push_back(L);
    }
}

static Scene load_scene(const std::string& s) {
    Scene sc;
    json j = json::parse(s);
    if (!j.contains("meshes")) return sc;
    for (const auto& mj : j["meshes"]) {
        Mesh m;
        if (mj.contains("vertices"))
            for (const auto& v : mj["vertices"]) m.verts.push_back(V3(v[0].get<float>(), v[1].get<float>(), v[2].get<float>()));
        std::vector<std::array<V3, 3>> tn;
        bool has_tn = false;
        if (mj.contains("triangle_normals")) {
            has_tn = true;
            for (const auto& t : mj["triangle_normals"]) {
                std::array<V3, 3> a;
                for (int k = 0; k < 3; ++k)
                    a[k] = make_normal_or(V3(static_cast<float>(t[k][0]), static_cast<float>(t[k][1]), static_cast<float>(t[k][2])), V3(0, 0, 1));
                tn.push_back(a);
            }
        }
        bool smooth = mj.contains("smooth") && mj["smooth"].get<bool>();
        std::vector<std::array<V2, 3>> tuv;
        if (mj.contains("triangle_uvs"))
            for (const auto& t : mj["triangle_uvs"]) {
                std::array<V2, 3> a;
                for (int k = 0; k < 3; ++k) a[k] = V2{t[k][0].get<float>(), t[k][1].get<float>()};
                tuv.push_back(a);
            }
        int ti = 0;
        if (mj.contains("triangles")) {
            for (const auto& t : mj["triangles"]) {
                Tri tr;
                tr.i0 = t[0]; tr.i1 = t[1]; tr.i2 = t[2];
                if (has_tn && (size_t)ti < tn.size()) { tr.n0 = tn[ti][0]; tr.n1 = tn[ti][1]; tr.n2 = tn[ti][2]; tr.smooth = smooth; }
                else tr.smooth = false;
                if ((size_t)ti < tuv.size()) { tr.uv0 = tuv[ti][0]; tr.uv1 = tuv[ti][1]; tr.uv2 = tuv[ti][2]; tr.has_uv = true; }
                m.tris.push_back(tr);
                ++ti;
            }
        }
        for (const Tri& t : m.tris) {
            int nv = (int)m.verts.size();
            if (t.i0 < 0 || t.i1 < 0 || t.i2 < 0 || t.i0 >= nv || t.i1 >= nv || t.i2 >= nv)
                throw std::runtime_error("triangle index out of range");
        }
        if (mj.contains("material")) {
            const auto& mat = mj["material"];
            RGB albedo(0.8f, 0.8f, 0.8f);
            float metallic = 0.0f, roughness = 0.5f;
            RGB emission(0, 0, 0);
            float transmission = 0.0f, ior = 1.45f;
            if (mat.contains("base_color")) albedo = RGB(mat["base_color"][0].get<float>(), mat["base_color"][1].get<float>(), mat["base_color"][2].get<float>());
            if (mat.contains("metallic")) metallic = mat["metallic"];
            if (mat.contains("roughness")) roughness = mat["roughness"];
            if (mat.contains("emission")) emission = RGB(mat["emission"][0].get<float>(), mat["emission"][1].get<float>(), mat["emission"][2].get<float>());
            if (mat.contains("transmission")) transmission = mat["transmission"];
            if (mat.contains("ior")) ior = mat["ior"];
            m.mat.albedo = albedo; m.mat.metallic = metallic; m.mat.roughness = roughness;
            m.mat.emission = emission; m.mat.transmission = transmission; m.mat.ior = ior;
            bool nt_valid = false;
            bool surf_linked = true;
            if (mat.contains("node_tree") && !mat["node_tree"].is_null()) {
                surf_linked = surface_socket_linked(mat["node_tree"], nt_valid);
                if (!nt_valid) surf_linked = true;
                m.mat.tree = parse_node_tree(mat["node_tree"]);
                m.mat.use_nodes = mat.value("use_nodes", false) && m.mat.tree.valid;
            }
            if (mat.contains("volume") && !mat["volume"].is_null()) {
                const auto& vol = mat["volume"];
                Volume& V = m.mat.volume;
                if (vol.contains("color") && vol["color"].is_array() && vol["color"].size() >= 3)
                    V.color = RGB(vol["color"][0].get<float>(), vol["color"][1].get<float>(), vol["color"][2].get<float>());
                if (vol.contains("absorption_color") && vol["absorption_color"].is_array() && vol["absorption_color"].size() >= 3)
                    V.absorption = RGB(vol["absorption_color"][0].get<float>(), vol["absorption_color"][1].get<float>(), vol["absorption_color"][2].get<float>());
                if (vol.contains("density")) V.density = vol["density"].get<float>();
                if (vol.contains("anisotropy")) V.anisotropy = vol["anisotropy"].get<float>();
                if (vol.contains("smoke_grid") && vol["smoke_grid"].is_object()) {
                    const auto& sg = vol["smoke_grid"];
                    if (sg.contains("dims") && sg["dims"].is_array() && sg["dims"].size() == 3 && sg.contains("world_min") &&
                        sg["world_min"].is_array() && sg.contains("world_max") && sg["world_max"].is_array() &&
                        sg.contains("sidecar_path")) {
                        for (int i = 0; i < 3; ++i) V.dims[i] = sg["dims"][i].get<int>();
                        for (int i = 0; i < 3; ++i) { V.wmin[i] = sg["world_min"][i].get<float>(); V.wmax[i] = sg["world_max"][i].get<float>(); }
                        std::string path = sg["sidecar_path"].get<std::string>();
                        size_t n = (size_t)V.dims[0] * V.dims[1] * V.dims[2];
                        V.grid.resize(n);
                        std::ifstream f(path, std::ios::binary);
                        if (f) {
                            f.read(reinterpret_cast<char*>(V.grid.data()), n * sizeof(float));
                            float mx = 0.0f;
                            for (float d : V.grid) if (d > mx) mx = d;
                            V.grid_max = mx;
                        } else {
                            V.grid.clear();
                            V.dims[0] = V.dims[1] = V.dims[2] = 0;
                        }
                    }
                }
            }
            if (m.mat.volume.present() && !surf_linked) m.mat.volume_boundary_only = true;
        }
        finalize_mesh(m);
        sc.meshes.push_back(std::move(m));
    }
    if (j.contains("native_lights") && j["native_lights"].is_array()) parse_native_lights(j["native_lights"], sc);
    else if (j.contains("lights") && j["lights"].is_array()) parse_native_lights(j["lights"], sc);
    if (j.contains("environment") && j["environment"].is_object()) {
        const auto& e = j["environment"];
        if (e.contains("color") && e["color"].is_array())
            sc.env_color = RGB(e["color"][0].get<float>(), e["color"][1].get<float>(), e["color"][2].get<float>());
        if (e.contains("strength")) sc.env_strength = e["strength"].get<float>();
    }
    return sc;
}

struct Renderer {
    Scene scene;
    Camera cam;
    bool scene_loaded = false, camera_set = false;
    std::string algorithm = "nee";   // PyRenderer() default (pybind_renderer.hpp:68)
};

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_create() { return new Renderer(); }
void orc_destroy(void* h) { delete static_cast<Renderer*>(h); }

void orc_set_options(int device_math, int canonical_ties) {
    opts().device_math = device_math != 0;
    opts().canonical_ties = canonical_ties != 0;
}

void orc_set_draw_order(int right_to_left) { opts().draw_rtl = right_to_left != 0; }

int orc_load_scene_json(void* h, const char* js) {
    Renderer* r = static_cast<Renderer*>(h);
    try {
        r->scene = load_scene(js);
        r->scene_loaded = true;
        return 1;
    } catch (const std::exception& e) {
        fprintf(stderr, "[oracle] failed to load scene: %s\n", e.what());
        r->scene_loaded = false;
        return 0;
    }
}

void orc_set_camera(void* h, float px, float py, float pz, float dx, float dy, float dz, float ux, float uy, float uz,
                    float fov_deg) {
    Renderer* r = static_cast<Renderer*>(h);
    set_camera(r->cam, px, py, pz, dx, dy, dz, ux, uy, uz, fov_deg);
    r->camera_set = true;
}

void orc_set_algorithm(void* h, const char* a) { static_cast<Renderer*>(h)->algorithm = a; }

// render_tile (pybind_renderer.hpp:185-361).  out_rgba: tile_w*tile_h*4 floats,
// Y-flipped, exposure/clamp applied.  recs (optional): tile_w*tile_h*samples
// SampleRec in (row-major unflipped pixel, sample) order.  Returns 0 on
// success, -1 when scene or camera are missing (the output is zeroed, as the
// reference returns a zero buffer).
int orc_render_tile(void* h, int tile_x, int tile_y, int tile_w, int tile_h, int full_w, int full_h, int samples,
                    int sample_offset, int max_depth, float* out_rgba, SampleRec* recs, int nthreads) {
    Renderer* r = static_cast<Renderer*>(h);
    size_t np = (size_t)tile_w * tile_h;
    std::fill(out_rgba, out_rgba + np * 4, 0.0f);
    if (!r->scene_loaded || !r->camera_set) return -1;
    r->cam.aspect = (float)full_w / (float)full_h;
    float scale = std::tan(r->cam.fov * 0.5f);
    SceneLights sl = build_lights(r->scene);
    Algo algo = algo_from_string(r->algorithm);
    std::vector<float> px(np * 4, 0.0f);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (long long idx = 0; idx < (long long)np; ++idx) {
        int py_ = (int)(idx / tile_w), px_ = (int)(idx % tile_w);
        int gx = tile_x + px_, gy = tile_y + py_;
        SampleRec* rr = recs ? recs + (size_t)idx * samples : nullptr;
        RGB rad = render_pixel(r->scene, sl, r->cam, gx, gy, full_w, full_h, samples, sample_offset, max_depth, algo,
                               scale, rr);
        // apply_camera_sensitivity with EV 0 (sensitivity 1), clamp_min_zero.
        RGB c(rad.r * 1.0f, rad.g * 1.0f, rad.b * 1.0f);
        c = RGB(smax(c.r, 0.0f), smax(c.g, 0.0f), smax(c.b, 0.0f));
        float* o = &px[(size_t)idx * 4];
        o[0] = c.r; o[1] = c.g; o[2] = c.b; o[3] = 1.0f;
    }
    for (int y = 0; y < tile_h; ++y)
        std::copy(px.begin() + (size_t)y * tile_w * 4, px.begin() + (size_t)(y + 1) * tile_w * 4,
                  out_rgba + (size_t)(tile_h - 1 - y) * tile_w * 4);
    return 0;
}

// FP64-accumulated render for converged references: every sample's FP32
// radiance (the same values render_tile sums in FP32) is summed per pixel in
// double, in sample order; clamp >= 0, alpha 1, Y-flipped like render_tile.
int orc_render_tile_f64(void* h, int tile_x, int tile_y, int tile_w, int tile_h, int full_w, int full_h, int samples,
                        int sample_offset, int max_depth, double* out_rgba, int nthreads) {
    Renderer* r = static_cast<Renderer*>(h);
    size_t np = (size_t)tile_w * tile_h;
    std::fill(out_rgba, out_rgba + np * 4, 0.0);
    if (!r->scene_loaded || !r->camera_set) return -1;
    r->cam.aspect = (float)full_w / (float)full_h;
    float scale = std::tan(r->cam.fov * 0.5f);
    SceneLights sl = build_lights(r->scene);
    Algo algo = algo_from_string(r->algorithm);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (long long idx = 0; idx < (long long)np; ++idx) {
        int py_ = (int)(idx / tile_w), px_ = (int)(idx % tile_w);
        double acc[3] = {0.0, 0.0, 0.0};
        render_pixel(r->scene, sl, r->cam, tile_x + px_, tile_y + py_, full_w, full_h, samples, sample_offset,
                     max_depth, algo, scale, nullptr, acc);
        double* o = out_rgba + ((size_t)(tile_h - 1 - py_) * tile_w + px_) * 4;
        for (int c = 0; c < 3; ++c) o[c] = (acc[c] < 0.0) ? 0.0 : acc[c];
        o[3] = 1.0;
    }
    return 0;
}

// render_debug (pybind_renderer.hpp:371-439): mode 0 normal, 1 albedo, 2 emission.
int orc_render_debug(void* h, int tile_x, int tile_y, int tile_w, int tile_h, int full_w, int full_h, int mode,
                     float* out) {
    Renderer* r = static_cast<Renderer*>(h);
    size_t np = (size_t)tile_w * tile_h;
    std::fill(out, out + np * 4, 0.0f);
    if (!r->scene_loaded || !r->camera_set) return -1;
    r->cam.aspect = (float)full_w / (float)full_h;
    float scale = std::tan(r->cam.fov * 0.5f);
    for (int py_ = 0; py_ < tile_h; ++py_)
        for (int px_ = 0; px_ < tile_w; ++px_) {
            int gx = tile_x + px_, gy = tile_y + py_;
            float ndc_x = (2.0f * ((float)gx + 0.5f) / (float)full_w - 1.0f) * r->cam.aspect;
            float ndc_y = 1.0f - 2.0f * ((float)gy + 0.5f) / (float)full_h;
            Ray ray{r->cam.pos, primary_dir(r->cam, ndc_x, ndc_y, scale)};
            RGB c = debug_pass(r->scene, ray, mode);
            float* o = out + ((size_t)(tile_h - 1 - py_) * tile_w + px_) * 4;
            o[0] = c.r; o[1] = c.g; o[2] = c.b; o[3] = 1.0f;
        }
    return 0;
}

// Scene statistics: [meshes, triangles, native lights, scene lights, boundary meshes, volumes]
void orc_scene_stats(void* h, int* out6) {
    Renderer* r = static_cast<Renderer*>(h);
    SceneLights sl = build_lights(r->scene);
    int tris = 0, bnd = 0, vols = 0;
    for (const Mesh& m : r->scene.meshes) {
        tris += (int)m.tris.size();
        bnd += m.mat.volume_boundary_only;
        vols += m.mat.volume.present() && m.mat.volume.has_grid();
    }
    out6[0] = (int)r->scene.meshes.size(); out6[1] = tris; out6[2] = (int)r->scene.native.size();
    out6[3] = (int)sl.lights.size(); out6[4] = bnd; out6[5] = vols;
}

// Light CDF and per-light (area, emission rgb) in SceneLights order.
int orc_scene_lights(void* h, float* cdf, float* area, float* emission, int cap) {
    Renderer* r = static_cast<Renderer*>(h);
    SceneLights sl = build_lights(r->scene);
    int n = (int)sl.lights.size();
    for (int i = 0; i < n && i < cap; ++i) {
        cdf[i] = sl.cdf[i]; area[i] = sl.lights[i].area;
        emission[3 * i] = sl.lights[i].emission.r; emission[3 * i + 1] = sl.lights[i].emission.g; emission[3 * i + 2] = sl.lights[i].emission.b;
    }
    return n;
}

// Closest hit of one ray through intersect_scene: returns mesh, tri, t.
void orc_closest_hit(void* h, const float* o, const float* d, float tmin, float tmax, int* mesh, int* tri, float* t) {
    Renderer* r = static_cast<Renderer*>(h);
    Hit hh = intersect_scene(r->scene, Ray{V3(o[0], o[1], o[2]), V3(d[0], d[1], d[2])}, tmin, tmax);
    *mesh = hh.hit ? hh.mesh : -1; *tri = hh.hit ? hh.tri : -1; *t = hh.t;
}

// ---- component functions for known-answer tests ----
uint32_t orc_sizeof_record() { return (uint32_t)sizeof(SampleRec); }
float orc_fresnel_schlick(float c, float f0) { return schlick_rgb(c, RGB(f0, f0, f0)).r; }
float orc_fresnel_dielectric(float c, float eta) { return fresnel_dielectric(c, eta); }
float orc_ggx_d(float nh, float r) { return ggxD(nh, r); }
float orc_ggx_g1(float nv, float r) { return ggxG1(nv, r); }
float orc_ggx_g2(float nl, float nv, float r) { return ggxG2(nl, nv, r); }
float orc_mis_power(float a, float b) { return mis_power(a, b); }
float orc_pdfw_from_area(float d, float a, float c) { return pdfw_from_area(d, a, c); }
float orc_inv_sq(float d) { return inv_sq(d); }
float orc_hg_eval(float g, float c) { return hg_eval(g, c); }
void orc_hg_sample(float g, const float* wo, float u1, float u2, float* wi, float* pdf) {
    V3 w = hg_sample(g, V3(wo[0], wo[1], wo[2]), u1, u2, *pdf);
    wi[0] = w.x; wi[1] = w.y; wi[2] = w.z;
}
void orc_rng_sequence(uint32_t x, uint32_t y, uint32_t s, int n, uint32_t* out_u32, float* out_f) {
    Rng a; seed_xyz(a, x, y, s);
    Rng b = a;
    for (int i = 0; i < n; ++i) { out_u32[i] = pcg32(a); out_f[i] = randf(b); }
}
int orc_isect_tri(const float* o, const float* d, const float* v, float tmin, float tmax, float* uvt) {
    float u, vv, t;
    bool hit = isect_tri(Ray{V3(o[0], o[1], o[2]), V3(d[0], d[1], d[2])}, V3(v[0], v[1], v[2]), V3(v[3], v[4], v[5]),
                         V3(v[6], v[7], v[8]), u, vv, t, tmin, tmax);
    if (hit) { uvt[0] = u; uvt[1] = vv; uvt[2] = t; }
    return hit;
}
int orc_isect_aabb(const float* o, const float* d, const float* bmin, const float* bmax) {
    Ray r{V3(o[0], o[1], o[2]), V3(d[0], d[1], d[2])};
    return isect_aabb(r, inv_dir(r.d), V3(bmin[0], bmin[1], bmin[2]), V3(bmax[0], bmax[1], bmax[2]));
}
int orc_isect_sphere(const float* o, const float* d, const float* c, float radius, float* t) {
    V3 n;
    return isect_sphere(Ray{V3(o[0], o[1], o[2]), V3(d[0], d[1], d[2])}, V3(c[0], c[1], c[2]), radius, *t, n);
}
// Evaluate the BSDF of a material (albedo rgb, metallic, roughness,
// transmission, ior) for (wo, wi, n): f rgb and pdf.
void orc_eval_bsdf(const float* mat7, const float* wo, const float* wi, const float* n, float* f3, float* pdf) {
    MatParams m;
    m.albedo = RGB(mat7[0], mat7[1], mat7[2]); m.metallic = mat7[3]; m.roughness = smax(mat7[4], MIN_ROUGHNESS);
    m.transmission = mat7[5]; m.ior = mat7[6];
    V3 a(wo[0], wo[1], wo[2]), b(wi[0], wi[1], wi[2]), nn(n[0], n[1], n[2]);
    RGB f = eval_bsdf(m, a, b, nn);
    f3[0] = f.r; f3[1] = f.g; f3[2] = f.b;
    *pdf = pdf_bsdf(m, a, b, nn);
}
// Sample the BSDF: returns kind (0 evaluated, 1 precomputed) and fills wi, f
// (or weight), pdf, type, valid.  The glass branch's extra draw comes from a
// generator seeded with (sx, sy, ss).
int orc_sample_bsdf(const float* mat7, const float* wo, const float* n, float u1, float u2, float u3, uint32_t sx,
                    uint32_t sy, uint32_t ss, float* wi, float* f3, float* pdf, int* type, int* valid) {
    MatParams m;
    m.albedo = RGB(mat7[0], mat7[1], mat7[2]); m.metallic = mat7[3]; m.roughness = smax(mat7[4], MIN_ROUGHNESS);
    m.transmission = mat7[5]; m.ior = mat7[6];
    Rng rng; seed_xyz(rng, sx, sy, ss);
    BsdfSample s = sample_bsdf(m, V3(wo[0], wo[1], wo[2]), V3(n[0], n[1], n[2]), u1, u2, u3, rng);
    wi[0] = s.wi.x; wi[1] = s.wi.y; wi[2] = s.wi.z;
    f3[0] = s.f.r; f3[1] = s.f.g; f3[2] = s.f.b;
    *pdf = s.pdf; *type = s.type; *valid = s.valid();
    return s.kind;
}
float orc_lm(int fn, float x) {
    switch (fn) {
        case 0: return lucid_math::lm_sinf(x);
        case 1: return lucid_math::lm_cosf(x);
        case 2: return lucid_math::lm_expf(x);
        case 3: return lucid_math::lm_logf(x);
        default: return lucid_math::lm_pow5(x);
    }
}

}  // extern "C"

// ------------------------------------------------------------------ diagnostics
#include "oracle_diag.hpp"

namespace orc {
struct DiagState {
    DiagFilm film;
    bool has = false;
};
static DiagState& diag_of(void* h) {
    static std::map<void*, DiagState> m;
    return m[h];
}
}  // namespace orc

extern "C" {

// One exported path group (layout shared with LucidDiagGroup in
// include/lucid_cuda.h).
struct OrcDiagGroup {
    uint64_t hash;
    uint32_t count;
    uint8_t depth, coarse_type, light_type, strategy;
    float mean_rgb[3], variance_rgb[3];
    float mean_luminance, total_variance;
    int32_t object_ids[16];
    uint8_t bsdf[16];
    uint8_t flags[16];
    float positions[16][3];
    float normals[16][3];
};
struct OrcDiagPixel {
    int32_t valid;
    uint32_t sample_count, group_count, outlier_count, overflow_count;
    float variance;
    float mean_rgb[3];
};

// render_tile with diagnostics enabled (pybind_renderer.hpp:205-316): the
// diagnostic integrators render every pixel; completed paths go to a fresh
// DiagnosticFilm(tile_w, tile_h, subsample) in the single-threaded loop order.
int orc_render_tile_diag(void* h, int tile_x, int tile_y, int tile_w, int tile_h, int full_w, int full_h, int samples,
                         int sample_offset, int max_depth, int subsample, float* out_rgba, int nthreads) {
    Renderer* r = static_cast<Renderer*>(h);
    size_t np = (size_t)tile_w * tile_h;
    std::fill(out_rgba, out_rgba + np * 4, 0.0f);
    if (!r->scene_loaded || !r->camera_set) return -1;
    DiagState& ds = diag_of(h);
    ds.film.init(tile_w, tile_h, subsample);
    ds.has = true;
    r->cam.aspect = (float)full_w / (float)full_h;
    float scale = std::tan(r->cam.fov * 0.5f);
    SceneLights sl = build_lights(r->scene);
    DiagAlgo algo = diag_algo_from(algo_from_string(r->algorithm));
    std::vector<std::vector<PTrace>> per_pixel(np);
    std::vector<float> px(np * 4, 0.0f);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (long long idx = 0; idx < (long long)np; ++idx) {
        int py_ = (int)(idx / tile_w), px_ = (int)(idx % tile_w);
        int gx = tile_x + px_, gy = tile_y + py_;
        float ndc_x = (2.0f * ((float)gx + 0.5f) / (float)full_w - 1.0f) * r->cam.aspect;
        float ndc_y = 1.0f - 2.0f * ((float)gy + 0.5f) / (float)full_h;
        V3 wd = primary_dir(r->cam, ndc_x, ndc_y, scale);
        RGB rad(0, 0, 0);
        Recorder rec;
        for (int si = 0; si < samples; ++si) {
            Rng rng;
            seed_xyz(rng, (uint32_t)gx, (uint32_t)gy, (uint32_t)(sample_offset + si));
            Ray ray{r->cam.pos, wd};
            if (samples > 1) {
                float jx = (randf(rng) - 0.5f) / (float)full_w;
                float jy = (randf(rng) - 0.5f) / (float)full_h;
                ray.d = primary_dir(r->cam, ndc_x + jx, ndc_y + jy, scale);
            }
            rec.begin();
            rad = rad + trace_diag(r->scene, sl, ray, max_depth, algo, rng, rec);
            for (const PTrace& t : rec.completed) per_pixel[idx].push_back(t);
        }
        float* o = &px[(size_t)idx * 4];
        o[0] = smax(rad.r * 1.0f, 0.0f); o[1] = smax(rad.g * 1.0f, 0.0f); o[2] = smax(rad.b * 1.0f, 0.0f); o[3] = 1.0f;
    }
    // film in the single-threaded loop order: 8x8 micro-tiles, pixels, samples, records
    for (int my = 0; my < tile_h; my += 8)
        for (int mx = 0; mx < tile_w; mx += 8)
            for (int j = 0; j < std::min(8, tile_h - my); ++j)
                for (int i = 0; i < std::min(8, tile_w - mx); ++i) {
                    int pxx = mx + i, pyy = my + j;
                    for (const PTrace& t : per_pixel[(size_t)pyy * tile_w + pxx]) ds.film.record(pxx, pyy, t);
                }
    for (int y = 0; y < tile_h; ++y)
        std::copy(px.begin() + (size_t)y * tile_w * 4, px.begin() + (size_t)(y + 1) * tile_w * 4,
                  out_rgba + (size_t)(tile_h - 1 - y) * tile_w * 4);
    return 0;
}

// get_pixel_diagnostic (pybind_renderer.hpp:1008-1102): sorts the cell's
// groups in place (by variance, or by mean when sort_by_mean) and exports them.
int orc_diag_pixel(void* h, int x, int y, int sort_by_mean, OrcDiagPixel* info, OrcDiagGroup* groups, int cap) {
    DiagState& ds = diag_of(h);
    info->valid = 0;
    if (!ds.has) return 0;
    PixelData* p = const_cast<PixelData*>(ds.film.at(x, y));
    if (!p) return 0;
    if (sort_by_mean)
        std::sort(p->groups, p->groups + p->num_groups,
                  [](const PGroup& a, const PGroup& b) { return a.stats.mean_luminance() > b.stats.mean_luminance(); });
    else
        std::sort(p->groups, p->groups + p->num_groups,
                  [](const PGroup& a, const PGroup& b) { return a.stats.total_variance() > b.stats.total_variance(); });
    info->valid = 1;
    info->sample_count = (uint32_t)p->total;
    info->group_count = (uint32_t)p->num_groups;
    info->outlier_count = (uint32_t)p->num_outliers;
    info->overflow_count = (uint32_t)p->overflow;
    info->variance = p->total_stats.total_variance();
    info->mean_rgb[0] = p->total_stats.mean.r; info->mean_rgb[1] = p->total_stats.mean.g; info->mean_rgb[2] = p->total_stats.mean.b;
    int n = (int)std::min<size_t>(p->num_groups, (size_t)cap);
    for (int i = 0; i < n; ++i) {
        const PGroup& g = p->groups[i];
        OrcDiagGroup& o = groups[i];
        std::memset(&o, 0, sizeof(o));
        o.hash = g.hash; o.count = g.stats.count; o.depth = g.depth; o.coarse_type = g.coarse;
        o.light_type = g.light_type; o.strategy = g.strategy;
        o.mean_rgb[0] = g.stats.mean.r; o.mean_rgb[1] = g.stats.mean.g; o.mean_rgb[2] = g.stats.mean.b;
        o.variance_rgb[0] = g.stats.variance.r; o.variance_rgb[1] = g.stats.variance.g; o.variance_rgb[2] = g.stats.variance.b;
        o.mean_luminance = g.stats.mean_luminance();
        o.total_variance = g.stats.total_variance();
        for (int k = 0; k < g.depth; ++k) {
            o.object_ids[k] = g.v[k].object_id; o.bsdf[k] = g.v[k].bsdf; o.flags[k] = g.v[k].flags;
            o.positions[k][0] = g.pos[k].x; o.positions[k][1] = g.pos[k].y; o.positions[k][2] = g.pos[k].z;
            o.normals[k][0] = g.nrm[k].x; o.normals[k][1] = g.nrm[k].y; o.normals[k][2] = g.nrm[k].z;
        }
    }
    return n;
}

static void export_group(const PGroup& g, OrcDiagGroup& o) {
    std::memset(&o, 0, sizeof(o));
    o.hash = g.hash; o.count = g.stats.count; o.depth = g.depth; o.coarse_type = g.coarse;
    o.light_type = g.light_type; o.strategy = g.strategy;
    o.mean_rgb[0] = g.stats.mean.r; o.mean_rgb[1] = g.stats.mean.g; o.mean_rgb[2] = g.stats.mean.b;
    o.variance_rgb[0] = g.stats.variance.r; o.variance_rgb[1] = g.stats.variance.g; o.variance_rgb[2] = g.stats.variance.b;
    o.mean_luminance = g.stats.mean_luminance();
    o.total_variance = g.stats.total_variance();
    for (int k = 0; k < g.depth; ++k) {
        o.object_ids[k] = g.v[k].object_id; o.bsdf[k] = g.v[k].bsdf; o.flags[k] = g.v[k].flags;
        o.positions[k][0] = g.pos[k].x; o.positions[k][1] = g.pos[k].y; o.positions[k][2] = g.pos[k].z;
        o.normals[k][0] = g.nrm[k].x; o.normals[k][1] = g.nrm[k].y; o.normals[k][2] = g.nrm[k].z;
    }
}

// top_groups_by_variance / top_groups_by_mean (diagnostic_film.hpp:160-222):
// every cell's groups (>= 2 samples for variance, >= 1 for mean) in cell
// order, then std::partial_sort of the first n.
int orc_diag_top_groups(void* h, int n, int by_mean, OrcDiagGroup* out, int32_t* xy, int cap) {
    DiagState& ds = diag_of(h);
    if (!ds.has) return 0;
    struct Ref { size_t x, y; const PGroup* g; };
    std::vector<Ref> all;
    const DiagFilm& f = ds.film;
    for (size_t sy = 0; sy < f.shh; ++sy)
        for (size_t sx = 0; sx < f.sw; ++sx) {
            const PixelData& px = f.px[sy * f.sw + sx];
            for (size_t i = 0; i < px.num_groups; ++i)
                if (px.groups[i].stats.count >= (by_mean ? 1u : 2u)) all.push_back({sx * f.sf, sy * f.sf, &px.groups[i]});
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
        export_group(*all[i].g, out[i]);
        xy[2 * i] = (int32_t)all[i].x;
        xy[2 * i + 1] = (int32_t)all[i].y;
    }
    return m;
}

// GlobalDiagnosticStats (diagnostic_film.hpp:124-154): total samples, active
// pixels, groups, overflow, paths recorded.
void orc_diag_stats(void* h, uint64_t* out5) {
    DiagState& ds = diag_of(h);
    uint64_t ts = 0, act = 0, grp = 0, ovf = 0;
    for (const PixelData& p : ds.film.px)
        if (p.total > 0) { ++act; ts += p.total; grp += p.num_groups; ovf += p.overflow; }
    out5[0] = ts; out5[1] = act; out5[2] = grp; out5[3] = ovf; out5[4] = ds.film.recorded;
}

// DiagnosticExporter::get_coarse_stats (diagnostic_export.hpp:110-157): for
// every sampled cell the film is read at (sx * 2, sy * 2) (the exporter's
// fixed factor), and each coarse type is merged with a count-weighted mean and
// the largest variance.  Layout shared with LucidDiagCoarse.
struct OrcDiagCoarse {
    int32_t type_id;
    char name[32];
    uint64_t sample_count;
    float mean_luminance, variance_luminance;
    float mean_rgb[3], variance_rgb[3];
};
void orc_diag_coarse(void* h, OrcDiagCoarse* out) {
    static const char* names[8] = {"Direct-NoDelta-BSDF",   "Direct-NoDelta-NEE",   "Direct-Delta-BSDF",
                                   "Direct-Delta-NEE",      "Indirect-NoDelta-BSDF", "Indirect-NoDelta-NEE",
                                   "Indirect-Delta-BSDF",   "Indirect-Delta-NEE"};   // path_stats.hpp:26-40
    DiagState& ds = diag_of(h);
    const DiagFilm& f = ds.film;
    size_t count[8] = {};
    RGB mean[8], var[8];
    for (size_t sy = 0; sy < f.shh; ++sy)
        for (size_t sx = 0; sx < f.sw; ++sx) {
            const PixelData* px = f.at(sx * 2, sy * 2);
            if (!px) continue;
            for (int t = 0; t < 8; ++t) {
                const PStats& cs = px->coarse[t];
                if (cs.count > 0) {
                    count[t] += cs.count;
                    float w = static_cast<float>(cs.count) / static_cast<float>(count[t]);
                    mean[t].r = mean[t].r * (1.0f - w) + cs.mean.r * w;
                    mean[t].g = mean[t].g * (1.0f - w) + cs.mean.g * w;
                    mean[t].b = mean[t].b * (1.0f - w) + cs.mean.b * w;
                    var[t].r = std::max(var[t].r, cs.variance.r);
                    var[t].g = std::max(var[t].g, cs.variance.g);
                    var[t].b = std::max(var[t].b, cs.variance.b);
                }
            }
        }
    for (int t = 0; t < 8; ++t) {
        OrcDiagCoarse& o = out[t];
        std::memset(&o, 0, sizeof(o));
        o.type_id = t;
        std::snprintf(o.name, sizeof(o.name), "%s", names[t]);
        o.sample_count = count[t];
        o.mean_luminance = 0.2126f * mean[t].r + 0.7152f * mean[t].g + 0.0722f * mean[t].b;   // path_stats.hpp:110-112
        o.variance_luminance = 0.2126f * 0.2126f * var[t].r + 0.7152f * 0.7152f * var[t].g +
                               0.0722f * 0.0722f * var[t].b;                                 // path_stats.hpp:117-123
        o.mean_rgb[0] = mean[t].r; o.mean_rgb[1] = mean[t].g; o.mean_rgb[2] = mean[t].b;
        o.variance_rgb[0] = var[t].r; o.variance_rgb[1] = var[t].g; o.variance_rgb[2] = var[t].b;
    }
}

// DiagnosticExporter::generate_suggestions (diagnostic_export.hpp:178-248):
// returns how many suggestions there are and, for up to cap of them, the
// index of each (0 glossy, 1 indirect, 2 diffuse, 3 capacity) in order.
int orc_diag_suggestions(void* h, int32_t* kinds, int cap) {
    DiagState& ds = diag_of(h);
    OrcDiagGroup top[10];
    int32_t xy[20];
    int n = orc_diag_top_groups(h, 10, 0, top, xy, 10);
    if (n == 0) return 0;
    size_t glossy = 0, indirect = 0, diffuse = 0;
    for (int i = 0; i < n; ++i) {
        bool has_glossy = false, has_indirect = top[i].depth > 2;
        for (int v = 0; v < top[i].depth; ++v)
            if (top[i].bsdf[v] == B_GLOSSY) has_glossy = true;
        if (has_glossy) ++glossy;
        if (has_indirect) ++indirect;
        if (!has_glossy && !has_indirect) ++diffuse;
    }
    std::vector<int32_t> out;
    if (glossy > 3) out.push_back(0);
    if (indirect > 3) out.push_back(1);
    if (diffuse > 3) out.push_back(2);
    uint64_t st[5];
    orc_diag_stats(h, st);
    if (st[0] > 0 && st[3] > st[1] * 0.1) out.push_back(3);
    for (int i = 0; i < (int)out.size() && i < cap; ++i) kinds[i] = out[i];
    (void)ds;
    return (int)out.size();
}

// DiagnosticFilm::export_binary (diagnostic_film.hpp:243-299); returns the
// size and copies min(size, cap) bytes.
long long orc_diag_export_binary(void* h, int max_groups, int max_outliers, uint8_t* out, size_t cap) {
    DiagState& ds = diag_of(h);
    const DiagFilm& f = ds.film;
    std::string b;
    auto w = [&](const void* p, size_t n) { b.append(static_cast<const char*>(p), n); };
    w("PVAR", 4);
    uint32_t version = 1, fw = (uint32_t)f.w, fh = (uint32_t)f.h, sw = (uint32_t)f.sw, sh = (uint32_t)f.shh;
    w(&version, 4); w(&fw, 4); w(&fh, 4); w(&sw, 4); w(&sh, 4);
    uint8_t sf = (uint8_t)f.sf, mg = (uint8_t)max_groups, mo = (uint8_t)max_outliers;
    char padding = 0;
    w(&sf, 1); w(&mg, 1); w(&mo, 1); w(&padding, 1);
    for (const PixelData& px : f.px) {
        uint16_t gc = (uint16_t)px.num_groups;
        uint32_t ts = (uint32_t)px.total;
        float mean[3] = {px.total_stats.mean.r, px.total_stats.mean.g, px.total_stats.mean.b};
        float var = px.total_stats.total_variance();
        w(&gc, 2); w(&ts, 4); w(mean, 12); w(&var, 4);
    }
    if (out) std::memcpy(out, b.data(), std::min(cap, b.size()));
    return (long long)b.size();
}

}  // extern "C"
