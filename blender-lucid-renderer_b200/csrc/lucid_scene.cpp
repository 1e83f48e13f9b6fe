// lucid_scene.cpp — JSON scene → flattened device-ready arrays.
//
// Semantics follow PyRenderer::loadSceneFromJsonString
// (include/pybind_renderer.hpp:1258-1542), parseNativeLights (:1544-1746),
// finalizeMeshBounds (core/scene.hpp:191-227) and SceneLights::buildFromScene
// (light/scene_lights.hpp:56-122): the same keys, defaults and float
// conversions, so the uploaded lights, CDF and normals equal the CPU
// renderer's bit for bit.  Compiled with -ffp-contract=off.
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <nlohmann/json.hpp>
#include <stdexcept>

#include <vector_functions.h>

#include "lucid_host.h"
#include "lucid_math.h"
#include "lucid_nodes.h"

namespace lucid {
static_assert(LUCID_LIGHT_POINT == LIGHT_POINT && LUCID_LIGHT_SUN == LIGHT_SUN && LUCID_LIGHT_SPOT == LIGHT_SPOT &&
                  LUCID_LIGHT_AREA == LIGHT_AREA, "light type ids");
static_assert(LUCID_AREA_SQUARE == AREA_SQUARE && LUCID_AREA_RECTANGLE == AREA_RECTANGLE && LUCID_AREA_DISK == AREA_DISK &&
                  LUCID_AREA_ELLIPSE == AREA_ELLIPSE, "area shape ids");
namespace {

using json = nlohmann::json;

struct F3 {
    float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 cross3(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len2(F3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// make_direction_or_default / make_normal_or_default (render_units.hpp:485-503, 776-791)
inline F3 dir_or(F3 v, F3 fb) {
    float l2 = len2(v);
    if (l2 < 1e-6f * 1e-6f) return fb;
    float l = std::sqrt(l2);
    return {v.x / l, v.y / l, v.z / l};
}
inline float4 f4(F3 v, float w) { float4 r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }
inline float ibits(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline F3 arr3(const json& a) { return {a[0].get<float>(), a[1].get<float>(), a[2].get<float>()}; }

// Is the Material Output's Surface input linked?  (node_evaluator.cpp:82-163
// builds the links map; pybind_renderer.hpp:1377-1388 reads the socket.)
bool surface_linked(const json& nt, bool& valid) {
    valid = false;
    if (!nt.contains("nodes") || !nt.is_object()) return true;
    const auto& nodes = nt["nodes"];
    valid = !nodes.empty();
    if (!valid) return true;
    std::map<std::pair<std::string, std::string>, bool> links;
    if (nt.contains("links"))
        for (const auto& l : nt["links"])
            links[{l["to_node"].get<std::string>(), l["to_socket"].get<std::string>()}] = true;
    for (const auto& n : nodes) {
        if (n.value("type", "") != "ShaderNodeOutputMaterial") continue;
        const std::string name = n.value("name", "");
        if (!n.contains("inputs")) return false;
        for (const auto& in : n["inputs"])
            if (in.value("name", "") == "Surface") return links.count({name, "Surface"}) > 0;
        return false;
    }
    return true;
}

struct NativeLight {
    int type = LIGHT_POINT;
    F3 pos{0, 0, 0}, normal{0, 0, 1};
    float em[3] = {0, 0, 0};
    float area = 0, radius = 0, spot_angle = 0, spot_blend = 0;
    F3 right{1, 0, 0}, up{0, 1, 0};
    float sx = 1, sy = 1;
    int shape = AREA_SQUARE;
};

// One native light from its parameters (parseNativeLights,
// pybind_renderer.hpp:1544-1746, W -> radiance conversions).  type: a
// LightTypeId (0 for a name the reference does not know); dir, right and up
// are null when the JSON omits them.
NativeLight make_light(int type, F3 pos, const F3* dir, float cr, float cg, float cb, float energy, float radius,
                       float spot_size, float spot_blend, float sx, float sy, int shape, const F3* right,
                       const F3* up) {
    const double PI = M_PI;
    const float EPS = 1e-6f;
    NativeLight L;
    L.pos = pos;
    if (dir) L.normal = dir_or(*dir, F3{0, 0, -1});
    if (type == LIGHT_POINT) {
        L.type = LIGHT_POINT;
        L.radius = radius;
        float area = 4.0f * PI * radius * radius;
        if (area < EPS) area = 1.0f;
        L.area = area;
        if (radius > EPS) {
            L.em[0] = (float)(cr * (energy / (PI * area)));
            L.em[1] = (float)(cg * (energy / (PI * area)));
            L.em[2] = (float)(cb * (energy / (PI * area)));
        } else {
            float factor = energy / (4.0f * PI);
            L.em[0] = cr * factor; L.em[1] = cg * factor; L.em[2] = cb * factor;
        }
    } else if (type == LIGHT_SUN) {
        L.type = LIGHT_SUN;
        L.area = 1.0f;
        L.em[0] = cr * energy; L.em[1] = cg * energy; L.em[2] = cb * energy;
    } else if (type == LIGHT_SPOT) {
        L.type = LIGHT_SPOT;
        L.radius = radius;
        L.spot_angle = spot_size;
        L.spot_blend = spot_blend;
        L.area = 1.0f;
        float half = spot_size * 0.5f;
        float solid = 2.0f * PI * (1.0f - std::cos(half));
        float factor = energy / solid;
        L.em[0] = cr * factor; L.em[1] = cg * factor; L.em[2] = cb * factor;
    } else if (type == LIGHT_AREA) {
        L.type = LIGHT_AREA;
        L.sx = sx; L.sy = sy;
        float area;
        if (shape == AREA_DISK) { L.shape = AREA_DISK; float r = sx * 0.5f; area = PI * r * r; }
        else if (shape == AREA_ELLIPSE) { L.shape = AREA_ELLIPSE; float rx = sx * 0.5f, ry = sy * 0.5f; area = PI * rx * ry; }
        else if (shape == AREA_RECTANGLE) { L.shape = AREA_RECTANGLE; area = sx * sy; }
        else { L.shape = AREA_SQUARE; area = sx * sy; }
        L.area = area;
        if (right) L.right = dir_or(*right, F3{1, 0, 0});
        if (up) L.up = dir_or(*up, F3{0, 1, 0});
        float factor = energy / (PI * area);
        L.em[0] = cr * factor; L.em[1] = cg * factor; L.em[2] = cb * factor;
    } else {
        // An unknown type keeps the reference's default-constructed Light
        // (EMISSIVE_MESH with zero area and emission).
        L.type = LIGHT_EMISSIVE;
        L.area = 0.0f;
    }
    return L;
}

// parseNativeLights (pybind_renderer.hpp:1544-1746): JSON keys and defaults.
void parse_lights(const json& arr, std::vector<NativeLight>& out) {
    for (const auto& lj : arr) {
        std::string type = lj.value("type", "POINT");
        int t = type == "POINT" ? LIGHT_POINT : type == "SUN" ? LIGHT_SUN : type == "SPOT" ? LIGHT_SPOT
              : type == "AREA" ? LIGHT_AREA : LIGHT_EMISSIVE;
        F3 pos{0, 0, 0}, dir{0, 0, -1}, right{1, 0, 0}, up{0, 1, 0};
        if (lj.contains("position")) pos = arr3(lj["position"]);
        const bool has_dir = lj.contains("direction");
        if (has_dir) dir = arr3(lj["direction"]);
        float cr = 1, cg = 1, cb = 1;
        if (lj.contains("color")) { F3 c = arr3(lj["color"]); cr = c.x; cg = c.y; cb = c.z; }
        float energy = lj.value("energy", 1.0f);
        float radius = lj.value("radius", 0.0f);
        float spot_size = lj.value("spot_size", static_cast<float>(M_PI / 4.0f));
        float spot_blend = lj.value("spot_blend", 0.0f);
        float sx = lj.value("size", 1.0f);
        float sy = lj.value("size_y", sx);
        std::string shape = lj.value("shape", "SQUARE");
        int sh = shape == "DISK" ? AREA_DISK : shape == "ELLIPSE" ? AREA_ELLIPSE
               : shape == "RECTANGLE" ? AREA_RECTANGLE : AREA_SQUARE;
        const bool has_right = t == LIGHT_AREA && lj.contains("right");
        const bool has_up = t == LIGHT_AREA && lj.contains("up");
        if (has_right) right = arr3(lj["right"]);
        if (has_up) up = arr3(lj["up"]);
        out.push_back(make_light(t, pos, has_dir ? &dir : nullptr, cr, cg, cb, energy, radius, spot_size, spot_blend,
                                 sx, sy, sh, has_right ? &right : nullptr, has_up ? &up : nullptr));
    }
}

DevLight pack_native(const NativeLight& L) {
    DevLight d;
    std::memset(&d, 0, sizeof(d));
    d.pos_type = f4(L.pos, ibits(L.type));
    // point-like lights get 1 m^2 in the CDF (scene_lights.hpp:106-108)
    float area = L.area < 1e-6f ? 1.0f : L.area;
    d.normal_area = f4(L.normal, area);
    d.emission_radius = f4(F3{L.em[0], L.em[1], L.em[2]}, L.radius);
    d.v0_shape = f4(F3{0, 0, 0}, ibits(L.shape));
    d.v1_cosc = f4(F3{0, 0, 0}, lucid_math::lm_cosf(L.spot_angle * 0.5f));
    d.v2_blend = f4(F3{0, 0, 0}, L.spot_blend);
    d.right_sx = f4(L.right, L.sx);
    d.up_sy = f4(L.up, L.sy);
    return d;
}

// is_emissive (render_units.hpp:1200-1202): luminance above 1e-6.
bool is_emissive(const float em[3]) { return (0.2126f * em[0] + 0.7152f * em[1] + 0.0722f * em[2]) > 1e-6f; }

// A mesh's material record (getMaterialParams / getEmission inputs,
// integrator/path_tracer.hpp:45-72); node programs are set by the caller.
DevMaterial make_material(const float alb[3], float metallic, float roughness, const float em[3], float transmission,
                          float ior, bool boundary, bool textured) {
    const bool emissive = is_emissive(em);
    DevMaterial dm;
    std::memset(&dm, 0, sizeof(dm));
    dm.albedo_metallic = f4(F3{alb[0], alb[1], alb[2]}, metallic);
    dm.rough_trans_ior_flags.x = roughness;
    dm.rough_trans_ior_flags.y = transmission;
    dm.rough_trans_ior_flags.z = ior;
    dm.rough_trans_ior_flags.w =
        ibits((emissive ? MAT_EMISSIVE : 0) | (boundary ? MAT_BOUNDARY_ONLY : 0) | (textured ? MAT_TEXTURED : 0));
    dm.emission = f4(F3{em[0], em[1], em[2]}, emissive ? 1.0f : 0.0f);
    return dm;
}

// One native light of the array form (LucidLightDesc).
NativeLight light_from_desc(const LucidLightDesc& l) {
    const int t = (l.type == LUCID_LIGHT_POINT || l.type == LUCID_LIGHT_SUN || l.type == LUCID_LIGHT_SPOT ||
                   l.type == LUCID_LIGHT_AREA) ? l.type : LIGHT_EMISSIVE;
    const F3 dir{l.direction[0], l.direction[1], l.direction[2]};
    const F3 right{l.right[0], l.right[1], l.right[2]}, up{l.up[0], l.up[1], l.up[2]};
    return make_light(t, F3{l.position[0], l.position[1], l.position[2]}, &dir, l.color[0], l.color[1], l.color[2],
                      l.energy, l.radius, l.spot_size, l.spot_blend, l.size, l.size_y, l.shape,
                      t == LIGHT_AREA ? &right : nullptr, t == LIGHT_AREA ? &up : nullptr);
}

// SceneLights' CDF over the light list by cumulative area / total
// (scene_lights.hpp:103-121; the total summed in list order, as
// buildFromScene sums it) and the CDF search guide.
void light_cdf(HostScene& S) {
    float total = 0.0f;
    for (const auto& d : S.lights) total += d.normal_area.w;
    S.total_light_area = total;
    S.cdf.resize(S.lights.size());
    float cum = 0.0f;
    for (size_t i = 0; i < S.lights.size(); ++i) {
        cum += S.lights[i].normal_area.w;
        S.cdf[i] = (total < 1e-6f) ? 0.0f : cum / total;
    }
    S.light_guide.resize(kLightGuide + 1);
    for (int k = 0; k <= kLightGuide; ++k) {
        float x = (float)k / (float)kLightGuide;   // exact: power-of-two denominator
        S.light_guide[k] = (int)(std::lower_bound(S.cdf.begin(), S.cdf.end(), x) - S.cdf.begin());
    }
}

// Scene assembly shared by the JSON and the array loaders: meshes in order,
// then the native lights, then SceneLights (emissive triangles first).
struct Assembly {
    std::vector<DevLight> emissive_lights;
    float total = 0.0f;
    int mesh_index = 0;
};

// One mesh's material, prims, face/vertex normals and emissive-triangle
// lights (pybind_renderer.hpp:1346-1503, scene.hpp:214-222,
// scene_lights.hpp:79-101).  tn: normalised per-triangle vertex normals
// (used when smooth), or empty.
void emit_mesh(HostScene& S, Assembly& A, const std::vector<F3>& verts, const std::vector<std::array<int, 3>>& tris,
               const std::vector<std::array<F3, 3>>& tn, bool has_tn, bool smooth, const float alb_in[3],
               float metallic, float roughness, const float em_in[3], float transmission, float ior, bool boundary,
               DevVolume vol, bool vol_has_grid, const std::vector<float>& grid,
               const std::vector<std::array<float, 6>>& uvs = {}, const NodeMaterial* nm = nullptr) {
    const int mesh_index = A.mesh_index;
    // use_nodes: every parameter comes from the node graph
    // (getMaterialParams / getEmission, integrator/path_tracer.hpp:45-72)
    float alb[3] = {alb_in[0], alb_in[1], alb_in[2]}, em[3] = {em_in[0], em_in[1], em_in[2]};
    if (nm) {
        for (int c = 0; c < 3; ++c) { alb[c] = nm->albedo[c]; em[c] = nm->emission[c]; }
        metallic = nm->metallic; roughness = nm->roughness; transmission = nm->transmission; ior = nm->ior;
    }
    const bool textured = nm && (nm->albedo_n > 0 || nm->emission_n > 0);
    for (const auto& t : tris)
        for (int k = 0; k < 3; ++k)
            if (t[k] < 0 || t[k] >= (int)verts.size())
                throw std::runtime_error("mesh " + std::to_string(mesh_index) + ": triangle index out of range");
    if (vol_has_grid) {
        vol.grid_offset = (long long)S.grid.size();
        S.grid.insert(S.grid.end(), grid.begin(), grid.end());
        S.volumes.push_back(vol);
    }
    S.num_boundary_meshes += boundary;
    const bool emissive = is_emissive(em);
    DevMaterial dm = make_material(alb, metallic, roughness, em, transmission, ior, boundary, textured);
    dm.program.x = nm ? nm->albedo_start : 0;
    dm.program.y = nm ? nm->albedo_n : 0;
    dm.program.z = nm ? nm->emission_start : 0;
    dm.program.w = nm ? nm->emission_n : 0;
    S.materials.push_back(dm);
    for (size_t ti = 0; ti < tris.size(); ++ti) {
        const auto& t = tris[ti];
        F3 a = verts[t[0]], b = verts[t[1]], c = verts[t[2]];
        F3 e1 = sub(b, a), e2 = sub(c, a);
        F3 fn = dir_or(cross3(e1, e2), F3{0, 1, 0});
        int prim = S.num_prims++;
        S.tri.push_back(f4(a, ibits(prim)));
        S.tri.push_back(f4(e1, 0.0f));
        S.tri.push_back(f4(e2, 0.0f));
        S.verts.push_back(f4(a, 0.0f));
        S.verts.push_back(f4(b, 0.0f));
        S.verts.push_back(f4(c, 0.0f));
        bool sm = has_tn && ti < tn.size() && smooth;
        int light_index = -1;
        if (emissive) {
            float area = std::sqrt(len2(cross3(e1, e2))) * 0.5f;
            if (area > 1e-6f) {
                DevLight d;
                std::memset(&d, 0, sizeof(d));
                d.pos_type = f4(F3{0, 0, 0}, ibits(LIGHT_EMISSIVE));
                d.normal_area = f4(fn, area);
                d.emission_radius = f4(F3{em[0], em[1], em[2]}, 0.0f);
                d.v0_shape = f4(a, ibits(0));
                d.v1_cosc = f4(b, 0.0f);
                d.v2_blend = f4(c, 0.0f);
                light_index = (int)A.emissive_lights.size();
                A.emissive_lights.push_back(d);
                A.total += area;
            }
        }
        int4 pi;
        pi.x = mesh_index; pi.y = (int)ti; pi.z = light_index; pi.w = sm ? 1 : 0;
        S.prim_info.push_back(pi);
        S.prim_fn.push_back(f4(fn, 0.0f));
        for (int k = 0; k < 3; ++k) S.prim_vn.push_back(sm ? f4(tn[ti][k], 0.0f) : f4(fn, 0.0f));
        S.prim_boundary.push_back(boundary ? 1 : 0);
        // UVs (pybind_renderer.hpp:1296-1336); dropped in finish_scene when no prim has any
        float4 u0 = {0, 0, 0, 0}, u1 = {0, 0, 0, 0};
        if (ti < uvs.size()) {
            const auto& q = uvs[ti];
            u0.x = q[0]; u0.y = q[1]; u0.z = q[2]; u0.w = q[3]; u1.x = q[4]; u1.y = q[5]; u1.z = 1.0f;
        }
        S.prim_uv.push_back(u0);
        S.prim_uv.push_back(u1);
    }
    ++A.mesh_index;
}

// SceneLights: emissive triangles, then native lights; CDF by cumulative
// area / total (scene_lights.hpp:103-121) and the CDF search guide.
void finish_scene(HostScene& S, Assembly& A, const std::vector<NativeLight>& native, const float env[3]) {
    S.num_meshes = A.mesh_index;
    bool any_uv = false;
    for (size_t i = 1; i < S.prim_uv.size() && !any_uv; i += 2) any_uv = S.prim_uv[i].z != 0.0f;
    if (!any_uv) std::vector<float4>().swap(S.prim_uv);
    for (int k = 0; k < 3; ++k) S.env[k] = env[k];
    S.lights = A.emissive_lights;
    S.native_start = (int)S.lights.size();
    S.num_native = (int)native.size();
    for (const auto& L : native) S.lights.push_back(pack_native(L));
    light_cdf(S);
}

// One "meshes" entry read as loadSceneFromJsonString reads it
// (pybind_renderer.hpp:1266-1536): geometry, normals, UVs, the material (node
// programs compiled into M.ops, offsets relative to M.ops) and the volume.
struct MeshIn {
    std::vector<F3> verts;
    std::vector<std::array<F3, 3>> tn;
    bool has_tn = false, smooth = false;
    std::vector<std::array<int, 3>> tris;
    std::vector<std::array<float, 6>> uvs;
    bool use_nodes = false;
    NodeMaterial nm;
    std::vector<float4> ops;
    float alb[3] = {0.8f, 0.8f, 0.8f}, metallic = 0.0f, roughness = 0.5f, em[3] = {0, 0, 0};
    float transmission = 0.0f, ior = 1.45f;
    bool boundary = false;
    DevVolume vol;
    bool vol_has_grid = false;
    std::vector<float> grid;
};

void read_mesh(const json& mj, MeshIn& M) {
    std::vector<F3> verts;
    if (mj.contains("vertices"))
        for (const auto& v : mj["vertices"]) verts.push_back(arr3(v));
    std::vector<std::array<F3, 3>> tn;
    bool has_tn = false;
    if (mj.contains("triangle_normals")) {
        has_tn = true;
        for (const auto& t : mj["triangle_normals"]) {
            std::array<F3, 3> a;
            for (int k = 0; k < 3; ++k)
                a[k] = dir_or(F3{static_cast<float>(t[k][0]), static_cast<float>(t[k][1]),
                                 static_cast<float>(t[k][2])}, F3{0, 0, 1});
            tn.push_back(a);
        }
    }
    bool smooth = mj.contains("smooth") && mj["smooth"].get<bool>();
    std::vector<std::array<int, 3>> tris;
    if (mj.contains("triangles"))
        for (const auto& t : mj["triangles"]) tris.push_back({t[0].get<int>(), t[1].get<int>(), t[2].get<int>()});
    std::vector<std::array<float, 6>> uvs;
    if (mj.contains("triangle_uvs"))
        for (const auto& t : mj["triangle_uvs"])
            uvs.push_back({t[0][0].get<float>(), t[0][1].get<float>(), t[1][0].get<float>(),
                           t[1][1].get<float>(), t[2][0].get<float>(), t[2][1].get<float>()});
    bool use_nodes = false;
    NodeMaterial nm;

    // material (pybind_renderer.hpp:1346-1503)
    float alb[3] = {0.8f, 0.8f, 0.8f}, metallic = 0.0f, roughness = 0.5f, em[3] = {0, 0, 0};
    float transmission = 0.0f, ior = 1.45f;
    bool boundary = false;
    DevVolume vol;
    std::memset(&vol, 0, sizeof(vol));
    vol.color[0] = vol.color[1] = vol.color[2] = 1.0f;
    bool vol_has_grid = false;
    std::vector<float> grid;
    if (mj.contains("material")) {
        const auto& mat = mj["material"];
        if (mat.contains("base_color")) { F3 c = arr3(mat["base_color"]); alb[0] = c.x; alb[1] = c.y; alb[2] = c.z; }
        if (mat.contains("metallic")) metallic = mat["metallic"];
        if (mat.contains("roughness")) roughness = mat["roughness"];
        if (mat.contains("emission")) { F3 c = arr3(mat["emission"]); em[0] = c.x; em[1] = c.y; em[2] = c.z; }
        if (mat.contains("transmission")) transmission = mat["transmission"];
        if (mat.contains("ior")) ior = mat["ior"];
        bool nt_valid = false, surf = true;
        if (mat.contains("node_tree") && !mat["node_tree"].is_null()) {
            surf = surface_linked(mat["node_tree"], nt_valid);
            if (!nt_valid) surf = true;
            use_nodes = nt_valid && mat.value("use_nodes", false);
            if (use_nodes) nm = compile_node_material(mat["node_tree"], M.ops);
        }
        if (mat.contains("volume") && !mat["volume"].is_null()) {
            const auto& v = mat["volume"];
            if (v.contains("color") && v["color"].is_array() && v["color"].size() >= 3) {
                F3 c = arr3(v["color"]); vol.color[0] = c.x; vol.color[1] = c.y; vol.color[2] = c.z;
            }
            if (v.contains("absorption_color") && v["absorption_color"].is_array() && v["absorption_color"].size() >= 3) {
                F3 c = arr3(v["absorption_color"]); vol.absorption[0] = c.x; vol.absorption[1] = c.y; vol.absorption[2] = c.z;
            }
            if (v.contains("density")) vol.density = v["density"].get<float>();
            if (v.contains("anisotropy")) vol.anisotropy = v["anisotropy"].get<float>();
            if (v.contains("smoke_grid") && v["smoke_grid"].is_object()) {
                const auto& sg = v["smoke_grid"];
                if (sg.contains("dims") && sg["dims"].is_array() && sg["dims"].size() == 3 && sg.contains("world_min") &&
                    sg["world_min"].is_array() && sg.contains("world_max") && sg["world_max"].is_array() &&
                    sg.contains("sidecar_path")) {
                    for (int i = 0; i < 3; ++i) vol.dims[i] = sg["dims"][i].get<int>();
                    for (int i = 0; i < 3; ++i) {
                        vol.wmin[i] = sg["world_min"][i].get<float>();
                        vol.wmax[i] = sg["world_max"][i].get<float>();
                    }
                    if (vol.dims[0] < 2 || vol.dims[1] < 2 || vol.dims[2] < 2)
                        throw std::runtime_error("volume grid dims must be >= 2 per axis");
                    size_t n = (size_t)vol.dims[0] * vol.dims[1] * vol.dims[2];
                    std::ifstream f(sg["sidecar_path"].get<std::string>(), std::ios::binary);
                    if (f) {
                        grid.resize(n);
                        f.read(reinterpret_cast<char*>(grid.data()), n * sizeof(float));
                        float mx = 0.0f;
                        for (float d : grid) if (d > mx) mx = d;
                        vol.grid_max = mx;
                        vol_has_grid = true;
                    } else {
                        vol.dims[0] = vol.dims[1] = vol.dims[2] = 0;
                    }
                }
            }
        }
        bool present = vol.density > 0.0f || vol_has_grid;
        if (present && !surf) boundary = true;
    }
    M.verts = std::move(verts); M.tn = std::move(tn); M.has_tn = has_tn; M.smooth = smooth; M.tris = std::move(tris);
    M.uvs = std::move(uvs); M.use_nodes = use_nodes; M.nm = nm;
    for (int c = 0; c < 3; ++c) { M.alb[c] = alb[c]; M.em[c] = em[c]; }
    M.metallic = metallic; M.roughness = roughness; M.transmission = transmission; M.ior = ior;
    M.boundary = boundary; M.vol = vol; M.vol_has_grid = vol_has_grid; M.grid = std::move(grid);
}

// Appends a read mesh (its node programs relocated after the scene's).
void emit_read_mesh(HostScene& S, Assembly& A, MeshIn& M) {
    const int base = (int)S.tex_ops.size() / 2;
    if (M.use_nodes) {
        if (M.nm.albedo_n) M.nm.albedo_start += base;
        if (M.nm.emission_n) M.nm.emission_start += base;
        S.tex_ops.insert(S.tex_ops.end(), M.ops.begin(), M.ops.end());
    }
    emit_mesh(S, A, M.verts, M.tris, M.tn, M.has_tn, M.smooth, M.alb, M.metallic, M.roughness, M.em, M.transmission,
              M.ior, M.boundary, M.vol, M.vol_has_grid, M.grid, M.uvs, M.use_nodes ? &M.nm : nullptr);
}

// Byte ranges of the elements of the document's top-level "meshes" array
// and of the array itself, found by a structural scan (strings and escapes
// respected).  False when the text is not a plain object with exactly one
// "meshes" array (the caller then parses it whole).
bool scan_meshes(const char* t, size_t n, size_t& arr_begin, size_t& arr_end,
                 std::vector<std::pair<size_t, size_t>>& elems) {
    size_t i = 0;
    auto ws = [&] { while (i < n && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) ++i; };
    auto skip_string = [&]() -> bool {   // at '"'
        for (++i; i < n; ++i) {
            if (t[i] == '\\') { ++i; continue; }
            if (t[i] == '"') { ++i; return true; }
        }
        return false;
    };
    auto skip_value = [&]() -> bool {
        ws();
        if (i >= n) return false;
        if (t[i] == '"') return skip_string();
        if (t[i] == '{' || t[i] == '[') {
            int depth = 0;
            while (i < n) {
                const char c = t[i];
                if (c == '"') { if (!skip_string()) return false; continue; }
                if (c == '{' || c == '[') ++depth;
                else if (c == '}' || c == ']') { if (--depth == 0) { ++i; return true; } }
                ++i;
            }
            return false;
        }
        while (i < n && t[i] != ',' && t[i] != '}' && t[i] != ']') ++i;   // number / literal
        return true;
    };
    ws();
    if (i >= n || t[i] != '{') return false;
    ++i;
    bool found = false;
    for (;;) {
        ws();
        if (i < n && t[i] == '}') break;
        if (i >= n || t[i] != '"') return false;
        const size_t k0 = i;
        if (!skip_string()) return false;
        const bool is_meshes = (i - k0 == 8) && std::memcmp(t + k0, "\"meshes\"", 8) == 0;
        ws();
        if (i >= n || t[i] != ':') return false;
        ++i;
        ws();
        if (is_meshes) {
            if (found || i >= n || t[i] != '[') return false;
            found = true;
            arr_begin = i++;
            for (;;) {
                ws();
                if (i < n && t[i] == ']') { ++i; break; }
                const size_t e0 = i;
                if (!skip_value()) return false;
                elems.push_back({e0, i});
                ws();
                if (i < n && t[i] == ',') { ++i; continue; }
                if (i < n && t[i] == ']') { ++i; break; }
                return false;
            }
            arr_end = i;
        } else if (!skip_value()) {
            return false;
        }
        ws();
        if (i < n && t[i] == ',') { ++i; continue; }
        if (i < n && t[i] == '}') break;
        return false;
    }
    return found;
}

}  // namespace

bool parse_scene_json(const char* text, size_t length, HostScene& S, std::string& err) {
    S = HostScene();
    // Large scenes: the mesh entries are parsed on all host threads, then
    // assembled in order (the result is the same as one whole parse).
    size_t ab = 0, ae = 0;
    std::vector<std::pair<size_t, size_t>> elems;
    std::vector<MeshIn> parsed;
    bool split = length > (8u << 20) && scan_meshes(text, length, ab, ae, elems) && elems.size() > 1;
    json j;
    try {
        if (split) {
            std::string rest(text, ab);
            rest += "[]";
            rest.append(text + ae, length - ae);
            j = json::parse(rest);
        } else {
            j = json::parse(text, text + length);
        }
    } catch (const std::exception& e) {
        err = std::string("scene JSON parse error: ") + e.what();
        return false;
    }
    if (split) {
        parsed.resize(elems.size());
        std::vector<std::string> errors(elems.size());
        std::atomic<size_t> next{0};
        auto work = [&] {
            for (size_t k; (k = next.fetch_add(1)) < elems.size();) {
                try {
                    read_mesh(json::parse(text + elems[k].first, text + elems[k].second), parsed[k]);
                } catch (const json::parse_error& e) {
                    errors[k] = std::string("scene JSON parse error: ") + e.what();
                } catch (const std::exception& e) {
                    errors[k] = std::string("malformed scene: ") + e.what();
                }
            }
        };
        const unsigned nt = std::max(1u, std::min((unsigned)elems.size(), std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        for (const auto& e : errors)
            if (!e.empty()) { err = e; return false; }
    }
    try {
        Assembly A;
        if (split) {
            for (auto& M : parsed) emit_read_mesh(S, A, M);
        } else if (j.contains("meshes")) {
            for (const auto& mj : j["meshes"]) {
                MeshIn M;
                read_mesh(mj, M);
                emit_read_mesh(S, A, M);
            }
        }
        std::vector<NativeLight> native;
        if (j.contains("native_lights") && j["native_lights"].is_array()) parse_lights(j["native_lights"], native);
        else if (j.contains("lights") && j["lights"].is_array()) parse_lights(j["lights"], native);
        float env[3] = {0.05f * 1.0f, 0.05f * 1.0f, 0.05f * 1.0f};
        if (j.contains("environment") && j["environment"].is_object()) {
            const auto& e = j["environment"];
            float col[3] = {0.05f, 0.05f, 0.05f}, strength = 1.0f;
            if (e.contains("color") && e["color"].is_array()) { F3 c = arr3(e["color"]); col[0] = c.x; col[1] = c.y; col[2] = c.z; }
            if (e.contains("strength")) strength = e["strength"].get<float>();
            for (int k = 0; k < 3; ++k) env[k] = col[k] * strength;
        }
        finish_scene(S, A, native, env);
    } catch (const std::exception& e) {
        err = std::string("malformed scene: ") + e.what();
        return false;
    }
    return true;
}

bool build_scene_arrays(const LucidSceneDesc& d, HostScene& S, std::string& err) {
    S = HostScene();
    try {
        if (d.num_meshes < 0 || d.num_lights < 0) throw std::runtime_error("negative mesh or light count");
        if ((d.num_meshes > 0 && !d.meshes) || (d.num_lights > 0 && !d.lights))
            throw std::runtime_error("null mesh or light array");
        Assembly A;
        for (int mi = 0; mi < d.num_meshes; ++mi) {
            const LucidMeshDesc& m = d.meshes[mi];
            if (m.num_vertices < 0 || m.num_triangles < 0) throw std::runtime_error("negative vertex or triangle count");
            if ((m.num_vertices > 0 && !m.vertices) || (m.num_triangles > 0 && !m.triangles))
                throw std::runtime_error("mesh " + std::to_string(mi) + ": null vertex or triangle array");
            std::vector<F3> verts((size_t)m.num_vertices);
            for (int i = 0; i < m.num_vertices; ++i)
                verts[i] = F3{m.vertices[3 * i], m.vertices[3 * i + 1], m.vertices[3 * i + 2]};
            std::vector<std::array<int, 3>> tris((size_t)m.num_triangles);
            for (int i = 0; i < m.num_triangles; ++i)
                tris[i] = {m.triangles[3 * i], m.triangles[3 * i + 1], m.triangles[3 * i + 2]};
            std::vector<std::array<F3, 3>> tn;
            const bool has_tn = m.triangle_normals != nullptr;
            if (has_tn) {
                tn.resize((size_t)m.num_triangles);
                for (int i = 0; i < m.num_triangles; ++i)
                    for (int k = 0; k < 3; ++k) {
                        const float* q = m.triangle_normals + 9 * i + 3 * k;
                        tn[i][k] = dir_or(F3{q[0], q[1], q[2]}, F3{0, 0, 1});
                    }
            }
            DevVolume vol;
            std::memset(&vol, 0, sizeof(vol));
            for (int k = 0; k < 3; ++k) {
                vol.color[k] = m.volume_color[k];
                vol.absorption[k] = m.volume_absorption[k];
            }
            vol.density = m.volume_density;
            vol.anisotropy = m.volume_anisotropy;
            bool vol_has_grid = false;
            std::vector<float> grid;
            if (m.volume_dims[0] != 0 || m.volume_dims[1] != 0 || m.volume_dims[2] != 0) {
                for (int k = 0; k < 3; ++k) {
                    vol.dims[k] = m.volume_dims[k];
                    vol.wmin[k] = m.volume_world_min[k];
                    vol.wmax[k] = m.volume_world_max[k];
                }
                if (vol.dims[0] < 2 || vol.dims[1] < 2 || vol.dims[2] < 2)
                    throw std::runtime_error("volume grid dims must be >= 2 per axis");
                if (m.volume_grid) {
                    const size_t n = (size_t)vol.dims[0] * vol.dims[1] * vol.dims[2];
                    grid.assign(m.volume_grid, m.volume_grid + n);
                    float mx = 0.0f;
                    for (float g : grid) if (g > mx) mx = g;
                    vol.grid_max = mx;
                    vol_has_grid = true;
                } else {
                    vol.dims[0] = vol.dims[1] = vol.dims[2] = 0;
                }
            }
            const bool present = vol.density > 0.0f || vol_has_grid;
            const bool boundary = present && !m.surface;
            emit_mesh(S, A, verts, tris, tn, has_tn, m.smooth != 0, m.base_color, m.metallic, m.roughness, m.emission,
                      m.transmission, m.ior, boundary, vol, vol_has_grid, grid);
        }
        std::vector<NativeLight> native;
        for (int li = 0; li < d.num_lights; ++li) native.push_back(light_from_desc(d.lights[li]));
        finish_scene(S, A, native, d.environment);
    } catch (const std::exception& e) {
        err = std::string("malformed scene arrays: ") + e.what();
        return false;
    }
    return true;
}

unsigned char prim_shading_class(const DevMaterial& dm) {
    const float rough = dm.rough_trans_ior_flags.x, trans = dm.rough_trans_ior_flags.y, metal = dm.albedo_metallic.w;
    return dm.emission.w != 0.0f ? 1 : trans > 0.5f ? 2 : (metal > 0.5f && rough < 0.05f) ? 3 : (metal > 0.5f ? 4 : 5);
}

bool apply_scene_edits(HostScene& S, const LucidSceneEdit* e, int n, std::string& err) {
    if (n < 0 || (n > 0 && !e)) { err = "scene edit: bad edit list"; return false; }
    // check every edit first: all or none
    for (int i = 0; i < n; ++i) {
        const LucidSceneEdit& x = e[i];
        if (x.kind == LUCID_EDIT_MATERIAL) {
            if (x.index < 0 || x.index >= (int)S.materials.size()) {
                err = "scene edit: no mesh " + std::to_string(x.index);
                return false;
            }
            int fl;
            std::memcpy(&fl, &S.materials[x.index].rough_trans_ior_flags.w, 4);
            if (fl & MAT_TEXTURED) {
                err = "scene edit: mesh " + std::to_string(x.index) + " has a textured node-graph material";
                return false;
            }
            if (((fl & MAT_EMISSIVE) != 0) != is_emissive(x.emission)) {
                err = "scene edit: mesh " + std::to_string(x.index) +
                      " would start or stop emitting, which changes the light list; reload the scene";
                return false;
            }
        } else if (x.kind == LUCID_EDIT_LIGHT) {
            if (x.index < 0 || x.index >= S.num_native) {
                err = "scene edit: no native light " + std::to_string(x.index);
                return false;
            }
        } else {
            err = "scene edit: unknown kind " + std::to_string(x.kind);
            return false;
        }
    }
    for (int i = 0; i < n; ++i) {
        const LucidSceneEdit& x = e[i];
        if (x.kind == LUCID_EDIT_MATERIAL) {
            DevMaterial& dm = S.materials[x.index];
            int fl;
            std::memcpy(&fl, &dm.rough_trans_ior_flags.w, 4);
            DevMaterial nd = make_material(x.base_color, x.metallic, x.roughness, x.emission, x.transmission, x.ior,
                                           (fl & MAT_BOUNDARY_ONLY) != 0, false);
            nd.program = dm.program;
            dm = nd;
            if (fl & MAT_EMISSIVE)   // the mesh's emissive-triangle lights carry its emission
                for (size_t p = 0; p < S.prim_info.size(); ++p)
                    if (S.prim_info[p].x == x.index && S.prim_info[p].z >= 0) {
                        float4& er = S.lights[S.prim_info[p].z].emission_radius;
                        er.x = x.emission[0]; er.y = x.emission[1]; er.z = x.emission[2];
                    }
        } else {
            S.lights[S.native_start + x.index] = pack_native(light_from_desc(x.light));
        }
    }
    light_cdf(S);
    return true;
}

namespace {
template <class T>
uint64_t fnv_bytes(const T* p, size_t n, uint64_t h) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n * sizeof(T); ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}
template <class T>
uint64_t fnv_vec(const std::vector<T>& v, uint64_t h) { return fnv_bytes(v.data(), v.size(), h); }
}  // namespace

uint64_t scene_digest(const HostScene& S) {
    uint64_t h = 1469598103934665603ull;
    const int counts[6] = {S.num_meshes, S.num_prims, S.native_start, S.num_native, S.num_boundary_meshes, 0};
    h = fnv_bytes(counts, 6, h);
    h = fnv_bytes(S.env, 3, h);
    h = fnv_bytes(&S.total_light_area, 1, h);
    h = fnv_vec(S.tri, h); h = fnv_vec(S.verts, h); h = fnv_vec(S.prim_info, h); h = fnv_vec(S.prim_fn, h);
    h = fnv_vec(S.prim_vn, h); h = fnv_vec(S.prim_boundary, h); h = fnv_vec(S.materials, h); h = fnv_vec(S.lights, h);
    h = fnv_vec(S.cdf, h); h = fnv_vec(S.light_guide, h); h = fnv_vec(S.volumes, h); h = fnv_vec(S.grid, h);
    h = fnv_vec(S.tex_ops, h); h = fnv_vec(S.prim_uv, h);
    return h;
}

void make_camera(HostCamera& c, float px, float py, float pz, float dx, float dy, float dz, float ux, float uy,
                 float uz, float fov_deg) {
    c.pos[0] = px; c.pos[1] = py; c.pos[2] = pz;
    F3 dir = dir_or(F3{dx, dy, dz}, F3{0, 0, -1});
    F3 up = dir_or(F3{ux, uy, uz}, F3{0, 1, 0});
    c.fov = fov_deg * (3.14159274101257324219f / 180.0f);
    F3 right = dir_or(cross3(dir, up), F3{1, 0, 0});
    F3 upc = dir_or(cross3(right, dir), F3{0, 1, 0});
    c.forward[0] = dir.x; c.forward[1] = dir.y; c.forward[2] = dir.z;
    c.right[0] = right.x; c.right[1] = right.y; c.right[2] = right.z;
    c.up[0] = upc.x; c.up[1] = upc.y; c.up[2] = upc.z;
}

std::vector<float4> native_light_bounds(const HostScene& S) {
    std::vector<float4> out((size_t)std::max(0, S.num_native));
    for (int i = 0; i < S.num_native; ++i) {
        const DevLight& L = S.lights[(size_t)(S.native_start + i)];
        int type;
        std::memcpy(&type, &L.pos_type.w, 4);
        float r = -1.0f;
        if (type == LIGHT_POINT && L.emission_radius.w > 1e-6f) {   // the device's MIN_LENGTH test
            r = L.emission_radius.w;
        } else if (type == LIGHT_AREA) {
            // circumscribed radius of the rectangle / ellipse, widened by
            // 0.1 % for the rounding of the unit right / up vectors
            const double hx = 0.5 * (double)L.right_sx.w, hy = 0.5 * (double)L.up_sy.w;
            r = (float)(std::sqrt(hx * hx + hy * hy) * 1.001);
        }
        out[(size_t)i] = make_float4(L.pos_type.x, L.pos_type.y, L.pos_type.z, r);
    }
    return out;
}

}  // namespace lucid
