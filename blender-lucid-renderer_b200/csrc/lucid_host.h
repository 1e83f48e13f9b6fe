// lucid_host.h — host-side scene and camera of the CUDA engine.
#pragma once

#include <array>
#include <string>
#include <vector>

#include "lucid_types.h"
#include "../../include/lucid_cuda.h"

namespace lucid {

// Flattened scene ready for upload.  Triangles are numbered globally in
// mesh-major order ("prim id"), which is also the reference's hit-order
// tie-break (later mesh wins on equal distance, geometry/bvh.hpp:167-174).
struct HostScene {
    int num_meshes = 0;
    int num_prims = 0;
    // per prim
    std::vector<float4> tri;        // 3 per prim: v0 | prim id bits, e1 = v1 - v0, e2 = v2 - v0
    std::vector<float4> verts;      // 3 per prim: v0, v1, v2 (bounds for the BVH build)
    std::vector<int4> prim_info;    // mesh, local tri, light index, smooth
    std::vector<float4> prim_fn;    // face normal
    std::vector<float4> prim_vn;    // 3 per prim: vertex normals
    std::vector<unsigned char> prim_boundary;
    std::vector<DevMaterial> materials;
    std::vector<float4> tex_ops;    // node program steps of textured materials
    std::vector<float4> prim_uv;    // 2 per prim when any mesh has UVs, else empty
    std::vector<DevLight> lights;
    std::vector<float> cdf;
    std::vector<int> light_guide;   // kLightGuide + 1 entries
    float total_light_area = 0.0f;
    int native_start = 0;
    int num_native = 0;
    std::vector<DevVolume> volumes;
    std::vector<float> grid;
    float env[3] = {0.05f, 0.05f, 0.05f};
    int num_boundary_meshes = 0;
};

// Parses the reference's scene JSON (pybind_renderer.hpp:1258-1746).
// Returns false and sets err on malformed input.
bool parse_scene_json(const char* json, size_t len, HostScene& out, std::string& err);
// The same scene from arrays (lucid_cuda_load_scene_arrays).
bool build_scene_arrays(const LucidSceneDesc& desc, HostScene& out, std::string& err);
// FNV-1a 64 over every uploaded array and count of a flattened scene.
uint64_t scene_digest(const HostScene& s);
// Parameter edits of a flattened scene (lucid_cuda_update_scene), all or
// none: materials and native lights, no geometry.  False (err set, scene
// unchanged) for an index out of range, a material that varies over its
// surface (a textured node graph), or an edit that would add or remove an
// emitting mesh.
bool apply_scene_edits(HostScene& s, const LucidSceneEdit* edits, int count, std::string& err);
// The shading class of a surface hit on a prim with this material (the
// material part of the shading-queue bins): 1 emitter, 2 glass, 3 near-delta
// metal, 4 metal, 5 other.
unsigned char prim_shading_class(const DevMaterial& dm);
// Bounding spheres of the native lights a ray can hit (centre, radius; a
// negative radius for lights the camera-side intersection skips: spot, sun
// and point lights without a radius), one per native light: the cheap
// rejection before the exact native-light tests.
std::vector<float4> native_light_bounds(const HostScene& s);

struct HostCamera {
    float pos[3] = {0, 0, 0};
    float forward[3] = {0, 0, 1};
    float right[3] = {1, 0, 0};
    float up[3] = {0, 1, 0};
    float fov = 1.04719758f;   // 60 degrees (ray.hpp:54)
};
// PyRenderer::set_camera (pybind_renderer.hpp:131-160).
void make_camera(HostCamera& c, float px, float py, float pz, float dx, float dy, float dz, float ux, float uy,
                 float uz, float fov_deg);

}  // namespace lucid
