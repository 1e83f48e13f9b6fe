// lucid_types.h — POD layouts shared by the host engine and the CUDA kernels.
// Every device array is 16-byte aligned and read with float4/int4 loads.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector_types.h>   // float4 / int4 (CUDA's aligned vector structs)

namespace lucid {

enum LightTypeId { LIGHT_EMISSIVE = 0, LIGHT_POINT = 1, LIGHT_SUN = 2, LIGHT_SPOT = 3, LIGHT_AREA = 4 };
enum AreaShapeId { AREA_SQUARE = 0, AREA_RECTANGLE = 1, AREA_DISK = 2, AREA_ELLIPSE = 3 };
constexpr int kLightGuide = 1024;
enum AlgoId { ALGO_SIMPLE = 0, ALGO_NEE = 1, ALGO_MIS = 2, ALGO_VOLUME_SIMPLE = 3, ALGO_VOLUME_MIS = 4 };

// One scene light in SceneLights order (emissive triangles, then native
// lights) — the fields of the reference's Light (light/light.hpp:43-90)
// packed into eight float4s (128 B).
struct alignas(16) DevLight {
    float4 pos_type;         // position xyz, type (int bits)
    float4 normal_area;      // normal xyz, area (1 m^2 substituted for point-like lights)
    float4 emission_radius;  // emission rgb, radius
    float4 v0_shape;         // emissive-triangle v0 xyz, area-light shape (int bits)
    float4 v1_cosc;          // v1 xyz, spot cos(angle/2)
    float4 v2_blend;         // v2 xyz, spot blend
    float4 right_sx;         // area right xyz, size_x
    float4 up_sy;            // area up xyz, size_y
};
static_assert(sizeof(DevLight) == 128, "DevLight layout");

// Per-mesh material (material.hpp:207-242), constant-folded.
struct alignas(16) DevMaterial {
    float4 albedo_metallic;        // albedo rgb, metallic
    float4 rough_trans_ior_flags;  // roughness, transmission, ior, flags (int bits)
    float4 emission;               // emission rgb, emissive flag
    int4 program;                  // node programs: albedo start, steps, emission start, steps (0: constant)
};
enum MaterialFlags { MAT_EMISSIVE = 1, MAT_BOUNDARY_ONLY = 2, MAT_TEXTURED = 4 };
// Steps of a material node program (two float4 each: {kind, operand a,
// operand b, k}, {rgb, 0}; operands index earlier steps of the program).
enum TexOpKind { TEX_CONST = 0, TEX_CHECKER = 1, TEX_MIX = 2, TEX_SCALE = 3 };
constexpr int kTexMaxOps = 24;   // steps in one material program

// A participating medium with a dense grid (material.hpp:149-188).
struct DevVolume {
    float wmin[3], wmax[3];
    int dims[3];
    float density, anisotropy, grid_max;
    float color[3], absorption[3];
    long long grid_offset;
};

// Flattened BVH2 node: both children's boxes inline (64 B).  A child index
// >= 0 is an internal node; < 0 encodes a leaf ~((start << 3) | (count - 1))
// over the BVH-ordered triangle array.
struct alignas(16) DevNode {
    float4 lmin_lc;   // left box min xyz, left child (int bits)
    float4 lmax_rc;   // left box max xyz, right child (int bits)
    float4 rmin;      // right box min xyz
    float4 rmax;      // right box max xyz
};

// 4-wide BVH node (128 B): the four children's boxes as x/y/z min/max lanes
// and their codes (>= 0 node index, < 0 leaf ~(start << 3 | count - 1),
// kEmptyChild for an unused slot).
struct alignas(16) DevNode4 {
    float4 xmin, xmax, ymin, ymax, zmin, zmax;
    int4 child;
    int4 pad;
};
constexpr int kEmptyChild = 0x7fffffff;

struct DevScene {
    // geometry in BVH order: 3 float4 per triangle (v0 | prim id, e1, e2)
    const float4* bvh_tris;
    const DevNode4* nodes;    // 4-wide tree (any-hit queries), root `root`
    const DevNode* nodes2;    // binary tree (closest-hit queries), root `root2`
    int root2;
    int num_bvh_tris;
    int root;                       // root child code (node index or leaf code)
    // boundary-only triangles (tested by brute force): 3 float4 each, in
    // groups of one mesh each with a padded bounding box (2 float4 per
    // group: min xyz | first triangle, max xyz | triangle count)
    const float4* bnd_tris;
    int num_bnd_tris;
    const float4* bnd_box;
    int num_bnd_groups;
    // the few triangles whose bounds span a large part of the scene (ground
    // planes, walls) are kept out of the BVH and tested first by brute force:
    // in a Morton-ordered hierarchy they would inflate every box on their
    // root path
    const float4* big_tris;
    int num_big_tris;
    // per global prim (mesh-major order)
    const int4* prim_info;          // mesh, local tri, light index (-1), smooth flag
    const unsigned char* prim_cls;  // shading class of a surface hit on the prim (1..5)
    const float4* prim_fn;          // face normal
    const float4* prim_vn;          // 3 vertex normals per prim (smooth prims)
    const DevMaterial* materials;   // per mesh
    const float4* tex_ops;          // node program steps (two float4 each)
    const float4* prim_uv;          // 2 per prim: (uv0, uv1), (uv2, has uv, 0); null without UVs
    // lights
    const DevLight* lights;
    const float* light_cdf;
    // guide[k] = lower_bound(cdf, k / kLightGuide) for k = 0..kLightGuide:
    // brackets std::lower_bound(cdf, u) for u in [k, k+1) / kLightGuide
    const int* light_guide;
    int num_lights;
    int native_start;
    int num_native;
    const float4* light_bsph;       // per native light: bounding sphere (radius < 0: never hit by rays)
    float total_light_area;
    // environment
    float env[3];
    // volumes
    const DevVolume* volumes;
    int num_volumes;
    const float* grid;
    int has_boundary;
    // scene box -> shading-bin cells (the spatial part of the shading sort)
    float bin_lo[3], bin_scale[3];
    // the largest coordinate magnitude of the scene (the BVH boxes' padding
    // is 2^-20 of it): rays starting within it may use the FMA slab test
    float coord_bound;
};

}  // namespace lucid
