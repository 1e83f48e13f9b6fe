/*
 * lucid_cuda.h — C ABI of the B200 (sm_100a) wavefront path tracer.
 *
 * This is the drop-in boundary for the Lucid renderer's progressive render
 * entry point.  Each entry point replaces one method of the reference's
 * PyRenderer façade (LucidRenderer/cpp_renderer/include/pybind_renderer.hpp),
 * which the pybind11 module (src/pybind_module.cpp) exposes to Blender.  All
 * signatures use plain C types, caller-owned host buffers and integer status
 * codes; no C++ type or exception crosses the boundary.
 *
 * Threading: a context may be used from one thread at a time, except
 * lucid_cuda_cancel(), which may be called from any thread (the reference's
 * std::atomic cancel flag, pybind_renderer.hpp:86-102).
 */
#ifndef LUCID_CUDA_H
#define LUCID_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports scene-load failure as `false` and
 * silently returns zero buffers otherwise (pybind_renderer.hpp:121-125,
 * 200-203); this ABI returns explicit codes instead and never falls back to
 * a CPU path. */
#define LUCID_OK 0
#define LUCID_ERR_NO_SCENE (-1)   /* render before load_scene_json / set_camera */
#define LUCID_ERR_OOM (-2)        /* device allocation failed                    */
#define LUCID_ERR_TIMEOUT (-3)    /* a bounded device wait gave up               */
#define LUCID_ERR_CANCELLED (-4)  /* lucid_cuda_cancel() observed; partial image */
#define LUCID_ERR_INVALID (-5)    /* bad argument or malformed scene             */
#define LUCID_ERR_CUDA (-6)       /* CUDA runtime error (see last_error)         */
#define LUCID_ERR_OVERFLOW (-7)   /* a traversal stack or queue bound was hit    */

typedef struct LucidCudaCtx LucidCudaCtx;

/* Render parameters of PyRenderer::render_tile / render_tile_gpu
 * (pybind_renderer.hpp:185-194, 538-547). */
typedef struct LucidRenderParams {
    int tile_x, tile_y, tile_w, tile_h;
    int full_w, full_h;
    int samples;        /* samples in this call (jitter only when > 1) */
    int sample_offset;  /* RNG sample index offset                      */
    int max_depth;
    int flags;          /* LUCID_RENDER_* bits                          */
} LucidRenderParams;

#define LUCID_RENDER_PROFILE 1   /* time every kernel launch (lucid_cuda_get_stats) */

/* One record per (pixel, sample) for parity checking against a CPU
 * implementation of the same integrator.  hash = FNV-1a 64 over the path's
 * event words: per bounce [hit mesh, hit tri, native light] (-1 when absent),
 * [scatter flag] under volume_mis, and [0x5EED0000 | occluded] per shadow
 * ray. */
typedef struct LucidSampleRecord {
    float rgb[3];
    int32_t primary_mesh, primary_tri;
    uint32_t bounces;
    uint32_t nee_tests, nee_occluded;
    uint64_t hash;
} LucidSampleRecord;

/* Per-render statistics (the last render call with LUCID_RENDER_PROFILE). */
#define LUCID_MAX_KERNEL_KINDS 12
typedef struct LucidKernelStat {
    char name[32];
    int launches;
    double total_ms;          /* sum of CUDA-event durations on the render stream */
    double algo_bytes;        /* algorithmic bytes moved by all launches           */
    double units;             /* rays / paths / pixels processed                    */
} LucidKernelStat;

typedef struct LucidRenderStats {
    double total_ms;
    double paths;             /* (pixel, sample) pairs traced          */
    double segments;          /* extension rays traced (path segments) */
    double shadow_rays;
    int waves;
    int num_kinds;
    LucidKernelStat kinds[LUCID_MAX_KERNEL_KINDS];
} LucidRenderStats;

/* ---- context -------------------------------------------------------- */
/* Replaces PyRenderer::PyRenderer (pybind_renderer.hpp:64-76). */
int lucid_cuda_create(int device, LucidCudaCtx** out);
void lucid_cuda_destroy(LucidCudaCtx* ctx);
/* Message of the last failing call on this context ("" when none). */
const char* lucid_cuda_last_error(LucidCudaCtx* ctx);
/* Device name and compute capability, e.g. "NVIDIA B200 (sm_100)". */
int lucid_cuda_device_info(LucidCudaCtx* ctx, char* buf, size_t cap);

/* ---- scene / camera / algorithm ------------------------------------- */
/* Replaces PyRenderer::load_scene_json (pybind_renderer.hpp:111-126) and
 * loadSceneFromJsonString (:1258-1746): parses the JSON scene, builds the
 * light CDF, uploads geometry and builds the device BVH. */
int lucid_cuda_load_scene_json(LucidCudaCtx* ctx, const char* json, size_t len);

/* Binary scene upload: the same scene as loadSceneFromJsonString
 * (pybind_renderer.hpp:1258-1746) given as arrays instead of JSON text, so
 * a host that already holds vertex buffers (Blender's depsgraph export,
 * engine.py) skips formatting and parsing ~150 MB of JSON per million
 * triangles.  A scene described the same way in both forms renders
 * bit-identically.  Each field mirrors the JSON key named beside it; every
 * field is required (the JSON loader's defaults for absent keys are the
 * caller's to fill in). */
typedef struct {
    const float* vertices;          /* "vertices": 3 * num_vertices floats */
    int32_t num_vertices;
    const int32_t* triangles;       /* "triangles": 3 * num_triangles indices */
    int32_t num_triangles;
    const float* triangle_normals;  /* "triangle_normals": 9 * num_triangles floats, or NULL */
    int32_t smooth;                 /* "smooth" */
    float base_color[3];            /* "material": "base_color", "metallic", ... */
    float metallic, roughness;
    float emission[3];
    float transmission, ior;
    int32_t surface;                /* 0: the material's Surface output is unlinked (a volume domain) */
    /* "material"."volume": density > 0 or a grid makes the mesh a medium */
    float volume_density, volume_anisotropy;
    float volume_color[3], volume_absorption[3];
    int32_t volume_dims[3];         /* "smoke_grid": dims (0: no grid), world_min/max, the grid itself */
    float volume_world_min[3], volume_world_max[3];
    const float* volume_grid;       /* dims[0] * dims[1] * dims[2] densities, x fastest, or NULL */
} LucidMeshDesc;

/* One "native_lights" entry (parseNativeLights, pybind_renderer.hpp:1544-1746):
 * energy in W, converted to radiance as the JSON loader does. */
#define LUCID_LIGHT_POINT 1
#define LUCID_LIGHT_SUN 2
#define LUCID_LIGHT_SPOT 3
#define LUCID_LIGHT_AREA 4
#define LUCID_AREA_SQUARE 0
#define LUCID_AREA_RECTANGLE 1
#define LUCID_AREA_DISK 2
#define LUCID_AREA_ELLIPSE 3
typedef struct {
    int32_t type;                   /* LUCID_LIGHT_*; any other value: a light with no area or emission */
    float position[3];
    float direction[3];             /* normalised, (0, 0, -1) when degenerate */
    float color[3];
    float energy;
    float radius;                   /* point and spot */
    float spot_size, spot_blend;    /* spot */
    float size, size_y;             /* area */
    int32_t shape;                  /* area: LUCID_AREA_* */
    float right[3], up[3];          /* area */
} LucidLightDesc;

typedef struct {
    const LucidMeshDesc* meshes;
    int32_t num_meshes;
    const LucidLightDesc* lights;
    int32_t num_lights;
    float environment[3];           /* "environment": color * strength */
} LucidSceneDesc;

/* Loads a scene given as arrays (no counterpart in the reference; the
 * loadSceneFromJsonString semantics above).  Replaces the current scene. */
int lucid_cuda_load_scene_arrays(LucidCudaCtx* ctx, const LucidSceneDesc* scene);

/* Parameter edits of the loaded scene without a re-upload or BVH rebuild.
 * The reference has no such call: every scene change re-exports, re-parses
 * and re-packs the whole scene (PyRenderer keys its packed GPU scene on
 * scene_version_, pybind_renderer.hpp:116, 502-504; the viewport pushes
 * edits through scene_update_pending, LucidRenderer/viewport.py:108-111).
 * An edited scene renders bit-identically to loading the edited scene. */
#define LUCID_EDIT_MATERIAL 1   /* mesh `index` ("meshes" order) gets the material fields below */
#define LUCID_EDIT_LIGHT 2      /* native light `index` ("native_lights" order) becomes `light` */
typedef struct {
    int32_t kind, index;
    /* LUCID_EDIT_MATERIAL: the Principled fields of a LucidMeshDesc */
    float base_color[3], metallic, roughness, emission[3], transmission, ior;
    /* LUCID_EDIT_LIGHT: the whole light, as lucid_cuda_load_scene_arrays takes it */
    LucidLightDesc light;
} LucidSceneEdit;
/* Applies `count` edits in order, all or none: LUCID_ERR_INVALID (nothing
 * changed) when an index is out of range, a material varies over its
 * surface (a node graph with a texture), or an edit would add or remove an
 * emitting mesh (that changes
 * the light list: reload the scene instead).  Renders and jobs started
 * after the call see the edited scene; a context rendering another
 * context's scene (the request loop's slots) keeps the version it took. */
int lucid_cuda_update_scene(LucidCudaCtx* ctx, const LucidSceneEdit* edits, int count);
/* Replaces PyRenderer::set_camera (pybind_renderer.hpp:131-160). */
int lucid_cuda_set_camera(LucidCudaCtx* ctx, float pos_x, float pos_y, float pos_z, float dir_x, float dir_y,
                          float dir_z, float up_x, float up_y, float up_z, float fov_deg);
/* Replaces PyRenderer::set_algorithm (pybind_renderer.hpp:165-167):
 * "simple", "nee", "mis", "volume_simple", "volume_mis" (others act as
 * "nee", as in the reference's dispatch at :296-328). */
int lucid_cuda_set_algorithm(LucidCudaCtx* ctx, const char* name);
/* Scene statistics: meshes, triangles, native lights, scene lights,
 * boundary-only meshes, volumes, BVH nodes, BVH leaves. */
int lucid_cuda_scene_stats(LucidCudaCtx* ctx, int out8[8]);

/* Host-only scene inspection (no GPU needed): parses the JSON exactly as
 * lucid_cuda_load_scene_json does and reports counts (meshes, triangles,
 * native lights, scene lights, boundary-only meshes, volumes, 0, 0) and, for
 * up to `cap` scene lights in SceneLights order (scene_lights.hpp:56-122),
 * the CDF value, area and emission rgb.  Returns the scene light count or a
 * negative status. */
int lucid_cuda_inspect_scene(const char* json, size_t len, int counts8[8], float* cdf, float* area,
                             float* emission_rgb, int cap);
/* Host-only (no GPU needed, no reference counterpart): a 64-bit FNV-1a digest
 * of the device-ready scene that lucid_cuda_load_scene_json (json, len) or
 * lucid_cuda_load_scene_arrays (arrays) would upload: geometry, per-prim
 * normals, materials, lights and their CDF, volumes.  Give exactly one of
 * json and arrays.  Equal digests mean identical uploads (and renders). */
int lucid_scene_digest(const char* json, size_t len, const LucidSceneDesc* arrays, uint64_t* digest);

/* ---- rendering ------------------------------------------------------- */
/* Replaces PyRenderer::render_tile / render_tile_gpu
 * (pybind_renderer.hpp:185-361, 538-666).  out_rgba: host buffer of
 * tile_w*tile_h*4 floats: the SUM over the call's samples of each pixel's
 * radiance, camera sensitivity applied, clamped >= 0, alpha 1, rows
 * Y-flipped; all zeros when the call fails before the image is copied out
 * (no scene or camera, invalid samples / depth, device errors).
 * records (optional, may be NULL): tile_w*tile_h*samples entries
 * in (row-major unflipped pixel, sample) order. */
int lucid_cuda_render(LucidCudaCtx* ctx, const LucidRenderParams* params, float* out_rgba,
                      LucidSampleRecord* records);
/* Same render with the image left in device memory (d_out_rgba: a device
 * pointer of tile_w*tile_h*4 floats); no host copies. */
int lucid_cuda_render_device(LucidCudaCtx* ctx, const LucidRenderParams* params, float* d_out_rgba);
/* Render without allocating any device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc/cudaFree while they
 * render: hosts whose device memory belongs to another allocator, and
 * latency-critical threads (a viewport draw callback) that must not make
 * calls which can synchronise the whole device.  Same result as
 * lucid_cuda_render_device (d_out_rgba: device pointer, tile_w*tile_h*4
 * floats), but all working memory sits in one fixed static device array of
 * about 12 MB that every GPU loading this library holds until exit.
 * Limits: tile_w*tile_h <= 65536 pixels, 1 <= max_depth <= 64, no sample
 * records; larger requests return LUCID_ERR_INVALID.  Path diagnostics and
 * path guiding keep buffers of their own: while either is on for the
 * context, the call returns LUCID_ERR_INVALID.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.
 * Every call on a device shares the array: calls that overlap on the GPU
 * (from several threads or contexts) race and must be serialised by the
 * caller.  The scene must already be loaded (lucid_cuda_load_scene_json
 * allocates). */
int lucid_cuda_render_noalloc(LucidCudaCtx* ctx, const LucidRenderParams* params, float* d_out_rgba);
/* Batched jobs.  No counterpart in the reference: the add-on gives every
 * session its own Renderer and renders each job with its own calls
 * (LucidRenderer/render_session.py:77-106, pybind_renderer.hpp:185-361).
 * Renders n jobs, each on the scene of its own context (`scene`: that
 * context's scene version current at the call; `ctx` may be one of them),
 * with its own camera, tile, image size, samples and sample offset, in one
 * set of wavefront launches over a device job table: the jobs' samples fill
 * waves of up to the context's wave capacity in job order, every path
 * carries its job's scene index, and each kernel launch of a wave serves all
 * its jobs.  Every job's image (out_rgba: host, tile_w*tile_h*4 floats) is
 * bit for bit the lucid_cuda_render of the same params on its own context
 * with that camera and `algorithm`.  All jobs need the same max_depth.  No
 * sample records, path diagnostics or path guiding.  A call that fails or
 * is cancelled (lucid_cuda_cancel on ctx, checked between waves) leaves
 * every job's image zero. */
typedef struct LucidBatchJob {
    LucidCudaCtx* scene;        /* context whose loaded scene the job renders */
    float camera[10];           /* position, direction, up, vertical fov (degrees) */
    LucidRenderParams params;   /* tile, image size, samples, sample_offset, max_depth */
    float* out_rgba;            /* host image, the layout of lucid_cuda_render */
} LucidBatchJob;
int lucid_cuda_render_batch(LucidCudaCtx* ctx, const LucidBatchJob* jobs, int n, const char* algorithm);
/* Concurrent small renders.  The reference gives each Blender session its
 * own Renderer (render_session.py:77-106), so a viewport, several material
 * previews and an F12 render call render_tile at the same time.  Here every
 * context of a device meets in one process-wide combiner: a
 * lucid_cuda_render call of at most 2^22 paths (tile_w * tile_h * samples)
 * with a host image, no sample records, diagnostics or guiding, made while
 * no other such call runs, renders on its own context as before; calls made
 * while one runs wait, and the first of them to find the device free renders
 * all waiting calls with its integrator and max_depth as one batch
 * (lucid_cuda_render_batch), every image unchanged bit for bit.  Larger
 * calls never wait for the combiner.  lucid_cuda_get_stats after a combined
 * call describes its batch (paths: this call's).  On by default;
 * on = 0 takes this context's calls out. */
int lucid_cuda_set_combining(LucidCudaCtx* ctx, int on);
/* Batches the combiner of `device` has run and the render calls in them. */
int lucid_cuda_combine_stats(int device, long long* batches, long long* calls);
/* Replaces PyRenderer::render_debug / render_debug_gpu
 * (pybind_renderer.hpp:371-525): mode "normal", "albedo" or "emission" at
 * the primary hit, no jitter, Y-flipped RGBA. */
int lucid_cuda_render_debug(LucidCudaCtx* ctx, int tile_x, int tile_y, int tile_w, int tile_h, int full_w,
                            int full_h, const char* mode, float* out_rgba);
/* Launch profile of the wavefront kernels for this context's renders
 * (no counterpart in the reference): 0 (default) runs closest-hit, shading
 * and shadow kernels at 9 / 8 / 9 resident CTAs per SM, the measured optimum
 * on large scenes; 1 at 8 / 6 / 8, more registers per thread and fewer
 * spills.  Images are identical under both. */
int lucid_cuda_set_launch_profile(LucidCudaCtx* ctx, int profile);
/* Statistics of the last render (kernel times need LUCID_RENDER_PROFILE). */
int lucid_cuda_get_stats(LucidCudaCtx* ctx, LucidRenderStats* out);
/* Path-pool capacity in paths (0 = automatic).  A render processes
 * samples in waves of at most this many paths. */
int lucid_cuda_set_wave_capacity(LucidCudaCtx* ctx, long long paths);

/* ---- progressive accumulator (viewport) -------------------------------- */
/* Replaces PyRenderer::render_start_async / render_poll_async /
 * render_snapshot_revision_async / render_reset_async / render_stop_async /
 * is_render_async_running (pybind_renderer.hpp:689-856).  A worker thread
 * adds one 1-spp render per iteration (iteration n uses sample offset n)
 * into a device accumulator and publishes an averaged snapshot after 1, 2,
 * 4, 8 and then every 16 samples. */
int lucid_cuda_async_start(LucidCudaCtx* ctx, int width, int height, int max_depth);
/* Latest snapshot: *samples = samples averaged (0 = none yet); out_rgba gets
 * width*height*4 floats (averaged, exposure applied, clamped >= 0, alpha 1,
 * Y-flipped) when *samples > 0. */
int lucid_cuda_async_poll(LucidCudaCtx* ctx, int* samples, float* out_rgba, size_t cap_floats);
/* Monotonic snapshot counter (>= 0). */
int lucid_cuda_async_revision(LucidCudaCtx* ctx);
/* Non-blocking wipe of the accumulator; picks up the current camera.  A
 * larger resolution needs stop + start. */
int lucid_cuda_async_reset(LucidCudaCtx* ctx, int width, int height, int max_depth);
int lucid_cuda_async_stop(LucidCudaCtx* ctx);
/* 1 while the worker runs, else 0. */
int lucid_cuda_async_running(LucidCudaCtx* ctx);

/* ---- converged references ---------------------------------------------- */
/* No reference counterpart (the reference sums in FP32 only).  Renders like
 * lucid_cuda_render but sums each pixel's per-sample FP32 radiance in FP64,
 * in sample order, for the 4096-spp references that relMSE is measured
 * against.  out_rgba: tile_w * tile_h * 4 doubles, clamp >= 0, alpha 1,
 * Y-flipped (the layout of lucid_cuda_render). */
int lucid_cuda_render_f64(LucidCudaCtx* ctx, const LucidRenderParams* params, double* out_rgba);

/* ---- path diagnostics (DiagnosticFilm) ---------------------------------- */
/* PathRecordingConfig (diagnostics/path_stats_config.hpp:24-105).  The film
 * uses subsample_factor; the others are carried for the caller, as in the
 * reference.  record_capacity is the initial size of the device record
 * buffer in completed paths per wave (0 = 1,048,576, with eight 16-byte
 * units per path for their vertices); a wave that produces more grows the
 * buffers and runs again. */
typedef struct LucidDiagConfig {
    int subsample_factor, max_groups_per_pixel, max_outliers_per_pixel, max_depth;
    float variance_threshold, outlier_threshold;
    long long record_capacity;
} LucidDiagConfig;

/* GlobalDiagnosticStats (diagnostic_film.hpp:124-154) + paths recorded. */
typedef struct LucidDiagStats {
    uint64_t total_samples, active_pixels, total_groups, total_overflow, paths_recorded;
} LucidDiagStats;

/* PixelDiagnosticInfo (pybind_renderer.hpp:971-981). */
typedef struct LucidDiagPixel {
    int32_t valid;
    uint32_t sample_count, group_count, outlier_count, overflow_count;
    float variance;
    float mean_rgb[3];
} LucidDiagPixel;

/* One path group (PathGroup, path_stats.hpp:142-232): hash, Welford stats,
 * vertex list (object id: mesh index, -1 environment, -(light+2) lights),
 * BSDF class and flags per vertex, representative positions and normals. */
typedef struct LucidDiagGroup {
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
} LucidDiagGroup;

/* Replaces PyRenderer::enable_diagnostics / disable_diagnostics /
 * is_diagnostics_enabled / clear_diagnostics (pybind_renderer.hpp:893-937).
 * While enabled, lucid_cuda_render uses the diagnostic integrators
 * (path_tracer.hpp:880-1514: "simple", "mis", everything else as "nee") and
 * rebuilds the film for each call.  config may be NULL (standard preset). */
int lucid_cuda_diag_enable(LucidCudaCtx* ctx, const LucidDiagConfig* config);
int lucid_cuda_diag_disable(LucidCudaCtx* ctx);
int lucid_cuda_diag_enabled(LucidCudaCtx* ctx);
int lucid_cuda_diag_clear(LucidCudaCtx* ctx);
/* get_diagnostic_stats (pybind_renderer.hpp:939-946). */
int lucid_cuda_diag_stats(LucidCudaCtx* ctx, LucidDiagStats* out);
/* get_pixel_diagnostic (pybind_renderer.hpp:1008-1102): tile-local pixel
 * (x, y); the cell's groups are sorted in place by variance (or by mean
 * luminance when sort_by_mean) and up to cap are copied; returns the number
 * copied. */
int lucid_cuda_diag_pixel(LucidCudaCtx* ctx, int x, int y, int sort_by_mean, LucidDiagPixel* info,
                          LucidDiagGroup* groups, int cap);
/* get_diagnostic_variance_map (pybind_renderer.hpp:952-972): film width *
 * height floats; returns the number written. */
int lucid_cuda_diag_variance_map(LucidCudaCtx* ctx, float* out, size_t cap);
/* get_top_variance_groups / top mean groups (diagnostic_film.hpp:160-222,
 * diagnostic_export.hpp:94-105): the n groups of the whole film with the
 * largest variance (groups with >= 2 samples) or mean luminance (>= 1),
 * with the film position (x, y) of their cell in xy[2 * i].  Returns the
 * number copied. */
int lucid_cuda_diag_top_groups(LucidCudaCtx* ctx, int n, int by_mean, LucidDiagGroup* groups, int32_t* xy, int cap);

/* DiagnosticExporter (diagnostics/diagnostic_export.hpp:78-220) over the
 * current diagnostic film. */
/* ExportedCoarseStats: one of the eight coarse path types aggregated over the
 * film the way get_coarse_stats does it (:110-157, sample-weighted means,
 * largest per-cell variance, cells read at (2 sx, 2 sy) as the reference
 * reads them). */
typedef struct LucidDiagCoarse {
    int32_t type_id;
    char name[32];
    uint64_t sample_count;
    float mean_luminance, variance_luminance;
    float mean_rgb[3], variance_rgb[3];
} LucidDiagCoarse;
/* DiagnosticSuggestion (:62-72, generate_suggestions :178-248). */
typedef struct LucidDiagSuggestion {
    char category[16];
    char severity[16];
    char message[128];
    char action[128];
} LucidDiagSuggestion;
/* Writes the eight coarse types (out[8]); returns 8. */
int lucid_cuda_diag_coarse_stats(LucidCudaCtx* ctx, LucidDiagCoarse* out);
/* Writes up to cap suggestions; returns how many there are. */
int lucid_cuda_diag_suggestions(LucidCudaCtx* ctx, LucidDiagSuggestion* out, int cap);
/* export_binary (diagnostic_film.hpp:243-299): the "PVAR" blob.  Copies
 * min(size, cap) bytes and returns its size (out may be NULL to ask). */
long long lucid_cuda_diag_export_binary(LucidCudaCtx* ctx, uint8_t* out, size_t cap);
/* metadata_json (diagnostic_film.hpp:228-241): copies the text (NUL-
 * terminated when it fits) and returns its length. */
long long lucid_cuda_diag_metadata_json(LucidCudaCtx* ctx, char* out, size_t cap);

/* ---- standalone diagnostic films (host only, no device) ---------------- */
/* The reference module's DiagnosticFilm / DiagnosticPathTracer /
 * DiagnosticExporter / PathTrace / PathDiagnosticRecorder classes
 * (src/pybind_module.cpp:433-539): a film built by the caller and fed one
 * completed path at a time, as the add-on's DiagnosticsManager does
 * (LucidRenderer/diagnostics.py:111-330).  These calls need no GPU. */
typedef struct LucidDiagFilm LucidDiagFilm;
/* PathVertex (diagnostics/path_types.hpp:195-246): object id (mesh index,
 * -1 environment, -(light + 2) a light), material id, BsdfType (0 Diffuse,
 * 1 Glossy, 2 Mirror, 3 Glass, 4 Emission, 5 Environment), flags (1 delta,
 * 2 light sampled). */
typedef struct LucidPathVertex {
    int32_t object_id;
    int16_t material_id;
    uint8_t bsdf_type, flags;
} LucidPathVertex;
/* PathTrace (path_types.hpp:249-257): up to 16 vertices with positions and
 * normals, the contribution, LightSourceType (0 Unknown, 1 Point, 2 Area,
 * 3 Directional, 4 Spot, 5 Environment, 6 Emissive) and SamplingStrategy
 * (0 BSDF, 1 NEE, 2 MIS_BSDF, 3 MIS_NEE). */
typedef struct LucidPathTrace {
    LucidPathVertex vertices[16];
    float positions[16][3];
    float normals[16][3];
    uint32_t depth;
    float contribution[3];
    uint8_t light_type, strategy, pad[2];
} LucidPathTrace;
/* DiagnosticFilm(width, height, config) (diagnostic_film.hpp:66-75);
 * config may be NULL (standard preset).  Free with lucid_diag_film_destroy. */
int lucid_diag_film_create(long long width, long long height, const LucidDiagConfig* config, LucidDiagFilm** out);
void lucid_diag_film_destroy(LucidDiagFilm* film);
/* DiagnosticFilm::record_path (diagnostic_film.hpp:94-106): pixel (x, y) of
 * the film (cells of subsample_factor^2 pixels; pixels outside are ignored). */
int lucid_diag_film_record_path(LucidDiagFilm* film, long long x, long long y, const LucidPathTrace* trace);
/* DiagnosticFilm::clear (:308-313). */
int lucid_diag_film_clear(LucidDiagFilm* film);
/* width, height, sampled_width, sampled_height, total_paths_recorded
 * (diagnostic_film.hpp:80-113) into out[5]. */
int lucid_diag_film_info(LucidDiagFilm* film, long long* out5);
/* global_stats (:130-154) + paths recorded. */
int lucid_diag_film_stats(LucidDiagFilm* film, LucidDiagStats* out);
/* PixelPathData of film pixel (x, y), groups sorted by variance (or mean
 * luminance), as lucid_cuda_diag_pixel. */
int lucid_diag_film_pixel(LucidDiagFilm* film, long long x, long long y, int sort_by_mean, LucidDiagPixel* info,
                          LucidDiagGroup* groups, int cap);
/* DiagnosticExporter over the film (diagnostic_export.hpp:78-220), as the
 * lucid_cuda_diag_* exporter calls over a renderer's film. */
int lucid_diag_film_top_groups(LucidDiagFilm* film, int n, int by_mean, LucidDiagGroup* groups, int32_t* xy, int cap);
int lucid_diag_film_coarse_stats(LucidDiagFilm* film, LucidDiagCoarse* out);
int lucid_diag_film_suggestions(LucidDiagFilm* film, LucidDiagSuggestion* out, int cap);
long long lucid_diag_film_export_binary(LucidDiagFilm* film, uint8_t* out, size_t cap);
long long lucid_diag_film_metadata_json(LucidDiagFilm* film, char* out, size_t cap);
/* PathTrace::hash and coarse_type (path_types.hpp:321-372). */
uint64_t lucid_path_trace_hash(const LucidPathTrace* trace);
int lucid_path_trace_coarse_type(const LucidPathTrace* trace);

/* ---- request loop (several jobs on one device) ------------------------- */
/* No reference counterpart: the reference runs one Renderer per Blender
 * session (viewport, F12 render, material preview; render_session.py:77-106),
 * each rendering on its own.  Here those sessions submit jobs to one server:
 * jobs are admitted in arrival order as slots and device memory free up,
 * run concurrently on per-slot CUDA streams, and each job's image is the
 * same, bit for bit, as one lucid_cuda_render call with all its samples. */
typedef struct LucidServer LucidServer;

typedef struct LucidJobDesc {
    int scene;            /* id returned by lucid_server_add_scene */
    float camera[10];     /* position, direction, up, vertical fov (degrees) */
    char algorithm[16];   /* "simple", "nee", "mis", "volume_simple", "volume_mis" */
    int width, height, samples, max_depth;
    int interactive;      /* 1: keep each iteration short (viewport); 0: throughput */
    int guided;           /* 1: "mis" with online path guiding (lucid_cuda_guide_enable), trained per job */
    int guide_seed;       /* the guide network's initialisation seed */
} LucidJobDesc;

enum { LUCID_JOB_QUEUED = 0, LUCID_JOB_RUNNING = 1, LUCID_JOB_DONE = 2, LUCID_JOB_REFUSED = 3,
       LUCID_JOB_FAILED = 4, LUCID_JOB_CANCELLED = 5 };

typedef struct LucidServerStats {
    int submitted, done, refused, running, queued;
    double latency_p50_ms, latency_p99_ms;   /* submit -> image ready, finished jobs */
    double first_p50_ms, first_p99_ms;       /* submit -> first iteration finished */
    double samples_per_s;                    /* samples of finished jobs / busy wall time */
    long long bytes_reserved, bytes_running, budget_bytes;
    int batches, batched_jobs;               /* batches run (lucid_server_set_batching) and the jobs in them */
} LucidServerStats;

/* slots: concurrent jobs; budget_bytes: device memory the jobs may use
 * (0 = 70 % of the free memory; slots keep their path pools between jobs
 * outside this budget). */
int lucid_server_create(int device, int slots, long long budget_bytes, LucidServer** out);
void lucid_server_destroy(LucidServer* srv);
const char* lucid_server_last_error(LucidServer* srv);
/* Parses, uploads and builds the BVH once; jobs name the scene by its id. */
int lucid_server_add_scene(LucidServer* srv, const char* json, size_t len, int* scene_id);
/* The same from arrays (lucid_cuda_load_scene_arrays). */
int lucid_server_add_scene_arrays(LucidServer* srv, const LucidSceneDesc* scene, int* scene_id);
/* lucid_cuda_update_scene on a server scene: jobs submitted after the call
 * render the edited scene; jobs already queued or running keep the version
 * they were submitted with. */
int lucid_server_update_scene(LucidServer* srv, int scene_id, const LucidSceneEdit* edits, int count);
/* Queues a job (LUCID_ERR_OOM and state REFUSED when it can never fit). */
int lucid_server_submit(LucidServer* srv, const LucidJobDesc* job, int* job_id);
/* Returns the job's LUCID_JOB_* state; samples_done may be NULL. */
int lucid_server_job_state(LucidServer* srv, int job_id, int* samples_done);
/* Waits until the job has finished (or timeout_ms, < 0 = no limit): returns its state. */
int lucid_server_wait(LucidServer* srv, int job_id, int timeout_ms);
/* The finished image: width * height * 4 floats, sum over samples, Y-flipped
 * (the layout of lucid_cuda_render). */
int lucid_server_result(LucidServer* srv, int job_id, float* out_rgba, size_t cap_floats);
int lucid_server_cancel(LucidServer* srv, int job_id);
int lucid_server_stats(LucidServer* srv, LucidServerStats* out);
/* Batched throughput jobs (no counterpart in the reference).  Jobs that are
 * neither interactive nor guided and wait in the queue together with the
 * same algorithm and max_depth run as one batch (lucid_cuda_render_batch:
 * one set of wavefront launches over a device job table) of at most
 * max_paths paths (width * height * samples summed over the batch; default
 * 2^25); a job of max_paths paths or more runs on its own.  A batch's jobs
 * finish together, each image unchanged.  0 turns batching off. */
int lucid_server_set_batching(LucidServer* srv, long long max_paths);
/* The server's batching policy on its own (host only, no GPU; no
 * counterpart in the reference): jobs[0] is the job a slot takes from the
 * head of the queue, jobs[1..n-1] the jobs waiting behind it in queue order,
 * cancelled[i] (may be NULL) marks jobs cancelled while queued, room_bytes
 * is the device-memory budget left.  member[i] = 1 for every job of the
 * batch the head forms (member[0] = 1 when one forms); returns the number of
 * jobs the head runs with (1: alone) or a negative status. */
int lucid_batch_plan(long long max_paths, long long room_bytes, const LucidJobDesc* jobs, const int* cancelled, int n,
                     int* member);
/* The server's admission policy on its own (host only, no GPU): n jobs of
 * job_bytes[i] arrive in order; decision[i] = the start order of job i
 * (0, 1, ...) when jobs finish in start order, or -1 when it is refused. */
int lucid_admission_plan(long long budget, long long reserved, int slots, const long long* job_bytes, int n,
                         int* decision);

/* ---- path-guiding network ------------------------------------------------ */
/* No reference counterpart.  The guide of the `mis` integrator (see
 * lucid_cuda_guide_enable) on its own: an MLP from 176 encoded inputs
 * (position in [0,1]^3 of the scene box: sin/cos of pi 2^j x, j < 16, per
 * axis; normal; one-blob(32) of (cos theta + 1)/2 and phi/(2 pi) + 1/2 of the
 * outgoing direction; zero padding) through three 64-wide ReLU layers to 48
 * raw outputs (8 lobe logits, 8 softplus concentrations, 8 x 3 mean
 * directions, padding), BF16 on the tensor cores with FP32 accumulation and
 * FP32 master weights.  Parameter layout: W1[64][176] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[48][64] b4[48].  A training record is 16 floats:
 * position01[3], normal[3], wo[3], wi[3], pdf, radiance[3]; the loss is
 * -sum_s c_s log q(wi_s) with c_s proportional to luminance / pdf, summing
 * to 1 over the batch. */
typedef struct LucidGuide LucidGuide;
int lucid_guide_create(int device, int seed, LucidGuide** out);
void lucid_guide_destroy(LucidGuide* guide);
const char* lucid_guide_last_error(LucidGuide* guide);
int lucid_guide_num_params(void);
int lucid_guide_get_params(LucidGuide* guide, float* out, size_t cap);
int lucid_guide_set_params(LucidGuide* guide, const float* params, size_t n);
/* n x 176 inputs -> n x 48 raw outputs */
int lucid_guide_forward(LucidGuide* guide, const float* inputs, int n, float* outputs);
/* n (position01, normal, wo) triples -> n x 176 inputs */
int lucid_guide_encode(LucidGuide* guide, const float* p01, const float* normal, const float* wo, int n,
                       float* out);
/* loss gradient of n records (parameter layout above); the network is unchanged */
int lucid_guide_gradient(LucidGuide* guide, const float* records, int n, float* grad_out);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8) on n records */
int lucid_guide_train(LucidGuide* guide, const float* records, int n, float lr);

/* Online path guiding for the `mis` integrator (no reference counterpart):
 * while on, every render call samples guidable surfaces (no transmission,
 * not near-delta metal) from the BSDF or from the guide network with
 * probability 1/2 each, weighted by the balance heuristic (NEE's MIS weight
 * uses the same mixed pdf), records the guided vertices with the radiance
 * that arrives along their samples, and takes Adam steps (lr 1e-2, up to
 * 2^18 records each) after each wave.  The estimator stays unbiased; its noise
 * changes.  Enabling (re)initialises the network from `seed`. */
int lucid_cuda_guide_enable(LucidCudaCtx* ctx, int on, int seed);
/* Training steps taken since the network was initialised. */
int lucid_cuda_guide_steps(LucidCudaCtx* ctx);
/* Adam steps per wave (1..64, each on up to 2^18 records; default 2) and
 * the learning rate (default 1e-2). */
int lucid_cuda_guide_config(LucidCudaCtx* ctx, int steps_per_wave, float lr);
/* Guided vertices: those at path depth < max_depth (1..1024; default 1, the
 * camera-ray hits only, which gave the best error at equal time on the
 * hard-indirect test room); deeper vertices sample the BSDF as without
 * guiding but still credit radiance to the guided vertices before them. */
int lucid_cuda_guide_max_depth(LucidCudaCtx* ctx, int max_depth);
/* The context's guide network as trained so far: its FP32 master weights
 * (out: cap >= lucid_guide_num_params() floats, the layout lucid_guide_*
 * uses) and the scene box its position encoding maps to [0,1]^3 (box6: lo
 * x y z, hi x y z; may be NULL).  Returns the number of weights copied. */
int lucid_cuda_guide_params(LucidCudaCtx* ctx, float* out, size_t cap, float* box6);

/* ---- cancellation ---------------------------------------------------- */
/* Replaces PyRenderer::cancel / is_cancelled / reset_cancel
 * (pybind_renderer.hpp:86-102).  Thread-safe. */
int lucid_cuda_cancel(LucidCudaCtx* ctx);
int lucid_cuda_is_cancelled(LucidCudaCtx* ctx);
int lucid_cuda_reset_cancel(LucidCudaCtx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* LUCID_CUDA_H */
