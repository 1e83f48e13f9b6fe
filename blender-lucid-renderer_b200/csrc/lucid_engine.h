// lucid_engine.h — host orchestration of the wavefront path tracer.
#pragma once

#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lucid_cuda.h"
#include "lucid_diag.h"
#include "lucid_host.h"
#include "lucid_types.h"

namespace lucid {

struct DeviceScene;   // device allocations of one uploaded scene
struct PathPool;      // wavefront SoA path state
struct DiagDevice;    // device record buffer of the path diagnostics
struct JobState;      // progressive job (film, captured iteration graph)
struct GuideState;    // path-guiding network and its per-path buffers

// One version of an uploaded scene, as other engines share it: the device
// scene and the counts and bounds that go with it.
struct SceneSnapshot {
    std::shared_ptr<DeviceScene> ds;
    int stats[8] = {};
    float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
};

class Engine {
public:
    explicit Engine(int device);
    ~Engine();

    int load_scene_json(const char* json, size_t len);
    int load_scene_arrays(const LucidSceneDesc& desc);
    int set_camera(float px, float py, float pz, float dx, float dy, float dz, float ux, float uy, float uz,
                   float fov_deg);
    int set_algorithm(const char* name);
    int render(const LucidRenderParams& p, float* out_host, LucidSampleRecord* recs, float* out_device);
    // Converged references: the per-pixel sum of the samples in FP64.
    int render_f64(const LucidRenderParams& p, double* out_host);
    // Progressive accumulator (PyRenderer render_*_async, pybind_renderer.hpp:689-856).
    int async_start(int w, int h, int max_depth);
    int async_poll(int* samples, float* out, size_t cap_floats);
    int async_reset(int w, int h, int max_depth);
    int async_stop();
    int async_revision() const { return async_revision_.load(); }
    bool async_running() const { return async_run_.load(); }
    int render_noalloc(const LucidRenderParams& p, float* d_out);
    // Jobs on other engines' scenes in one set of wavefront launches over a
    // device job table (lucid_cuda_render_batch); the scenes must stay
    // loaded until the call returns.
    struct BatchItem {
        const void* scene;        // DeviceScene: scene_ptr() of the engine or snapshot holding it
        float camera[10];         // position, direction, up, vertical fov (degrees)
        LucidRenderParams p;      // the same max_depth for every job
        float* out_host;          // tile_w * tile_h * 4 floats (the layout of render)
    };
    int render_batch(const BatchItem* items, int n, const char* algorithm, long long wave_paths);
    // Small render calls of concurrent contexts combined into batches
    // (lucid_cuda_set_combining); on by default.
    void set_combining(bool on) { combine_ = on; }
    static void combine_stats(int device, long long* batches, long long* calls);
    static constexpr long long kCombinePaths = 1LL << 22;
    // Device memory of a batch: path state for wave_paths paths and films of `pixels`.
    static long long batch_bytes(long long pixels, long long wave_paths);
    int render_debug(int tx, int ty, int tw, int th, int fw, int fh, const char* mode, float* out_host);
    // Path diagnostics (PyRenderer's diagnostics API, pybind_renderer.hpp:893-1102).
    int diag_enable(const LucidDiagConfig* cfg);
    int diag_disable();
    bool diag_enabled() const { return diag_enabled_; }
    int diag_clear();
    int diag_stats(LucidDiagStats* out);
    int diag_pixel(int x, int y, bool by_mean, LucidDiagPixel* info, LucidDiagGroup* groups, int cap);
    int diag_variance_map(float* out, size_t cap);
    int diag_top(int n, bool by_mean, LucidDiagGroup* groups, int32_t* xy, int cap);
    int diag_coarse(LucidDiagCoarse* out);
    int diag_suggestions(LucidDiagSuggestion* out, int cap);
    long long diag_export_binary(uint8_t* out, size_t cap);
    long long diag_metadata_json(char* out, size_t cap);
    int scene_stats(int out8[8]) const;
    // Online-trained path guiding for the `mis` integrator (reseeds the network).
    int guide_enable(bool on, int seed);
    int guide_steps() const;
    int guide_config(int steps_per_wave, float lr);
    int guide_max_depth(int max_depth);
    int guide_params(float* out, size_t cap, float* box6);
    // Uses `owner`'s uploaded scene (BVH, materials, lights) without a copy.
    int share_scene(Engine& owner);
    // The current version of this engine's scene, and rendering a version
    // taken from another engine.
    int snapshot_scene(SceneSnapshot& out);
    int use_snapshot(const SceneSnapshot& snap);
    const void* scene_ptr() const { return ds_.get(); }
    // Parameter edits (lucid_cuda_update_scene): a new scene version that
    // shares the geometry of the current one.
    int update_scene(const LucidSceneEdit* edits, int count);
    // Guided progressive jobs: render_impl iterations (guiding and training
    // per wave) summed into a per-pixel accumulator.
    static long long guide_job_bytes(long long paths);
    int accum_begin(int w, int h);
    int render_accumulate(const LucidRenderParams& p);
    int accum_output(float* out_host);
    void accum_end();          // frees the accumulator
    void guide_free();         // frees the guide network and its buffers
    // Progressive jobs (the request loop's unit of work).
    static long long job_bytes(int w, int h, int chunk);
    int job_begin(int w, int h, int spp, int max_depth, int chunk, bool use_graph);
    int job_set_chunk(int chunk, bool use_graph);
    // Launch profile (resident CTAs per SM of the wavefront kernels; 0 the
    // default, 1 more registers per thread) of renders and of the job.
    int set_launch_profile(int profile);
    int job_set_profile(int profile, bool use_graph);
    int launch_profile() const { return launch_profile_; }
    int job_iterate(int sample_offset, int n);
    int job_wait();
    int job_output(float* out_host);
    void job_end();
    void release_pool();
    int stats(LucidRenderStats* out) const;
    int set_wave_capacity(long long paths);
    int device_info(char* buf, size_t cap) const;

    void cancel() { cancel_.store(true); }
    bool is_cancelled() const { return cancel_.load(); }
    void reset_cancel() { cancel_.store(false); }

    const std::string& last_error() const { return err_; }
    int fail(int code, const std::string& msg) { err_ = msg; return code; }

private:
    int render_impl(const LucidRenderParams& p, float* out_host, LucidSampleRecord* recs, float* out_device,
                    void* accumulate, bool from_async, double* out_f64 = nullptr);
    int render_diag_impl(const LucidRenderParams& p, float* out_host, float* out_device);
    int render_combined(const LucidRenderParams& p, float* out_host);
    void async_worker();
    int ensure_pool(long long paths, bool records);
    long long default_wave_paths(bool records) const;
    int build_bvh();
    int upload_scene(HostScene&& hs);
    int ensure_stream();
    int guide_buffers(long long paths);
    void scene_stats_locked(int out8[8]) const;
    void enqueue_iteration(void* frame_params, int n);
    void job_end_locked();
    int capture_locked(int chunk);
    void job_grids_locked();
    int build_ploc(const float4* verts, const int* sorted_ids, int n, int2* child, int2* range, float* nbox,
                   int* slot_ids, int& root);
    void free_scene();

    int device_ = 0;
    void* stream_ = nullptr;   // cudaStream_t
    int num_sms_ = 0;
    HostScene host_;
    HostCamera cam_;
    float cam_raw_[10] = {};   // set_camera's arguments (batched renders rebuild the camera from them)
    bool combine_ = true;
    bool scene_loaded_ = false, camera_set_ = false;
    int algo_ = 1;            // "nee": PyRenderer's default (pybind_renderer.hpp:68)
    std::shared_ptr<DeviceScene> ds_;
    bool shared_ = false;         // ds_ belongs to another engine (share_scene)
    int shared_stats_[8] = {};
    JobState* job_ = nullptr;
    GuideState* guide_ = nullptr;
    void* jacc_ = nullptr;        // device float4 accumulator of a guided job
    size_t jacc_n_ = 0;
    int jacc_w_ = 0, jacc_h_ = 0;
    float scene_lo_[3] = {0, 0, 0}, scene_hi_[3] = {1, 1, 1};
    PathPool* pool_ = nullptr;
    long long wave_cap_ = 0;  // 0 = automatic
    int launch_profile_ = 0;
    std::atomic<bool> cancel_{false};
    std::string err_;
    LucidRenderStats stats_{};
    int bvh_nodes_ = 0, bvh_leaves_ = 0, bvh_depth_ = 0, num_big_ = 0, ploc_rounds_ = 0;
    double bvh_sah_ = 0.0;
    // one GPU call at a time per context (the reference's gpu_mutex_); API
    // calls take it through GpuLock, which the async worker yields to
    std::mutex gpu_mu_;
    std::atomic<int> gpu_waiters_{0};
    struct GpuLock {
        Engine& e;
        explicit GpuLock(Engine& en) : e(en) {
            e.gpu_waiters_.fetch_add(1);
            e.gpu_mu_.lock();
            e.gpu_waiters_.fetch_sub(1);
        }
        ~GpuLock() { e.gpu_mu_.unlock(); }
        GpuLock(const GpuLock&) = delete;
        GpuLock& operator=(const GpuLock&) = delete;
    };
    // path diagnostics
    bool diag_enabled_ = false;
    LucidDiagConfig diag_cfg_{};
    DiagFilm diag_film_;
    DiagDevice* diag_dev_ = nullptr;
    // async accumulator
    std::thread async_thread_;
    std::atomic<bool> async_run_{false}, async_reset_{false};
    std::atomic<int> async_revision_{0};
    int async_w_ = 0, async_h_ = 0, async_depth_ = 8;
    void* async_acc_ = nullptr;       // device float4[w*h] sum of samples
    size_t async_acc_n_ = 0;
    float* async_pinned_ = nullptr;   // pinned host copy of the accumulator
    std::mutex snap_mu_;
    std::vector<float> snap_;
    int snap_samples_ = 0;
    std::string async_err_;
};

}  // namespace lucid
