// lucid_capi.cpp — extern "C" entry points of liblucid_cuda.so.
// Exceptions never cross the boundary: every call returns a status code and
// records its message for lucid_cuda_last_error().
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/lucid_cuda.h"
#include "lucid_engine.h"
#include "lucid_host.h"
#include "lucid_server.h"

struct LucidCudaCtx {
    lucid::Engine* engine;
};

struct LucidServer {
    lucid::Server* server;
};

namespace {
template <class F>
int guarded(LucidCudaCtx* ctx, F&& f) {
    if (!ctx || !ctx->engine) return LUCID_ERR_INVALID;
    try {
        return f(*ctx->engine);
    } catch (const std::bad_alloc&) {
        return ctx->engine->fail(LUCID_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return ctx->engine->fail(LUCID_ERR_INVALID, e.what());
    } catch (...) {
        return ctx->engine->fail(LUCID_ERR_INVALID, "unknown error");
    }
}
template <class F>
int server_guarded(LucidServer* srv, F&& f) {
    if (!srv || !srv->server) return LUCID_ERR_INVALID;
    try {
        return f(*srv->server);
    } catch (const std::bad_alloc&) {
        return srv->server->fail(LUCID_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return srv->server->fail(LUCID_ERR_INVALID, e.what());
    }
}
}  // namespace

extern "C" {

int lucid_cuda_create(int device, LucidCudaCtx** out) {
    if (!out) return LUCID_ERR_INVALID;
    *out = nullptr;
    try {
        LucidCudaCtx* c = new LucidCudaCtx;
        c->engine = new lucid::Engine(device);
        *out = c;
        return LUCID_OK;
    } catch (...) {
        return LUCID_ERR_OOM;
    }
}

void lucid_cuda_destroy(LucidCudaCtx* ctx) {
    if (!ctx) return;
    delete ctx->engine;
    delete ctx;
}

const char* lucid_cuda_last_error(LucidCudaCtx* ctx) {
    if (!ctx || !ctx->engine) return "invalid context";
    return ctx->engine->last_error().c_str();
}

int lucid_cuda_device_info(LucidCudaCtx* ctx, char* buf, size_t cap) {
    if (!buf || cap == 0) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.device_info(buf, cap); });
}

int lucid_cuda_load_scene_json(LucidCudaCtx* ctx, const char* json, size_t len) {
    if (!json) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.load_scene_json(json, len); });
}

int lucid_cuda_load_scene_arrays(LucidCudaCtx* ctx, const LucidSceneDesc* scene) {
    if (!scene) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.load_scene_arrays(*scene); });
}

int lucid_cuda_set_camera(LucidCudaCtx* ctx, float px, float py, float pz, float dx, float dy, float dz, float ux,
                          float uy, float uz, float fov_deg) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.set_camera(px, py, pz, dx, dy, dz, ux, uy, uz, fov_deg); });
}

int lucid_cuda_set_algorithm(LucidCudaCtx* ctx, const char* name) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.set_algorithm(name); });
}

int lucid_cuda_scene_stats(LucidCudaCtx* ctx, int out8[8]) {
    if (!out8) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.scene_stats(out8); });
}

int lucid_cuda_inspect_scene(const char* json, size_t len, int counts8[8], float* cdf, float* area,
                             float* emission_rgb, int cap) {
    if (!json || !counts8) return LUCID_ERR_INVALID;
    try {
        lucid::HostScene hs;
        std::string err;
        if (!lucid::parse_scene_json(json, len, hs, err)) return LUCID_ERR_INVALID;
        counts8[0] = hs.num_meshes; counts8[1] = hs.num_prims; counts8[2] = hs.num_native;
        counts8[3] = (int)hs.lights.size(); counts8[4] = hs.num_boundary_meshes; counts8[5] = (int)hs.volumes.size();
        counts8[6] = 0; counts8[7] = 0;
        for (int i = 0; i < (int)hs.lights.size() && i < cap; ++i) {
            if (cdf) cdf[i] = hs.cdf[i];
            if (area) area[i] = hs.lights[i].normal_area.w;
            if (emission_rgb) {
                emission_rgb[3 * i] = hs.lights[i].emission_radius.x;
                emission_rgb[3 * i + 1] = hs.lights[i].emission_radius.y;
                emission_rgb[3 * i + 2] = hs.lights[i].emission_radius.z;
            }
        }
        return (int)hs.lights.size();
    } catch (...) {
        return LUCID_ERR_INVALID;
    }
}

int lucid_scene_digest(const char* json, size_t len, const LucidSceneDesc* arrays, uint64_t* digest) {
    if (!digest || (json == nullptr) == (arrays == nullptr)) return LUCID_ERR_INVALID;
    try {
        lucid::HostScene hs;
        std::string err;
        const bool ok = json ? lucid::parse_scene_json(json, len, hs, err) : lucid::build_scene_arrays(*arrays, hs, err);
        if (!ok) return LUCID_ERR_INVALID;
        *digest = lucid::scene_digest(hs);
        return LUCID_OK;
    } catch (...) {
        return LUCID_ERR_INVALID;
    }
}

int lucid_cuda_render(LucidCudaCtx* ctx, const LucidRenderParams* params, float* out_rgba, LucidSampleRecord* records) {
    if (!params || !out_rgba) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.render(*params, out_rgba, records, nullptr); });
}

int lucid_cuda_render_device(LucidCudaCtx* ctx, const LucidRenderParams* params, float* d_out_rgba) {
    if (!params || !d_out_rgba) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.render(*params, nullptr, nullptr, d_out_rgba); });
}

int lucid_cuda_render_noalloc(LucidCudaCtx* ctx, const LucidRenderParams* params, float* d_out_rgba) {
    if (!params || !d_out_rgba) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.render_noalloc(*params, d_out_rgba); });
}

int lucid_cuda_set_combining(LucidCudaCtx* ctx, int on) {
    return guarded(ctx, [&](lucid::Engine& e) { e.set_combining(on != 0); return LUCID_OK; });
}

int lucid_cuda_combine_stats(int device, long long* batches, long long* calls) {
    lucid::Engine::combine_stats(device, batches, calls);
    return LUCID_OK;
}

int lucid_cuda_render_batch(LucidCudaCtx* ctx, const LucidBatchJob* jobs, int n, const char* algorithm) {
    if (!jobs || n <= 0) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) {
        // a job that cannot start leaves every image zero, as a failed render does
        auto refuse = [&](int code, const std::string& msg) {
            for (int j = 0; j < n; ++j) {
                const LucidRenderParams& p = jobs[j].params;
                if (jobs[j].out_rgba && p.tile_w > 0 && p.tile_h > 0)
                    std::memset(jobs[j].out_rgba, 0, (size_t)p.tile_w * p.tile_h * 4 * sizeof(float));
            }
            return e.fail(code, msg);
        };
        // each distinct scene context's current version, held for the call
        std::vector<LucidCudaCtx*> owners;
        std::vector<lucid::SceneSnapshot> snaps;
        std::vector<lucid::Engine::BatchItem> items((size_t)n);
        for (int j = 0; j < n; ++j) {
            LucidCudaCtx* sc = jobs[j].scene;
            if (!sc || !sc->engine) return refuse(LUCID_ERR_INVALID, "batch: job " + std::to_string(j) + " has no scene context");
            size_t k = 0;
            while (k < owners.size() && owners[k] != sc) ++k;
            if (k == owners.size()) {
                snaps.emplace_back();
                if (sc->engine->snapshot_scene(snaps.back()) != LUCID_OK)
                    return refuse(LUCID_ERR_NO_SCENE, "batch: job " + std::to_string(j) + ": " + sc->engine->last_error());
                owners.push_back(sc);
            }
            lucid::Engine::BatchItem& it = items[(size_t)j];
            it.scene = snaps[k].ds.get();
            std::memcpy(it.camera, jobs[j].camera, sizeof(it.camera));
            it.p = jobs[j].params;
            it.out_host = jobs[j].out_rgba;
        }
        return e.render_batch(items.data(), n, algorithm, 0);
    });
}

int lucid_cuda_render_debug(LucidCudaCtx* ctx, int tile_x, int tile_y, int tile_w, int tile_h, int full_w, int full_h,
                            const char* mode, float* out_rgba) {
    if (!out_rgba) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) {
        return e.render_debug(tile_x, tile_y, tile_w, tile_h, full_w, full_h, mode, out_rgba);
    });
}

int lucid_cuda_get_stats(LucidCudaCtx* ctx, LucidRenderStats* out) {
    if (!out) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.stats(out); });
}

int lucid_cuda_set_wave_capacity(LucidCudaCtx* ctx, long long paths) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.set_wave_capacity(paths); });
}

int lucid_cuda_async_start(LucidCudaCtx* ctx, int width, int height, int max_depth) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_start(width, height, max_depth); });
}

int lucid_cuda_async_poll(LucidCudaCtx* ctx, int* samples, float* out_rgba, size_t cap_floats) {
    if (!samples) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_poll(samples, out_rgba, cap_floats); });
}

int lucid_cuda_async_revision(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_revision(); });
}

int lucid_cuda_async_reset(LucidCudaCtx* ctx, int width, int height, int max_depth) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_reset(width, height, max_depth); });
}

int lucid_cuda_async_stop(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_stop(); });
}

int lucid_cuda_async_running(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.async_running() ? 1 : 0; });
}

int lucid_cuda_render_f64(LucidCudaCtx* ctx, const LucidRenderParams* params, double* out_rgba) {
    if (!params || !out_rgba) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.render_f64(*params, out_rgba); });
}

int lucid_cuda_diag_enable(LucidCudaCtx* ctx, const LucidDiagConfig* config) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_enable(config); });
}

int lucid_cuda_diag_disable(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_disable(); });
}

int lucid_cuda_diag_enabled(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_enabled() ? 1 : 0; });
}

int lucid_cuda_diag_clear(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_clear(); });
}

int lucid_cuda_diag_stats(LucidCudaCtx* ctx, LucidDiagStats* out) {
    if (!out) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_stats(out); });
}

int lucid_cuda_diag_pixel(LucidCudaCtx* ctx, int x, int y, int sort_by_mean, LucidDiagPixel* info,
                          LucidDiagGroup* groups, int cap) {
    if (!info) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_pixel(x, y, sort_by_mean != 0, info, groups, cap); });
}

int lucid_cuda_diag_variance_map(LucidCudaCtx* ctx, float* out, size_t cap) {
    if (!out) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_variance_map(out, cap); });
}

int lucid_cuda_diag_top_groups(LucidCudaCtx* ctx, int n, int by_mean, LucidDiagGroup* groups, int32_t* xy, int cap) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_top(n, by_mean != 0, groups, xy, cap); });
}

int lucid_cuda_diag_coarse_stats(LucidCudaCtx* ctx, LucidDiagCoarse* out) {
    if (!out) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_coarse(out); });
}

int lucid_cuda_diag_suggestions(LucidCudaCtx* ctx, LucidDiagSuggestion* out, int cap) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.diag_suggestions(out, cap); });
}

long long lucid_cuda_diag_export_binary(LucidCudaCtx* ctx, uint8_t* out, size_t cap) {
    long long n = LUCID_ERR_INVALID;
    int rc = guarded(ctx, [&](lucid::Engine& e) { n = e.diag_export_binary(out, cap); return LUCID_OK; });
    return rc == LUCID_OK ? n : rc;
}

long long lucid_cuda_diag_metadata_json(LucidCudaCtx* ctx, char* out, size_t cap) {
    long long n = LUCID_ERR_INVALID;
    int rc = guarded(ctx, [&](lucid::Engine& e) { n = e.diag_metadata_json(out, cap); return LUCID_OK; });
    return rc == LUCID_OK ? n : rc;
}

// ---- request loop ----
int lucid_server_create(int device, int slots, long long budget_bytes, LucidServer** out) {
    if (!out || slots <= 0 || slots > 64) return LUCID_ERR_INVALID;
    *out = nullptr;
    try {
        LucidServer* s = new LucidServer;
        s->server = new lucid::Server(device, slots, budget_bytes);
        *out = s;
        return LUCID_OK;
    } catch (...) {
        return LUCID_ERR_OOM;
    }
}

void lucid_server_destroy(LucidServer* srv) {
    if (!srv) return;
    delete srv->server;
    delete srv;
}

const char* lucid_server_last_error(LucidServer* srv) {
    if (!srv || !srv->server) return "invalid server";
    return srv->server->last_error().c_str();
}

int lucid_server_add_scene(LucidServer* srv, const char* json, size_t len, int* scene_id) {
    if (!json || !scene_id) return LUCID_ERR_INVALID;
    return server_guarded(srv, [&](lucid::Server& s) { return s.add_scene(json, len, scene_id); });
}

int lucid_server_add_scene_arrays(LucidServer* srv, const LucidSceneDesc* scene, int* scene_id) {
    if (!scene || !scene_id) return LUCID_ERR_INVALID;
    return server_guarded(srv, [&](lucid::Server& s) { return s.add_scene_arrays(*scene, scene_id); });
}

int lucid_server_update_scene(LucidServer* srv, int scene_id, const LucidSceneEdit* edits, int count) {
    return server_guarded(srv, [&](lucid::Server& s) { return s.update_scene(scene_id, edits, count); });
}

int lucid_server_submit(LucidServer* srv, const LucidJobDesc* job, int* job_id) {
    if (!job || !job_id) return LUCID_ERR_INVALID;
    return server_guarded(srv, [&](lucid::Server& s) { return s.submit(*job, job_id); });
}

int lucid_server_job_state(LucidServer* srv, int job_id, int* samples_done) {
    return server_guarded(srv, [&](lucid::Server& s) { return s.state(job_id, samples_done); });
}

int lucid_server_wait(LucidServer* srv, int job_id, int timeout_ms) {
    return server_guarded(srv, [&](lucid::Server& s) { return s.wait(job_id, timeout_ms); });
}

int lucid_server_result(LucidServer* srv, int job_id, float* out_rgba, size_t cap_floats) {
    if (!out_rgba) return LUCID_ERR_INVALID;
    return server_guarded(srv, [&](lucid::Server& s) { return s.result(job_id, out_rgba, cap_floats); });
}

int lucid_server_cancel(LucidServer* srv, int job_id) {
    return server_guarded(srv, [&](lucid::Server& s) { return s.cancel(job_id); });
}

int lucid_server_set_batching(LucidServer* srv, long long max_paths) {
    return server_guarded(srv, [&](lucid::Server& s) { return s.set_batching(max_paths); });
}

int lucid_server_stats(LucidServer* srv, LucidServerStats* out) {
    if (!out) return LUCID_ERR_INVALID;
    return server_guarded(srv, [&](lucid::Server& s) { return s.stats(out); });
}

int lucid_admission_plan(long long budget, long long reserved, int slots, const long long* job_bytes, int n,
                         int* decision) {
    if (n < 0 || slots <= 0 || (n > 0 && (!job_bytes || !decision))) return LUCID_ERR_INVALID;
    lucid::Admission a;
    a.budget = budget;
    a.reserved = reserved;
    a.slots = slots;
    std::vector<int> running;   // job indices in start order
    int started = 0;
    for (int i = 0; i < n; ++i) {
        if (a.never_fits(job_bytes[i])) { decision[i] = -1; continue; }
        while (!a.can_start(job_bytes[i])) {   // the earliest started job finishes first
            int k = running.front();
            running.erase(running.begin());
            a.finish(job_bytes[k]);
        }
        a.start(job_bytes[i]);
        running.push_back(i);
        decision[i] = started++;
    }
    return LUCID_OK;
}

int lucid_batch_plan(long long max_paths, long long room_bytes, const LucidJobDesc* jobs, const int* cancelled, int n,
                     int* member) {
    if (n <= 0 || !jobs || !member) return LUCID_ERR_INVALID;
    try {
        std::vector<const LucidJobDesc*> waiting;
        std::vector<char> canc;
        for (int i = 1; i < n; ++i) {
            waiting.push_back(&jobs[i]);
            canc.push_back(cancelled && cancelled[i] ? 1 : 0);
        }
        std::vector<int> take = lucid::plan_batch(jobs[0], waiting, canc, max_paths, room_bytes, 256, nullptr);
        for (int i = 0; i < n; ++i) member[i] = 0;
        for (int k : take) member[k + 1] = 1;
        member[0] = take.empty() ? 0 : 1;
        return (int)take.size() + 1;
    } catch (...) {
        return LUCID_ERR_INVALID;
    }
}

int lucid_cuda_guide_enable(LucidCudaCtx* ctx, int on, int seed) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.guide_enable(on != 0, seed); });
}

int lucid_cuda_guide_config(LucidCudaCtx* ctx, int steps_per_wave, float lr) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.guide_config(steps_per_wave, lr); });
}

int lucid_cuda_guide_max_depth(LucidCudaCtx* ctx, int max_depth) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.guide_max_depth(max_depth); });
}

int lucid_cuda_set_launch_profile(LucidCudaCtx* ctx, int profile) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.set_launch_profile(profile); });
}

int lucid_cuda_update_scene(LucidCudaCtx* ctx, const LucidSceneEdit* edits, int count) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.update_scene(edits, count); });
}

int lucid_cuda_guide_params(LucidCudaCtx* ctx, float* out, size_t cap, float* box6) {
    if (!out) return LUCID_ERR_INVALID;
    return guarded(ctx, [&](lucid::Engine& e) { return e.guide_params(out, cap, box6); });
}

int lucid_cuda_guide_steps(LucidCudaCtx* ctx) {
    return guarded(ctx, [&](lucid::Engine& e) { return e.guide_steps(); });
}

int lucid_cuda_cancel(LucidCudaCtx* ctx) {
    if (!ctx || !ctx->engine) return LUCID_ERR_INVALID;
    ctx->engine->cancel();
    return LUCID_OK;
}

int lucid_cuda_is_cancelled(LucidCudaCtx* ctx) {
    if (!ctx || !ctx->engine) return LUCID_ERR_INVALID;
    return ctx->engine->is_cancelled() ? 1 : 0;
}

int lucid_cuda_reset_cancel(LucidCudaCtx* ctx) {
    if (!ctx || !ctx->engine) return LUCID_ERR_INVALID;
    ctx->engine->reset_cancel();
    return LUCID_OK;
}

}  // extern "C"
