// lucid_server.cpp — the request loop (see lucid_server.h).
#include "lucid_server.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "lucid_engine.h"

namespace lucid {

namespace {
// Largest wave a job may use (paths per iteration) and the iteration time
// an interactive job aims for.
constexpr long long kJobWavePaths = 1LL << 24;
constexpr double kInteractiveMs = 33.0;
// Default paths per batch (one wave: 32 Mi paths, 6 GB of path state) and
// the most jobs one batch takes.  On the batched configuration (56 jobs on
// 56 scenes, 175 M samples), same box: 2^25 455 M samples/s on 4 slots,
// 2^26 398 M, 2^27 379 M, 2^28 362 M (two or more smaller batches in flight
// overlap each other's wave tails and host gaps; large retained pools crowd
// the device).
constexpr long long kBatchPaths = 1LL << 25;
constexpr int kBatchJobs = 256;
long long job_paths(const LucidJobDesc& d) { return (long long)d.width * d.height * d.samples; }

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double pos = q * (double)(v.size() - 1);
    size_t lo = (size_t)pos, hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}
}  // namespace

std::vector<int> plan_batch(const LucidJobDesc& head, const std::vector<const LucidJobDesc*>& queue,
                            const std::vector<char>& cancelled, long long max_paths, long long room_bytes,
                            int max_jobs, long long* bytes) {
    std::vector<int> take;
    long long paths = job_paths(head), pixels = (long long)head.width * head.height;
    long long bb = Engine::batch_bytes(pixels, paths);
    if (max_paths > 0 && !head.interactive && !head.guided && paths < max_paths) {
        for (int k = 0; k < (int)queue.size() && (int)take.size() + 1 < max_jobs; ++k) {
            const LucidJobDesc& c = *queue[(size_t)k];
            const long long p2 = paths + job_paths(c), px2 = pixels + (long long)c.width * c.height;
            const long long b2 = Engine::batch_bytes(px2, p2);
            if (cancelled[(size_t)k] || c.interactive || c.guided || c.max_depth != head.max_depth ||
                std::strncmp(c.algorithm, head.algorithm, sizeof(c.algorithm)) != 0 || p2 > max_paths || b2 > room_bytes)
                continue;
            take.push_back(k);
            paths = p2;
            pixels = px2;
            bb = b2;
        }
    }
    if (bytes) *bytes = bb;
    return take;
}

double Server::now() const {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

Server::Server(int device, int slots, long long budget_bytes) : device_(device), batch_paths_(kBatchPaths) {
    slots = std::max(1, slots);
    if (budget_bytes <= 0) {
        // 70 % of the free memory: the rest holds the path pools slots keep
        // between jobs
        size_t free_b = 0, total_b = 0;
        cudaSetDevice(device);
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget_bytes = (long long)(free_b * 0.7);
        else budget_bytes = 1LL << 30;
    }
    budget_ = budget_bytes;
    adm_.budget = budget_bytes;
    adm_.slots = slots;
    t0_ = now();
    for (int s = 0; s < slots; ++s) {
        slot_eng_.emplace_back(new Engine(device));
        pre_eng_.emplace_back(nullptr);
    }
    for (int s = 0; s < slots; ++s) threads_.emplace_back([this, s] { slot_loop(s); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
        for (auto& kv : jobs_) kv.second.cancel = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
    pre_eng_.clear();
    slot_eng_.clear();
    scenes_.clear();
}

int Server::add_scene(const char* json, size_t len, int* scene_id) {
    return add_scene_with([&](Engine& e) { return e.load_scene_json(json, len); }, scene_id);
}

int Server::add_scene_arrays(const LucidSceneDesc& desc, int* scene_id) {
    return add_scene_with([&](Engine& e) { return e.load_scene_arrays(desc); }, scene_id);
}

// Loads a scene into a new engine with `load` and registers it with the
// device memory it took.
template <class Load>
int Server::add_scene_with(Load&& load, int* scene_id) {
    size_t f0 = 0, f1 = 0, tot = 0;
    cudaSetDevice(device_);
    cudaMemGetInfo(&f0, &tot);
    std::unique_ptr<Engine> e(new Engine(device_));
    int rc = load(*e);
    if (rc != LUCID_OK) return fail(rc, e->last_error());
    cudaMemGetInfo(&f1, &tot);
    std::lock_guard<std::mutex> lk(mu_);
    long long bytes = f0 > f1 ? (long long)(f0 - f1) : 0;
    scenes_.push_back(std::move(e));
    scene_bytes_.push_back(bytes);
    adm_.reserved += bytes;
    *scene_id = (int)scenes_.size() - 1;
    return LUCID_OK;
}

int Server::update_scene(int scene_id, const LucidSceneEdit* edits, int count) {
    std::lock_guard<std::mutex> lk(mu_);   // ordered with submissions: later jobs see the edit
    if (scene_id < 0 || scene_id >= (int)scenes_.size()) return fail(LUCID_ERR_INVALID, "update: unknown scene");
    int rc = scenes_[scene_id]->update_scene(edits, count);
    if (rc != LUCID_OK) return fail(rc, scenes_[scene_id]->last_error());
    return LUCID_OK;
}

// Bytes of a job: path state and film for `chunk` samples per iteration,
// plus the guide's buffers for a guided job.
static long long job_total_bytes(const LucidJobDesc& d, int chunk) {
    long long b = Engine::job_bytes(d.width, d.height, chunk);
    if (d.guided) b += Engine::guide_job_bytes((long long)d.width * d.height * chunk);
    return b;
}

int Server::submit(const LucidJobDesc& d, int* job_id) {
    if (d.width <= 0 || d.height <= 0 || d.samples <= 0 || d.max_depth <= 0 || d.max_depth > 1024)
        return fail(LUCID_ERR_INVALID, "job: sizes must be positive (max_depth <= 1024)");
    if (d.guided && std::string(d.algorithm, strnlen(d.algorithm, sizeof(d.algorithm))) != "mis")
        return fail(LUCID_ERR_INVALID, "job: path guiding needs the \"mis\" integrator");
    std::unique_lock<std::mutex> lk(mu_);
    if (d.scene < 0 || d.scene >= (int)scenes_.size()) return fail(LUCID_ERR_INVALID, "job: unknown scene");
    auto snap = std::make_shared<SceneSnapshot>();
    if (scenes_[d.scene]->snapshot_scene(*snap) != LUCID_OK) return fail(LUCID_ERR_NO_SCENE, "job: scene not loaded");
    int id = next_id_++;
    Job& j = jobs_[id];
    j.d = d;
    j.d.algorithm[sizeof(j.d.algorithm) - 1] = 0;
    j.snap = std::move(snap);
    j.t_submit = now();
    const long long np = (long long)d.width * d.height;
    // the largest samples per iteration within the wave limit and the budget
    int cmax = (int)std::max(1LL, std::min<long long>(d.samples, kJobWavePaths / std::max(1LL, np)));
    while (cmax > 1 && adm_.never_fits(job_total_bytes(d, cmax))) cmax /= 2;
    j.chunk_max = cmax;
    j.bytes = job_total_bytes(d, j.chunk_max);
    *job_id = id;
    if (adm_.never_fits(j.bytes)) {
        j.state = LUCID_JOB_REFUSED;
        j.t_end = now();
        j.error = "job needs " + std::to_string(j.bytes) + " bytes; the budget leaves " +
                  std::to_string(adm_.budget - adm_.reserved);
        done_cv_.notify_all();
        return fail(LUCID_ERR_OOM, j.error);
    }
    // interactive jobs (viewport ticks) queue ahead of batch jobs; arrival
    // order holds within each class
    if (d.interactive) {
        auto it = std::find_if(queue_.begin(), queue_.end(), [&](int q) { return !jobs_[q].d.interactive; });
        queue_.insert(it, id);
    } else {
        queue_.push_back(id);
    }
    lk.unlock();
    cv_.notify_all();
    return LUCID_OK;
}

void Server::slot_loop(int slot) {
    for (;;) {
        int id = -1;
        Job* j = nullptr;
        std::vector<Job*> batch;
        long long batch_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] {
                if (stop_) return true;
                while (!queue_.empty() && jobs_[queue_.front()].cancel) {   // drop cancelled queued jobs
                    Job& c = jobs_[queue_.front()];
                    c.state = LUCID_JOB_CANCELLED;
                    c.t_end = now();
                    queue_.pop_front();
                    done_cv_.notify_all();
                }
                return !queue_.empty() && adm_.can_start(jobs_[queue_.front()].bytes);
            });
            if (stop_) return;
            id = queue_.front();
            queue_.pop_front();
            j = &jobs_[id];
            // a throughput job takes the compatible jobs waiting behind it
            // (same integrator and depth, in queue order) into one batch
            // while the batch stays within a wave and the budget
            std::vector<Job*> members{j};
            long long bbytes = 0;
            {
                std::vector<const LucidJobDesc*> waiting;
                std::vector<char> cancelled;
                for (int q : queue_) {
                    waiting.push_back(&jobs_[q].d);
                    cancelled.push_back(jobs_[q].cancel ? 1 : 0);
                }
                std::vector<int> take = plan_batch(j->d, waiting, cancelled, batch_paths_,
                                                   adm_.budget - adm_.reserved - adm_.running, kBatchJobs, &bbytes);
                for (int k = (int)take.size() - 1; k >= 0; --k) {   // erase from the back: indices stay valid
                    auto it = queue_.begin() + take[(size_t)k];
                    members.push_back(&jobs_[*it]);
                    queue_.erase(it);
                }
                std::reverse(members.begin() + 1, members.end());   // queue order
            }
            const double t = now();
            if (busy_from_ < 0) busy_from_ = t;
            if (members.size() > 1) {
                adm_.start(bbytes);
                for (Job* m : members) {
                    m->state = LUCID_JOB_RUNNING;
                    m->t_start = t;
                }
                batch = std::move(members);
            } else {
                adm_.start(j->bytes);
                j->state = LUCID_JOB_RUNNING;
                j->t_start = t;
            }
            batch_bytes = bbytes;
        }
        cv_.notify_all();   // another slot may start the next job too
        if (!batch.empty()) {
            int rc = run_batch(*slot_eng_[slot], batch);
            if (rc == LUCID_ERR_OOM) {   // retained pools may be in the way: release them and retry once
                slot_eng_[slot]->guide_free();
                slot_eng_[slot]->accum_end();
                slot_eng_[slot]->release_pool();
                if (pre_eng_[slot]) pre_eng_[slot]->release_pool();
                rc = run_batch(*slot_eng_[slot], batch);
            }
            finish_batch(batch, batch_bytes, rc);
            continue;
        }
        // the slot keeps its path pool (and a guided job's buffers) for the
        // next job: freeing device memory synchronises the whole device and
        // would stall every other slot's work
        int rc = run_job(*slot_eng_[slot], *j, slot, true);
        if (rc == LUCID_ERR_OOM) {   // a pool grown by earlier jobs may be in the way: release it and retry once
            slot_eng_[slot]->guide_free();
            slot_eng_[slot]->accum_end();
            slot_eng_[slot]->release_pool();
            if (pre_eng_[slot]) pre_eng_[slot]->release_pool();
            {
                std::lock_guard<std::mutex> lk(mu_);
                j->error.clear();
            }
            rc = run_job(*slot_eng_[slot], *j, slot, true);
        }
        finish_job(*j, rc);
    }
}

void Server::finish_job(Job& j, int rc) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        adm_.finish(j.bytes);
        j.t_end = now();
        busy_to_ = std::max(busy_to_, j.t_end);
        if (rc == LUCID_OK && !j.cancel) {
            j.state = LUCID_JOB_DONE;
            samples_done_ += (long long)j.d.samples * j.d.width * j.d.height;
        } else {
            j.state = j.cancel ? LUCID_JOB_CANCELLED : LUCID_JOB_FAILED;
        }
        j.snap.reset();   // the scene version may go once no job needs it
    }
    cv_.notify_all();
    done_cv_.notify_all();
}

// Between two iterations of a batch job: while an interactive job waits at
// the head of the queue and its memory fits, run it to completion on the
// slot's second engine (the batch job's iterations in flight keep running on
// their own stream), so interactive work never waits for a long render.
void Server::run_waiting_interactive(int slot) {
    for (;;) {
        Job* j = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (stop_ || queue_.empty()) return;
            Job& head = jobs_[queue_.front()];
            if (!head.d.interactive || head.cancel) return;
            if (adm_.reserved + adm_.running + head.bytes > adm_.budget) return;
            queue_.pop_front();
            j = &head;
            adm_.running += j->bytes;   // admitted beside the slot's batch job (no slot of its own)
            ++adm_.busy;
            j->state = LUCID_JOB_RUNNING;
            j->t_start = now();
        }
        if (!pre_eng_[slot]) pre_eng_[slot].reset(new Engine(device_));
        // the second engine keeps its path pool from one interactive job to the next
        // (freeing device memory synchronises the device and would stall the batch job)
        int rc = run_job(*pre_eng_[slot], *j, slot, true);
        finish_job(*j, rc);
    }
}

// Autotuner: the first iterations of a job shape (scene, size, integrator,
// depth, interactivity) try 1, 2, 4, ... samples per iteration; the size with
// the most samples per second wins (for interactive jobs among those whose
// iteration stays under kInteractiveMs) and is cached for the shape.  The
// trial iterations are part of the job's own samples.
int Server::pick_chunk(Engine& e, Job& j, int id, int& offset) {
    const LucidJobDesc& d = j.d;
    std::string key = std::to_string(d.scene) + ":" + std::to_string(d.width) + "x" + std::to_string(d.height) + ":" +
                      d.algorithm + ":" + std::to_string(d.max_depth) + ":" + std::to_string(d.interactive);
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = tuned_.find(key);
        if (it != tuned_.end()) {
            if (it->second.second != 0) {
                int rc = e.job_set_profile(it->second.second, false);
                if (rc != LUCID_OK) return -rc;
            }
            return std::min(it->second.first, j.chunk_max);
        }
    }
    auto timed = [&](int c, double& ms) {
        auto t = std::chrono::steady_clock::now();
        int rc = e.job_iterate(offset, c);
        if (rc == LUCID_OK) rc = e.job_wait();
        if (rc != LUCID_OK) return rc;
        ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
        offset += c;
        std::lock_guard<std::mutex> lk(mu_);
        j.done = offset;
        if (j.t_first == 0) j.t_first = now();
        return LUCID_OK;
    };
    int best = 1;
    double best_rate = -1.0, best_ms = 0.0;
    for (int c = 1; c <= j.chunk_max && offset + c <= d.samples; c *= 2) {
        double ms = 0.0;
        int rc = timed(c, ms);
        if (rc != LUCID_OK) return -rc;
        double rate = c / std::max(ms, 1e-3);
        bool ok = !d.interactive || ms <= kInteractiveMs || c == 1;
        if (ok && rate > best_rate) { best_rate = rate; best = c; best_ms = ms; }
        if (d.interactive && ms > kInteractiveMs) break;
    }
    // then the launch profiles (resident CTAs per SM) at that size, when the
    // job has samples left for a trial of each
    int best_profile = 0, cur_profile = 0;
    for (int prof = 1; prof < 2 && offset + best <= d.samples; ++prof) {
        int rc = e.job_set_profile(prof, false);
        if (rc != LUCID_OK) return -rc;
        cur_profile = prof;
        double ms = 0.0;
        rc = timed(best, ms);
        if (rc != LUCID_OK) return -rc;
        if (ms < best_ms) { best_ms = ms; best_profile = prof; }
    }
    if (cur_profile != best_profile) {
        int rc = e.job_set_profile(best_profile, false);
        if (rc != LUCID_OK) return -rc;
    }
    (void)id;
    std::lock_guard<std::mutex> lk(mu_);
    tuned_[key] = {best, best_profile};
    return best;
}

int Server::run_job(Engine& e, Job& j, int slot, bool keep_pool) {
    const LucidJobDesc& d = j.d;
    int rc = LUCID_OK;
    if (e.scene_ptr() != j.snap->ds.get()) {   // another scene, or another version of it
        rc = e.use_snapshot(*j.snap);
        if (rc != LUCID_OK) { j.error = e.last_error(); return rc; }
    }
    const float* c = d.camera;
    e.set_camera(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9]);
    e.set_algorithm(d.algorithm);
    if (d.guided) return run_guided_job(e, j, slot, keep_pool);
    rc = e.job_begin(d.width, d.height, d.samples, d.max_depth, j.chunk_max, false);
    if (rc != LUCID_OK) { j.error = e.last_error(); e.job_end(); if (!keep_pool) e.release_pool(); return rc; }
    int offset = 0;
    int chunk = pick_chunk(e, j, slot, offset);
    if (chunk < 0) { j.error = e.last_error(); e.job_end(); if (!keep_pool) e.release_pool(); return -chunk; }
    if (offset < d.samples) {
        rc = e.job_set_chunk(chunk, d.samples - offset >= 2 * chunk);
        while (rc == LUCID_OK && offset < d.samples) {
            if (j.cancel) break;
            int n = std::min(chunk, d.samples - offset);
            rc = e.job_iterate(offset, n);
            offset += n;
            {
                std::lock_guard<std::mutex> lk(mu_);
                // iteration k returns once iteration k - 2 has finished
                j.done = std::max(j.done, std::max(0, offset - 2 * chunk));
                if (j.t_first == 0 && offset > 2 * chunk) j.t_first = now();
            }
            if (!d.interactive && rc == LUCID_OK) run_waiting_interactive(slot);
        }
    }
    if (rc == LUCID_OK) rc = e.job_wait();
    if (rc == LUCID_OK && !j.cancel) {
        std::vector<float> img((size_t)d.width * d.height * 4);
        rc = e.job_output(img.data());
        std::lock_guard<std::mutex> lk(mu_);
        if (rc == LUCID_OK) {
            j.image.swap(img);
            j.done = d.samples;
            if (j.t_first == 0) j.t_first = now();
        }
    }
    if (rc != LUCID_OK) j.error = e.last_error();
    e.job_end();
    if (!keep_pool) e.release_pool();
    return rc;
}

// A guided job: iterations of chunk_max samples through the engine's render
// path (guided sampling, and training after every wave, on the job's own
// network), summed per pixel; batch jobs let waiting interactive jobs run
// between their iterations as unguided jobs do.
int Server::run_guided_job(Engine& e, Job& j, int slot, bool keep_pool) {
    const LucidJobDesc& d = j.d;
    int rc = e.guide_enable(true, d.guide_seed);
    if (rc == LUCID_OK) rc = e.accum_begin(d.width, d.height);
    int offset = 0;
    while (rc == LUCID_OK && offset < d.samples) {
        if (j.cancel) break;
        const int n = std::min(j.chunk_max, d.samples - offset);
        LucidRenderParams p{0, 0, d.width, d.height, d.width, d.height, n, offset, d.max_depth, 0};
        rc = e.render_accumulate(p);
        offset += n;
        {
            std::lock_guard<std::mutex> lk(mu_);
            j.done = offset;
            if (j.t_first == 0) j.t_first = now();
        }
        if (!d.interactive && rc == LUCID_OK) run_waiting_interactive(slot);
    }
    if (rc == LUCID_OK && !j.cancel) {
        std::vector<float> img((size_t)d.width * d.height * 4);
        rc = e.accum_output(img.data());
        std::lock_guard<std::mutex> lk(mu_);
        if (rc == LUCID_OK) j.image.swap(img);
    }
    if (rc != LUCID_OK) j.error = e.last_error();
    e.guide_enable(false, 0);
    if (!keep_pool) {
        e.guide_free();
        e.accum_end();
        e.release_pool();
    }
    return rc;
}

// A batch: every member's whole image in one Engine::render_batch call on
// the slot's engine (each member on the scene version of its submission).
int Server::run_batch(Engine& e, const std::vector<Job*>& members) {
    std::vector<Engine::BatchItem> items(members.size());
    for (size_t k = 0; k < members.size(); ++k) {
        Job& j = *members[k];
        const LucidJobDesc& d = j.d;
        j.image.assign((size_t)d.width * d.height * 4, 0.0f);
        Engine::BatchItem& it = items[k];
        it.scene = j.snap->ds.get();
        std::memcpy(it.camera, d.camera, sizeof(it.camera));
        it.p = LucidRenderParams{0, 0, d.width, d.height, d.width, d.height, d.samples, 0, d.max_depth, 0};
        it.out_host = j.image.data();
    }
    int rc = e.render_batch(items.data(), (int)items.size(), members[0]->d.algorithm, batch_paths_);
    if (rc != LUCID_OK) {
        std::lock_guard<std::mutex> lk(mu_);
        for (Job* m : members) m->error = e.last_error();
    }
    return rc;
}

void Server::finish_batch(const std::vector<Job*>& members, long long bytes, int rc) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        adm_.finish(bytes);
        ++batches_;
        batched_jobs_ += (int)members.size();
        const double t = now();
        busy_to_ = std::max(busy_to_, t);
        for (Job* m : members) {
            Job& j = *m;
            j.t_end = t;
            if (rc == LUCID_OK && !j.cancel) {
                j.state = LUCID_JOB_DONE;
                j.done = j.d.samples;
                j.t_first = t;
                j.error.clear();
                samples_done_ += (long long)j.d.samples * j.d.width * j.d.height;
            } else {
                j.state = j.cancel ? LUCID_JOB_CANCELLED : LUCID_JOB_FAILED;
                j.image.clear();
            }
            j.snap.reset();
        }
    }
    cv_.notify_all();
    done_cv_.notify_all();
}

int Server::set_batching(long long max_paths) {
    if (max_paths < 0) return fail(LUCID_ERR_INVALID, "batching: max_paths must be >= 0");
    std::lock_guard<std::mutex> lk(mu_);
    batch_paths_ = max_paths;
    return LUCID_OK;
}

int Server::state(int job, int* samples_done) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) return fail(LUCID_ERR_INVALID, "unknown job");
    if (samples_done) *samples_done = it->second.done;
    return it->second.state;
}

int Server::wait(int job, int timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) return fail(LUCID_ERR_INVALID, "unknown job");
    auto finished = [&] { int s = jobs_[job].state; return s != LUCID_JOB_QUEUED && s != LUCID_JOB_RUNNING; };
    if (timeout_ms < 0) done_cv_.wait(lk, finished);
    else done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished);
    return jobs_[job].state;
}

int Server::result(int job, float* out, size_t cap_floats) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) return fail(LUCID_ERR_INVALID, "unknown job");
    Job& j = it->second;
    if (j.state != LUCID_JOB_DONE) return fail(LUCID_ERR_INVALID, "job has no image" + (j.error.empty() ? "" : ": " + j.error));
    if (cap_floats < j.image.size()) return fail(LUCID_ERR_INVALID, "result buffer too small");
    std::memcpy(out, j.image.data(), j.image.size() * sizeof(float));
    return LUCID_OK;
}

int Server::cancel(int job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) return fail(LUCID_ERR_INVALID, "unknown job");
    it->second.cancel = true;
    cv_.notify_all();
    return LUCID_OK;
}

int Server::stats(LucidServerStats* out) {
    std::lock_guard<std::mutex> lk(mu_);
    std::memset(out, 0, sizeof(*out));
    std::vector<double> lat, first;
    for (auto& kv : jobs_) {
        const Job& j = kv.second;
        ++out->submitted;
        switch (j.state) {
            case LUCID_JOB_DONE:
                ++out->done;
                lat.push_back(j.t_end - j.t_submit);
                first.push_back(j.t_first - j.t_submit);
                break;
            case LUCID_JOB_REFUSED: ++out->refused; break;
            case LUCID_JOB_RUNNING: ++out->running; break;
            case LUCID_JOB_QUEUED: ++out->queued; break;
            default: break;
        }
    }
    out->latency_p50_ms = percentile(lat, 0.50);
    out->latency_p99_ms = percentile(lat, 0.99);
    out->first_p50_ms = percentile(first, 0.50);
    out->first_p99_ms = percentile(first, 0.99);
    double busy = busy_to_ - busy_from_;
    out->samples_per_s = (busy_from_ >= 0 && busy > 0) ? (double)samples_done_ / (busy / 1000.0) : 0.0;
    out->bytes_reserved = adm_.reserved;
    out->bytes_running = adm_.running;
    out->budget_bytes = adm_.budget;
    out->batches = batches_;
    out->batched_jobs = batched_jobs_;
    return LUCID_OK;
}

}  // namespace lucid
