// lucid_server.h — the device-resident request loop.
//
// Lucid's concurrent sessions (viewport, F12 render, material previews: one
// Renderer each in the Blender add-on, render_session.py:77-106) become jobs
// of one server.  A job renders a whole image progressively on one of a few
// slots; each slot is an engine with its own CUDA stream sharing the
// uploaded scenes, so iterations of different jobs overlap on the device.
// Jobs are admitted in arrival order (interactive jobs ahead of batch jobs)
// as slots and device memory free up; a slot running a batch job also runs
// waiting interactive jobs between the batch job's iterations, on a second
// engine, so that they never wait for a long render
// (HBM budget = uploaded scenes + every running job's path state and film;
// slots keep their path pools between jobs, since freeing device memory
// synchronises the device, and the default budget leaves room for them);
// a job that could never fit is refused at submission.  Throughput jobs
// (not interactive, not guided) waiting together with the same integrator
// and depth run as one batch: one set of wavefront launches over a device
// job table (Engine::render_batch), up to a wave of paths.  The autotuner also
// picks the kernels' launch profile (resident CTAs per SM).  Scene edits make a
// new scene version; a job renders the version current when it was
// submitted.  Guided jobs (the "mis" integrator with online path guiding)
// train their own guide and count its buffers in their bytes.  Each slot picks the
// samples per iteration (the queue capacity of its waves) with a small
// autotuner and replays the iteration as a CUDA graph.  A job's image
// depends only on its own sample indices, so it is the same alone and in
// any mix, bit for bit, and equals one render call with all its samples.
#pragma once

#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lucid_cuda.h"

namespace lucid {

class Engine;
struct SceneSnapshot;

// FIFO admission under a byte budget: the head job starts when a slot is
// free and reserved + running + its bytes fit; a job larger than budget -
// reserved is refused.  Shared by the server and by the host-only planner.
struct Admission {
    long long budget = 0, reserved = 0, running = 0;
    int slots = 1, busy = 0;
    bool never_fits(long long bytes) const { return reserved + bytes > budget; }
    bool can_start(long long bytes) const { return busy < slots && reserved + running + bytes <= budget; }
    void start(long long bytes) { running += bytes; ++busy; }
    void finish(long long bytes) { running -= bytes; --busy; }
};

// The batch a slot forms when it takes `head` from the queue: the indices
// of the jobs of `queue` (the jobs waiting behind it, in queue order) that
// join it — throughput jobs (not interactive, not guided, not cancelled)
// with the head's integrator and depth, taken in order while the batch
// stays within max_paths paths (width * height * samples), the byte room
// left in the budget (Engine::batch_bytes) and max_jobs jobs.  An empty
// result: the head runs on its own.  `bytes` receives the batch's bytes.
// Shared by the server and by the host-only planner (lucid_batch_plan).
std::vector<int> plan_batch(const LucidJobDesc& head, const std::vector<const LucidJobDesc*>& queue,
                            const std::vector<char>& cancelled, long long max_paths, long long room_bytes,
                            int max_jobs, long long* bytes);

class Server {
public:
    Server(int device, int slots, long long budget_bytes);
    ~Server();
    int add_scene(const char* json, size_t len, int* scene_id);
    int add_scene_arrays(const LucidSceneDesc& desc, int* scene_id);
    int update_scene(int scene_id, const LucidSceneEdit* edits, int count);
    int submit(const LucidJobDesc& d, int* job_id);
    int state(int job, int* samples_done);
    int wait(int job, int timeout_ms);
    int result(int job, float* out, size_t cap_floats);
    int cancel(int job);
    int stats(LucidServerStats* out);
    // Batched throughput jobs: at most `max_paths` paths (samples x pixels)
    // per batch, 0 = every job its own launches.
    int set_batching(long long max_paths);
    const std::string& last_error() const { return err_; }
    int fail(int code, const std::string& m) { err_ = m; return code; }

private:
    struct Job {
        LucidJobDesc d{};
        int state = LUCID_JOB_QUEUED;
        int done = 0;
        long long bytes = 0;
        int chunk_max = 1;
        bool cancel = false;
        double t_submit = 0, t_start = 0, t_first = 0, t_end = 0;
        std::vector<float> image;
        std::string error;
        std::shared_ptr<SceneSnapshot> snap;   // the scene version current at submission
    };
    template <class Load>
    int add_scene_with(Load&& load, int* scene_id);
    void slot_loop(int slot);
    int run_job(Engine& e, Job& j, int slot, bool keep_pool);
    int run_guided_job(Engine& e, Job& j, int slot, bool keep_pool);
    int run_batch(Engine& e, const std::vector<Job*>& members);
    void finish_batch(const std::vector<Job*>& members, long long bytes, int rc);
    void finish_job(Job& j, int rc);
    void run_waiting_interactive(int slot);
    int pick_chunk(Engine& e, Job& j, int slot, int& offset);
    double now() const;

    int device_;
    long long budget_;
    std::vector<std::unique_ptr<Engine>> scenes_;
    std::vector<long long> scene_bytes_;
    std::vector<std::unique_ptr<Engine>> slot_eng_;
    std::vector<std::unique_ptr<Engine>> pre_eng_;   // per slot: interactive jobs run between batch iterations
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<int> queue_;
    std::map<int, Job> jobs_;
    std::map<std::string, std::pair<int, int>> tuned_;   // autotuned samples per iteration and launch profile
    Admission adm_;
    int next_id_ = 1;
    bool stop_ = false;
    double t0_ = 0, busy_from_ = -1, busy_to_ = 0;
    long long samples_done_ = 0;
    long long batch_paths_;
    int batches_ = 0, batched_jobs_ = 0;
    std::string err_;
};

}  // namespace lucid
