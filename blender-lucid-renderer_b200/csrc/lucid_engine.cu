// lucid_engine.cu — B200 wavefront path tracer: device LBVH build, persistent
// traversal, shading, shadow rays, film; host orchestration.
//
// Pipeline per wave (a block of (pixel, sample) paths, sample-major):
//   k_raygen                      seed PCG32 per (x, y, sample), jitter, primary ray
//   for depth in [0, max_depth):
//     k_trace   (persistent)      closest hit + native lights      -> hit SoA
//     k_shade   (persistent)      volume / emission / NEE / BSDF   -> next queue,
//                                                                     shadow queue
//     k_shadow  (persistent)      any-hit, adds unoccluded NEE
//   k_film                        per-pixel sum in sample order (deterministic)
// Queues are compacted with warp ballots + one atomic per warp.  Work counts
// stay on the device; the host enqueues a whole wave without synchronising.
#include <cooperative_groups.h>
#include <cooperative_groups/scan.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <future>
#include <cub/cub.cuh>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "lucid_diag.h"
#include "lucid_engine.h"
#include "lucid_guide.cuh"
#include "lucid_guide_host.h"
#include "lucid_kernels.cuh"

namespace lucid {
namespace cg = cooperative_groups;

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(e_ == cudaErrorMemoryAllocation ? LUCID_ERR_OOM     \
                                                                           : LUCID_ERR_CUDA,  \
                                           std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------- buffers
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count; else p = nullptr;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

struct DeviceScene {
    DBuf<float4> bvh_tris, bnd_tris, bnd_box, big_tris, prim_fn, prim_vn, light_bsph;
    DBuf<int4> prim_info;
    DBuf<unsigned char> prim_cls;
    DBuf<int> guide;
    DBuf<DevNode4> nodes;
    DBuf<DevNode> nodes2;
    DBuf<DevMaterial> materials;
    DBuf<float4> tex_ops, prim_uv;
    DBuf<DevLight> lights;
    DBuf<float> cdf, grid;
    DBuf<DevVolume> volumes;
    DevScene view{};
    // an edited version (Engine::update_scene) owns only its material, light
    // and class arrays and keeps the version whose geometry it renders alive
    std::shared_ptr<DeviceScene> base;
    void release() {
        base.reset();
        bvh_tris.release(); bnd_tris.release(); bnd_box.release(); light_bsph.release(); big_tris.release(); prim_fn.release(); prim_vn.release(); prim_info.release();
        prim_cls.release(); nodes.release(); nodes2.release(); guide.release(); materials.release(); tex_ops.release(); prim_uv.release(); lights.release(); cdf.release(); grid.release(); volumes.release();
    }
};

// Per-path SoA state, indexed by path id (sample-major within a wave).
struct PathView {
    ulonglong2* rng;   // PCG state, increment
    float4* ray_o;     // origin, tMin
    float4* ray_d;     // direction, depth (int bits)
    float4* thr;       // throughput rgb, pdf of the sampler that chose the ray
    float4* rad;       // accumulated radiance
    float4* hit;       // t, u, v, prim (int bits, -1 = miss)
    float2* lhit;      // native light index (int bits, -1 = none), t
    float4* sh_o;      // shadow ray origin, length
    float4* sh_d;      // shadow ray direction
    float4* sh_c;      // radiance added when unoccluded
    int* q0;
    int* q1;
    int* qs;
    int* qb;           // shading queue binned by event / material class
    unsigned short* cls;  // shading bin of each path's pending event
    int* counters;     // per depth: [0] active, [1] shadow, [2..4] fetch cursors,
                       // [8, 8 + kBins) bin counts, then kBins bin cursors
    int* errors;       // [0] traversal stack overflow
    int2* rec_prim;
    int4* rec_cnt;     // bounces, nee tests, nee occluded
    unsigned long long* rec_hash;
    // path guiding (null when off)
    float* gmix;       // compact guide mixture per path (k_guide_infer, kGMixFloats)
    int4* gslot;       // training records of the path's 3 latest guided vertices (-1: none)
    float4* ginv;      // 3 per path: 1 / throughput after each of those vertices
    GuideRec* grec;    // training records of this wave
    int* gcount;       // [0] records written, [1] guided vertices
    int gcap;
    unsigned gkeep;    // a guided vertex is recorded when its hash < gkeep
    int gdepth;        // vertices at path depth < gdepth are guided
    float glo[3], gscale[3];   // scene box -> [0,1]^3
    // batched jobs (null otherwise): the device table of the batch's scenes
    // and each path's index into it, set with its camera ray
    const DevScene* scenes;
    unsigned short* sid;
};
// Shading bins: the event / material class (bin_class, 16 values) times
// the cell of the hit point in a 4 x 4 x 4 grid over the scene box.
constexpr int kClassBins = 16;
constexpr int kCellBits = 2;                       // per axis
constexpr int kCellDim = 1 << kCellBits;
constexpr int kCells = 1 << (3 * kCellBits);
constexpr int kBins = kClassBins * kCells;
constexpr int kCountersPerDepth = 8 + 2 * kBins;
constexpr int kMaxDepth = 1024;

struct PathPool {
    long long cap = 0;
    bool records = false;
    DBuf<ulonglong2> rng;
    DBuf<float4> ray_o, ray_d, thr, rad, hit, sh_o, sh_d, sh_c;
    DBuf<float2> lhit;
    DBuf<int> q0, q1, qs, qb, counters, errors;
    DBuf<unsigned short> cls;
    DBuf<int2> rec_prim;
    DBuf<int4> rec_cnt;
    DBuf<unsigned long long> rec_hash;
    DBuf<float4> film;
    DBuf<float4> out;
    size_t film_n = 0;
    DBuf<double> film64, out64;   // FP64 accumulation (converged references)
    size_t film64_n = 0;
    DBuf<unsigned short> sid;     // batched jobs: scene index per path (render_batch)
    DBuf<unsigned char> btab;     // batched jobs: the scene table, then a wave's job table
    PathView view{};
    void release() {
        sid.release();
        btab.release();
        rng.release(); ray_o.release(); ray_d.release(); thr.release(); rad.release(); hit.release();
        sh_o.release(); sh_d.release(); sh_c.release(); lhit.release(); q0.release(); q1.release(); qs.release();
        qb.release(); cls.release();
        counters.release(); errors.release(); rec_prim.release(); rec_cnt.release(); rec_hash.release();
        film.release(); out.release(); film64.release(); out64.release();
        film_n = 0;
        film64_n = 0;
        cap = 0;
    }
};

// Path guiding: the network and the per-path / per-wave buffers.
constexpr int kGuideBatch = 1 << 18;   // training records per step
constexpr long long kGuideWave = 1LL << 24;
struct GuideState {
    GuideNet net;
    DBuf<float> gmix;
    DBuf<int4> gslot;
    DBuf<float4> ginv;
    DBuf<GuideRec> recs;
    DBuf<int> count;
    long long cap = 0;
    float keep = 1.0f;
    float lr = 1e-2f;
    int steps = 2;   // Adam steps per wave, each on its own batch of records
    int max_depth = 1;   // vertices at path depth < max_depth are guided (camera hits: depth 0)
    bool on = false;
};

// Completed-path records of the path diagnostics (compact form: 16-B units
// and an index of each record's first unit) and their counts.
struct DiagDevice {
    DBuf<uint4> units;
    DBuf<uint32_t> index;
    DBuf<unsigned long long> count;   // [0] records, [1] units
    // pinned host copies of a band's records, two of them: the host replays
    // one band while the device renders the next into the other (kept
    // between calls: page-locked copies run at full link speed and the
    // buffers are not zero-filled)
    uint8_t* host_units[2] = {nullptr, nullptr};
    uint32_t* host_index[2] = {nullptr, nullptr};
    size_t host_units_cap[2] = {0, 0}, host_index_cap[2] = {0, 0};
    ~DiagDevice() {
        for (int b = 0; b < 2; ++b) {
            if (host_units[b]) cudaFreeHost(host_units[b]);
            if (host_index[b]) cudaFreeHost(host_index[b]);
        }
    }
    // grows a pinned buffer of `elem`-byte entries to hold n, keeping the first `keep`
    template <typename T>
    static cudaError_t grow(T*& buf, size_t& cap, size_t n, size_t keep, size_t elem) {
        if (n <= cap) return cudaSuccess;
        const size_t c = n + n / 4;
        T* h = nullptr;
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&h), c * elem, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        if (buf && keep) std::memcpy(h, buf, keep * elem);
        if (buf) cudaFreeHost(buf);
        buf = h;
        cap = c;
        return cudaSuccess;
    }
    cudaError_t reserve_host(int b, size_t n_rec, size_t keep_rec, size_t n_units, size_t keep_units) {
        cudaError_t e = grow(host_index[b], host_index_cap[b], n_rec, keep_rec, sizeof(uint32_t));
        if (e != cudaSuccess) return e;
        return grow(host_units[b], host_units_cap[b], n_units, keep_units, kDiagUnitBytes);
    }
};

struct FrameParams {
    float pos[3], fwd[3], right[3], up[3];
    float aspect, scale;
    int tile_x, tile_y, tile_w, tile_h, full_w, full_h;
    int samples, sample_offset, max_depth, algo;
    int npix;
    int s0;          // first sample (within the call) of this wave
    int n_wave;      // paths in this wave
    int records;
    int jitter;      // jitter camera rays even when `samples` is 1 (progressive jobs)
    const int* dyn;  // when set, dyn[0] replaces sample_offset (graph-replayed iterations)
};

// ---------------------------------------------------------------- warp helpers
LD unsigned lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated append: one atomic per warp, ranks from the ballot.
LD void warp_append(int* queue, int* counter, int value, bool pred) {
    unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0) return;
    int leader = __ffs(mask) - 1;
    int base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) queue[base + __popc(mask & ((1u << lane_id()) - 1u))] = value;
}

// Persistent-thread work fetch: a warp claims 32 consecutive items.
LD int warp_fetch(int* cursor) {
    int base = 0;
    if (lane_id() == 0) base = atomicAdd(cursor, 32);
    return __shfl_sync(0xffffffffu, base, 0);
}

// ---------------------------------------------------------------- raygen
LD V3 primary_dir(const FrameParams& f, float nx, float ny) {
    V3 v = v3(f.fwd[0] + f.right[0] * (nx * f.scale) + f.up[0] * (ny * f.scale),
              f.fwd[1] + f.right[1] * (nx * f.scale) + f.up[1] * (ny * f.scale),
              f.fwd[2] + f.right[2] * (nx * f.scale) + f.up[2] * (ny * f.scale));
    return make_dir_or(v, v3(f.fwd[0], f.fwd[1], f.fwd[2]));
}

// Primary ray of wave path `id` (pybind_renderer.hpp:250-293): NDC, seed
// (x, y, offset + s), two jitter draws when the call has more than one
// sample; writes the path's initial state and returns the direction (the
// origin is the camera position, tMin 0).
LD V3 camera_ray_at(const FrameParams& f, const PathView& pv, int local, int id);
LD V3 camera_ray(const FrameParams& f, const PathView& pv, int id) { return camera_ray_at(f, pv, id, id); }

// The same for path `local` of the frame `f` stored at wave path `id`
// (a batched job's paths start at its base in the wave).
LD V3 camera_ray_at(const FrameParams& f, const PathView& pv, int local, int id) {
    int p = local % f.npix, sl = local / f.npix;
    int gx = f.tile_x + p % f.tile_w, gy = f.tile_y + p / f.tile_w;
    float nx = (2.0f * ((float)gx + 0.5f) / (float)f.full_w - 1.0f) * f.aspect;
    float ny = 1.0f - 2.0f * ((float)gy + 0.5f) / (float)f.full_h;
    const int offset = f.dyn ? f.dyn[0] : f.sample_offset;
    Rng rng = seed_xyz((uint32_t)gx, (uint32_t)gy, (uint32_t)(offset + f.s0 + sl));
    V3 d;
    if (f.samples > 1 || f.jitter) {
        float jx = (randf(rng) - 0.5f) / (float)f.full_w;
        float jy = (randf(rng) - 0.5f) / (float)f.full_h;
        d = primary_dir(f, nx + jx, ny + jy);
    } else {
        d = primary_dir(f, nx, ny);
    }
    pv.rng[id] = make_ulonglong2(rng.state, rng.inc);
    pv.ray_o[id] = make_float4(f.pos[0], f.pos[1], f.pos[2], 0.0f);
    pv.ray_d[id] = make_float4(d.x, d.y, d.z, __int_as_float(0));
    pv.thr[id] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    pv.rad[id] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (f.records) {
        pv.rec_prim[id] = make_int2(-1, -1);
        pv.rec_cnt[id] = make_int4(0, 0, 0, 0);
        pv.rec_hash[id] = 1469598103934665603ULL;
    }
    return d;
}

// Primary rays alone, for the passes that do not trace them at once.
__global__ void k_raygen(FrameParams f, PathView pv) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id == 0) pv.counters[0] = f.n_wave;
    if (id >= f.n_wave) return;
    camera_ray(f, pv, id);
}

// ---------------------------------------------------------------- trace
// closest hit: descend/test rounds per lane between refills (five frames on
// the 1M-triangle scene: 3 -> 321 ms, 4 -> 317 ms, 6 -> 362 ms)
constexpr int kRounds = 4;
// any hit: node visits per lane between refills (6: 3x slower; five frames:
// 16 -> 229.7 ms, 24 -> 231.9 ms, 32 -> 240.4 ms)
constexpr int kShadowSteps = 16;

LD unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// Per-lane dynamic refill: lanes without a ray claim new ones together (one
// atomic per warp per round); `exhausted` stops claiming once the queue is
// drained.  Returns the claimed index or -1.
LD int refill(int* cursor, int n, bool need, bool& exhausted) {
    unsigned m = __ballot_sync(0xffffffffu, need && !exhausted);
    if (m == 0) return -1;
    int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(cursor, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!(need && !exhausted)) return -1;
    int r = base + __popc(m & lanemask_lt());
    if (r >= n) { exhausted = true; return -1; }
    return r;
}

// ---------------------------------------------------------------- shading bins
// The shading kernel is limited by instruction fetch: divergent warps run
// different parts of it (light/environment hits, emitters, glass, near-delta
// metal, general Principled lobes, volume delta tracking).  Before each
// shading launch the queue is binned by that class — a counting sort whose
// histogram the trace kernels build as each ray finishes (the hit, the
// native-light hit and the ray are still in registers there) and whose
// scatter pass is k_bin_scatter — so neighbouring warps shade the same kind
// of event.  The order of paths in a queue does not change any result.
LD int bin_class(const DevScene& sc, int prim, float t, int li, float lt, V3 o, V3 d, bool vol) {
    // 0: light or environment reached; else the prim's material class
    // (emitter, glass, near-delta metal, metal, dielectric), set at upload
    int c = (prim >= 0 && !(li >= 0 && lt < t)) ? (int)__ldg(sc.prim_cls + prim) : 0;
    if (vol && sc.num_volumes > 0) {
        float ts = 1e6f;
        if (prim >= 0) ts = smin(ts, t);
        if (li >= 0) ts = smin(ts, lt);
        for (int k = 0; k < sc.num_volumes && k < 4; ++k) {
            float te, tx;
            if (ray_aabb_segment(o, d, ts, sc.volumes[k], te, tx)) { c += 8; break; }
        }
    }
    return c;
}

// Cell of a surface hit point: its Morton index in the kCellDim^3 grid over
// the scene box, so that neighbouring bins hold neighbouring cells.  Paths
// shaded in bin order hand the trace and shadow kernels rays whose origins
// lie close together (neighbouring lanes then walk similar BVH nodes).
LD int bin_cell(const DevScene& sc, V3 p) {
    const float c[3] = {p.x, p.y, p.z};
    int m = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int q = (int)((c[a] - sc.bin_lo[a]) * sc.bin_scale[a]);
        q = min(max(q, 0), kCellDim - 1);
#pragma unroll
        for (int b = 0; b < kCellBits; ++b) m |= ((q >> b) & 1) << (3 * b + a);
    }
    return m;
}

// Per-block histogram of the shading bins of the rays a trace kernel
// finished, flushed to the depth's bin counters when the block ends.  bins
// < 0: no binning; else a set of kBin* flags: the volume bit of the class,
// and the hit-point cell (without it every ray of a class takes cell 0).
// The cells pay off on large waves only: each block flushes up to kBins
// counters, which a small wave (a few thousand rays per block) does not
// amortise (a 256x256 16-spp Cornell render: 546 M samples/s without the
// cells, 478 M with them; the 1M-triangle 1080p frame gains 1.5 % with
// them).
constexpr int kBinVolume = 1, kBinCells = 2;
constexpr long long kCellBinPaths = 1LL << 24;   // waves from this size on use the cells
struct BinHist {
    int* h;
    LD void clear(int bins) {
        if (bins >= 0)
            for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
        __syncthreads();
    }
    LD void add(const DevScene& sc, const PathView& pv, int id, int bins, int prim, float t, int li, float lt, V3 o,
                V3 d) {
        if (bins < 0) return;
        const int c = bin_class(sc, prim, t, li, lt, o, d, (bins & kBinVolume) != 0);
        const int key = c * kCells + ((bins & kBinCells) && (c & 7) != 0 ? bin_cell(sc, o + d * t) : 0);
        pv.cls[id] = (unsigned short)key;
        atomicAdd(&h[key], 1);
    }
    LD void flush(int bins, int* cnt) {
        if (bins < 0) return;
        __syncthreads();
        for (int i = threadIdx.x; i < kBins; i += blockDim.x)
            if (h[i]) atomicAdd(&cnt[8 + i], h[i]);
    }
};

// Camera rays, generated and traced in one pass: neighbouring pixels trace
// similar paths, so a warp claims 32 consecutive rays at a time and keeps
// them together.  Also publishes the wave's path count as the depth-0 queue
// length for the kernels after it.
template <bool FMA>
__global__ void __launch_bounds__(128) k_trace_primary_t(DevScene sc, FrameParams f, PathView pv, int* cnt,
                                                       int records, int bins) {
    __shared__ int hist[kBins];
    BinHist bh{hist};
    bh.clear(bins);
    const int n = f.n_wave;
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[0] = n;
    const V3 o = v3(f.pos[0], f.pos[1], f.pos[2]);
    // a warp traces the 8 x 4 pixels of one screen tile (one sample each):
    // a compact footprint keeps its lanes on the same BVH nodes longer than
    // a 32-pixel row.  Slots run over the tiles of the first sample, then of
    // the next; lanes past the tile's edge idle.
    const int tiles_x = (f.tile_w + 7) / 8, tiles_y = (f.tile_h + 3) / 4;
    const long long per_sample = (long long)tiles_x * tiles_y * 32;
    const long long slots = per_sample * (long long)(n / max(f.npix, 1));
    const int lane = (int)lane_id();
    bool ok = true;
    for (;;) {
        const int base = warp_fetch(&cnt[2]);
        if (base >= slots) break;
        const long long slot = (long long)base + lane;
        const int sl = (int)(slot / per_sample), tile = (int)((slot % per_sample) >> 5);
        const int px = (tile % tiles_x) * 8 + (lane & 7), py = (tile / tiles_x) * 4 + (lane >> 3);
        if (slot >= slots || px >= f.tile_w || py >= f.tile_h) continue;
        const int id = sl * f.npix + py * f.tile_w + px;
        const V3 d = camera_ray(f, pv, id);
        HitRec h = closest_skip_boundaries<FMA>(sc, o, d, 0.0f, ok);
        if (h.prim < 0) { h.t = 1e30f; h.u = 0.0f; h.v = 0.0f; }
        pv.hit[id] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
        pv.lhit[id] = make_float2(__int_as_float(-1), 1e30f);   // native lights are invisible to camera rays
        bh.add(sc, pv, id, bins, h.prim, h.t, -1, 1e30f, o, d);
        if (records) {
            int4 pi = h.prim >= 0 ? sc.prim_info[h.prim] : make_int4(-1, -1, -1, 0);
            pv.rec_prim[id] = make_int2(pi.x, pi.y);
            pv.rec_cnt[id].x += 1;
            unsigned long long hs = pv.rec_hash[id];
            hs = hpush(hs, (uint32_t)pi.x);
            hs = hpush(hs, (uint32_t)pi.y);
            hs = hpush(hs, 0xffffffffu);
            pv.rec_hash[id] = hs;
        }
    }
    bh.flush(bins, cnt);
    if (!ok) atomicAdd(&pv.errors[0], 1);
}

// Camera rays take the FMA slab test when the camera lies within the
// scene's coordinate bound (its error analysis then holds as for secondary
// rays), else the subtraction form.
using PrimaryKernel = void (*)(DevScene, FrameParams, PathView, int*, int, int);
static PrimaryKernel k_trace_primary_for(const DevScene& sc, const float pos[3]) {
    const float m = std::max(std::fabs(pos[0]), std::max(std::fabs(pos[1]), std::fabs(pos[2])));
    return m <= sc.coord_bound ? k_trace_primary_t<true> : k_trace_primary_t<false>;
}

// ---------------------------------------------------------------- batched jobs
// One entry of the device job table of a batch wave: a piece of one job (a
// range of its samples) with its camera and image (f: s0 = the piece's first
// sample, n_wave = its paths), the scene it renders (index into the wave's
// scene table), where its paths start in the wave, and where its camera-ray
// slots start (each piece has whole warps of slots: 8 x 4 pixel tiles per
// sample).
struct BatchJob {
    FrameParams f;
    int sid;
    int path_base;
    int slot_base;
    int pad;
};
constexpr int kMaxBatchPieces = 1024;

// Camera rays of a batch wave, generated and traced in one pass over every
// piece: a warp's 32 slots lie in one piece (found by binary search over the
// slot bases, staged in shared memory), whose camera and sample range give
// the rays and whose scene the rays are traced in.  Each path's scene index
// is stored for the kernels after this one.  The subtraction form of the
// slab test is used throughout (the FMA form's error bound needs the camera
// inside its scene's coordinate bound, which varies from job to job); both
// give the same hits.
__global__ void __launch_bounds__(128) k_trace_primary_batch(PathView pv, const BatchJob* jobs, int njobs, int slots,
                                                           int n, int* cnt, int bins) {
    __shared__ int hist[kBins];
    __shared__ int sbase[kMaxBatchPieces];
    for (int i = threadIdx.x; i < njobs; i += blockDim.x) sbase[i] = jobs[i].slot_base;
    BinHist bh{hist};
    bh.clear(bins);   // ends with a block barrier, which also publishes sbase
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[0] = n;
    const int lane = (int)lane_id();
    bool ok = true;
    for (;;) {
        const int base = warp_fetch(&cnt[2]);
        if (base >= slots) break;
        int lo = 0, hi = njobs - 1;   // the last piece whose slots start at or before base
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sbase[mid] <= base) lo = mid; else hi = mid - 1;
        }
        const BatchJob& J = jobs[lo];
        const FrameParams& f = J.f;
        const int tw = f.tile_w, th = f.tile_h;
        const int tiles_x = (tw + 7) / 8, tiles_y = (th + 3) / 4;
        const int per_sample = tiles_x * tiles_y * 32;
        const int slot = base - sbase[lo] + lane;
        const int sl = slot / per_sample, tile = (slot % per_sample) >> 5;
        const int px = (tile % tiles_x) * 8 + (lane & 7), py = (tile / tiles_x) * 4 + (lane >> 3);
        if (px >= tw || py >= th) continue;
        const int local = sl * f.npix + py * tw + px;
        const int id = J.path_base + local;
        const int sid = J.sid;
        const DevScene& sc = pv.scenes[sid];
        const V3 d = camera_ray_at(f, pv, local, id);
        const V3 o = v3(f.pos[0], f.pos[1], f.pos[2]);
        pv.sid[id] = (unsigned short)sid;
        HitRec h = closest_skip_boundaries<false>(sc, o, d, 0.0f, ok);
        if (h.prim < 0) { h.t = 1e30f; h.u = 0.0f; h.v = 0.0f; }
        pv.hit[id] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
        pv.lhit[id] = make_float2(__int_as_float(-1), 1e30f);   // native lights are invisible to camera rays
        bh.add(sc, pv, id, bins, h.prim, h.t, -1, 1e30f, o, d);
    }
    bh.flush(bins, cnt);
    if (!ok) atomicAdd(&pv.errors[0], 1);
}

// The scene of path `id`: the kernel's scene, or in a batch wave the entry
// of the wave's scene table the path's camera ray chose.
template <bool MULTI>
LD const DevScene& path_scene(const DevScene& sc, const PathView& pv, int id) {
    if constexpr (MULTI) return pv.scenes[pv.sid[id]];
    else return sc;
}

// Closest hit of extension rays (persistent, dynamic refill), including the
// skip-volume-boundary rule (path_tracer.hpp:82-95) and native lights.
// Nine resident CTAs per SM (at most 56 registers): one more warp group to
// hide node-fetch latency than the unconstrained 61 registers allow
// (1M-triangle scene: 8 CTAs 232 ms, 9 CTAs 221 ms, 10 CTAs 225 ms).
template <int MINB, bool MULTI = false>
__global__ void __launch_bounds__(128, MINB) k_trace_lb(DevScene sc0, PathView pv, int* cnt, int identity, int records,
                                                      int bins) {
    __shared__ int hist[kBins];
    BinHist bh{hist};
    bh.clear(bins);
    const int n = *(volatile int*)&cnt[0];
    const int* q = identity ? nullptr : pv.q0;
    int stack[kStack];
    float stack_t[kStack];
    Trav s;
    bool active = false, exhausted = false, ok = true;
    int id = 0, depth = 0, peek = 0, sid = 0;
    float search = 0.0f;
    // the lane's scene: the kernel's, or in a batch wave its ray's entry of
    // the wave's scene table (kept in a register between refills)
    auto scene = [&]() -> const DevScene& {
        if constexpr (MULTI) return pv.scenes[sid];
        else return sc0;
    };
    for (;;) {
        int r = refill(&cnt[2], n, !active, exhausted);
        if (r >= 0) {
            id = q ? q[r] : r;
            if constexpr (MULTI) sid = pv.sid[id];
            const DevScene& sc = scene();
            float4 ro = pv.ray_o[id], rd = pv.ray_d[id];
            depth = __float_as_int(rd.w);
            trav_begin<false>(s, sc, f3(ro), f3(rd), ro.w, 1e30f);
            search = ro.w;
            peek = 0;
            active = true;
        }
        if (__ballot_sync(0xffffffffu, active) == 0) break;
        if (!active) continue;
        const DevScene& sc = scene();
        if (!trav_run<false>(s, stack, stack_t, sc, ok, kRounds)) continue;
        HitRec res = s.h;
        if (sc.num_bnd_tris) {
            // resolve the closest real surface against boundary-only hits
            bool restart = false;
            for (;;) {
                HitRec real = s.h;
                HitRec b = real;
                if (real.prim < 0) b.t = 1e30f;
                boundary_closest<true>(sc, s.o, s.d, s.inv, search, b);
                if (b.prim < 0) { res.prim = -1; res.t = 1e30f; break; }
                if (b.prim == real.prim) { res = real; break; }
                search = b.t + 1e-3f;
                if (++peek == 8) { res.prim = -1; res.t = 1e30f; break; }
                if (real.prim >= 0 && real.t < search) {
                    trav_begin<false>(s, sc, s.o, s.d, search, 1e30f);
                    restart = true;
                    break;
                }
            }
            if (restart) continue;
        }
        if (res.prim < 0) { res.t = 1e30f; res.u = 0.0f; res.v = 0.0f; }
        float lt = 1e30f;
        // a native light counts only in front of the surface hit (the shading
        // kernel's `lh.y < hh.x`): lights beyond it are not tested
        int li = (depth == 0) ? -1 : native_lights_closest(sc, s.o, s.d, res.t, lt);
        pv.hit[id] = make_float4(res.t, res.u, res.v, __int_as_float(res.prim));
        pv.lhit[id] = make_float2(__int_as_float(li), lt);
        bh.add(sc, pv, id, bins, res.prim, res.t, li, lt, s.o, s.d);
        if (records) {
            int4 pi = res.prim >= 0 ? sc.prim_info[res.prim] : make_int4(-1, -1, -1, 0);
            if (depth == 0) pv.rec_prim[id] = make_int2(pi.x, pi.y);
            pv.rec_cnt[id].x += 1;
            unsigned long long hs = pv.rec_hash[id];
            hs = hpush(hs, (uint32_t)pi.x);
            hs = hpush(hs, (uint32_t)pi.y);
            hs = hpush(hs, (uint32_t)li);
            pv.rec_hash[id] = hs;
        }
        active = false;
    }
    bh.flush(bins, cnt);
    if (!ok) atomicAdd(&pv.errors[0], 1);
}

// ---------------------------------------------------------------- shade
struct ShadeResult {
    bool cont, shadow;
};

// One path segment: volume sampling, native-light / environment / emission
// terms, NEE, BSDF sampling and Russian roulette.  ALGO is the integrator as
// a compile-time constant, so each integrator's kernel carries only its own
// branches.
// Adds a radiance contribution c (already weighted by the path throughput)
// to the training records of the path's guided vertices from slot `from` on
// (c / throughput-after-vertex = radiance that arrived along its sample).
LD void guide_credit(const PathView& pv, int id, RGB c, int from) {
    int4 s = pv.gslot[id];
    const int r[3] = {s.x, s.y, s.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k < from || r[k] < 0) continue;
        float4 iv = pv.ginv[3 * id + k];
        GuideRec& g = pv.grec[r[k]];
        g.L[0] += c.r * iv.x; g.L[1] += c.g * iv.y; g.L[2] += c.b * iv.z;
    }
}

// Hit UV (bvh.hpp:67-72): the triangle's UVs at the hit's barycentrics,
// (0, 0) when it has none.
LD void hit_uv(const DevScene& sc, int prim, float bu, float bv, float& su, float& sv) {
    su = 0.0f;
    sv = 0.0f;
    if (!sc.prim_uv) return;
    const float4 a = sc.prim_uv[2 * prim], b = sc.prim_uv[2 * prim + 1];
    if (b.z == 0.0f) return;
    const float w = 1.0f - bu - bv;
    su = a.x * w + a.z * bu + b.x * bv;
    sv = a.y * w + a.w * bu + b.y * bv;
}

// A material node program (the loader's folding, lucid_nodes.cpp, in the
// same float operations) at (u, v).  Out of line: only textured materials
// run it, and its step array stays out of the shading kernels' frames.
static __device__ __noinline__ RGB tex_eval(const float4* ops, int start, int n, float u, float v) {
    float val[kTexMaxOps][3];
    n = min(n, kTexMaxOps);
    for (int i = 0; i < n; ++i) {
        const float4 s0 = ops[2 * (start + i)], s1 = ops[2 * (start + i) + 1];
        const int kind = __float_as_int(s0.x), a = __float_as_int(s0.y), b = __float_as_int(s0.z);
        const float k = s0.w;
        if (kind == TEX_CONST) {
            val[i][0] = s1.x; val[i][1] = s1.y; val[i][2] = s1.z;
        } else if (kind == TEX_CHECKER) {   // node_evaluator.cpp:385-396
            int cu = (int)floorf(u * k) % 2, cv = (int)floorf(v * k) % 2;
            if (cu < 0) cu += 2;
            if (cv < 0) cv += 2;
            const int src = (cu + cv) % 2 == 0 ? a : b;
            for (int c = 0; c < 3; ++c) val[i][c] = val[src][c];
        } else if (kind == TEX_MIX) {
            for (int c = 0; c < 3; ++c) val[i][c] = val[a][c] * (1.0f - k) + val[b][c] * k;
        } else {
            for (int c = 0; c < 3; ++c) val[i][c] = val[a][c] * k;
        }
    }
    return n > 0 ? rgb(val[n - 1][0], val[n - 1][1], val[n - 1][2]) : rgb(0.0f, 0.0f, 0.0f);
}

// Albedo and emission of a textured material at the hit (getMaterialParams
// / getEmission, integrator/path_tracer.hpp:45-72); the other parameters
// are constants of the material.
LD void apply_textures(const DevScene& sc, const DevMaterial& dm, int prim, float bu, float bv, RGB& albedo, RGB& em,
                       bool& has_em) {
    if (!(__float_as_int(dm.rough_trans_ior_flags.w) & MAT_TEXTURED)) return;
    float u, v;
    hit_uv(sc, prim, bu, bv, u, v);
    if (dm.program.y > 0) albedo = tex_eval(sc.tex_ops, dm.program.x, dm.program.y, u, v);
    if (dm.program.w > 0) {
        em = tex_eval(sc.tex_ops, dm.program.z, dm.program.w, u, v);
        has_em = (0.2126f * em.r + 0.7152f * em.g + 0.0722f * em.b) > 1e-6f;
    }
}

// A surface the guide may sample: no transmission lobe and not the
// near-delta metal that sample_bsdf weights in closed form.
LD bool guide_eligible(const DevMaterial& dm) {
    float rough = smax(dm.rough_trans_ior_flags.x, MIN_ROUGHNESS);
    return dm.rough_trans_ior_flags.y == 0.0f && !(rough < 0.05f && dm.albedo_metallic.w > 0.5f);
}

template <int ALGO, bool GUIDE = false>
LD ShadeResult shade_path(const DevScene& sc, const FrameParams& f, const PathView& pv, int id) {
    ShadeResult out;
    out.cont = false;
    out.shadow = false;
    int pushed = 0;
    constexpr int algo = ALGO;
    constexpr bool nee = algo == ALGO_NEE || algo == ALGO_MIS || algo == ALGO_VOLUME_MIS;
    constexpr bool mis = algo == ALGO_MIS || algo == ALGO_VOLUME_MIS;
    float4 ro = pv.ray_o[id], rd = pv.ray_d[id];
    V3 o = f3(ro), d = f3(rd);
    int depth = __float_as_int(rd.w);
    float4 th = pv.thr[id];
    RGB T = c3(th);
    float last_pdf = th.w;
    RGB result = c3(pv.rad[id]);
    ulonglong2 rs = pv.rng[id];
    Rng rng;
    rng.state = rs.x;
    rng.inc = rs.y;
    float4 hh = pv.hit[id];
    int prim = __float_as_int(hh.w);
    bool has_hit = prim >= 0;
    float2 lh = pv.lhit[id];
    int lidx = __float_as_int(lh.x);
    bool has_lh = lidx >= 0;
    V3 new_o = o, new_d = d;
    V3 sh_o = o, sh_d = d;
    float sh_len = 0.0f;
    RGB sh_inc = rgb(0.f, 0.f, 0.f);

    do {
        if (algo == ALGO_VOLUME_SIMPLE) {
            float ts = 1e6f;
            if (has_hit) ts = smin(ts, hh.x);
            if (has_lh) ts = smin(ts, lh.y);
            T = mul(T, volume_transmittance(sc, o, d, ts, false));
        }
        if (algo == ALGO_VOLUME_MIS) {
            float ts = 1e6f;
            if (has_hit) ts = smin(ts, hh.x);
            if (has_lh) ts = smin(ts, lh.y);
            float vt = 0.0f;
            int vi = sample_volume_distance(sc, o, d, ts, rng, vt);
            if (f.records) pv.rec_hash[id] = hpush(pv.rec_hash[id], vi >= 0 ? 1u : 0u);
            if (vi >= 0) {
                // scatter event (path_tracer.hpp:616-700)
                const DevVolume& v = sc.volumes[vi];
                T = mul(T, rgb(v.color[0] / (1.0f + v.absorption[0]), v.color[1] / (1.0f + v.absorption[1]),
                               v.color[2] / (1.0f + v.absorption[2])));
                V3 x = o + d * vt;
                V3 wo = -d;
                float g = v.anisotropy;
                if (sc.num_lights > 0) {
                    float usel = randf(rng);
                    int li = select_light(sc, usel);
                    const DevLight& L = sc.lights[li];
                    float lsp = area_ratio(L.normal_area.w, sc.total_light_area);
                    if (lsp > 1e-6f) {
                        float u1 = randf(rng), u2 = randf(rng);
                        LightSample ls = sample_light(L, x, u1, u2);
                        if (ls.pdf > MIN_PDF) {
                            RGB Tsh = volume_transmittance(sc, x, ls.dir, ls.dist, true);
                            float ct = dot(wo, ls.dir);
                            float pe = hg_eval(g, ct);
                            float pl = ls.pdf * lsp;
                            float mw = mis_power(pl, pe);
                            RGB pw = bsdf_weight(rgb(pe, pe, pe), 1.0f, pl);
                            RGB c = mul(pw * mw, mul(Tsh, ls.emission));
                            sh_inc = mul(T, c);
                            sh_o = x; sh_d = ls.dir; sh_len = ls.dist;
                            out.shadow = true;
                        }
                    }
                }
                float u1 = randf(rng), u2 = randf(rng);
                float ppdf;
                V3 wi = hg_sample(g, wo, u1, u2, ppdf);
                last_pdf = ppdf;
                new_o = x; new_d = wi;
                if (depth >= 3) {
                    float rr = smin(smax3(T.r, T.g, T.b), 0.95f);
                    if (randf(rng) > rr) break;
                    T = T * (1.0f / rr);
                }
                if (!rgb_valid(T)) break;
                out.cont = true;
                break;
            }
        }
        if (has_lh && (!has_hit || lh.y < hh.x)) {
            // native light hit (path_tracer.hpp:429-452)
            const DevLight& L = sc.lights[sc.native_start + lidx];
            RGB em = c3(L.emission_radius);
            if (mis) {
                float lpdf = 0.0f;
                if (sc.num_lights > 0) {
                    float sp = area_ratio(L.normal_area.w, sc.total_light_area);
                    if (sp > 0.0f) {
                        V3 lp = o + d * lh.y;
                        V3 ln = (__float_as_int(L.pos_type.w) == LIGHT_POINT) ? normalize_nz(lp - f3(L.pos_type))
                                                                              : f3(L.normal_area);
                        lpdf = pdf_light(L.normal_area.w, o, lp, ln) * sp;
                    }
                }
                float mw = (last_pdf > MIN_PDF && lpdf > MIN_PDF) ? mis_power(last_pdf, lpdf) : 1.0f;
                result = result + mul(T, em) * mw;
                if (GUIDE) guide_credit(pv, id, mul(T, em) * mw, 0);
            } else {
                result = result + mul(T, em);
            }
            break;
        }
        if (!has_hit) {
            result = result + mul(T, rgb(sc.env[0], sc.env[1], sc.env[2]));
            if (GUIDE) guide_credit(pv, id, mul(T, rgb(sc.env[0], sc.env[1], sc.env[2])), 0);
            break;
        }
        // surface hit: point and normal from (t, u, v, prim) as in bvh.hpp:108-128
        V3 p = o + d * hh.x;
        int4 pi = sc.prim_info[prim];
        V3 fn = f3(sc.prim_fn[prim]);
        V3 n = fn;
        if (pi.w) {
            float u = hh.y, v = hh.z;
            float w = 1.0f - u - v;
            V3 ni = f3(sc.prim_vn[3 * prim]) * w + f3(sc.prim_vn[3 * prim + 1]) * u + f3(sc.prim_vn[3 * prim + 2]) * v;
            n = make_dir_or(ni, fn);
        }
        const DevMaterial& dm = sc.materials[pi.x];
        Mat m;
        m.albedo = c3(dm.albedo_metallic);
        m.metallic = dm.albedo_metallic.w;
        m.roughness = smax(dm.rough_trans_ior_flags.x, MIN_ROUGHNESS);
        m.transmission = dm.rough_trans_ior_flags.y;
        m.ior = dm.rough_trans_ior_flags.z;
        RGB em = c3(dm.emission);
        bool has_em = dm.emission.w != 0.0f;
        apply_textures(sc, dm, prim, hh.y, hh.z, m.albedo, em, has_em);
        V3 wo = -d;
        bool front = dot(wo, n) > 0;
        V3 sn = n;
        if (m.transmission < 0.5f && !front) sn = -n;
        if (!nee) {
            result = result + mul(T, em);
        } else if (!mis) {
            if (has_em && depth == 0) result = result + mul(T, em);
        } else if (has_em) {
            float mw = 1.0f;
            if (sc.num_lights > 0 && last_pdf > MIN_PDF && pi.z >= 0) {
                const DevLight& L = sc.lights[pi.z];
                float sp = area_ratio(L.normal_area.w, sc.total_light_area);
                if (sp > 0.0f) {
                    float lpdf = pdf_light(L.normal_area.w, o, p, n) * sp;
                    if (lpdf > MIN_PDF) mw = mis_power(last_pdf, lpdf);
                }
            }
            result = result + mul(T, em) * mw;
            if (GUIDE) guide_credit(pv, id, mul(T, em) * mw, 0);
        }
        bool transmissive = m.transmission > 0.5f;
        const bool guided = GUIDE && depth < pv.gdepth && guide_eligible(dm);
        const float* gm = GUIDE ? pv.gmix + (size_t)id * kGMixFloats : nullptr;
        if (nee && sc.num_lights > 0 && !has_em && !transmissive) {
            float usel = randf(rng);
            int li = select_light(sc, usel);
            const DevLight& L = sc.lights[li];
            float lsp = area_ratio(L.normal_area.w, sc.total_light_area);
            if (lsp > 1e-6f) {
                float u1 = randf(rng), u2 = randf(rng);
                LightSample ls = sample_light(L, p, u1, u2);
                if (ls.pdf > MIN_PDF) {
                    float nl = dot(sn, ls.dir);
                    if (nl > 1e-6f) {
                        RGB fb = eval_bsdf(m, wo, ls.dir, sn);
                        float pl = ls.pdf * lsp;
                        RGB c;
                        if (mis) {
                            float pb = pdf_bsdf(m, wo, ls.dir, sn);
                            if (guided) pb = 0.5f * pb + 0.5f * guide_pdf_c(gm, ls.dir);
                            float mw = mis_power(pl, pb);
                            RGB bw = bsdf_weight(fb, nl, pl);
                            if (algo == ALGO_VOLUME_MIS) {
                                RGB Tsh = volume_transmittance(sc, p, ls.dir, ls.dist, true);
                                c = mul(bw * mw, mul(Tsh, ls.emission));
                            } else {
                                c = mul(bw * mw, ls.emission);
                            }
                        } else {
                            c = mul(bsdf_weight(fb, nl, pl), ls.emission);
                        }
                        sh_inc = mul(T, c);
                        sh_o = p; sh_d = ls.dir; sh_len = ls.dist;
                        out.shadow = true;
                    }
                }
            }
        }
        V3 smp_n = (m.transmission > 0.5f) ? n : sn;
        V3 wi;
        float gpdf = 0.0f;
        if (guided) {
            // one-sample MIS of BSDF and guide sampling, 1/2 each (balance heuristic)
            float usel = randf(rng);
            float u1 = randf(rng), u2 = randf(rng), u3 = randf(rng);
            if (usel < 0.5f) wi = sample_bsdf(m, wo, smp_n, u1, u2, u3, rng).wi;
            else wi = guide_sample_c(gm, u1, u2, u3);
            float c = dot(smp_n, wi);
            if (c <= 1e-6f) break;
            gpdf = 0.5f * pdf_bsdf(m, wo, wi, smp_n) + 0.5f * guide_pdf_c(gm, wi);
            if (!(gpdf > MIN_PDF)) break;
            T = mul(T, bsdf_weight(eval_bsdf(m, wo, wi, smp_n), c, gpdf));
            last_pdf = gpdf;
        } else {
            float u1 = randf(rng), u2 = randf(rng), u3 = randf(rng);
            BsdfSample bs = sample_bsdf(m, wo, smp_n, u1, u2, u3, rng);
            if (!(bs.kind == BS_PRECOMP || bs.pdf > MIN_PDF)) break;
            RGB w;
            if (bs.kind == BS_PRECOMP) {
                w = bs.f;
            } else {
                float c = fabsf(dot(smp_n, bs.wi));
                if (c <= 1e-6f || bs.pdf < MIN_PDF) break;
                w = bsdf_weight(bs.f, c, bs.pdf);
            }
            T = mul(T, w);
            if (mis) last_pdf = (bs.kind == BS_EVAL) ? bs.pdf : 0.0f;
            wi = bs.wi;
        }
        if (depth >= 3) {
            float rr = smin(smax3(T.r, T.g, T.b), 0.95f);
            if (randf(rng) > rr) break;
            T = T * (1.0f / rr);
        }
        if (!rgb_valid(T)) break;
        new_o = p; new_d = wi;
        out.cont = true;
        if (guided) {
            // warp-aggregated counters: guided vertices, then record slots
            unsigned am = __activemask();
            int leader = __ffs(am) - 1;
            if ((int)lane_id() == leader) atomicAdd(&pv.gcount[1], __popc(am));
            unsigned hsh = murmur3_finalize((unsigned)id * 0x9E3779B9u ^ (unsigned)(depth + 1) * 0x85EBCA6Bu);
            if (hsh < pv.gkeep) {
                unsigned km = __activemask();
                int kl = __ffs(km) - 1, rb = 0;
                if ((int)lane_id() == kl) rb = atomicAdd(&pv.gcount[0], __popc(km));
                int r = __shfl_sync(km, rb, kl) + __popc(km & lanemask_lt());
                if (r < pv.gcap) {
                    GuideRec g;
                    g.p[0] = (p.x - pv.glo[0]) * pv.gscale[0];
                    g.p[1] = (p.y - pv.glo[1]) * pv.gscale[1];
                    g.p[2] = (p.z - pv.glo[2]) * pv.gscale[2];
                    g.n[0] = n.x; g.n[1] = n.y; g.n[2] = n.z;
                    g.wo[0] = wo.x; g.wo[1] = wo.y; g.wo[2] = wo.z;
                    g.wi[0] = wi.x; g.wi[1] = wi.y; g.wi[2] = wi.z;
                    g.pdf = gpdf;
                    g.L[0] = g.L[1] = g.L[2] = 0.0f;
                    pv.grec[r] = g;
                    int4 sl = pv.gslot[id];
                    pv.gslot[id] = make_int4(r, sl.x, sl.y, -1);
                    pv.ginv[3 * id + 2] = pv.ginv[3 * id + 1];
                    pv.ginv[3 * id + 1] = pv.ginv[3 * id];
                    pv.ginv[3 * id] = make_float4(T.r > 0.0f ? 1.0f / T.r : 0.0f, T.g > 0.0f ? 1.0f / T.g : 0.0f,
                                                  T.b > 0.0f ? 1.0f / T.b : 0.0f, 0.0f);
                    pushed = 1;
                }
            }
        }
    } while (0);

    if (out.cont && depth + 1 >= f.max_depth) out.cont = false;
    pv.rng[id] = make_ulonglong2(rng.state, rng.inc);
    pv.rad[id] = make_float4(result.r, result.g, result.b, 0.0f);
    if (out.cont) {
        pv.thr[id] = make_float4(T.r, T.g, T.b, last_pdf);
        pv.ray_o[id] = make_float4(new_o.x, new_o.y, new_o.z, RAY_T_MIN);
        pv.ray_d[id] = make_float4(new_d.x, new_d.y, new_d.z, __int_as_float(depth + 1));
    }
    if (out.shadow) {
        pv.sh_o[id] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_len);
        // w: the first guide slot the NEE contribution credits (a vertex's
        // own light sample did not arrive along its sampled direction)
        pv.sh_d[id] = make_float4(sh_d.x, sh_d.y, sh_d.z, __int_as_float(pushed));
        pv.sh_c[id] = make_float4(sh_inc.r, sh_inc.g, sh_inc.b, 0.0f);
    }
    return out;
}

// Eight resident CTAs per SM (at most 64 registers per thread, a few
// hundred bytes of spills): the extra warps hide more of the shading
// kernel's instruction-fetch and memory latency than the spills cost
// (measured on the 1M-triangle scene: 4, 5, 6, 7, 8 CTAs per SM).
template <int ALGO, bool GUIDE = false, int MINB = 8, bool MULTI = false>
__global__ void __launch_bounds__(128, MINB) k_shade(DevScene sc, FrameParams f, PathView pv, int* cnt, int* cnt_next,
                                                  int identity, int* qin, int* qout) {
    const int n = *(volatile int*)&cnt[0];
    for (;;) {
        int base = warp_fetch(&cnt[3]);
        if (base >= n) break;
        int i = base + (int)lane_id();
        int id = -1;
        ShadeResult r;
        r.cont = false;
        r.shadow = false;
        if (i < n) {
            id = identity ? i : qin[i];
            r = shade_path<ALGO, GUIDE>(path_scene<MULTI>(sc, pv, id), f, pv, id);
        }
        warp_append(qout, &cnt_next[0], id, r.cont);
        warp_append(pv.qs, &cnt[1], id, r.shadow);
    }
}

using ShadeKernel = void (*)(DevScene, FrameParams, PathView, int*, int*, int, int*, int*);
template <int MINB>
static ShadeKernel shade_kernel_lb(int algo, bool guide) {
    if (guide && algo == ALGO_MIS) return k_shade<ALGO_MIS, true, MINB>;
    switch (algo) {
        case ALGO_SIMPLE: return k_shade<ALGO_SIMPLE, false, MINB>;
        case ALGO_MIS: return k_shade<ALGO_MIS, false, MINB>;
        case ALGO_VOLUME_SIMPLE: return k_shade<ALGO_VOLUME_SIMPLE, false, MINB>;
        case ALGO_VOLUME_MIS: return k_shade<ALGO_VOLUME_MIS, false, MINB>;
        default: return k_shade<ALGO_NEE, false, MINB>;
    }
}
static ShadeKernel shade_kernel(int algo, bool guide = false) { return shade_kernel_lb<8>(algo, guide); }
// Batch waves (unguided): each path shaded in its own job's scene.
static ShadeKernel shade_kernel_batch(int algo) {
    switch (algo) {
        case ALGO_SIMPLE: return k_shade<ALGO_SIMPLE, false, 8, true>;
        case ALGO_MIS: return k_shade<ALGO_MIS, false, 8, true>;
        case ALGO_VOLUME_SIMPLE: return k_shade<ALGO_VOLUME_SIMPLE, false, 8, true>;
        case ALGO_VOLUME_MIS: return k_shade<ALGO_VOLUME_MIS, false, 8, true>;
        default: return k_shade<ALGO_NEE, false, 8, true>;
    }
}

// ---------------------------------------------------------------- shading bins
// The scatter half of the counting sort whose histogram the trace kernels
// build (bin_class): one atomic per class per warp, paths of a class kept
// together so neighbouring warps shade the same kind of event.
constexpr int kBinThreads = 256;
static_assert(kBins % kBinThreads == 0, "bins per scatter thread");
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(PathView pv, int* cnt, int identity, const int* qin,
                                                             int* qb) {
    __shared__ int base[kBins];
    __shared__ int wsum[kBinThreads / 32];
    {
        // exclusive prefix sum of the bin counts: kPer bins per thread, then a
        // block scan of the per-thread sums
        constexpr int kPer = kBins / kBinThreads;
        int loc[kPer], sum = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) { loc[j] = sum; sum += cnt[8 + threadIdx.x * kPer + j]; }
        const int lane = (int)(threadIdx.x & 31), w = (int)(threadIdx.x >> 5);
        int x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        int before = 0;
        for (int k = 0; k < w; ++k) before += wsum[k];
        const int excl = before + x - sum;
#pragma unroll
        for (int j = 0; j < kPer; ++j) base[threadIdx.x * kPer + j] = excl + loc[j];
    }
    __syncthreads();
    const int n = *(volatile int*)&cnt[0];
    // whole warps iterate together (match/shuffle below need every lane)
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        int i = i0 + (int)threadIdx.x;
        bool act = i < n;
        int id = act ? (identity ? i : qin[i]) : 0;
        int c = act ? (int)pv.cls[id] : -1;
        unsigned peers = __match_any_sync(0xffffffffu, c);
        int leader = __ffs(peers) - 1;
        int pos = 0;
        if (act && (int)lane_id() == leader) pos = atomicAdd(&cnt[8 + kBins + c], __popc(peers));
        pos = __shfl_sync(0xffffffffu, pos, leader);
        if (act) qb[base[c] + pos + __popc(peers & lanemask_lt())] = id;
    }
}

// ---------------------------------------------------------------- guide inference
// Raw guide outputs for every queued path whose next event is a guidable
// surface hit: 16 paths per warp-tile through the BF16 tensor-core MLP
// (16 warps per block, one block per SM), the weights staged once per block
// in shared memory.  Two lanes encode each path (lanes r and r + 16, half of
// the features each).
constexpr int kInferWarps = 16;
constexpr size_t kInferSmem = sizeof(GuideSmemW) + kInferWarps * sizeof(GuideLeanTile);

__global__ void __launch_bounds__(32 * kInferWarps, 1) k_guide_infer(DevScene sc, PathView pv, int* cnt, int identity,
                                                                     const int* qin, const __nv_bfloat16* wq,
                                                                     const float* master) {
    extern __shared__ __align__(16) unsigned char smem[];
    GuideSmemW& W = *reinterpret_cast<GuideSmemW*>(smem);
    GuideLeanTile* tiles = reinterpret_cast<GuideLeanTile*>(smem + sizeof(GuideSmemW));
    guide_load_weights(W, wq, master);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, rl = lane & 15, half = lane >> 4;
    GuideLeanTile& T = tiles[warp];
    const int n = *(volatile int*)&cnt[0];
    const int ntiles = (n + 15) / 16;
    for (int tile = blockIdx.x * kInferWarps + warp; tile < ntiles; tile += gridDim.x * kInferWarps) {
        int id = -1;
        bool elig = false;
        __nv_bfloat16* row = T.x + rl * kLdIn;
        const int i = tile * 16 + rl;
        if (i < n) {
            id = identity ? i : qin[i];
            float4 hh = pv.hit[id];
            int prim = __float_as_int(hh.w);
            float2 lh = pv.lhit[id];
            int li = __float_as_int(lh.x);
            if (prim >= 0 && !(li >= 0 && lh.y < hh.x)) {
                int4 pi = sc.prim_info[prim];
                elig = guide_eligible(sc.materials[pi.x]);
                if (elig) {
                    float4 ro = pv.ray_o[id], rd = pv.ray_d[id];
                    V3 o = f3(ro), d = f3(rd);
                    V3 p = o + d * hh.x;
                    V3 p01 = v3((p.x - pv.glo[0]) * pv.gscale[0], (p.y - pv.glo[1]) * pv.gscale[1],
                                (p.z - pv.glo[2]) * pv.gscale[2]);
                    V3 fn = f3(sc.prim_fn[prim]);
                    V3 nn = fn;
                    if (pi.w) {
                        float w = 1.0f - hh.y - hh.z;
                        V3 ni = f3(sc.prim_vn[3 * prim]) * w + f3(sc.prim_vn[3 * prim + 1]) * hh.y +
                                f3(sc.prim_vn[3 * prim + 2]) * hh.z;
                        nn = make_dir_or(ni, fn);
                    }
                    guide_encode_half(p01, nn, -d, half, [&](int k, float v) { row[k] = __float2bfloat16(v); });
                }
            }
        }
        if (!elig)
            for (int k = half * 88; k < half * 88 + 88; ++k) row[k] = __float2bfloat16(0.0f);
        __syncwarp();
        guide_forward_lean(W, T);
        // the compact mixture of each path, half by each of its two lanes
        if (elig) {
            float4 o[5];
            guide_compact_half(T.raw() + rl * kGOut, half, o);
            float4* dst = reinterpret_cast<float4*>(pv.gmix + (size_t)id * kGMixFloats);
#pragma unroll
            for (int k = 0; k < 4; ++k) dst[4 * half + k] = o[k];
            dst[8 + half] = o[4];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- shadow
// Shadow rays (persistent, dynamic refill): is_shadowed_skipping_volume_
// boundaries (path_tracer.hpp:103-119) with any-hit BVH queries; a segment
// ends at the nearest boundary-only hit, past which the probe advances 1 mm.
// The boundary triangles are tested one after another, without the group
// boxes the closest-hit kernels use: on the 1M-triangle scene the box tests
// made this kernel 4 % slower (more registers at its 56-register cap),
// while they save the closest-hit kernels 7 %.
// Nine resident CTAs per SM as for k_trace (shadow time -0.7 %; 10: +4 %).
template <int MINB, bool MULTI = false>
__global__ void __launch_bounds__(128, MINB) k_shadow_lb(DevScene sc0, PathView pv, int* cnt, int records) {
    const int n = *(volatile int*)&cnt[1];
    int stack[kStack];
    Trav s;
    bool active = false, exhausted = false, ok = true;
    int id = 0, peek = 0, sid = 0;
    float tmax = 0.0f, off = 0.0f, bt = -1.0f;
    V3 po = v3(0.f, 0.f, 0.f), d = v3(0.f, 0.f, 1.f);
    // the lane's scene (a batch wave: its ray's entry of the scene table)
    auto scene = [&]() -> const DevScene& {
        if constexpr (MULTI) return pv.scenes[sid];
        else return sc0;
    };
    for (;;) {
        int r = refill(&cnt[4], n, !active, exhausted);
        int outcome = -1;   // -1 running, 0 unoccluded, 1 occluded
        if (r >= 0) {
            id = pv.qs[r];
            if constexpr (MULTI) sid = pv.sid[id];
            const DevScene& sc = scene();
            float4 so = pv.sh_o[id], sd = pv.sh_d[id];
            po = f3(so); d = f3(sd); tmax = so.w; off = 0.0f; peek = 0;
            active = true;
            // first segment
            float rem = tmax - off;
            if (rem <= 0.0f) outcome = 0;
            else {
                bt = -1.0f;
                if (sc.num_bnd_tris) {
                    HitRec b; b.t = rem; b.u = 0.f; b.v = 0.f; b.prim = -1;
                    boundary_closest_all(sc, po, d, RAY_T_MIN, b);
                    if (b.prim >= 0) bt = b.t;
                }
                trav_begin<true>(s, sc, po, d, RAY_T_MIN, bt >= 0.0f ? bt : rem);
                if (s.any_hit) outcome = 1;
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0) break;
        if (!active) continue;
        if (outcome < 0) {
            const DevScene& sc = scene();
            if (!trav_run_any(s, stack, sc, ok, kShadowSteps)) continue;
            if (s.any_hit) outcome = 1;
            else if (bt < 0.0f) outcome = 0;
            else {
                // skip past the boundary hit and start the next segment
                float skip = bt + 1e-3f;
                off += skip;
                po = po + d * skip;
                if (++peek == 8) outcome = 0;
                else {
                    float rem = tmax - off;
                    if (rem <= 0.0f) outcome = 0;
                    else {
                        bt = -1.0f;
                        HitRec b; b.t = rem; b.u = 0.f; b.v = 0.f; b.prim = -1;
                        boundary_closest_all(sc, po, d, RAY_T_MIN, b);
                        if (b.prim >= 0) bt = b.t;
                        trav_begin<true>(s, sc, po, d, RAY_T_MIN, bt >= 0.0f ? bt : rem);
                        if (s.any_hit) outcome = 1;
                    }
                }
            }
            if (outcome < 0) continue;
        }
        bool occ = outcome == 1;
        if (!occ) {
            float4 ra = pv.rad[id], c = pv.sh_c[id];
            pv.rad[id] = make_float4(ra.x + c.x, ra.y + c.y, ra.z + c.z, 0.0f);
            if (pv.grec) guide_credit(pv, id, rgb(c.x, c.y, c.z), __float_as_int(pv.sh_d[id].w));
        }
        if (records) {
            int4 rc = pv.rec_cnt[id];
            rc.y += 1;
            rc.z += occ ? 1 : 0;
            pv.rec_cnt[id] = rc;
            pv.rec_hash[id] = hpush(pv.rec_hash[id], 0x5EED0000u | (occ ? 1u : 0u));
        }
        active = false;
    }
    if (!ok) atomicAdd(&pv.errors[0], 1);
}

// ---------------------------------------------------------------- launch profiles
// Resident CTAs per SM of the wavefront kernels (their register caps):
// profile 0 is the measured optimum on the 1M-triangle scene (closest hit 9,
// shading 8, shadow 9); profile 1 gives each kernel more registers and fewer
// spills (8, 6, 8), which scenes with short paths or few triangles can
// prefer.  The request loop's autotuner picks per job shape.
using TraceKernel = void (*)(DevScene, PathView, int*, int, int, int);
using ShadowKernel = void (*)(DevScene, PathView, int*, int);
struct LaunchSet {
    TraceKernel trace;
    ShadeKernel shade;
    ShadowKernel shadow;
};
constexpr int kLaunchProfiles = 2;
static LaunchSet launch_set(int algo, bool guide, int profile) {
    if (profile == 1) return {k_trace_lb<8>, shade_kernel_lb<6>(algo, guide), k_shadow_lb<8>};
    return {k_trace_lb<9>, shade_kernel_lb<8>(algo, guide), k_shadow_lb<9>};
}
// Batch waves: the same kernels reading each path's scene from the wave's
// scene table (profile 0's resident CTAs).
static LaunchSet launch_set_batch(int algo) {
    return {k_trace_lb<9, true>, shade_kernel_batch(algo), k_shadow_lb<9, true>};
}

// ---------------------------------------------------------------- film
// Per-pixel radiance sum in sample order: film += rad(s0), rad(s0+1), ...
// (the reference's `radiance = radiance + sample_radiance`, :318-327).
__global__ void k_film(int npix, int spw, const float4* rad, float4* film) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float4 a = film[p];
    for (int s = 0; s < spw; ++s) {
        float4 r = rad[(size_t)s * npix + p];
        a.x = a.x + r.x; a.y = a.y + r.y; a.z = a.z + r.z;
    }
    film[p] = a;
}

// FP64 accumulation for converged references: the same per-sample FP32
// radiance, summed per pixel in double in sample order.
__global__ void k_film_f64(int npix, int spw, const float4* rad, double* film) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    double a0 = film[3 * (size_t)p], a1 = film[3 * (size_t)p + 1], a2 = film[3 * (size_t)p + 2];
    for (int s = 0; s < spw; ++s) {
        float4 r = rad[(size_t)s * npix + p];
        a0 += (double)r.x; a1 += (double)r.y; a2 += (double)r.z;
    }
    film[3 * (size_t)p] = a0; film[3 * (size_t)p + 1] = a1; film[3 * (size_t)p + 2] = a2;
}
__global__ void k_output_f64(int tw, int th, const double* film, double* out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tw * th) return;
    int x = p % tw, y = p / tw;
    double* o = out + ((size_t)(th - 1 - y) * tw + x) * 4;
    for (int c = 0; c < 3; ++c) {
        double v = film[3 * (size_t)p + c];
        o[c] = (v < 0.0) ? 0.0 : v;
    }
    o[3] = 1.0;
}

// Camera sensitivity (EV 0 => 1), clamp >= 0 keeping NaN, alpha 1, Y flip
// (pybind_renderer.hpp:330-360).
__global__ void k_output(int tw, int th, const float4* film, float4* out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= tw * th) return;
    int x = p % tw, y = p / tw;
    float4 a = film[p];
    float r = a.x * 1.0f, g = a.y * 1.0f, b = a.z * 1.0f;
    out[(size_t)(th - 1 - y) * tw + x] = make_float4(smax(r, 0.0f), smax(g, 0.0f), smax(b, 0.0f), 1.0f);
}

__global__ void k_records(FrameParams f, PathView pv, LucidSampleRecord* out) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= f.n_wave) return;
    int p = id % f.npix, sl = id / f.npix;
    LucidSampleRecord r;
    float4 ra = pv.rad[id];
    r.rgb[0] = ra.x; r.rgb[1] = ra.y; r.rgb[2] = ra.z;
    int2 pp = pv.rec_prim[id];
    int4 c = pv.rec_cnt[id];
    r.primary_mesh = pp.x; r.primary_tri = pp.y;
    r.bounces = (uint32_t)c.x; r.nee_tests = (uint32_t)c.y; r.nee_occluded = (uint32_t)c.z;
    r.hash = pv.rec_hash[id];
    out[(size_t)p * f.samples + f.s0 + sl] = r;
}

// ---------------------------------------------------------------- path diagnostics
// trace{Simple,NEE,MIS}WithDiagnostics (integrator/path_tracer.hpp:880-1514)
// with the PathDiagnosticRecorder (diagnostics/diagnostic_integrator.hpp:
// 87-389): one thread follows one (pixel, sample) path through every bounce;
// intersectScene covers every triangle (no volume-boundary skipping), shadow
// rays are any-hit queries over every triangle, volumes are ignored.  Each
// completed path (light, environment or emitter reached) is appended to the
// record buffer; the host replays the records into the DiagnosticFilm.
enum DiagBsdf { DB_DIFFUSE = 0, DB_GLOSSY = 1, DB_MIRROR = 2, DB_GLASS = 3, DB_EMISSION = 4 };
enum DiagLight { DL_UNKNOWN = 0, DL_POINT = 1, DL_AREA = 2, DL_DIRECTIONAL = 3, DL_SPOT = 4, DL_ENV = 5, DL_EMISSIVE = 6 };
enum DiagStrategy { DS_BSDF = 0, DS_NEE = 1, DS_MIS_BSDF = 2, DS_MIS_NEE = 3 };

LD uint8_t diag_light_type(int type) {   // to_light_source_type (diagnostics/path_types.hpp)
    switch (type) {
        case LIGHT_EMISSIVE: return DL_AREA;
        case LIGHT_POINT: return DL_POINT;
        case LIGHT_SUN: return DL_DIRECTIONAL;
        case LIGHT_SPOT: return DL_SPOT;
        case LIGHT_AREA: return DL_AREA;
    }
    return DL_UNKNOWN;
}

struct DiagPath {   // the recorder's current PathTrace
    int depth;
    int32_t obj[kDiagMaxDepth];
    uint8_t bsdf[kDiagMaxDepth], flags[kDiagMaxDepth];
    V3 pos[kDiagMaxDepth], nrm[kDiagMaxDepth];
};

struct DiagOut {
    uint4* units;
    uint32_t* index;
    unsigned long long* count;   // [0] records, [1] units
    long long cap, cap_units;
    uint32_t unit_base;          // the band's units before this wave (index entries are band offsets)
};

LD void diag_vertex(DiagPath& P, int32_t obj, uint8_t type, bool delta, V3 p, V3 n) {
    if (P.depth >= kDiagMaxDepth) return;
    P.obj[P.depth] = obj; P.bsdf[P.depth] = type; P.flags[P.depth] = delta ? 1 : 0;
    P.pos[P.depth] = p; P.nrm[P.depth] = n;
    ++P.depth;
}

// record_completed_path_with_geometry (diagnostic_integrator.hpp:349-389):
// the path plus a final Emission vertex (object -1 for the environment, else
// -(light + 2)) when there is room, in the compact form (lucid_diag.h).
// A record slot and its units per calling thread with one atomic each per
// group of converged lanes (the lanes that complete a path at the same point
// of the loop; the units by an exclusive scan of the record sizes); each
// thread's slots still increase in its own program order, which the host's
// sort uses to keep records of one (pixel, sample, bounce) in order.
LD void diag_vertex_store(uint4* u, int32_t obj, uint32_t bsdf, uint32_t flags, V3 p, V3 n) {
    u[0] = make_uint4((uint32_t)obj, bsdf | (flags << 8), __float_as_uint(p.x), __float_as_uint(p.y));
    u[1] = make_uint4(__float_as_uint(p.z), __float_as_uint(n.x), __float_as_uint(n.y), __float_as_uint(n.z));
}

LD void diag_complete(const DiagOut& o, const DiagPath& P, uint32_t pixel, uint32_t sample, uint32_t seq,
                      uint8_t strategy, int light_id, uint8_t ltype, RGB c, V3 lpos) {
    const int d = P.depth;
    const bool emission = d < kDiagMaxDepth;
    const int dv = d + (emission ? 1 : 0);
    const unsigned size = 2u + 2u * (unsigned)dv;
    cg::coalesced_group g = cg::coalesced_threads();
    const unsigned before = cg::exclusive_scan(g, size);
    const unsigned total = g.shfl(before + size, g.size() - 1);
    unsigned long long rb = 0, ub = 0;
    if (g.thread_rank() == 0) {
        rb = atomicAdd(&o.count[0], (unsigned long long)g.size());
        ub = atomicAdd(&o.count[1], (unsigned long long)total);
    }
    const unsigned long long slot = g.shfl(rb, 0) + g.thread_rank();
    const unsigned long long uoff = g.shfl(ub, 0) + before;
    // past either capacity the host grows the buffers and runs the wave again
    if ((long long)slot >= o.cap || (long long)(uoff + size) > o.cap_units) return;
    o.index[slot] = o.unit_base + (uint32_t)uoff;
    uint4* u = o.units + uoff;
    u[0] = make_uint4(pixel, sample, seq, (uint32_t)strategy | ((uint32_t)ltype << 8) | ((uint32_t)dv << 16));
    u[1] = make_uint4(__float_as_uint(c.r), __float_as_uint(c.g), __float_as_uint(c.b), 0u);
    for (int k = 0; k < d; ++k) diag_vertex_store(u + 2 + 2 * k, P.obj[k], P.bsdf[k], P.flags[k], P.pos[k], P.nrm[k]);
    if (emission)
        diag_vertex_store(u + 2 + 2 * d, (ltype == DL_ENV) ? -1 : -(light_id + 2), DB_EMISSION, 0u, lpos,
                          v3(0.0f, 0.0f, 0.0f));
}

__global__ void __launch_bounds__(128) k_diag_paths(DevScene sc, FrameParams f, PathView pv, DiagOut out,
                                                    int pixel_base) {
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= f.n_wave) return;
    const int algo = f.algo;   // ALGO_SIMPLE, ALGO_MIS, else NEE (pybind_renderer.hpp:300-309)
    const bool simple = algo == ALGO_SIMPLE, mis = algo == ALGO_MIS, nee_only = !simple && !mis;
    const uint32_t pixel = (uint32_t)(pixel_base + id % f.npix);
    const uint32_t sample = (uint32_t)(f.s0 + id / f.npix);
    ulonglong2 rs = pv.rng[id];
    Rng rng;
    rng.state = rs.x;
    rng.inc = rs.y;
    float4 ro = pv.ray_o[id], rd = pv.ray_d[id];
    V3 o = f3(ro), d = f3(rd);
    float tmin = 0.0f;
    RGB result = rgb(0.f, 0.f, 0.f), T = rgb(1.f, 1.f, 1.f);
    float last_pdf = 0.0f;
    bool ok = true;
    DiagPath P;
    P.depth = 0;
    for (int depth = 0; depth < f.max_depth; ++depth) {
        const uint32_t seq = (uint32_t)depth * 2u;
        HitRec h = scene_closest(sc, o, d, tmin, 1e30f, ok);
        float lt = 1e30f;
        int li = (depth == 0) ? -1 : native_lights_closest(sc, o, d, h.prim >= 0 ? h.t : 1e30f, lt);
        if (li >= 0) {   // in front of the surface hit (the bound above)
            if (!nee_only || depth == 0) {
                const DevLight& L = sc.lights[sc.native_start + li];
                uint8_t ltype = diag_light_type(__float_as_int(L.pos_type.w));
                V3 lp = o + d * lt;
                float mw = 1.0f;
                if (mis) {
                    float lpdf = 0.0f;
                    if (sc.num_lights > 0) {
                        float sp = area_ratio(L.normal_area.w, sc.total_light_area);
                        if (sp > 0.0f) {
                            V3 ln = (__float_as_int(L.pos_type.w) == LIGHT_POINT) ? normalize_nz(lp - f3(L.pos_type))
                                                                                  : f3(L.normal_area);
                            lpdf = pdf_light(L.normal_area.w, o, lp, ln) * sp;
                        }
                    }
                    mw = (last_pdf > MIN_PDF && lpdf > MIN_PDF) ? mis_power(last_pdf, lpdf) : 1.0f;
                }
                RGB em = c3(L.emission_radius);
                RGB pc = mis ? mul(T, em) * mw : mul(T, em);
                diag_complete(out, P, pixel, sample, seq, mis ? DS_MIS_BSDF : DS_BSDF, li, ltype, pc, lp);
                result = result + pc;
            }
            break;
        }
        if (h.prim < 0) {
            if (!nee_only || depth == 0) {
                RGB env = mul(T, rgb(sc.env[0], sc.env[1], sc.env[2]));
                diag_complete(out, P, pixel, sample, seq, mis ? DS_MIS_BSDF : DS_BSDF, -1, DL_ENV, env,
                              o + d * 1000.0f);
                result = result + env;
            }
            break;
        }
        V3 p = o + d * h.t;
        int4 pi = sc.prim_info[h.prim];
        V3 fn = f3(sc.prim_fn[h.prim]);
        V3 n = fn;
        if (pi.w) {
            float w = 1.0f - h.u - h.v;
            V3 ni = f3(sc.prim_vn[3 * h.prim]) * w + f3(sc.prim_vn[3 * h.prim + 1]) * h.u +
                    f3(sc.prim_vn[3 * h.prim + 2]) * h.v;
            n = make_dir_or(ni, fn);
        }
        const DevMaterial& dm = sc.materials[pi.x];
        Mat m;
        m.albedo = c3(dm.albedo_metallic);
        m.metallic = dm.albedo_metallic.w;
        m.roughness = smax(dm.rough_trans_ior_flags.x, MIN_ROUGHNESS);
        m.transmission = dm.rough_trans_ior_flags.y;
        m.ior = dm.rough_trans_ior_flags.z;
        RGB em = c3(dm.emission);
        bool has_em = dm.emission.w != 0.0f;
        apply_textures(sc, dm, h.prim, h.u, h.v, m.albedo, em, has_em);
        // classify_bsdf / is_delta_bsdf (diagnostic_integrator.hpp:25-60)
        uint8_t bt = m.transmission > 0.5f                       ? DB_GLASS
                     : (m.roughness < 0.01f && m.metallic > 0.5f) ? DB_MIRROR
                     : (m.metallic > 0.5f || m.roughness < 0.5f)  ? DB_GLOSSY
                                                                  : DB_DIFFUSE;
        bool delta = (m.transmission > 0.5f && m.roughness < 0.01f) || (m.metallic > 0.5f && m.roughness < 0.01f);
        V3 wo = -d;
        bool front = dot(wo, n) > 0;
        V3 sn = n;
        if (m.transmission < 0.5f && !front) sn = -n;
        if (simple) {
            if (has_em) {
                RGB ec = mul(T, em);
                diag_complete(out, P, pixel, sample, seq, DS_BSDF, pi.x, DL_EMISSIVE, ec, p);
                result = result + ec;
                break;
            }
            diag_vertex(P, pi.x, bt, delta, p, n);
        } else {
            bool do_nee = false;
            if (has_em && (mis || depth == 0)) {
                float mw = 1.0f;
                if (mis && sc.num_lights > 0 && last_pdf > MIN_PDF && pi.z >= 0) {
                    const DevLight& L = sc.lights[pi.z];
                    float sp = area_ratio(L.normal_area.w, sc.total_light_area);
                    if (sp > 0.0f) {
                        float lpdf = pdf_light(L.normal_area.w, o, p, n) * sp;
                        if (lpdf > MIN_PDF) mw = mis_power(last_pdf, lpdf);
                    }
                }
                RGB ec = mis ? mul(T, em) * mw : mul(T, em);
                diag_complete(out, P, pixel, sample, seq, mis ? DS_MIS_BSDF : DS_BSDF, pi.x, DL_EMISSIVE, ec, p);
                result = result + ec;
            } else if (!has_em) {
                diag_vertex(P, pi.x, bt, delta, p, n);
                do_nee = true;
            }
            const bool transmissive = m.transmission > 0.5f;
            if (do_nee && sc.num_lights > 0 && !transmissive) {
                float usel = randf(rng);
                int sli = select_light(sc, usel);
                const DevLight& L = sc.lights[sli];
                float lsp = area_ratio(L.normal_area.w, sc.total_light_area);
                if (lsp > 1e-6f) {
                    float u1 = randf(rng), u2 = randf(rng);
                    LightSample ls = sample_light(L, p, u1, u2);
                    if (ls.pdf > MIN_PDF) {
                        float nl = dot(sn, ls.dir);
                        if (nl > 1e-6f) {
                            bool occ = bvh_any(sc, p, ls.dir, RAY_T_MIN, ls.dist, ok) ||
                                       (sc.num_bnd_tris &&
                                        list_any(sc.bnd_tris, sc.num_bnd_tris, p, ls.dir, RAY_T_MIN, ls.dist));
                            if (!occ) {
                                RGB fb = eval_bsdf(m, wo, ls.dir, sn);
                                float pl = ls.pdf * lsp;
                                RGB nr;
                                if (mis) {
                                    float pb = pdf_bsdf(m, wo, ls.dir, sn);
                                    float mw = mis_power(pl, pb);
                                    nr = mul(bsdf_weight(fb, nl, pl) * mw, ls.emission);
                                } else {
                                    nr = mul(bsdf_weight(fb, nl, pl), ls.emission);
                                }
                                RGB tot = mul(T, nr);
                                diag_complete(out, P, pixel, sample, seq + 1u, mis ? DS_MIS_NEE : DS_NEE,
                                              sli - sc.native_start, diag_light_type(__float_as_int(L.pos_type.w)),
                                              tot, ls.pos);
                                result = result + tot;
                            }
                        }
                    }
                }
            }
        }
        V3 smp_n = (m.transmission > 0.5f) ? n : sn;
        float u1 = randf(rng), u2 = randf(rng), u3 = randf(rng);
        BsdfSample bs = sample_bsdf(m, wo, smp_n, u1, u2, u3, rng);
        if (!(bs.kind == BS_PRECOMP || bs.pdf > MIN_PDF)) break;
        RGB w;
        if (bs.kind == BS_PRECOMP) {
            w = bs.f;
        } else {
            float c = fabsf(dot(smp_n, bs.wi));
            if (c <= 1e-6f || bs.pdf < MIN_PDF) break;
            w = bsdf_weight(bs.f, c, bs.pdf);
        }
        T = mul(T, w);
        if (mis) last_pdf = (bs.kind == BS_EVAL) ? bs.pdf : 0.0f;
        if (depth >= 3) {
            float rr = smin(smax3(T.r, T.g, T.b), 0.95f);
            if (randf(rng) > rr) break;
            T = T * (1.0f / rr);
        }
        if (!rgb_valid(T)) break;
        o = p;
        d = bs.wi;
        tmin = RAY_T_MIN;
    }
    pv.rad[id] = make_float4(result.r, result.g, result.b, 0.0f);
    if (!ok) atomicAdd(&pv.errors[0], 1);
}

// ---------------------------------------------------------------- debug passes
// render_debug (renderer.hpp:59-93): intersectScene from t = 0 over every
// triangle (boundary meshes included), no jitter.
__global__ void k_debug(DevScene sc, FrameParams f, int mode, float4* out, int* errors) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= f.npix) return;
    int px = p % f.tile_w, py = p / f.tile_w;
    int gx = f.tile_x + px, gy = f.tile_y + py;
    float nx = (2.0f * ((float)gx + 0.5f) / (float)f.full_w - 1.0f) * f.aspect;
    float ny = 1.0f - 2.0f * ((float)gy + 0.5f) / (float)f.full_h;
    V3 d = primary_dir(f, nx, ny);
    bool ok = true;
    HitRec h = scene_closest(sc, v3(f.pos[0], f.pos[1], f.pos[2]), d, 0.0f, 1e30f, ok);
    if (!ok) atomicAdd(&errors[0], 1);
    // a miss is black, except in the normal pass, which maps its colour to
    // 0..1 after the lookup (pybind_renderer.hpp:412-415): grey
    float4 c = mode == 0 ? make_float4(0.5f, 0.5f, 0.5f, 1.f) : make_float4(0.f, 0.f, 0.f, 1.f);
    if (h.prim >= 0) {
        int4 pi = sc.prim_info[h.prim];
        V3 fn = f3(sc.prim_fn[h.prim]);
        V3 n = fn;
        if (pi.w) {
            float w = 1.0f - h.u - h.v;
            V3 ni = f3(sc.prim_vn[3 * h.prim]) * w + f3(sc.prim_vn[3 * h.prim + 1]) * h.u +
                    f3(sc.prim_vn[3 * h.prim + 2]) * h.v;
            n = make_dir_or(ni, fn);
        }
        const DevMaterial& dm = sc.materials[pi.x];
        RGB alb = c3(dm.albedo_metallic), em = c3(dm.emission);
        bool has_em = false;
        apply_textures(sc, dm, h.prim, h.u, h.v, alb, em, has_em);
        if (mode == 0) c = make_float4(n.x * 0.5f + 0.5f, n.y * 0.5f + 0.5f, n.z * 0.5f + 0.5f, 1.0f);
        else if (mode == 1) c = make_float4(alb.r, alb.g, alb.b, 1.0f);
        else c = make_float4(em.r * 1.0f, em.g * 1.0f, em.b * 1.0f, 1.0f);
    }
    out[(size_t)(f.tile_h - 1 - py) * f.tile_w + px] = c;
}

// ---------------------------------------------------------------- LBVH build
// Karras 2012 ("Maximizing parallelism in the construction of BVHs"):
// 63-bit Morton codes of triangle centroids, radix sort, one thread per
// internal node, bottom-up refit with arrival counters; subtrees of at most
// four triangles are collapsed into leaves when the nodes are flattened.
LD int ord_f(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
LD float unord_f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }
LD V3 centroid(const float4* verts, int prim) {
    V3 a = f3(verts[3 * prim]), b = f3(verts[3 * prim + 1]), c = f3(verts[3 * prim + 2]);
    return (a + b + c) * (1.0f / 3.0f);
}

__global__ void k_centroid_bounds(const float4* verts, const int* ids, int n, int* bounds) {
    __shared__ int s[6][128];
    int t = threadIdx.x;
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
    for (int i = blockIdx.x * blockDim.x + t; i < n; i += gridDim.x * blockDim.x) {
        V3 c = centroid(verts, ids[i]);
        int o[3] = {ord_f(c.x), ord_f(c.y), ord_f(c.z)};
        for (int k = 0; k < 3; ++k) { mn[k] = min(mn[k], o[k]); mx[k] = max(mx[k], o[k]); }
    }
    for (int k = 0; k < 3; ++k) { s[k][t] = mn[k]; s[3 + k][t] = mx[k]; }
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
        if (t < w)
            for (int k = 0; k < 3; ++k) {
                s[k][t] = min(s[k][t], s[k][t + w]);
                s[3 + k][t] = max(s[3 + k][t], s[3 + k][t + w]);
            }
        __syncthreads();
    }
    if (t == 0)
        for (int k = 0; k < 3; ++k) { atomicMin(&bounds[k], s[k][0]); atomicMax(&bounds[3 + k], s[3 + k][0]); }
}

LD unsigned long long expand21(unsigned long long v) {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

__global__ void k_morton(const float4* verts, const int* ids, int n, const int* bounds, unsigned long long* keys,
                         int* vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 c = centroid(verts, ids[i]);
    float lo[3] = {unord_f(bounds[0]), unord_f(bounds[1]), unord_f(bounds[2])};
    float hi[3] = {unord_f(bounds[3]), unord_f(bounds[4]), unord_f(bounds[5])};
    float cc[3] = {c.x, c.y, c.z};
    unsigned long long code = 0;
    for (int k = 0; k < 3; ++k) {
        float ext = hi[k] - lo[k];
        float u = ext > 0.0f ? (cc[k] - lo[k]) / ext : 0.5f;
        unsigned long long q = (unsigned long long)fminf(fmaxf(u * 2097152.0f, 0.0f), 2097151.0f);
        code |= expand21(q) << (2 - k);
    }
    keys[i] = code;
    vals[i] = ids[i];
}

LD int delta_k(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    unsigned long long a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(i ^ j);
    return __clzll(a ^ b);
}

// children: code >= 0 internal node, < 0 ~leaf index
__global__ void k_karras(const unsigned long long* keys, int n, int2* child, int* parent, int* leaf_parent,
                         int2* range) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta_k(keys, n, i, i + 1) - delta_k(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta_k(keys, n, i, i - d);
    int lmax = 2;
    while (delta_k(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta_k(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta_k(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta_k(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    int cl = (first == gamma) ? ~gamma : gamma;
    int cr = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    child[i] = make_int2(cl, cr);
    range[i] = make_int2(first, last);
    if (cl >= 0) parent[cl] = i; else leaf_parent[~cl] = i;
    if (cr >= 0) parent[cr] = i; else leaf_parent[~cr] = i;
}

LD void leaf_box(const float4* verts, int prim, float* b) {
    V3 a = f3(verts[3 * prim]), c = f3(verts[3 * prim + 1]), e = f3(verts[3 * prim + 2]);
    b[0] = fminf(fminf(a.x, c.x), e.x); b[1] = fminf(fminf(a.y, c.y), e.y); b[2] = fminf(fminf(a.z, c.z), e.z);
    b[3] = fmaxf(fmaxf(a.x, c.x), e.x); b[4] = fmaxf(fmaxf(a.y, c.y), e.y); b[5] = fmaxf(fmaxf(a.z, c.z), e.z);
}

__global__ void k_refit(const float4* verts, const int* sorted_ids, int n, const int2* child, const int* parent,
                        const int* leaf_parent, int* arrive, float* nbox) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = leaf_parent[k];
    // A Karras tree is at most 64 + log2(n) levels deep; the bound only
    // guards against a malformed hierarchy.
    for (int level = 0; node >= 0 && level < 256; ++level) {
        __threadfence();
        if (atomicAdd(&arrive[node], 1) == 0) return;   // the sibling subtree finishes this node
        __threadfence();
        int2 c = child[node];
        float b[6], bb[6];
        if (c.x < 0) leaf_box(verts, sorted_ids[~c.x], b);
        else for (int q = 0; q < 6; ++q) b[q] = __ldcg(&nbox[6 * c.x + q]);
        if (c.y < 0) leaf_box(verts, sorted_ids[~c.y], bb);
        else for (int q = 0; q < 6; ++q) bb[q] = __ldcg(&nbox[6 * c.y + q]);
        for (int q = 0; q < 3; ++q) {
            __stcg(&nbox[6 * node + q], fminf(b[q], bb[q]));
            __stcg(&nbox[6 * node + 3 + q], fmaxf(b[3 + q], bb[3 + q]));
        }
        node = parent[node];
    }
}

__host__ __device__ __forceinline__ int leaf_code(int start, int count) { return ~((start << 3) | (count - 1)); }

__global__ void k_flatten(const float4* verts, const int* sorted_ids, int n, const int2* child, const int2* range,
                          const float* nbox, float pad, DevNode* nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int2 c = child[i];
    int cc[2] = {c.x, c.y};
    float bx[2][6];
    int code[2];
    for (int s = 0; s < 2; ++s) {
        int ch = cc[s];
        if (ch < 0) {
            leaf_box(verts, sorted_ids[~ch], bx[s]);
            code[s] = leaf_code(~ch, 1);
        } else {
            for (int q = 0; q < 6; ++q) bx[s][q] = nbox[6 * ch + q];
            int2 r = range[ch];
            int cnt = r.y - r.x + 1;
            code[s] = cnt <= 4 ? leaf_code(r.x, cnt) : ch;
        }
        for (int q = 0; q < 3; ++q) { bx[s][q] -= pad; bx[s][3 + q] += pad; }
    }
    DevNode nd;
    nd.lmin_lc = make_float4(bx[0][0], bx[0][1], bx[0][2], __int_as_float(code[0]));
    nd.lmax_rc = make_float4(bx[0][3], bx[0][4], bx[0][5], __int_as_float(code[1]));
    nd.rmin = make_float4(bx[1][0], bx[1][1], bx[1][2], 0.0f);
    nd.rmax = make_float4(bx[1][3], bx[1][4], bx[1][5], 0.0f);
    nodes[i] = nd;
}

// ---------------------------------------------------------------- PLOC build
// Parallel locally-ordered clustering (Meister & Bittner, "Parallel Locally-
// Ordered Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG
// 2018): clusters start as the Morton-sorted triangles; each round every
// cluster finds the neighbour within +-kPlocRadius positions whose merged box
// has the smallest surface area, mutual nearest neighbours merge into a new
// node, and the cluster array is compacted in order.  Candidate pairs are
// totally ordered (area, then a tie key of the pair), so the best pair of a
// round is always mutual and every round merges at least one pair.  Node ids follow
// creation order (root last); a top-down pass then gives every subtree a
// contiguous range of triangle slots so that k_flatten can collapse small
// subtrees into leaves exactly as for the Karras tree.
constexpr int kPlocRadius = 32;
constexpr int kPlocBlock = 256;

struct PlocBox { float lo[3], hi[3]; };

LD float ploc_area(const float* a, const float* b) {
    float dx = fmaxf(a[3], b[3]) - fminf(a[0], b[0]);
    float dy = fmaxf(a[4], b[4]) - fminf(a[1], b[1]);
    float dz = fmaxf(a[5], b[5]) - fminf(a[2], b[2]);
    return dx * dy + dy * dz + dz * dx;
}

// Initial clusters: leaf i (Morton order) with its triangle's box.
__global__ void k_ploc_init(const float4* verts, const int* sorted_ids, int n, int* cl, float* cbox, int* cnt_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cl[i] = ~i;
    leaf_box(verts, sorted_ids[i], cbox + 6 * (size_t)i);
    cnt_leaf[i] = 1;
}

// Nearest neighbour of every cluster within the window (boxes staged in
// shared memory with a halo of kPlocRadius on both sides).
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const float* cbox, int count, int* nn) {
    __shared__ float sb[(kPlocBlock + 2 * kPlocRadius) * 6];
    const int b0 = blockIdx.x * kPlocBlock;
    for (int t = threadIdx.x; t < (kPlocBlock + 2 * kPlocRadius) * 6; t += kPlocBlock) {
        int j = b0 - kPlocRadius + t / 6;
        sb[t] = (j >= 0 && j < count) ? cbox[6 * (size_t)j + t % 6] : 0.0f;
    }
    __syncthreads();
    int i = b0 + threadIdx.x;
    if (i >= count) return;
    const float* bi = sb + 6 * (threadIdx.x + kPlocRadius);
    float best = 3.0e38f;
    int bj = -1, bgap = 0, ba = 0;
    int lo = max(0, i - kPlocRadius), hi = min(count - 1, i + kPlocRadius);
    for (int j = lo; j <= hi; ++j) {
        if (j == i) continue;
        float d = ploc_area(bi, sb + 6 * (j - b0 + kPlocRadius));
        // pair key (area, index gap, parity of the lower index, lower index):
        // it depends on the pair only, so the best pair is mutual; on equal
        // areas neighbours pair up (0,1), (2,3), ... instead of chaining
        int a = min(i, j), gap = abs(i - j);
        bool better = bj < 0 || d < best ||
                      (d == best && (gap < bgap || (gap == bgap && ((a & 1) < (ba & 1) ||
                                                                    ((a & 1) == (ba & 1) && a < ba)))));
        if (better) { best = d; bj = j; bgap = gap; ba = a; }
    }
    nn[i] = bj;
}

// flag[i]: 1 = creates a node (mutual pair, lower index), keep[i]: cluster
// survives (unmerged, or the lower index of a merged pair).
__global__ void k_ploc_flags(const int* nn, int count, int* create, int* keep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    int j = nn[i];
    bool mutual = j >= 0 && nn[j] == i;
    create[i] = (mutual && i < j) ? 1 : 0;
    keep[i] = (!mutual || i < j) ? 1 : 0;
}

// Merges (node id = base + exclusive scan of create) and compacts the
// clusters (position = exclusive scan of keep) into the other buffers.
__global__ void k_ploc_merge(const int* cl, const float* cbox, const int* nn, const int* create, const int* keep,
                             const int* create_pos, const int* keep_pos, int count, int base, int2* child,
                             float* nbox, int* cnt_node, const int* cnt_leaf, int* cl_out, float* cbox_out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || !keep[i]) return;
    int o = keep_pos[i];
    if (!create[i]) {
        cl_out[o] = cl[i];
        for (int q = 0; q < 6; ++q) cbox_out[6 * (size_t)o + q] = cbox[6 * (size_t)i + q];
        return;
    }
    int j = nn[i];
    int id = base + create_pos[i];
    int a = cl[i], b = cl[j];
    child[id] = make_int2(a, b);
    float m[6];
    for (int q = 0; q < 3; ++q) {
        m[q] = fminf(cbox[6 * (size_t)i + q], cbox[6 * (size_t)j + q]);
        m[3 + q] = fmaxf(cbox[6 * (size_t)i + 3 + q], cbox[6 * (size_t)j + 3 + q]);
    }
    for (int q = 0; q < 6; ++q) { nbox[6 * (size_t)id + q] = m[q]; cbox_out[6 * (size_t)o + q] = m[q]; }
    cnt_node[id] = (a >= 0 ? cnt_node[a] : cnt_leaf[~a]) + (b >= 0 ? cnt_node[b] : cnt_leaf[~b]);
    cl_out[o] = id;
}

// Top-down slot assignment for the nodes created in one round (processed in
// reverse creation order, so a node's own offset is already known).
__global__ void k_ploc_offsets(const int2* child, const int* cnt_node, int base, int m, int* off_node, int* leaf_pos) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    int id = base + k;
    int2 c = child[id];
    int o = off_node[id];
    int ca = c.x >= 0 ? cnt_node[c.x] : 1;
    if (c.x >= 0) off_node[c.x] = o; else leaf_pos[~c.x] = o;
    if (c.y >= 0) off_node[c.y] = o + ca; else leaf_pos[~c.y] = o + ca;
}

// Children re-coded to triangle slots, subtree slot ranges, triangle ids in
// slot order.
__global__ void k_ploc_finish(const int* sorted_ids, const int* leaf_pos, int n, int2* child, const int* off_node,
                              const int* cnt_node, int2* range, int* slot_ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) slot_ids[leaf_pos[i]] = sorted_ids[i];
    if (i < n - 1) {
        int2 c = child[i];
        if (c.x < 0) c.x = ~leaf_pos[~c.x];
        if (c.y < 0) c.y = ~leaf_pos[~c.y];
        child[i] = c;
        range[i] = make_int2(off_node[i], off_node[i] + cnt_node[i] - 1);
    }
}

__global__ void k_gather_tris(const float4* tri, const int* sorted_ids, int n, float4* out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int prim = sorted_ids[k];
    out[3 * k] = tri[3 * prim];
    out[3 * k + 1] = tri[3 * prim + 1];
    out[3 * k + 2] = tri[3 * prim + 2];
}

// ---------------------------------------------------------------- Engine
static inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

Engine::Engine(int device) : device_(device) {
    ds_ = std::make_shared<DeviceScene>();
    pool_ = new PathPool();
}

Engine::~Engine() {
    async_stop();
    cudaSetDevice(device_);
    if (async_acc_) cudaFree(async_acc_);
    if (async_pinned_) cudaFreeHost(async_pinned_);
    if (jacc_) cudaFree(jacc_);
    job_end();
    delete guide_;
    ds_.reset();   // the device scene is freed with its last sharing engine
    if (pool_) { pool_->release(); delete pool_; }
    delete diag_dev_;
    if (stream_) cudaStreamDestroy(S(stream_));
}

int Engine::device_info(char* buf, size_t cap) const {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_) != cudaSuccess) return LUCID_ERR_CUDA;
    snprintf(buf, cap, "%s (sm_%d%d, %d SMs)", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    return LUCID_OK;
}

int Engine::set_camera(float px, float py, float pz, float dx, float dy, float dz, float ux, float uy, float uz,
                       float fov_deg) {
    GpuLock gl(*this);
    make_camera(cam_, px, py, pz, dx, dy, dz, ux, uy, uz, fov_deg);
    const float raw[10] = {px, py, pz, dx, dy, dz, ux, uy, uz, fov_deg};
    std::memcpy(cam_raw_, raw, sizeof(cam_raw_));
    camera_set_ = true;
    return LUCID_OK;
}

int Engine::set_algorithm(const char* name) {
    GpuLock gl(*this);
    std::string a = name ? name : "";
    if (a == "simple") algo_ = ALGO_SIMPLE;
    else if (a == "mis") algo_ = ALGO_MIS;
    else if (a == "volume_simple") algo_ = ALGO_VOLUME_SIMPLE;
    else if (a == "volume_mis") algo_ = ALGO_VOLUME_MIS;
    else algo_ = ALGO_NEE;   // the reference's dispatch falls through to traceNEE
    return LUCID_OK;
}

int Engine::set_wave_capacity(long long paths) {
    if (paths < 0) return fail(LUCID_ERR_INVALID, "wave capacity must be >= 0");
    wave_cap_ = paths;
    return LUCID_OK;
}

int Engine::scene_stats(int out8[8]) const {
    if (!scene_loaded_) return LUCID_ERR_NO_SCENE;
    scene_stats_locked(out8);
    return LUCID_OK;
}

void Engine::scene_stats_locked(int out8[8]) const {
    if (shared_) { std::memcpy(out8, shared_stats_, 8 * sizeof(int)); return; }
    int nvol = (int)host_.volumes.size();
    out8[0] = host_.num_meshes; out8[1] = host_.num_prims; out8[2] = host_.num_native;
    out8[3] = (int)host_.lights.size(); out8[4] = host_.num_boundary_meshes; out8[5] = nvol;
    out8[6] = bvh_nodes_; out8[7] = bvh_leaves_;
}

int Engine::stats(LucidRenderStats* out) const { *out = stats_; return LUCID_OK; }

void Engine::free_scene() {
    if (ds_.use_count() > 1) ds_ = std::make_shared<DeviceScene>();   // still used by a sharing engine
    else ds_->release();
    scene_loaded_ = false;
}

int Engine::ensure_stream() {
    if (stream_) return LUCID_OK;
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    stream_ = s;
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device_));
    num_sms_ = prop.multiProcessorCount;
    return LUCID_OK;
}

int Engine::share_scene(Engine& owner) {
    SceneSnapshot snap;
    int rc = owner.snapshot_scene(snap);
    if (rc != LUCID_OK) return fail(rc, owner.last_error());
    return use_snapshot(snap);
}

int Engine::snapshot_scene(SceneSnapshot& out) {
    GpuLock gl(*this);
    if (!scene_loaded_) return fail(LUCID_ERR_NO_SCENE, "the sharing source has no scene");
    out.ds = ds_;
    scene_stats_locked(out.stats);
    for (int k = 0; k < 3; ++k) { out.lo[k] = scene_lo_[k]; out.hi[k] = scene_hi_[k]; }
    return LUCID_OK;
}

int Engine::use_snapshot(const SceneSnapshot& snap) {
    if (!snap.ds) return fail(LUCID_ERR_NO_SCENE, "empty scene snapshot");
    GpuLock gl(*this);
    CK(cudaSetDevice(device_));
    int rc = ensure_stream();
    if (rc != LUCID_OK) return rc;
    ds_ = snap.ds;
    std::memcpy(shared_stats_, snap.stats, sizeof(shared_stats_));
    for (int k = 0; k < 3; ++k) { scene_lo_[k] = snap.lo[k]; scene_hi_[k] = snap.hi[k]; }
    shared_ = true;
    scene_loaded_ = true;
    return LUCID_OK;
}

// A new scene version: the edited materials, lights, light CDF and guide,
// and per-prim shading classes in buffers of its own; the BVH, triangles and
// everything else are the current version's, which it keeps alive.  Engines
// rendering the current version keep it until they take the new one.
int Engine::update_scene(const LucidSceneEdit* edits, int count) {
    GpuLock gl(*this);
    if (!scene_loaded_) return fail(LUCID_ERR_NO_SCENE, "no scene loaded");
    if (shared_) return fail(LUCID_ERR_INVALID, "this context renders a scene it does not own; edit the owner");
    CK(cudaSetDevice(device_));
    std::string err;
    if (!apply_scene_edits(host_, edits, count, err)) return fail(LUCID_ERR_INVALID, err);
    const HostScene& H = host_;
    std::vector<unsigned char> cls(H.prim_info.size());
    for (size_t p = 0; p < cls.size(); ++p) cls[p] = prim_shading_class(H.materials[H.prim_info[p].x]);
    auto nv = std::make_shared<DeviceScene>();
    cudaStream_t st = S(stream_);
    auto up = [&](auto& buf, const auto& vec) -> cudaError_t {
        cudaError_t e = buf.alloc(vec.size());
        if (e != cudaSuccess || vec.empty()) return e;
        return cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, st);
    };
    CK(up(nv->materials, H.materials));
    CK(up(nv->lights, H.lights));
    CK(up(nv->light_bsph, native_light_bounds(H)));
    CK(up(nv->cdf, H.cdf));
    CK(up(nv->guide, H.light_guide));
    CK(up(nv->prim_cls, cls));
    CK(cudaStreamSynchronize(st));   // complete before any other stream reads the version
    nv->view = ds_->view;
    nv->view.materials = nv->materials.p;
    nv->view.lights = nv->lights.p;
    nv->view.light_bsph = H.num_native > 0 ? nv->light_bsph.p : nullptr;
    nv->view.light_cdf = nv->cdf.p;
    nv->view.light_guide = nv->guide.p;
    nv->view.prim_cls = nv->prim_cls.p;
    nv->view.total_light_area = H.total_light_area;
    nv->base = ds_;
    ds_ = nv;
    return LUCID_OK;
}

int Engine::load_scene_json(const char* json, size_t len) {
    GpuLock gl(*this);
    CK(cudaSetDevice(device_));
    {
        int rc = ensure_stream();
        if (rc != LUCID_OK) return rc;
    }
    shared_ = false;
    HostScene hs;
    std::string err;
    free_scene();
    if (!parse_scene_json(json, len, hs, err)) return fail(LUCID_ERR_INVALID, err);
    return upload_scene(std::move(hs));
}

int Engine::load_scene_arrays(const LucidSceneDesc& desc) {
    GpuLock gl(*this);
    CK(cudaSetDevice(device_));
    {
        int rc = ensure_stream();
        if (rc != LUCID_OK) return rc;
    }
    shared_ = false;
    HostScene hs;
    std::string err;
    free_scene();
    if (!build_scene_arrays(desc, hs, err)) return fail(LUCID_ERR_INVALID, err);
    return upload_scene(std::move(hs));
}

// Uploads a flattened scene and builds its BVH (the caller holds the GPU
// lock with the device current and the stream created).
int Engine::upload_scene(HostScene&& hs) {
    host_ = std::move(hs);
    DeviceScene& D = *ds_;
    const HostScene& H = host_;
    // boundary triangles (brute force list) and per-prim shading data
    std::vector<float4> bnd;
    for (int p = 0; p < H.num_prims; ++p)
        if (H.prim_boundary[p])
            for (int k = 0; k < 3; ++k) bnd.push_back(H.tri[3 * p + k]);
    auto up = [&](auto& buf, const auto& vec) -> cudaError_t {
        cudaError_t e = buf.alloc(vec.size());
        if (e != cudaSuccess) return e;
        if (vec.empty()) return cudaSuccess;
        return cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, S(stream_));
    };
    // each prim's shading class for a surface hit (the material part of
    // bin_class, decided once here instead of per hit)
    std::vector<unsigned char> cls(H.prim_info.size());
    for (size_t p = 0; p < cls.size(); ++p) cls[p] = prim_shading_class(H.materials[H.prim_info[p].x]);
    CK(up(D.bnd_tris, bnd));
    CK(up(D.prim_info, H.prim_info));
    CK(up(D.prim_cls, cls));
    CK(up(D.prim_fn, H.prim_fn));
    CK(up(D.prim_vn, H.prim_vn));
    CK(up(D.materials, H.materials));
    CK(up(D.tex_ops, H.tex_ops));
    CK(up(D.prim_uv, H.prim_uv));
    CK(up(D.lights, H.lights));
    CK(up(D.light_bsph, native_light_bounds(H)));
    CK(up(D.cdf, H.cdf));
    CK(up(D.guide, H.light_guide));
    CK(up(D.volumes, H.volumes));
    CK(up(D.grid, H.grid));
    DevScene& v = D.view;
    v = DevScene{};
    v.bnd_tris = D.bnd_tris.p;
    v.num_bnd_tris = (int)(bnd.size() / 3);
    v.prim_info = D.prim_info.p;
    v.prim_cls = D.prim_cls.p;
    v.prim_fn = D.prim_fn.p;
    v.prim_vn = D.prim_vn.p;
    v.materials = D.materials.p;
    v.tex_ops = H.tex_ops.empty() ? nullptr : D.tex_ops.p;
    v.prim_uv = H.prim_uv.empty() ? nullptr : D.prim_uv.p;
    v.lights = D.lights.p;
    v.light_cdf = D.cdf.p;
    v.light_guide = D.guide.p;
    v.num_lights = (int)H.lights.size();
    v.native_start = H.native_start;
    v.num_native = H.num_native;
    v.light_bsph = H.num_native > 0 ? D.light_bsph.p : nullptr;
    v.total_light_area = H.total_light_area;
    for (int k = 0; k < 3; ++k) v.env[k] = H.env[k];
    v.volumes = D.volumes.p;
    v.num_volumes = (int)H.volumes.size();
    v.grid = D.grid.p;
    v.has_boundary = v.num_bnd_tris > 0;
    int rc = build_bvh();
    if (rc != LUCID_OK) return rc;
    CK(cudaStreamSynchronize(S(stream_)));
    scene_loaded_ = true;
    return LUCID_OK;
}

// PLOC rounds on the device; the host reads four integers per round to know
// the surviving cluster count.  Returns LUCID_OK with root = -1 when the
// clustering needs more than kPlocMaxRounds rounds (the caller then builds
// the Karras tree instead).
int Engine::build_ploc(const float4* verts, const int* sorted_ids, int n, int2* child, int2* range, float* nbox,
                       int* slot_ids, int& root) {
    constexpr int kPlocMaxRounds = 4096;
    cudaStream_t st = S(stream_);
    root = -1;
    DBuf<int> cl0, cl1, nn, create, keep, create_pos, keep_pos, cnt_leaf, cnt_node, off_node, leaf_pos;
    DBuf<float> cb0, cb1;
    CK(cl0.alloc(n)); CK(cl1.alloc(n)); CK(nn.alloc(n)); CK(create.alloc(n)); CK(keep.alloc(n));
    CK(create_pos.alloc(n)); CK(keep_pos.alloc(n)); CK(cnt_leaf.alloc(n)); CK(cnt_node.alloc(n - 1));
    CK(off_node.alloc(n - 1)); CK(leaf_pos.alloc(n)); CK(cb0.alloc((size_t)6 * n)); CK(cb1.alloc((size_t)6 * n));
    size_t temp = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, temp, create.p, create_pos.p, n, st));
    DBuf<unsigned char> d_temp;
    CK(d_temp.alloc(temp));
    k_ploc_init<<<(n + 255) / 256, 256, 0, st>>>(verts, sorted_ids, n, cl0.p, cb0.p, cnt_leaf.p);
    int* cl[2] = {cl0.p, cl1.p};
    float* cb[2] = {cb0.p, cb1.p};
    int cur = 0, count = n, base = 0;
    std::vector<std::pair<int, int>> rounds;
    int h[4];
    while (count > 1) {
        if ((int)rounds.size() >= kPlocMaxRounds) return LUCID_OK;
        k_ploc_nn<<<(count + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, st>>>(cb[cur], count, nn.p);
        k_ploc_flags<<<(count + 255) / 256, 256, 0, st>>>(nn.p, count, create.p, keep.p);
        size_t t1 = temp;
        CK(cub::DeviceScan::ExclusiveSum(d_temp.p, t1, create.p, create_pos.p, count, st));
        t1 = temp;
        CK(cub::DeviceScan::ExclusiveSum(d_temp.p, t1, keep.p, keep_pos.p, count, st));
        k_ploc_merge<<<(count + 255) / 256, 256, 0, st>>>(cl[cur], cb[cur], nn.p, create.p, keep.p, create_pos.p,
                                                         keep_pos.p, count, base, child, nbox, cnt_node.p,
                                                         cnt_leaf.p, cl[cur ^ 1], cb[cur ^ 1]);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&h[0], create_pos.p + count - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h[1], create.p + count - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h[2], keep_pos.p + count - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h[3], keep.p + count - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        int m = h[0] + h[1], survivors = h[2] + h[3];
        if (m <= 0 || survivors != count - m) return fail(LUCID_ERR_CUDA, "BVH clustering made no progress");
        rounds.push_back({base, m});
        base += m;
        count = survivors;
        cur ^= 1;
    }
    if (base != n - 1) return fail(LUCID_ERR_CUDA, "BVH clustering produced a wrong node count");
    const int r = n - 2;   // the last node created is the root
    CK(cudaMemsetAsync(off_node.p + r, 0, sizeof(int), st));
    for (auto it = rounds.rbegin(); it != rounds.rend(); ++it)
        k_ploc_offsets<<<(it->second + 255) / 256, 256, 0, st>>>(child, cnt_node.p, it->first, it->second, off_node.p,
                                                                 leaf_pos.p);
    k_ploc_finish<<<(n + 255) / 256, 256, 0, st>>>(sorted_ids, leaf_pos.p, n, child, off_node.p, cnt_node.p, range,
                                                  slot_ids);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    ploc_rounds_ = (int)rounds.size();
    root = r;
    return LUCID_OK;
}

int Engine::build_bvh() {
    DeviceScene& D = *ds_;
    const HostScene& H = host_;
    // Scene bounds, then split off the largest triangles: at most kMaxBig
    // whose bounding-box diagonal exceeds a quarter of the scene's.
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    float maxabs = 0.0f;
    std::vector<float> diag(H.num_prims, 0.0f);
    for (int p = 0; p < H.num_prims; ++p) {
        if (H.prim_boundary[p]) continue;
        float pl[3] = {1e30f, 1e30f, 1e30f}, ph[3] = {-1e30f, -1e30f, -1e30f};
        for (int k = 0; k < 3; ++k) {
            const float4& q = H.verts[3 * p + k];
            const float c[3] = {q.x, q.y, q.z};
            for (int a = 0; a < 3; ++a) {
                pl[a] = std::min(pl[a], c[a]); ph[a] = std::max(ph[a], c[a]);
                maxabs = std::max(maxabs, std::fabs(c[a]));
            }
        }
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], pl[a]); hi[a] = std::max(hi[a], ph[a]); }
        diag[p] = std::sqrt((ph[0] - pl[0]) * (ph[0] - pl[0]) + (ph[1] - pl[1]) * (ph[1] - pl[1]) +
                            (ph[2] - pl[2]) * (ph[2] - pl[2]));
    }
    // secondary-ray origins lie on triangles (boundary ones included) or
    // inside volume boxes: all of them bound the FMA slab test's error
    for (int p = 0; p < H.num_prims; ++p)
        if (H.prim_boundary[p])
            for (int k = 0; k < 3; ++k) {
                const float4& q = H.verts[3 * p + k];
                maxabs = std::max(maxabs, std::max(std::fabs(q.x), std::max(std::fabs(q.y), std::fabs(q.z))));
            }
    for (const DevVolume& vol : H.volumes)
        for (int a = 0; a < 3; ++a)
            maxabs = std::max(maxabs, std::max(std::fabs(vol.wmin[a]), std::fabs(vol.wmax[a])));
    for (int a = 0; a < 3; ++a) { scene_lo_[a] = lo[a]; scene_hi_[a] = hi[a]; }
    {
        // boundary-only triangles grouped by mesh (they are stored in prim
        // order), each group with its bounding box padded as the BVH's boxes
        std::vector<float4> boxes;
        const float bpad = maxabs * 9.5367431640625e-07f + 1e-30f;
        int k = 0;
        for (int p = 0; p < H.num_prims; ++p) {
            if (!H.prim_boundary[p]) continue;
            const int mesh = H.prim_info[(size_t)p].x;
            bool fresh = boxes.empty();
            if (!fresh) {
                int last_mesh;
                std::memcpy(&last_mesh, &boxes[boxes.size() - 1].w, 4);   // scratch: mesh id of the open group
                fresh = last_mesh != mesh;
            }
            if (fresh) {
                float first;
                std::memcpy(&first, &k, 4);
                float m;
                std::memcpy(&m, &mesh, 4);
                boxes.push_back(make_float4(1e30f, 1e30f, 1e30f, first));
                boxes.push_back(make_float4(-1e30f, -1e30f, -1e30f, m));
            }
            float4& blo = boxes[boxes.size() - 2];
            float4& bhi = boxes[boxes.size() - 1];
            for (int c = 0; c < 3; ++c) {
                const float4& q = H.verts[3 * p + c];
                blo.x = std::min(blo.x, q.x); blo.y = std::min(blo.y, q.y); blo.z = std::min(blo.z, q.z);
                bhi.x = std::max(bhi.x, q.x); bhi.y = std::max(bhi.y, q.y); bhi.z = std::max(bhi.z, q.z);
            }
            ++k;
        }
        // close the groups: pad the boxes, replace the mesh id by the count
        for (size_t g = 0; g < boxes.size(); g += 2) {
            int first, next;
            std::memcpy(&first, &boxes[g].w, 4);
            if (g + 2 < boxes.size()) std::memcpy(&next, &boxes[g + 2].w, 4);
            else next = k;
            const int count = next - first;
            boxes[g].x -= bpad; boxes[g].y -= bpad; boxes[g].z -= bpad;
            boxes[g + 1].x += bpad; boxes[g + 1].y += bpad; boxes[g + 1].z += bpad;
            std::memcpy(&boxes[g + 1].w, &count, 4);
        }
        DeviceScene& Db = D;
        cudaError_t e = Db.bnd_box.alloc(std::max<size_t>(1, boxes.size()));
        if (e != cudaSuccess) return fail(LUCID_ERR_OOM, "boundary box allocation failed");
        if (!boxes.empty())
            CK(cudaMemcpyAsync(Db.bnd_box.p, boxes.data(), boxes.size() * sizeof(float4), cudaMemcpyHostToDevice,
                               S(stream_)));
        Db.view.bnd_box = boxes.empty() ? nullptr : Db.bnd_box.p;
        Db.view.num_bnd_groups = (int)(boxes.size() / 2);
        if (k != Db.view.num_bnd_tris) return fail(LUCID_ERR_CUDA, "boundary triangle groups do not cover the list");
    }
    float sdiag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                            (hi[2] - lo[2]) * (hi[2] - lo[2]));
    const int kMaxBig = 32;
    std::vector<int> bigc;
    for (int p = 0; p < H.num_prims; ++p)
        if (!H.prim_boundary[p] && diag[p] > 0.25f * sdiag) bigc.push_back(p);
    std::sort(bigc.begin(), bigc.end(), [&](int a, int b) { return diag[a] > diag[b] || (diag[a] == diag[b] && a < b); });
    if ((int)bigc.size() > kMaxBig) bigc.resize(kMaxBig);
    // keep at least one triangle in the BVH so tiny scenes still build one
    int nonbnd = 0;
    for (int p = 0; p < H.num_prims; ++p) nonbnd += !H.prim_boundary[p];
    if ((int)bigc.size() == nonbnd) bigc.clear();
    std::vector<unsigned char> is_big(H.num_prims, 0);
    std::vector<float4> big;
    for (int p : bigc) is_big[p] = 1;
    for (int p = 0; p < H.num_prims; ++p)
        if (is_big[p]) for (int k = 0; k < 3; ++k) big.push_back(H.tri[3 * p + k]);
    std::vector<int> real;
    real.reserve(H.num_prims);
    for (int p = 0; p < H.num_prims; ++p)
        if (!H.prim_boundary[p] && !is_big[p]) real.push_back(p);
    int n = (int)real.size();
    DevScene& v = D.view;
    v.coord_bound = maxabs;
    for (int a = 0; a < 3; ++a) {
        const float ext = hi[a] - lo[a];
        v.bin_lo[a] = ext > 0.0f ? lo[a] : 0.0f;
        v.bin_scale[a] = ext > 0.0f ? (float)kCellDim / ext : 0.0f;
    }
    {
        cudaError_t e = D.big_tris.alloc(big.size());
        if (e != cudaSuccess) return fail(LUCID_ERR_OOM, "big triangle list allocation failed");
        if (!big.empty())
            CK(cudaMemcpyAsync(D.big_tris.p, big.data(), big.size() * sizeof(float4), cudaMemcpyHostToDevice, S(stream_)));
        v.big_tris = D.big_tris.p;
        v.num_big_tris = (int)(big.size() / 3);
        num_big_ = v.num_big_tris;
    }
    v.num_bvh_tris = n;
    bvh_nodes_ = 0; bvh_leaves_ = 0; bvh_depth_ = 0;
    if (n == 0) { v.root = v.root2 = 0; v.nodes = nullptr; v.nodes2 = nullptr; v.bvh_tris = nullptr; return LUCID_OK; }
    cudaStream_t st = S(stream_);
    DBuf<float4> d_tri, d_verts;
    DBuf<int> d_ids, d_vals, d_vals_sorted, d_parent, d_leaf_parent, d_arrive, d_bounds;
    DBuf<unsigned long long> d_keys, d_keys_sorted;
    DBuf<int2> d_child, d_range;
    DBuf<float> d_nbox;
    CK(d_tri.alloc(H.tri.size()));
    CK(cudaMemcpyAsync(d_tri.p, H.tri.data(), H.tri.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
    CK(d_verts.alloc(H.verts.size()));
    CK(cudaMemcpyAsync(d_verts.p, H.verts.data(), H.verts.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
    CK(d_ids.alloc(n));
    CK(cudaMemcpyAsync(d_ids.p, real.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(d_bounds.alloc(6));
    int init[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000, (int)0x80000000, (int)0x80000000};
    CK(cudaMemcpyAsync(d_bounds.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_centroid_bounds<<<std::max(1, std::min(4 * num_sms_, (n + 127) / 128)), 128, 0, st>>>(d_verts.p, d_ids.p, n,
                                                                                             d_bounds.p);
    CK(d_keys.alloc(n)); CK(d_keys_sorted.alloc(n)); CK(d_vals.alloc(n)); CK(d_vals_sorted.alloc(n));
    k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_verts.p, d_ids.p, n, d_bounds.p, d_keys.p, d_vals.p);
    size_t temp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, temp, d_keys.p, d_keys_sorted.p, d_vals.p, d_vals_sorted.p, n, 0, 63,
                                       st));
    DBuf<unsigned char> d_temp;
    CK(d_temp.alloc(temp));
    CK(cub::DeviceRadixSort::SortPairs(d_temp.p, temp, d_keys.p, d_keys_sorted.p, d_vals.p, d_vals_sorted.p, n, 0, 63,
                                       st));
    CK(D.bvh_tris.alloc((size_t)3 * n));
    v.bvh_tris = D.bvh_tris.p;
    if (n <= 4) {
        k_gather_tris<<<(n + 255) / 256, 256, 0, st>>>(d_tri.p, d_vals_sorted.p, n, D.bvh_tris.p);
        v.root = leaf_code(0, n);
        v.root2 = v.root;
        v.nodes = nullptr;
        v.nodes2 = nullptr;
        bvh_leaves_ = 1;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        return LUCID_OK;
    }
    CK(d_child.alloc(n - 1)); CK(d_range.alloc(n - 1)); CK(d_nbox.alloc((size_t)6 * (n - 1)));
    int root = -1;
    DBuf<int> d_slot;
    {
        CK(d_slot.alloc(n));
        int rc = build_ploc(d_verts.p, d_vals_sorted.p, n, d_child.p, d_range.p, d_nbox.p, d_slot.p, root);
        if (rc != LUCID_OK) return rc;
    }
    const int* slot_ids = root >= 0 ? d_slot.p : d_vals_sorted.p;
    if (root < 0) {   // Karras LBVH: the fallback when clustering does not converge
        CK(d_parent.alloc(n - 1)); CK(d_leaf_parent.alloc(n)); CK(d_arrive.alloc(n - 1));
        CK(cudaMemsetAsync(d_parent.p, 0xff, (n - 1) * sizeof(int), st));   // root's parent = -1
        CK(cudaMemsetAsync(d_arrive.p, 0, (n - 1) * sizeof(int), st));
        k_karras<<<(n - 1 + 255) / 256, 256, 0, st>>>(d_keys_sorted.p, n, d_child.p, d_parent.p, d_leaf_parent.p,
                                                      d_range.p);
        k_refit<<<(n + 255) / 256, 256, 0, st>>>(d_verts.p, d_vals_sorted.p, n, d_child.p, d_parent.p,
                                                d_leaf_parent.p, d_arrive.p, d_nbox.p);
        root = 0;
    }
    k_gather_tris<<<(n + 255) / 256, 256, 0, st>>>(d_tri.p, slot_ids, n, D.bvh_tris.p);
    DBuf<DevNode>& d_nodes2 = D.nodes2;
    CK(d_nodes2.alloc(n - 1));
    float pad = maxabs * 9.5367431640625e-07f + 1e-30f;   // 2^-20 of the scene's coordinate magnitude
    k_flatten<<<(n - 1 + 255) / 256, 256, 0, st>>>(d_verts.p, slot_ids, n, d_child.p, d_range.p, d_nbox.p, pad,
                                                  d_nodes2.p);
    CK(cudaGetLastError());
    // Reachable node count, leaves and depth (the traversal stack bound).
    std::vector<DevNode> hn(n - 1);
    CK(cudaMemcpyAsync(hn.data(), d_nodes2.p, (n - 1) * sizeof(DevNode), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // The walk also validates the hierarchy before any traversal kernel uses
    // it: child indices in range, leaf ranges inside the triangle array, and
    // no node reached twice.
    // The same walk sums the surface-area cost (node visits + triangle tests
    // weighted by box area relative to the root's) reported as bvh_sah_.
    std::vector<std::pair<int, int>> stack{{root, 1}};
    std::vector<unsigned char> seen(n - 1, 0);
    int nodes = 0, leaves = 0, depth = 0;
    long long leaf_tris = 0;
    auto area = [](const float4& lo, const float4& hi) {
        double dx = (double)hi.x - lo.x, dy = (double)hi.y - lo.y, dz = (double)hi.z - lo.z;
        return dx * dy + dy * dz + dz * dx;
    };
    double sah = 1.0, root_area = 0.0;
    {
        const DevNode& r = hn[root];
        float4 lo = make_float4(std::min(r.lmin_lc.x, r.rmin.x), std::min(r.lmin_lc.y, r.rmin.y),
                                std::min(r.lmin_lc.z, r.rmin.z), 0.0f);
        float4 hi = make_float4(std::max(r.lmax_rc.x, r.rmax.x), std::max(r.lmax_rc.y, r.rmax.y),
                                std::max(r.lmax_rc.z, r.rmax.z), 0.0f);
        root_area = std::max(area(lo, hi), 1e-30);
    }
    while (!stack.empty()) {
        auto [nd, dep] = stack.back();
        stack.pop_back();
        if (nd < 0 || nd >= n - 1 || seen[nd]) return fail(LUCID_ERR_CUDA, "BVH build produced an invalid hierarchy");
        seen[nd] = 1;
        ++nodes;
        depth = std::max(depth, dep);
        int c[2];
        std::memcpy(&c[0], &hn[nd].lmin_lc.w, 4);
        std::memcpy(&c[1], &hn[nd].lmax_rc.w, 4);
        const double ca[2] = {area(hn[nd].lmin_lc, hn[nd].lmax_rc) / root_area, area(hn[nd].rmin, hn[nd].rmax) / root_area};
        for (int s = 0; s < 2; ++s) {
            if (c[s] < 0) {
                int w = ~c[s], start = w >> 3, count = (w & 7) + 1;
                if (start < 0 || start + count > n) return fail(LUCID_ERR_CUDA, "BVH leaf out of range");
                leaf_tris += count;
                ++leaves;
                depth = std::max(depth, dep + 1);
                sah += ca[s] * count;
            } else {
                stack.push_back({c[s], dep + 1});
                sah += ca[s];
            }
        }
    }
    if (leaf_tris != n) return fail(LUCID_ERR_CUDA, "BVH leaves do not cover every triangle");
    // Collapse the binary tree into 4-wide nodes: starting from a node's two
    // children, the internal child with the largest box is replaced by its
    // own two children until there are four (or only leaves).
    std::vector<DevNode4> n4;
    n4.reserve((size_t)nodes / 2 + 1);
    std::vector<std::pair<int, int>> todo{{root, 0}};   // (binary node, index of its 4-wide node)
    n4.push_back(DevNode4{});
    int depth4 = 1;
    std::vector<int> level4{1};
    while (!todo.empty()) {
        auto [bn, idx] = todo.back();
        todo.pop_back();
        struct Ch { float4 lo, hi; int code; };
        Ch ch[4];
        int cnt = 0;
        auto children_of = [&](int b, Ch* out) {
            int c0, c1;
            std::memcpy(&c0, &hn[b].lmin_lc.w, 4);
            std::memcpy(&c1, &hn[b].lmax_rc.w, 4);
            out[0] = {hn[b].lmin_lc, hn[b].lmax_rc, c0};
            out[1] = {hn[b].rmin, hn[b].rmax, c1};
        };
        children_of(bn, ch);
        cnt = 2;
        while (cnt < 4) {
            int best = -1;
            double ba = -1.0;
            for (int k = 0; k < cnt; ++k)
                if (ch[k].code >= 0 && area(ch[k].lo, ch[k].hi) > ba) { ba = area(ch[k].lo, ch[k].hi); best = k; }
            if (best < 0) break;
            Ch two[2];
            children_of(ch[best].code, two);
            ch[best] = two[0];
            ch[cnt++] = two[1];
        }
        const int my_level = level4[idx];
        DevNode4 q;
        float* f[6] = {&q.xmin.x, &q.xmax.x, &q.ymin.x, &q.ymax.x, &q.zmin.x, &q.zmax.x};
        int codes[4];
        for (int k = 0; k < 4; ++k) {
            if (k < cnt) {
                f[0][k] = ch[k].lo.x; f[1][k] = ch[k].hi.x; f[2][k] = ch[k].lo.y; f[3][k] = ch[k].hi.y;
                f[4][k] = ch[k].lo.z; f[5][k] = ch[k].hi.z;
                if (ch[k].code >= 0) {
                    int ni = (int)n4.size();
                    n4.push_back(DevNode4{});
                    level4.push_back(my_level + 1);
                    depth4 = std::max(depth4, my_level + 1);
                    todo.push_back({ch[k].code, ni});
                    codes[k] = ni;
                } else {
                    codes[k] = ch[k].code;
                    depth4 = std::max(depth4, my_level + 1);
                }
            } else {
                for (int a = 0; a < 6; ++a) f[a][k] = 0.0f;
                codes[k] = kEmptyChild;
            }
        }
        q.child = make_int4(codes[0], codes[1], codes[2], codes[3]);
        q.pad = make_int4(0, 0, 0, 0);
        n4[idx] = q;
    }
    CK(D.nodes.alloc(n4.size()));
    CK(cudaMemcpyAsync(D.nodes.p, n4.data(), n4.size() * sizeof(DevNode4), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    // Binary nodes in depth-first order (a node, its left subtree, its right
    // subtree; root first): a ray's descent then reads nearby lines, and the
    // top of the tree shares a few cache lines.
    {
        std::vector<int> order(n - 1, -1), stk{root};
        std::vector<DevNode> dfs;
        dfs.reserve(nodes);
        while (!stk.empty()) {
            int nd = stk.back();
            stk.pop_back();
            order[nd] = (int)dfs.size();
            dfs.push_back(hn[nd]);
            int c0, c1;
            std::memcpy(&c0, &hn[nd].lmin_lc.w, 4);
            std::memcpy(&c1, &hn[nd].lmax_rc.w, 4);
            if (c1 >= 0) stk.push_back(c1);
            if (c0 >= 0) stk.push_back(c0);
        }
        for (DevNode& d : dfs) {
            int c0, c1;
            std::memcpy(&c0, &d.lmin_lc.w, 4);
            std::memcpy(&c1, &d.lmax_rc.w, 4);
            if (c0 >= 0) { c0 = order[c0]; std::memcpy(&d.lmin_lc.w, &c0, 4); }
            if (c1 >= 0) { c1 = order[c1]; std::memcpy(&d.lmax_rc.w, &c1, 4); }
        }
        CK(cudaMemcpyAsync(D.nodes2.p, dfs.data(), dfs.size() * sizeof(DevNode), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        root = 0;
    }
    v.nodes = D.nodes.p;
    v.root = 0;
    v.nodes2 = D.nodes2.p;
    v.root2 = root;
    bvh_nodes_ = (int)n4.size(); bvh_leaves_ = leaves; bvh_depth_ = depth4; bvh_sah_ = sah;
    if (std::getenv("LUCID_VERBOSE"))
        std::fprintf(stderr, "[lucid] BVH %s (%d rounds): %d binary nodes, %d leaves, depth %d, SAH cost %.2f; "
                     "%d 4-wide nodes, depth %d\n",
                     slot_ids == d_vals_sorted.p ? "lbvh" : "ploc", slot_ids == d_vals_sorted.p ? 0 : ploc_rounds_,
                     nodes, leaves, depth, sah, (int)n4.size(), depth4);
    if (3 * (depth4 - 1) >= kStack || depth >= kStack)
        return fail(LUCID_ERR_OVERFLOW, "BVH depth " + std::to_string(depth) + " exceeds the traversal stack");
    return LUCID_OK;
}

int Engine::ensure_pool(long long paths, bool records) {
    PathPool& P = *pool_;
    if (P.cap >= paths && (!records || P.records)) return LUCID_OK;
    long long cap = std::max(paths, P.cap);
    P.release();
    CK(P.rng.alloc(cap)); CK(P.ray_o.alloc(cap)); CK(P.ray_d.alloc(cap)); CK(P.thr.alloc(cap)); CK(P.rad.alloc(cap));
    CK(P.hit.alloc(cap)); CK(P.lhit.alloc(cap)); CK(P.sh_o.alloc(cap)); CK(P.sh_d.alloc(cap)); CK(P.sh_c.alloc(cap));
    CK(P.q0.alloc(cap)); CK(P.q1.alloc(cap)); CK(P.qs.alloc(cap)); CK(P.qb.alloc(cap)); CK(P.cls.alloc(cap));
    CK(P.counters.alloc((size_t)kCountersPerDepth * (kMaxDepth + 1)));
    CK(P.errors.alloc(4));
    if (records) { CK(P.rec_prim.alloc(cap)); CK(P.rec_cnt.alloc(cap)); CK(P.rec_hash.alloc(cap)); }
    P.cap = cap;
    P.records = records;
    PathView& v = P.view;
    v.rng = P.rng.p; v.ray_o = P.ray_o.p; v.ray_d = P.ray_d.p; v.thr = P.thr.p; v.rad = P.rad.p; v.hit = P.hit.p;
    v.lhit = P.lhit.p; v.sh_o = P.sh_o.p; v.sh_d = P.sh_d.p; v.sh_c = P.sh_c.p; v.q0 = P.q0.p; v.q1 = P.q1.p;
    v.qs = P.qs.p; v.qb = P.qb.p; v.cls = P.cls.p; v.counters = P.counters.p; v.errors = P.errors.p;
    v.rec_prim = P.rec_prim.p; v.rec_cnt = P.rec_cnt.p; v.rec_hash = P.rec_hash.p;
    return LUCID_OK;
}

namespace {
// Algorithmic bytes per unit of work (compulsory SoA traffic; BVH node and
// triangle fetches are scene-dependent and excluded):
//   trace : ray 32 + queue id 4 + hit 16 + light hit 8
//           + the hit prim's class 1 and the shading bin 2 (binning)   = 63 / ray
//   shade : queue 4 + hit 24 + ray 32 + throughput 16 + radiance 16 + rng 16
//           + prim info/normal 32 + material 48  (reads)
//           + rng 16 + radiance 16 + throughput 16 + ray 32 + queue 4
//           + shadow record 48 + shadow queue 4  (writes)           = 340 / path
//   shadow: queue 4 + shadow record 48 + radiance 16 read + 16 write  = 84 / ray
//   raygen: rng 16 + ray 32 + throughput 16 + radiance 16            = 80 / path
//   camera trace (generates its rays): the raygen writes 80 + hit 16
//           + light hit 8 + prim class 1 + shading bin 2               = 107 / ray
//   film  : radiance 16 / path + film 32 / pixel
//   bin   : queue id 4 + shading bin 2 + binned id 4 (scatter)       = 10 / path
constexpr double kBytesTrace0 = 107, kBytesTrace = 63, kBytesShade = 340, kBytesShadow = 84, kBytesRaygen = 80, kBytesFilm = 16,
                 kBytesBin = 10;
//   guide : queue 4 + hit 24 + ray 32 + raw outputs 160 w              = 220 / path
//   train : one record 64 / record (weights are read from shared memory)
enum Kind { K_RAYGEN, K_TRACE0, K_TRACE, K_SHADE, K_SHADOW, K_FILM, K_BIN, K_GUIDE, K_TRAIN, K_NUM };
const char* kKindNames[K_NUM] = {"k_raygen", "k_trace_primary", "k_trace", "k_shade", "k_shadow", "k_film", "k_bin",
                                 "k_guide_infer", "k_guide_train"};
const double kKindBytes[K_NUM] = {kBytesRaygen, kBytesTrace0, kBytesTrace, kBytesShade, kBytesShadow, kBytesFilm,
                                  kBytesBin, 220, 64};
static_assert(K_NUM <= LUCID_MAX_KERNEL_KINDS, "kernel kinds");
}  // namespace

// Default paths per wave: large waves keep every depth's launches full and
// amortise each persistent kernel's tail (measured on the 1M-triangle
// frame, samples/s: 4 Mi paths 287 M, 16 Mi 390 M, 64 Mi 429 M, the whole
// 133 M-path frame 435 M; with the current kernels 64 Mi 608 M against 622 M
// for the whole frame), so up to 256 Mi paths (43 GB of path state), bounded
// to a fifth of the free device memory (about 170 bytes per path).
long long Engine::default_wave_paths(bool records) const {
    constexpr long long kMaxWave = 1LL << 28;
    // path state: 8 float4 arrays, the PCG state 16, the native-light hit 8,
    // four int queues 16 and the shading bin 2 = 170 B (+ 32 B of records)
    const long long per_path = 170 + (records ? 32 : 0);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 1LL << 22;
    long long fit = (long long)(free_b / 5) / per_path;
    return std::max(1LL << 20, std::min(kMaxWave, fit));
}

int Engine::render(const LucidRenderParams& p, float* out_host, LucidSampleRecord* recs, float* out_device) {
    GpuLock gl(*this);
    if (diag_enabled_) {
        if (recs) return fail(LUCID_ERR_INVALID, "per-sample records are not produced while diagnostics are enabled");
        return render_diag_impl(p, out_host, out_device);
    }
    const long long paths = (long long)std::max(0, p.tile_w) * std::max(0, p.tile_h) * std::max(0, p.samples);
    if (combine_ && out_host && !recs && !out_device && !(guide_ && guide_->on) && scene_loaded_ && camera_set_ &&
        paths > 0 && paths <= kCombinePaths && p.full_w > 0 && p.full_h > 0 && p.max_depth >= 1 &&
        p.max_depth <= kMaxDepth)
        return render_combined(p, out_host);
    return render_impl(p, out_host, recs, out_device, nullptr, false);
}

// ---------------------------------------------------------------- combining concurrent small renders
// Concurrent sessions (the add-on's viewport, material previews and F12
// renders each own a Renderer) meet on one device.  Small render calls
// (at most kCombinePaths paths, image to host memory, no records,
// diagnostics or guiding) pass through a process-wide combiner per device:
// a call that finds no other small call running renders on its own
// context exactly as without the combiner; calls that arrive while one
// runs wait, and the first of them to find the device free renders every
// waiting call with the same integrator and depth as one batch
// (render_batch on the combiner's own engine), each call's image bit for
// bit its own render.  Large calls never wait here: they overlap on their
// own streams as before.
namespace {
const char* const kAlgoNames[5] = {"simple", "nee", "mis", "volume_simple", "volume_mis"};
struct CombineReq {
    Engine* e;
    Engine::BatchItem item;
    int algo;
    int rc = LUCID_OK;
    bool done = false;
    std::string err;
    LucidRenderStats stats{};
};
struct Combiner {
    std::mutex mu;
    std::condition_variable cv;
    bool busy = false;
    std::vector<CombineReq*> pending;
    std::unique_ptr<Engine> runner;   // renders the batches (its own stream and path pool)
    long long batches = 0, calls = 0;
};
// One per device for the life of the process (never destroyed, so no CUDA
// call runs from a static destructor at exit).
Combiner& combiner_for(int device) {
    static std::mutex mu;
    static std::map<int, Combiner*>* all = new std::map<int, Combiner*>();
    std::lock_guard<std::mutex> lk(mu);
    Combiner*& c = (*all)[device];
    if (!c) c = new Combiner();
    return *c;
}
}  // namespace

int Engine::render_combined(const LucidRenderParams& p, float* out_host) {
    reset_cancel();
    Combiner& C = combiner_for(device_);
    CombineReq r;
    r.e = this;
    r.item.scene = ds_.get();
    std::memcpy(r.item.camera, cam_raw_, sizeof(cam_raw_));
    r.item.p = p;
    r.item.p.flags = 0;
    r.item.out_host = out_host;
    r.algo = algo_;
    std::shared_ptr<DeviceScene> keep = ds_;   // this call's scene version, whoever renders it
    std::unique_lock<std::mutex> lk(C.mu);
    C.pending.push_back(&r);
    while (!r.done) {
        if (C.busy) {
            C.cv.wait(lk);
            continue;
        }
        // lead: every waiting call with this call's integrator and depth
        C.busy = true;
        std::vector<CombineReq*> group;
        for (auto it = C.pending.begin(); it != C.pending.end();) {
            CombineReq* q = *it;
            if (q->algo == r.algo && q->item.p.max_depth == r.item.p.max_depth && group.size() < 256) {
                group.push_back(q);
                it = C.pending.erase(it);
            } else {
                ++it;
            }
        }
        lk.unlock();
        if (group.size() == 1) {
            // alone: this context's own render, as without the combiner
            r.rc = render_impl(p, out_host, nullptr, nullptr, nullptr, false);
            if (r.rc != LUCID_OK) r.err = err_;
            r.stats = stats_;
        } else {
            int rc = LUCID_OK;
            if (!C.runner) C.runner.reset(new Engine(device_));
            std::vector<BatchItem> items;
            items.reserve(group.size());
            for (CombineReq* q : group) items.push_back(q->item);
            rc = C.runner->render_batch(items.data(), (int)items.size(), kAlgoNames[r.algo], kCombinePaths * 8);
            LucidRenderStats bst{};
            C.runner->stats(&bst);
            for (CombineReq* q : group) {
                q->rc = rc;
                if (rc != LUCID_OK) q->err = C.runner->last_error();
                q->stats = bst;
                q->stats.paths = (double)q->item.p.tile_w * q->item.p.tile_h * q->item.p.samples;
            }
        }
        lk.lock();
        for (CombineReq* q : group) q->done = true;
        if (group.size() > 1) {
            ++C.batches;
            C.calls += (long long)group.size();
        }
        C.busy = false;
        C.cv.notify_all();
    }
    lk.unlock();
    stats_ = r.stats;
    if (r.rc == LUCID_OK && is_cancelled()) return fail(LUCID_ERR_CANCELLED, "render cancelled");
    if (r.rc != LUCID_OK) return fail(r.rc, r.err);
    return LUCID_OK;
}

void Engine::combine_stats(int device, long long* batches, long long* calls) {
    Combiner& C = combiner_for(device);
    std::lock_guard<std::mutex> lk(C.mu);
    if (batches) *batches = C.batches;
    if (calls) *calls = C.calls;
}

int Engine::render_f64(const LucidRenderParams& p, double* out_host) {
    GpuLock gl(*this);
    if (diag_enabled_) return fail(LUCID_ERR_INVALID, "FP64 references are not rendered while diagnostics are enabled");
    return render_impl(p, nullptr, nullptr, nullptr, nullptr, false, out_host);
}

// ---------------------------------------------------------------- path diagnostics (host)
constexpr long long kDiagWavePaths = 1LL << 20;   // paths per diagnostic wave

// render_tile with diagnostics enabled (pybind_renderer.hpp:205-316): a
// fresh DiagnosticFilm per call.  The tile is processed in bands of whole
// 8-row micro-tile rows, so replaying each band's records (sorted into the
// reference's loop order) band after band gives the order of the whole tile.
int Engine::render_diag_impl(const LucidRenderParams& p, float* out_host, float* out_device) {
    reset_cancel();
    if (p.tile_w <= 0 || p.tile_h <= 0 || p.full_w <= 0 || p.full_h <= 0)
        return fail(LUCID_ERR_INVALID, "tile and image sizes must be positive");
    const size_t np = (size_t)p.tile_w * p.tile_h;
    if (out_host) std::fill(out_host, out_host + np * 4, 0.0f);
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    CK(cudaSetDevice(device_));
    if (p.samples <= 0) return fail(LUCID_ERR_INVALID, "samples must be >= 1");
    if (p.max_depth > kMaxDepth) return fail(LUCID_ERR_INVALID, "max_depth too large");
    if (np > (size_t)0x7fffffff / 2) return fail(LUCID_ERR_INVALID, "tile too large");
    diag_film_.init(p.tile_w, p.tile_h, diag_cfg_.subsample_factor);
    diag_film_.set_limits(diag_cfg_.max_groups_per_pixel, diag_cfg_.max_outliers_per_pixel);
    cudaStream_t st = S(stream_);
    const long long wave = wave_cap_ > 0 ? std::min(wave_cap_, kDiagWavePaths) : kDiagWavePaths;
    const long long row_paths = (long long)p.tile_w * p.samples;
    int band_rows = 8 * (int)std::max<long long>(1, wave / (8 * row_paths));
    band_rows = std::min(band_rows, (p.tile_h + 7) / 8 * 8);
    const long long band_np = (long long)band_rows * p.tile_w;
    const int spw = (int)std::max<long long>(1, std::min<long long>(p.samples, wave / band_np));
    int rc = ensure_pool((long long)spw * band_np, false);
    if (rc != LUCID_OK) return rc;
    PathPool& P = *pool_;
    if (P.film_n < np) {
        CK(P.film.alloc(np));
        CK(P.out.alloc(np));
        P.film_n = np;
    }
    if (!diag_dev_) diag_dev_ = new DiagDevice();
    DiagDevice& D = *diag_dev_;
    const long long want = diag_cfg_.record_capacity > 0 ? diag_cfg_.record_capacity : (1LL << 20);
    if ((long long)D.index.n < want) CK(D.index.alloc((size_t)want));
    if ((long long)D.units.n < 8 * want) CK(D.units.alloc((size_t)(8 * want)));   // a few bounces per record
    if (!D.count.p) CK(D.count.alloc(2));
    CK(cudaMemsetAsync(P.film.p, 0, np * sizeof(float4), st));
    CK(cudaMemsetAsync(P.errors.p, 0, 4 * sizeof(int), st));

    FrameParams f{};
    for (int k = 0; k < 3; ++k) { f.pos[k] = cam_.pos[k]; f.fwd[k] = cam_.forward[k]; f.right[k] = cam_.right[k]; f.up[k] = cam_.up[k]; }
    f.aspect = (float)p.full_w / (float)p.full_h;
    f.scale = std::tan(cam_.fov * 0.5f);
    f.tile_x = p.tile_x; f.tile_w = p.tile_w; f.full_w = p.full_w; f.full_h = p.full_h;
    f.samples = p.samples; f.sample_offset = p.sample_offset; f.max_depth = p.max_depth; f.algo = algo_;
    f.records = 0;

    stats_ = LucidRenderStats{};
    cudaEvent_t t0, t1, ka, kb, ca, cb;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    for (cudaEvent_t* e : {&ka, &kb, &ca, &cb}) cudaEventCreate(e);
    cudaEventRecord(t0, st);
    int status = LUCID_OK;
    int waves = 0;
    double kernel_ms = 0.0, copy_ms = 0.0, replay_ms = 0.0, records_total = 0.0, record_bytes = 0.0;
    size_t band_n = 0, band_units = 0;
    // the host replays band k (in band order) while the device renders band
    // k + 1 into the other pinned buffer; the film is touched by the replay
    // alone.  A pending replay is waited for before the next starts, and on
    // every return (the future's destructor).
    int hb = 0;
    std::future<double> replay;
    for (int y0 = 0; y0 < p.tile_h && status == LUCID_OK; y0 += band_rows) {
        const int bh = std::min(band_rows, p.tile_h - y0);
        f.tile_y = p.tile_y + y0;
        f.tile_h = bh;
        f.npix = bh * p.tile_w;
        band_n = 0;
        band_units = 0;
        for (int s0 = 0; s0 < p.samples; s0 += spw) {
            if (is_cancelled()) { status = LUCID_ERR_CANCELLED; break; }
            const int this_spw = std::min(spw, p.samples - s0);
            f.s0 = s0;
            f.n_wave = this_spw * f.npix;
            unsigned long long produced[2] = {0, 0};
            for (;;) {
                CK(cudaMemsetAsync(D.count.p, 0, 2 * sizeof(unsigned long long), st));
                cudaEventRecord(ka, st);
                k_raygen<<<(f.n_wave + 255) / 256, 256, 0, st>>>(f, P.view);
                DiagOut o{D.units.p, D.index.p, D.count.p, (long long)D.index.n, (long long)D.units.n,
                          (uint32_t)band_units};
                k_diag_paths<<<(f.n_wave + 127) / 128, 128, 0, st>>>(ds_->view, f, P.view, o, y0 * p.tile_w);
                cudaEventRecord(kb, st);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(produced, D.count.p, sizeof(produced), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                float kms = 0.0f;
                cudaEventElapsedTime(&kms, ka, kb);
                kernel_ms += kms;
                if (band_units + produced[1] >= (1ULL << 32))
                    return fail(LUCID_ERR_OVERFLOW, "path diagnostics: a band's records exceed 64 GB");
                if (produced[0] <= (unsigned long long)D.index.n && produced[1] <= (unsigned long long)D.units.n) break;
                // the wave is deterministic: grow the buffers and run it again
                if (produced[0] > (unsigned long long)D.index.n) CK(D.index.alloc((size_t)(produced[0] + produced[0] / 4)));
                if (produced[1] > (unsigned long long)D.units.n) CK(D.units.alloc((size_t)(produced[1] + produced[1] / 4)));
            }
            k_film<<<(f.npix + 255) / 256, 256, 0, st>>>(f.npix, this_spw, P.rad.p, P.film.p + (size_t)y0 * p.tile_w);
            CK(D.reserve_host(hb, band_n + (size_t)produced[0], band_n, band_units + (size_t)produced[1], band_units));
            cudaEventRecord(ca, st);
            if (produced[0]) {
                CK(cudaMemcpyAsync(D.host_index[hb] + band_n, D.index.p, (size_t)produced[0] * sizeof(uint32_t),
                                   cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(D.host_units[hb] + band_units * kDiagUnitBytes, D.units.p,
                                   (size_t)produced[1] * kDiagUnitBytes, cudaMemcpyDeviceToHost, st));
            }
            band_n += (size_t)produced[0];
            band_units += (size_t)produced[1];
            record_bytes += (double)produced[0] * sizeof(uint32_t) + (double)produced[1] * kDiagUnitBytes;
            cudaEventRecord(cb, st);
            CK(cudaStreamSynchronize(st));
            float cms = 0.0f;
            cudaEventElapsedTime(&cms, ca, cb);
            copy_ms += cms;
            records_total += (double)produced[0];
            ++waves;
        }
        if (status == LUCID_OK) {
            if (replay.valid()) replay_ms += replay.get();
            const uint8_t* units = D.host_units[hb];
            const uint32_t* index = D.host_index[hb];
            const size_t n_rec = band_n;
            const int tw = p.tile_w;
            const bool last = y0 + band_rows >= p.tile_h;
            // while the device renders the next band, this thread waits on it:
            // the replay leaves it a core
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            const unsigned nt = last ? hw : std::max(1u, hw - 1);
            auto run = [this, units, index, n_rec, tw, nt]() {
                const auto h0 = std::chrono::steady_clock::now();
                diag_film_.replay(units, index, n_rec, tw, nt);
                return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
            };
            if (last) replay_ms += run();   // the last band: nothing left to overlap
            else replay = std::async(std::launch::async, run);
            hb ^= 1;
        }
    }
    if (replay.valid()) replay_ms += replay.get();
    for (cudaEvent_t e : {ka, kb, ca, cb}) cudaEventDestroy(e);
    // where a diagnostic render's time goes: the path kernel (raygen
    // included), the record copies to the host, and the host replay
    const char* names[3] = {"k_diag_paths", "diag_record_copy", "diag_replay_host"};
    const double ms3[3] = {kernel_ms, copy_ms, replay_ms};
    stats_.num_kinds = 3;
    for (int k = 0; k < 3; ++k) {
        std::snprintf(stats_.kinds[k].name, sizeof(stats_.kinds[k].name), "%s", names[k]);
        stats_.kinds[k].launches = waves;
        stats_.kinds[k].total_ms = ms3[k];
        stats_.kinds[k].units = k == 0 ? (double)np * p.samples : records_total;
        stats_.kinds[k].algo_bytes = k == 1 ? record_bytes : 0.0;
    }
    const int np_i = (int)np;
    k_output<<<(np_i + 255) / 256, 256, 0, st>>>(p.tile_w, p.tile_h, P.film.p, out_device ? (float4*)out_device : P.out.p);
    CK(cudaGetLastError());
    cudaEventRecord(t1, st);
    int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, P.errors.p, sizeof(herr), cudaMemcpyDeviceToHost, st));
    if (out_host && !out_device)
        CK(cudaMemcpyAsync(out_host, P.out.p, np * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float tot = 0.0f;
    cudaEventElapsedTime(&tot, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    stats_.total_ms = tot;
    stats_.paths = (double)np * p.samples;
    stats_.waves = waves;
    if (herr[0] != 0) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    if (status == LUCID_ERR_CANCELLED) return fail(LUCID_ERR_CANCELLED, "render cancelled");
    return LUCID_OK;
}

// PathRecordingConfig::standard() (diagnostics/path_stats_config.hpp).
int Engine::diag_enable(const LucidDiagConfig* cfg) {
    GpuLock gl(*this);
    LucidDiagConfig c{2, 16, 4, 16, 0.001f, 3.0f, 0};
    if (cfg) c = *cfg;
    if (c.subsample_factor < 1) return fail(LUCID_ERR_INVALID, "subsample_factor must be >= 1");
    diag_cfg_ = c;
    diag_enabled_ = true;
    diag_film_.reset();
    return LUCID_OK;
}
int Engine::diag_disable() {
    GpuLock gl(*this);
    diag_enabled_ = false;
    diag_film_.reset();
    if (diag_dev_) { delete diag_dev_; diag_dev_ = nullptr; }
    return LUCID_OK;
}
int Engine::diag_clear() {
    GpuLock gl(*this);
    if (diag_film_.valid()) diag_film_.clear();
    return LUCID_OK;
}
int Engine::diag_stats(LucidDiagStats* out) {
    GpuLock gl(*this);
    std::memset(out, 0, sizeof(*out));
    if (diag_film_.valid()) diag_film_.stats(out);
    return LUCID_OK;
}
int Engine::diag_pixel(int x, int y, bool by_mean, LucidDiagPixel* info, LucidDiagGroup* groups, int cap) {
    GpuLock gl(*this);
    std::memset(info, 0, sizeof(*info));
    if (!diag_film_.valid()) return 0;
    return diag_film_.export_pixel(x, y, by_mean, info, groups, groups ? cap : 0);
}
int Engine::diag_variance_map(float* out, size_t cap) {
    GpuLock gl(*this);
    if (!diag_film_.valid()) return 0;
    size_t n = (size_t)diag_film_.width() * diag_film_.height();
    if (cap < n) return fail(LUCID_ERR_INVALID, "variance map buffer too small");
    diag_film_.variance_map(out);
    return (int)n;
}
int Engine::diag_top(int n, bool by_mean, LucidDiagGroup* groups, int32_t* xy, int cap) {
    GpuLock gl(*this);
    if (!diag_film_.valid()) return 0;
    return diag_film_.export_top(n, by_mean, groups, xy, groups ? cap : 0);
}

int Engine::diag_coarse(LucidDiagCoarse* out) {
    GpuLock gl(*this);
    if (!diag_film_.valid()) {
        DiagFilm empty;
        empty.coarse_export(out);
        return 8;
    }
    diag_film_.coarse_export(out);
    return 8;
}
int Engine::diag_suggestions(LucidDiagSuggestion* out, int cap) {
    GpuLock gl(*this);
    if (!diag_film_.valid()) return 0;
    return diag_film_.suggestions(out, out ? cap : 0);
}
long long Engine::diag_export_binary(uint8_t* out, size_t cap) {
    GpuLock gl(*this);
    const std::vector<uint8_t> b = diag_film_.export_binary();
    if (out) std::memcpy(out, b.data(), std::min(cap, b.size()));
    return (long long)b.size();
}
long long Engine::diag_metadata_json(char* out, size_t cap) {
    GpuLock gl(*this);
    const std::string m = diag_film_.metadata_json();
    if (out && cap > 0) {
        const size_t n = std::min(cap - 1, m.size());
        std::memcpy(out, m.data(), n);
        out[n] = 0;
    }
    return (long long)m.size();
}

// Adds one render's film into the async accumulator (float4 sum per pixel).
__global__ void k_accumulate(int npix, const float4* film, float4* acc) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float4 a = acc[p], f = film[p];
    acc[p] = make_float4(a.x + f.x, a.y + f.y, a.z + f.z, 0.0f);
}

int Engine::render_impl(const LucidRenderParams& p, float* out_host, LucidSampleRecord* recs, float* out_device,
                        void* accumulate, bool from_async, double* out_f64) {
    if (!from_async) reset_cancel();
    if (p.tile_w <= 0 || p.tile_h <= 0 || p.full_w <= 0 || p.full_h <= 0)
        return fail(LUCID_ERR_INVALID, "tile and image sizes must be positive");
    size_t np = (size_t)p.tile_w * p.tile_h;
    // A call that returns before its image is copied out leaves a zero image
    // (the reference's empty result); a finished copy is not written twice,
    // which at 1920x1080 saves a 33 MB host fill per call.
    struct ZeroUnlessCopied {
        float* f;
        double* d;
        size_t n;
        bool copied = false;
        ~ZeroUnlessCopied() {
            if (copied) return;
            if (f) std::fill(f, f + n * 4, 0.0f);
            if (d) std::fill(d, d + n * 4, 0.0);
        }
    } host_image{out_host, out_f64, np};
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    CK(cudaSetDevice(device_));
    if (p.samples <= 0) return fail(LUCID_ERR_INVALID, "samples must be >= 1");
    if (p.max_depth > kMaxDepth) return fail(LUCID_ERR_INVALID, "max_depth too large");
    if (np > (size_t)0x7fffffff / 2) return fail(LUCID_ERR_INVALID, "tile too large");
    cudaStream_t st = S(stream_);
    const bool profile = (p.flags & LUCID_RENDER_PROFILE) != 0;
    const bool records = recs != nullptr;
    const bool guide = guide_ && guide_->on && algo_ == ALGO_MIS && !from_async;
    // The wave cap needs a device memory query (a driver call that other
    // processes' driver traffic can hold up for tens of milliseconds); a
    // call that fits the path pool it already has skips it.
    const PathPool& P0 = *pool_;
    long long cap;
    if (wave_cap_ > 0)
        cap = wave_cap_;
    else if (P0.cap >= (long long)p.samples * (long long)np && (!records || P0.records))
        cap = P0.cap;
    else
        cap = default_wave_paths(records);
    if (guide) cap = std::min(cap, kGuideWave);
    int spw = (int)std::max<long long>(1, std::min<long long>(p.samples, cap / (long long)np));
    long long wave_paths = (long long)spw * (long long)np;
    // A progressive caller (the add-on's F12 loop: 4, 8, 16, 32, then 64
    // samples per call) grows the wave call by call; reserving 64 samples
    // per pixel of the tile (within the cap) at the first multi-sample call
    // keeps the later calls from reallocating the pool (50-60 ms each at
    // 1920x1080).  Async dispatches (1 sample each) keep their small pool.
    long long reserve = wave_paths;
    if (!from_async && !records && p.samples > 1)
        reserve = std::max(wave_paths, std::min(cap, 64LL * (long long)np));
    int rc = ensure_pool(reserve, records);
    if (rc != LUCID_OK) return rc;
    PathPool& P = *pool_;
    if (P.film_n < np) {
        CK(P.film.alloc(np));
        CK(P.out.alloc(np));
        P.film_n = np;
    }
    CK(cudaMemsetAsync(P.film.p, 0, np * sizeof(float4), st));
    CK(cudaMemsetAsync(P.errors.p, 0, 4 * sizeof(int), st));
    if (out_f64) {
        if (P.film64_n < np) {
            CK(P.film64.alloc(np * 3));
            CK(P.out64.alloc(np * 4));
            P.film64_n = np;
        }
        CK(cudaMemsetAsync(P.film64.p, 0, np * 3 * sizeof(double), st));
    }
    DBuf<LucidSampleRecord> d_recs;
    if (records) CK(d_recs.alloc(np * (size_t)p.samples));

    FrameParams f{};
    for (int k = 0; k < 3; ++k) { f.pos[k] = cam_.pos[k]; f.fwd[k] = cam_.forward[k]; f.right[k] = cam_.right[k]; f.up[k] = cam_.up[k]; }
    f.aspect = (float)p.full_w / (float)p.full_h;
    f.scale = std::tan(cam_.fov * 0.5f);
    f.tile_x = p.tile_x; f.tile_y = p.tile_y; f.tile_w = p.tile_w; f.tile_h = p.tile_h;
    f.full_w = p.full_w; f.full_h = p.full_h;
    f.samples = p.samples; f.sample_offset = p.sample_offset; f.max_depth = p.max_depth; f.algo = algo_;
    f.npix = (int)np;
    f.records = records ? 1 : 0;

    // persistent grids: a whole number of CTAs per SM
    int occ_t = 1, occ_s = 1, occ_h = 1, occ_t0 = 1;
    const LaunchSet ks = launch_set(algo_, guide, launch_profile_);
    const TraceKernel k_trace = ks.trace;
    const ShadowKernel k_shadow = ks.shadow;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t0, k_trace_primary_t<false>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, k_trace, 128, 0);
    const ShadeKernel shade = ks.shade;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, shade, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k_shadow, 128, 0);
    const int g_trace0 = num_sms_ * std::max(1, occ_t0);
    const int g_trace = num_sms_ * std::max(1, occ_t), g_shade = num_sms_ * std::max(1, occ_s),
              g_shadow = num_sms_ * std::max(1, occ_h);
    const int g_bin = num_sms_ * 8;
    PathView gv = P.view;   // the path view with the guide's buffers when guiding
    if (guide) {
        int rc2 = guide_buffers(wave_paths);
        if (rc2 != LUCID_OK) return rc2;
        GuideState& G = *guide_;
        gv.gmix = G.gmix.p; gv.gslot = G.gslot.p; gv.ginv = G.ginv.p; gv.grec = G.recs.p; gv.gcount = G.count.p;
        gv.gcap = G.steps * kGuideBatch;
        gv.gdepth = G.max_depth;
        for (int k = 0; k < 3; ++k) {
            gv.glo[k] = scene_lo_[k];
            float ext = scene_hi_[k] - scene_lo_[k];
            gv.gscale[k] = ext > 0.0f ? 1.0f / ext : 0.0f;
        }
        static bool attr = false;
        if (!attr) {
            CK(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
            attr = true;
        }
    }
    // the shading queue is binned at every depth (the volume bit only for
    // the integrators with media, the hit-point cells on large waves)
    const int bins = ((algo_ == ALGO_VOLUME_MIS || algo_ == ALGO_VOLUME_SIMPLE) ? kBinVolume : 0) |
                     (wave_paths >= kCellBinPaths ? kBinCells : 0);

    struct Launch { int kind; cudaEvent_t a, b; int depth; };
    std::vector<Launch> launches;
    auto ev_begin = [&](int kind, int depth) -> int {
        if (!profile) return -1;
        Launch l{kind, nullptr, nullptr, depth};
        cudaEventCreate(&l.a);
        cudaEventCreate(&l.b);
        cudaEventRecord(l.a, st);
        launches.push_back(l);
        return (int)launches.size() - 1;
    };
    auto ev_end = [&](int idx) { if (idx >= 0) cudaEventRecord(launches[idx].b, st); };

    stats_ = LucidRenderStats{};
    double seg = 0, shadows = 0;
    std::vector<int> hcnt((size_t)kCountersPerDepth * (p.max_depth + 1));
    std::vector<double> kind_units(K_NUM, 0.0);
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    int status = LUCID_OK;
    int waves = 0;
    for (int s0 = 0; s0 < p.samples; s0 += spw) {
        if (!from_async && is_cancelled()) { status = LUCID_ERR_CANCELLED; break; }
        int this_spw = std::min(spw, p.samples - s0);
        f.s0 = s0;
        f.n_wave = (int)((long long)this_spw * (long long)np);
        CK(cudaMemsetAsync(P.counters.p, 0, sizeof(int) * kCountersPerDepth * (p.max_depth + 1), st));
        if (guide) {
            GuideState& G = *guide_;
            gv.gkeep = (unsigned)std::min(4294967295.0, (double)G.keep * 4294967296.0);
            CK(cudaMemsetAsync(G.gslot.p, 0xff, (size_t)f.n_wave * sizeof(int4), st));
            CK(cudaMemsetAsync(G.count.p, 0, 2 * sizeof(int), st));
        }
        int e = 0;
        for (int depth = 0; depth < p.max_depth; ++depth) {
            int* cnt = P.counters.p + kCountersPerDepth * depth;
            int* cnt_next = P.counters.p + kCountersPerDepth * (depth + 1);
            PathView pv = gv;
            // queue ping-pong: depth d reads q[d&1] and writes q[(d+1)&1]
            int* qin = (depth & 1) ? P.q1.p : P.q0.p;
            int* qout = (depth & 1) ? P.q0.p : P.q1.p;
            pv.q0 = qin;
            if (depth == 0) {
                e = ev_begin(K_TRACE0, depth);
                k_trace_primary_for(ds_->view, f.pos)<<<g_trace0, 128, 0, st>>>(ds_->view, f, pv, cnt, f.records, bins);
            } else {
                e = ev_begin(K_TRACE, depth);
                k_trace<<<g_trace, 128, 0, st>>>(ds_->view, pv, cnt, 0, f.records, bins);
            }
            ev_end(e);
            if (guide && depth < guide_->max_depth) {
                e = ev_begin(K_GUIDE, depth);
                k_guide_infer<<<num_sms_, 32 * kInferWarps, kInferSmem, st>>>(
                    ds_->view, pv, cnt, depth == 0, qin, static_cast<const __nv_bfloat16*>(guide_->net.weights_bf16()),
                    guide_->net.master());
                ev_end(e);
            }
            e = ev_begin(K_BIN, depth);
            k_bin_scatter<<<g_bin, 256, 0, st>>>(pv, cnt, depth == 0, qin, P.qb.p);
            ev_end(e);
            e = ev_begin(K_SHADE, depth);
            shade<<<g_shade, 128, 0, st>>>(ds_->view, f, pv, cnt, cnt_next, 0, P.qb.p, qout);
            ev_end(e);
            e = ev_begin(K_SHADOW, depth);
            k_shadow<<<g_shadow, 128, 0, st>>>(ds_->view, pv, cnt, f.records);
            ev_end(e);
        }
        e = ev_begin(K_FILM, 0);
        if (out_f64)
            k_film_f64<<<(f.npix + 255) / 256, 256, 0, st>>>(f.npix, this_spw, P.rad.p, P.film64.p);
        else
            k_film<<<(f.npix + 255) / 256, 256, 0, st>>>(f.npix, this_spw, P.rad.p, P.film.p);
        ev_end(e);
        if (records) k_records<<<(f.n_wave + 255) / 256, 256, 0, st>>>(f, P.view, d_recs.p);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hcnt.data(), P.counters.p, hcnt.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
        int gcnt[2] = {0, 0};
        if (guide) CK(cudaMemcpyAsync(gcnt, guide_->count.p, sizeof(gcnt), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (guide) {
            // Adam steps on this wave's records, one batch each; the next
            // wave's sampling rate aims at 90 % of the batches
            GuideState& G = *guide_;
            int nrec = std::min(gcnt[0], G.steps * kGuideBatch);
            e = ev_begin(K_TRAIN, 0);
            for (int b = 0; b * kGuideBatch < nrec; ++b)
                if (G.net.train_step(G.recs.p + (size_t)b * kGuideBatch, std::min(kGuideBatch, nrec - b * kGuideBatch),
                                     st, G.lr) != 0)
                    return fail(LUCID_ERR_CUDA, "guide training: " + G.net.error());
            ev_end(e);
            if (profile) kind_units[K_TRAIN] += nrec;
            G.keep = (float)std::min(1.0, 0.9 * G.steps * kGuideBatch / std::max(1.0, (double)gcnt[1]));
        }
        for (int d = 0; d < p.max_depth; ++d) {
            seg += hcnt[kCountersPerDepth * d];
            shadows += hcnt[kCountersPerDepth * d + 1];
        }
        if (profile) {
            kind_units[K_FILM] += f.n_wave;
            for (int d = 0; d < p.max_depth; ++d) {
                kind_units[d == 0 ? K_TRACE0 : K_TRACE] += hcnt[kCountersPerDepth * d];
                kind_units[K_SHADE] += hcnt[kCountersPerDepth * d];
                kind_units[K_BIN] += hcnt[kCountersPerDepth * d];
                if (guide) kind_units[K_GUIDE] += hcnt[kCountersPerDepth * d];
                kind_units[K_SHADOW] += hcnt[kCountersPerDepth * d + 1];
            }
        }
        ++waves;
    }
    int np_i = (int)np;
    if (accumulate)
        k_accumulate<<<(np_i + 255) / 256, 256, 0, st>>>(np_i, P.film.p, (float4*)accumulate);
    else if (out_f64)
        k_output_f64<<<(np_i + 255) / 256, 256, 0, st>>>(p.tile_w, p.tile_h, P.film64.p, P.out64.p);
    else
        k_output<<<(np_i + 255) / 256, 256, 0, st>>>(p.tile_w, p.tile_h, P.film.p,
                                                     out_device ? (float4*)out_device : P.out.p);
    cudaEventRecord(t1, st);
    int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, P.errors.p, sizeof(herr), cudaMemcpyDeviceToHost, st));
    if (out_host && !out_device)
        CK(cudaMemcpyAsync(out_host, P.out.p, np * sizeof(float4), cudaMemcpyDeviceToHost, st));
    if (out_f64)
        CK(cudaMemcpyAsync(out_f64, P.out64.p, np * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (records)
        CK(cudaMemcpyAsync(recs, d_recs.p, np * (size_t)p.samples * sizeof(LucidSampleRecord), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    host_image.copied = true;
    if (guide && guide_->net.failed(st) != 0) return fail(LUCID_ERR_TIMEOUT, guide_->net.error());
    float tot = 0.0f;
    cudaEventElapsedTime(&tot, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    stats_.total_ms = tot;
    stats_.paths = (double)np * p.samples;
    stats_.segments = seg;
    stats_.shadow_rays = shadows;
    stats_.waves = waves;
    if (profile) {
        stats_.num_kinds = K_NUM;
        for (int k = 0; k < K_NUM; ++k) {
            std::snprintf(stats_.kinds[k].name, sizeof(stats_.kinds[k].name), "%s", kKindNames[k]);
            stats_.kinds[k].units = kind_units[k];
            stats_.kinds[k].algo_bytes = kind_units[k] * kKindBytes[k];
        }
        for (auto& l : launches) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, l.a, l.b);
            stats_.kinds[l.kind].launches += 1;
            stats_.kinds[l.kind].total_ms += ms;
            cudaEventDestroy(l.a);
            cudaEventDestroy(l.b);
        }
        stats_.kinds[K_FILM].algo_bytes += (double)np * 32.0 * waves;
    }
    if (herr[0] != 0) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    if (status == LUCID_ERR_CANCELLED) return fail(LUCID_ERR_CANCELLED, "render cancelled");
    return LUCID_OK;
}

// ---------------------------------------------------------------- batched jobs (host)
static int algo_from_name(const char* name) {
    std::string a = name ? name : "";
    if (a == "simple") return ALGO_SIMPLE;
    if (a == "mis") return ALGO_MIS;
    if (a == "volume_simple") return ALGO_VOLUME_SIMPLE;
    if (a == "volume_mis") return ALGO_VOLUME_MIS;
    return ALGO_NEE;   // the reference's dispatch falls through to traceNEE
}

long long Engine::batch_bytes(long long pixels, long long wave_paths) {
    // path state (170 B) and scene index (2 B) per path with slack, film and
    // output per pixel, the job and scene tables
    return wave_paths * 178 + pixels * 32 + (2 << 20);
}

// Jobs on different scenes (and cameras, image sizes, sample counts) in one
// set of wavefront launches: the jobs' samples are cut into pieces that fill
// waves of up to `wave_paths` paths in job order (a job larger than a wave
// continues in the next one, in sample order); a wave's device job table
// gives the camera-ray kernel each piece's camera, image, sample range,
// scene and first path, and every later kernel reads a path's scene from the
// wave's scene table.  Each job's film sums its samples in sample order, so
// its image is the one lucid_cuda_render gives for the same call on its own
// scene, bit for bit.
int Engine::render_batch(const BatchItem* items, int n, const char* algorithm, long long wave_paths) {
    GpuLock gl(*this);
    reset_cancel();
    if (n <= 0 || !items) return fail(LUCID_ERR_INVALID, "batch: no jobs");
    // a call that returns before the images are copied out leaves every
    // job's image zero, as a single render call does
    struct ZeroUnlessCopied {
        const BatchItem* it;
        int n;
        bool copied = false;
        ~ZeroUnlessCopied() {
            if (copied) return;
            for (int j = 0; j < n; ++j)
                if (it[j].out_host && it[j].p.tile_w > 0 && it[j].p.tile_h > 0)
                    std::fill(it[j].out_host, it[j].out_host + (size_t)it[j].p.tile_w * it[j].p.tile_h * 4, 0.0f);
        }
    } host_images{items, n};
    const int algo = algo_from_name(algorithm);
    const int depth = items[0].p.max_depth;
    if (depth < 1 || depth > kMaxDepth) return fail(LUCID_ERR_INVALID, "batch: max_depth must be 1..1024");
    std::vector<const DeviceScene*> scenes;
    std::vector<int> job_sid((size_t)n);
    std::vector<size_t> film_off((size_t)n + 1, 0);
    long long total_paths = 0, max_np = 1;
    for (int j = 0; j < n; ++j) {
        const LucidRenderParams& p = items[j].p;
        if (!items[j].scene || !items[j].out_host) return fail(LUCID_ERR_INVALID, "batch: a job has no scene or output");
        if (p.tile_w <= 0 || p.tile_h <= 0 || p.full_w <= 0 || p.full_h <= 0)
            return fail(LUCID_ERR_INVALID, "batch: tile and image sizes must be positive");
        if (p.samples <= 0) return fail(LUCID_ERR_INVALID, "batch: samples must be >= 1");
        if (p.max_depth != depth) return fail(LUCID_ERR_INVALID, "batch: every job needs the same max_depth");
        const long long np = (long long)p.tile_w * p.tile_h;
        if (np > (1LL << 28)) return fail(LUCID_ERR_INVALID, "batch: tile too large");
        const DeviceScene* ds = static_cast<const DeviceScene*>(items[j].scene);
        int k = 0;
        while (k < (int)scenes.size() && scenes[k] != ds) ++k;
        if (k == (int)scenes.size()) {
            if (scenes.size() >= 65535) return fail(LUCID_ERR_INVALID, "batch: more than 65535 scenes");
            scenes.push_back(ds);
        }
        job_sid[j] = k;
        film_off[j + 1] = film_off[j] + (size_t)np;
        total_paths += np * p.samples;
        max_np = std::max(max_np, np);
    }
    CK(cudaSetDevice(device_));
    int rc = ensure_stream();
    if (rc != LUCID_OK) return rc;
    cudaStream_t st = S(stream_);
    long long cap = wave_paths > 0 ? wave_paths : wave_cap_;
    if (cap <= 0) cap = pool_->cap >= total_paths ? pool_->cap : default_wave_paths(false);
    cap = std::max(cap, max_np);                 // one sample of the largest tile per wave at least
    cap = std::min(cap, std::max(total_paths, max_np));
    if (cap >= (1LL << 31) - 64) return fail(LUCID_ERR_INVALID, "batch: wave too large");
    rc = ensure_pool(cap, false);
    if (rc != LUCID_OK) return rc;
    PathPool& P = *pool_;
    if (P.sid.n < (size_t)P.cap) CK(P.sid.alloc((size_t)P.cap));
    const size_t npix_all = film_off[(size_t)n];
    if (P.film_n < npix_all) {
        CK(P.film.alloc(npix_all));
        CK(P.out.alloc(npix_all));
        P.film_n = npix_all;
    }
    CK(cudaMemsetAsync(P.film.p, 0, npix_all * sizeof(float4), st));
    CK(cudaMemsetAsync(P.errors.p, 0, 4 * sizeof(int), st));

    // the scene table, then room for the largest wave's job table
    std::vector<DevScene> scene_tab(scenes.size());
    for (size_t k = 0; k < scenes.size(); ++k) scene_tab[k] = scenes[k]->view;
    const size_t tab_off = (scene_tab.size() * sizeof(DevScene) + 255) & ~(size_t)255;
    const size_t tab_bytes = tab_off + (size_t)kMaxBatchPieces * sizeof(BatchJob);
    if (P.btab.n < tab_bytes) CK(P.btab.alloc(tab_bytes));
    CK(cudaMemcpyAsync(P.btab.p, scene_tab.data(), scene_tab.size() * sizeof(DevScene), cudaMemcpyHostToDevice, st));
    const DevScene* d_scenes = reinterpret_cast<const DevScene*>(P.btab.p);
    const BatchJob* d_jobs = reinterpret_cast<const BatchJob*>(P.btab.p + tab_off);

    std::vector<HostCamera> cams((size_t)n);
    for (int j = 0; j < n; ++j) {
        const float* c = items[j].camera;
        make_camera(cams[j], c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9]);
    }
    auto frame_of = [&](int j, int s0, int spw) {
        const LucidRenderParams& p = items[j].p;
        const HostCamera& cam = cams[j];
        FrameParams f{};
        for (int k = 0; k < 3; ++k) { f.pos[k] = cam.pos[k]; f.fwd[k] = cam.forward[k]; f.right[k] = cam.right[k]; f.up[k] = cam.up[k]; }
        f.aspect = (float)p.full_w / (float)p.full_h;
        f.scale = std::tan(cam.fov * 0.5f);
        f.tile_x = p.tile_x; f.tile_y = p.tile_y; f.tile_w = p.tile_w; f.tile_h = p.tile_h;
        f.full_w = p.full_w; f.full_h = p.full_h;
        f.samples = p.samples; f.sample_offset = p.sample_offset; f.max_depth = depth; f.algo = algo;
        f.npix = p.tile_w * p.tile_h;
        f.s0 = s0;
        f.n_wave = spw * f.npix;
        return f;
    };

    const LaunchSet ks = launch_set_batch(algo);
    int occ_t0 = 1, occ_t = 1, occ_s = 1, occ_h = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t0, k_trace_primary_batch, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, ks.trace, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, ks.shade, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, ks.shadow, 128, 0);
    const int g_trace0 = num_sms_ * std::max(1, occ_t0), g_trace = num_sms_ * std::max(1, occ_t),
              g_shade = num_sms_ * std::max(1, occ_s), g_shadow = num_sms_ * std::max(1, occ_h);
    const int g_bin = num_sms_ * 8;
    FrameParams fshade{};
    fshade.max_depth = depth;
    fshade.algo = algo;

    stats_ = LucidRenderStats{};
    double seg = 0, shadows = 0;
    std::vector<int> hcnt((size_t)kCountersPerDepth * (depth + 1));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    int waves = 0, status = LUCID_OK;
    std::vector<BatchJob> tab;
    struct PieceFilm { int job, spw, path_base; };
    std::vector<PieceFilm> films;
    int j = 0, s = 0;   // next sample s of job j still to render
    while (j < n) {
        if (is_cancelled()) { status = LUCID_ERR_CANCELLED; break; }
        // fill one wave with pieces, in job order
        tab.clear();
        films.clear();
        long long used = 0, slots = 0;
        while (j < n && (int)tab.size() < kMaxBatchPieces) {
            const LucidRenderParams& p = items[j].p;
            const long long np = (long long)p.tile_w * p.tile_h;
            const int take = (int)std::min<long long>(p.samples - s, (cap - used) / np);
            if (take < 1) break;
            const long long per_sample = (long long)((p.tile_w + 7) / 8) * ((p.tile_h + 3) / 4) * 32;
            if (slots + per_sample * take >= (1LL << 31) - 64) break;
            BatchJob b{};
            b.f = frame_of(j, s, take);
            b.sid = job_sid[j];
            b.path_base = (int)used;
            b.slot_base = (int)slots;
            tab.push_back(b);
            films.push_back({j, take, (int)used});
            used += np * take;
            slots += per_sample * take;
            s += take;
            if (s >= p.samples) { ++j; s = 0; }
        }
        if (tab.empty()) return fail(LUCID_ERR_INVALID, "batch: a job piece does not fit a wave");
        CK(cudaMemcpyAsync(const_cast<BatchJob*>(d_jobs), tab.data(), tab.size() * sizeof(BatchJob),
                           cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(P.counters.p, 0, sizeof(int) * kCountersPerDepth * (depth + 1), st));
        const int n_wave = (int)used;
        const int bins = ((algo == ALGO_VOLUME_MIS || algo == ALGO_VOLUME_SIMPLE) ? kBinVolume : 0) |
                         (n_wave >= kCellBinPaths ? kBinCells : 0);
        PathView pv = P.view;
        pv.scenes = d_scenes;
        pv.sid = P.sid.p;
        for (int dd = 0; dd < depth; ++dd) {
            int* cnt = P.counters.p + kCountersPerDepth * dd;
            int* cnt_next = P.counters.p + kCountersPerDepth * (dd + 1);
            int* qin = (dd & 1) ? P.q1.p : P.q0.p;
            int* qout = (dd & 1) ? P.q0.p : P.q1.p;
            pv.q0 = qin;
            if (dd == 0)
                k_trace_primary_batch<<<g_trace0, 128, 0, st>>>(pv, d_jobs, (int)tab.size(), (int)slots, n_wave, cnt, bins);
            else
                ks.trace<<<g_trace, 128, 0, st>>>(scene_tab[0], pv, cnt, 0, 0, bins);
            k_bin_scatter<<<g_bin, 256, 0, st>>>(pv, cnt, dd == 0, qin, P.qb.p);
            ks.shade<<<g_shade, 128, 0, st>>>(scene_tab[0], fshade, pv, cnt, cnt_next, 0, P.qb.p, qout);
            ks.shadow<<<g_shadow, 128, 0, st>>>(scene_tab[0], pv, cnt, 0);
        }
        for (const PieceFilm& pf : films) {
            const int np_j = (int)(film_off[(size_t)pf.job + 1] - film_off[(size_t)pf.job]);
            k_film<<<(np_j + 255) / 256, 256, 0, st>>>(np_j, pf.spw, P.rad.p + pf.path_base, P.film.p + film_off[pf.job]);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hcnt.data(), P.counters.p, hcnt.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int d = 0; d < depth; ++d) {
            seg += hcnt[kCountersPerDepth * d];
            shadows += hcnt[kCountersPerDepth * d + 1];
        }
        ++waves;
    }
    for (int k = 0; k < n && status == LUCID_OK; ++k) {
        const LucidRenderParams& p = items[k].p;
        const int np_k = p.tile_w * p.tile_h;
        k_output<<<(np_k + 255) / 256, 256, 0, st>>>(p.tile_w, p.tile_h, P.film.p + film_off[k], P.out.p + film_off[k]);
    }
    cudaEventRecord(t1, st);
    int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, P.errors.p, sizeof(herr), cudaMemcpyDeviceToHost, st));
    if (status == LUCID_OK)
        for (int k = 0; k < n; ++k)
            CK(cudaMemcpyAsync(items[k].out_host, P.out.p + film_off[k],
                               (film_off[(size_t)k + 1] - film_off[k]) * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    host_images.copied = status == LUCID_OK;
    float tot = 0.0f;
    cudaEventElapsedTime(&tot, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    stats_.total_ms = tot;
    stats_.paths = (double)total_paths;
    stats_.segments = seg;
    stats_.shadow_rays = shadows;
    stats_.waves = waves;
    if (herr[0] != 0) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    if (status == LUCID_ERR_CANCELLED) return fail(LUCID_ERR_CANCELLED, "render cancelled");
    return LUCID_OK;
}

// ---------------------------------------------------------------- path guiding (host)
int Engine::guide_buffers(long long paths) {
    GuideState& G = *guide_;
    if (G.cap < paths) {
        CK(G.gmix.alloc((size_t)paths * kGMixFloats));
        CK(G.gslot.alloc((size_t)paths));
        CK(G.ginv.alloc((size_t)paths * 3));
        G.cap = paths;
    }
    if ((long long)G.recs.n < (long long)G.steps * kGuideBatch) CK(G.recs.alloc((size_t)G.steps * kGuideBatch));
    if (!G.count.p) CK(G.count.alloc(2));
    return LUCID_OK;
}

int Engine::guide_enable(bool on, int seed) {
    GpuLock gl(*this);
    CK(cudaSetDevice(device_));
    if (!on) {
        if (guide_) guide_->on = false;
        return LUCID_OK;
    }
    int rc = ensure_stream();
    if (rc != LUCID_OK) return rc;
    if (!guide_) guide_ = new GuideState();
    if (guide_->net.init(seed, S(stream_)) != 0) return fail(LUCID_ERR_CUDA, "guide init: " + guide_->net.error());
    CK(cudaStreamSynchronize(S(stream_)));
    guide_->keep = 1.0f;
    guide_->on = true;
    return LUCID_OK;
}

int Engine::guide_steps() const { return guide_ ? guide_->net.steps() : 0; }

int Engine::guide_params(float* out, size_t cap, float* box6) {
    GpuLock gl(*this);
    if (!guide_) return fail(LUCID_ERR_INVALID, "guide: not enabled on this context");
    if (cap < (size_t)kGuideParams) return fail(LUCID_ERR_INVALID, "guide: output buffer too small");
    CK(cudaSetDevice(device_));
    if (guide_->net.get_params(out, S(stream_)) != 0) return fail(LUCID_ERR_CUDA, guide_->net.error());
    if (box6)
        for (int k = 0; k < 3; ++k) { box6[k] = scene_lo_[k]; box6[3 + k] = scene_hi_[k]; }
    return kGuideParams;
}

int Engine::guide_config(int steps_per_wave, float lr) {
    GpuLock gl(*this);
    if (steps_per_wave < 1 || steps_per_wave > 64 || !(lr > 0.0f)) return fail(LUCID_ERR_INVALID, "guide: bad config");
    if (!guide_) guide_ = new GuideState();
    guide_->steps = steps_per_wave;
    guide_->lr = lr;
    return LUCID_OK;
}

int Engine::guide_max_depth(int max_depth) {
    GpuLock gl(*this);
    if (max_depth < 1 || max_depth > kMaxDepth) return fail(LUCID_ERR_INVALID, "guide: bad guided depth");
    if (!guide_) guide_ = new GuideState();
    guide_->max_depth = max_depth;
    return LUCID_OK;
}

// ---------------------------------------------------------------- progressive jobs
// A job renders one image progressively: each iteration adds n samples to a
// film that keeps its sum across iterations, pixel by pixel in sample order,
// so a job's image is bit-identical to one render call with all its samples
// (camera rays are jittered whenever the job has more than one sample, as in
// that call).  Iterations of `chunk` samples are captured once into a CUDA
// graph and replayed; the sample offset comes from a device integer that a
// one-thread kernel sets before each replay.  Nothing in an iteration waits
// for the host, so iterations of jobs on different engines (streams) overlap
// on the device.
__global__ void k_set_int(int* p, int v) { *p = v; }

struct JobState {
    int w = 0, h = 0, spp = 0, depth = 8, chunk = 1;
    bool active = false;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};   // iteration k records ev[k & 1]
    long long issued = 0;
    DBuf<int> dyn;
    FrameParams f{};
    int g_trace0 = 0, g_trace = 0, g_shade = 0, g_shadow = 0, g_bin = 0;
    int profile = 0;   // launch profile of the job's kernels
};

long long Engine::job_bytes(int w, int h, int chunk) {
    const long long np = (long long)w * h;
    return (long long)chunk * np * 176 + np * 32 + (1 << 20);   // path state (170 B) with slack
}

void Engine::enqueue_iteration(void* fp, int n) {
    JobState& J = *job_;
    FrameParams f = *static_cast<const FrameParams*>(fp);
    PathPool& P = *pool_;
    cudaStream_t st = S(stream_);
    f.s0 = 0;
    f.samples = n;
    f.n_wave = n * f.npix;
    const LaunchSet ks = launch_set(algo_, false, J.profile);
    const ShadeKernel shade = ks.shade;
    const TraceKernel k_trace = ks.trace;
    const ShadowKernel k_shadow = ks.shadow;
    const int bins = ((algo_ == ALGO_VOLUME_MIS || algo_ == ALGO_VOLUME_SIMPLE) ? kBinVolume : 0) |
                     ((long long)f.n_wave >= kCellBinPaths ? kBinCells : 0);
    cudaMemsetAsync(P.counters.p, 0, sizeof(int) * kCountersPerDepth * (J.depth + 1), st);
    for (int depth = 0; depth < J.depth; ++depth) {
        int* cnt = P.counters.p + kCountersPerDepth * depth;
        int* cnt_next = P.counters.p + kCountersPerDepth * (depth + 1);
        PathView pv = P.view;
        int* qin = (depth & 1) ? P.q1.p : P.q0.p;
        int* qout = (depth & 1) ? P.q0.p : P.q1.p;
        pv.q0 = qin;
        if (depth == 0) k_trace_primary_for(ds_->view, f.pos)<<<J.g_trace0, 128, 0, st>>>(ds_->view, f, pv, cnt, 0, bins);
        else k_trace<<<J.g_trace, 128, 0, st>>>(ds_->view, pv, cnt, 0, 0, bins);
        k_bin_scatter<<<J.g_bin, 256, 0, st>>>(pv, cnt, depth == 0, qin, P.qb.p);
        shade<<<J.g_shade, 128, 0, st>>>(ds_->view, f, pv, cnt, cnt_next, 0, P.qb.p, qout);
        k_shadow<<<J.g_shadow, 128, 0, st>>>(ds_->view, pv, cnt, 0);
    }
    k_film<<<(f.npix + 255) / 256, 256, 0, st>>>(f.npix, n, P.rad.p, P.film.p);
}

int Engine::job_begin(int w, int h, int spp, int max_depth, int chunk, bool use_graph) {
    GpuLock gl(*this);
    if (w <= 0 || h <= 0 || spp <= 0 || chunk <= 0) return fail(LUCID_ERR_INVALID, "job: sizes must be positive");
    if (max_depth <= 0 || max_depth > kMaxDepth) return fail(LUCID_ERR_INVALID, "job: bad max_depth");
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    if ((long long)w * h * chunk > 0x7fffffffLL) return fail(LUCID_ERR_INVALID, "job: chunk too large");
    CK(cudaSetDevice(device_));
    job_end_locked();
    if (!job_) job_ = new JobState();
    JobState& J = *job_;
    J.w = w; J.h = h; J.spp = spp; J.depth = max_depth; J.chunk = std::min(chunk, spp);
    const size_t np = (size_t)w * h;
    int rc = ensure_pool((long long)J.chunk * (long long)np, false);
    if (rc != LUCID_OK) return rc;
    PathPool& P = *pool_;
    if (P.film_n < np) {
        CK(P.film.alloc(np));
        CK(P.out.alloc(np));
        P.film_n = np;
    }
    cudaStream_t st = S(stream_);
    CK(cudaMemsetAsync(P.film.p, 0, np * sizeof(float4), st));
    CK(cudaMemsetAsync(P.errors.p, 0, 4 * sizeof(int), st));
    if (!J.dyn.p) CK(J.dyn.alloc(1));
    FrameParams& f = J.f;
    f = FrameParams{};
    for (int k = 0; k < 3; ++k) { f.pos[k] = cam_.pos[k]; f.fwd[k] = cam_.forward[k]; f.right[k] = cam_.right[k]; f.up[k] = cam_.up[k]; }
    f.aspect = (float)w / (float)h;
    f.scale = std::tan(cam_.fov * 0.5f);
    f.tile_w = w; f.tile_h = h; f.full_w = w; f.full_h = h;
    f.max_depth = max_depth; f.algo = algo_;
    f.npix = (int)np;
    f.jitter = spp > 1 ? 1 : 0;
    J.profile = launch_profile_;
    job_grids_locked();
    for (int k = 0; k < 2; ++k)
        if (!J.ev[k]) CK(cudaEventCreateWithFlags(&J.ev[k], cudaEventDisableTiming));
    J.issued = 0;
    J.active = true;
    return use_graph ? capture_locked(J.chunk) : LUCID_OK;
}

// Captures one iteration of `chunk` samples into a graph (chunk <= the
// chunk the job's path state was sized for).
int Engine::capture_locked(int chunk) {
    JobState& J = *job_;
    cudaStream_t st = S(stream_);
    if (J.graph) { cudaGraphExecDestroy(J.graph); J.graph = nullptr; }
    FrameParams fg = J.f;
    fg.dyn = J.dyn.p;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    enqueue_iteration(&fg, chunk);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) return fail(LUCID_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&J.graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { J.graph = nullptr; return fail(LUCID_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
    J.chunk = chunk;
    return LUCID_OK;
}

// Persistent grids of the job's kernels for its launch profile: a whole
// number of CTAs per SM.
void Engine::job_grids_locked() {
    JobState& J = *job_;
    const LaunchSet ks = launch_set(algo_, false, J.profile);
    int occ_t = 1, occ_s = 1, occ_h = 1, occ_t0 = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t0, k_trace_primary_t<false>, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, ks.trace, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, ks.shade, 128, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, ks.shadow, 128, 0);
    J.g_trace0 = num_sms_ * std::max(1, occ_t0);
    J.g_trace = num_sms_ * std::max(1, occ_t);
    J.g_shade = num_sms_ * std::max(1, occ_s);
    J.g_shadow = num_sms_ * std::max(1, occ_h);
    J.g_bin = num_sms_ * 8;
}

int Engine::set_launch_profile(int profile) {
    GpuLock gl(*this);
    if (profile < 0 || profile >= kLaunchProfiles) return fail(LUCID_ERR_INVALID, "unknown launch profile");
    launch_profile_ = profile;
    return LUCID_OK;
}

int Engine::job_set_profile(int profile, bool use_graph) {
    GpuLock gl(*this);
    if (!job_ || !job_->active) return fail(LUCID_ERR_INVALID, "no job");
    if (profile < 0 || profile >= kLaunchProfiles) return fail(LUCID_ERR_INVALID, "unknown launch profile");
    CK(cudaSetDevice(device_));
    // iterations in flight were enqueued with the old grids; they finish first
    CK(cudaStreamSynchronize(S(stream_)));
    job_->profile = profile;
    job_grids_locked();
    if (use_graph) return capture_locked(job_->chunk);
    if (job_->graph) { cudaGraphExecDestroy(job_->graph); job_->graph = nullptr; }
    return LUCID_OK;
}

int Engine::job_set_chunk(int chunk, bool use_graph) {
    GpuLock gl(*this);
    if (!job_ || !job_->active) return fail(LUCID_ERR_INVALID, "no job");
    if (chunk <= 0 || (long long)chunk * job_->w * job_->h > pool_->cap)
        return fail(LUCID_ERR_INVALID, "job: chunk exceeds the job's path state");
    CK(cudaSetDevice(device_));
    if (use_graph) return capture_locked(chunk);
    if (job_->graph) { cudaGraphExecDestroy(job_->graph); job_->graph = nullptr; }
    job_->chunk = chunk;
    return LUCID_OK;
}

int Engine::job_iterate(int sample_offset, int n) {
    GpuLock gl(*this);
    if (!job_ || !job_->active) return fail(LUCID_ERR_INVALID, "no job");
    JobState& J = *job_;
    if (n <= 0 || n > J.chunk) return fail(LUCID_ERR_INVALID, "job: iteration size must be in [1, chunk]");
    CK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    // at most two iterations in flight per job: wait for iteration k - 2
    if (J.issued >= 2) CK(cudaEventSynchronize(J.ev[J.issued & 1]));
    if (J.graph && n == J.chunk) {
        k_set_int<<<1, 1, 0, st>>>(J.dyn.p, sample_offset);
        CK(cudaGraphLaunch(J.graph, st));
    } else {
        FrameParams f = J.f;
        f.sample_offset = sample_offset;
        enqueue_iteration(&f, n);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(J.ev[J.issued & 1], st));
    ++J.issued;
    return LUCID_OK;
}

int Engine::job_wait() {
    GpuLock gl(*this);
    CK(cudaSetDevice(device_));
    CK(cudaStreamSynchronize(S(stream_)));
    int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpy(herr, pool_->errors.p, sizeof(herr), cudaMemcpyDeviceToHost));
    if (herr[0] != 0) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    return LUCID_OK;
}

int Engine::job_output(float* out_host) {
    GpuLock gl(*this);
    if (!job_ || !job_->active) return fail(LUCID_ERR_INVALID, "no job");
    JobState& J = *job_;
    CK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    const int np = J.w * J.h;
    k_output<<<(np + 255) / 256, 256, 0, st>>>(J.w, J.h, pool_->film.p, pool_->out.p);
    CK(cudaMemcpyAsync(out_host, pool_->out.p, (size_t)np * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LUCID_OK;
}

long long Engine::guide_job_bytes(long long paths) {
    // per path: compact mixture (40 floats), slot and inverse-throughput
    // entries; fixed: two batches of records, the feature-major training
    // workspace and the per-block partial gradients
    return paths * (kGMixFloats * 4 + 16 + 48) + 2LL * kGuideBatch * (long long)sizeof(GuideRec) +
           608LL * kGuideBatch * 2 + 148LL * 51200 * 4 + (1 << 20);
}

int Engine::accum_begin(int w, int h) {
    GpuLock gl(*this);
    if (w <= 0 || h <= 0) return fail(LUCID_ERR_INVALID, "accumulator: sizes must be positive");
    CK(cudaSetDevice(device_));
    int rc = ensure_stream();
    if (rc != LUCID_OK) return rc;
    const size_t np = (size_t)w * h;
    if (jacc_n_ < np) {
        if (jacc_) cudaFree(jacc_);
        jacc_ = nullptr;
        jacc_n_ = 0;
        CK(cudaMalloc(&jacc_, np * sizeof(float4)));
        jacc_n_ = np;
    }
    jacc_w_ = w;
    jacc_h_ = h;
    CK(cudaMemsetAsync(jacc_, 0, np * sizeof(float4), S(stream_)));
    return LUCID_OK;
}

int Engine::render_accumulate(const LucidRenderParams& p) {
    GpuLock gl(*this);
    if (!jacc_ || p.tile_w != jacc_w_ || p.tile_h != jacc_h_) return fail(LUCID_ERR_INVALID, "accumulator size mismatch");
    return render_impl(p, nullptr, nullptr, nullptr, jacc_, false);
}

int Engine::accum_output(float* out_host) {
    GpuLock gl(*this);
    if (!jacc_) return fail(LUCID_ERR_INVALID, "no accumulator");
    CK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    const int np = jacc_w_ * jacc_h_;
    PathPool& P = *pool_;
    if (P.film_n < (size_t)np) { CK(P.film.alloc(np)); CK(P.out.alloc(np)); P.film_n = np; }
    k_output<<<(np + 255) / 256, 256, 0, st>>>(jacc_w_, jacc_h_, (const float4*)jacc_, P.out.p);
    CK(cudaMemcpyAsync(out_host, P.out.p, (size_t)np * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return LUCID_OK;
}

void Engine::accum_end() {
    GpuLock gl(*this);
    if (!jacc_) return;
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(S(stream_));
    cudaFree(jacc_);
    jacc_ = nullptr;
    jacc_n_ = 0;
}

void Engine::guide_free() {
    GpuLock gl(*this);
    if (!guide_) return;
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(S(stream_));
    delete guide_;
    guide_ = nullptr;
}

void Engine::job_end_locked() {
    if (!job_) return;
    if (stream_) cudaStreamSynchronize(S(stream_));
    if (job_->graph) { cudaGraphExecDestroy(job_->graph); job_->graph = nullptr; }
    job_->active = false;
}

void Engine::job_end() {
    GpuLock gl(*this);
    cudaSetDevice(device_);
    job_end_locked();
    if (job_)
        for (int k = 0; k < 2; ++k)
            if (job_->ev[k]) cudaEventDestroy(job_->ev[k]);
    delete job_;
    job_ = nullptr;
}

void Engine::release_pool() {
    GpuLock gl(*this);
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(S(stream_));
    pool_->release();
}

// ---------------------------------------------------------------- async accumulator
// The viewport's progressive mode (PyRenderer::render_start_async ..
// render_stop_async, pybind_renderer.hpp:689-856; the Dawn worker it drives,
// gpu/path_tracer.cpp:838-1090): a worker thread adds one 1-spp render per
// iteration (sample offset n, so iteration n seeds (x, y, n)) into a device
// accumulator and publishes an averaged snapshot after 1, 2, 4, 8 and then
// every 16 samples.  reset() wipes the accumulator without stopping.
int Engine::async_start(int w, int h, int max_depth) {
    async_stop();
    if (w <= 0 || h <= 0) return fail(LUCID_ERR_INVALID, "async: size must be positive");
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    {
        GpuLock gl(*this);
        CK(cudaSetDevice(device_));
        size_t n = (size_t)w * h;
        if (async_acc_n_ < n) {
            if (async_acc_) cudaFree(async_acc_);
            if (async_pinned_) cudaFreeHost(async_pinned_);
            async_acc_ = nullptr;
            async_pinned_ = nullptr;
            async_acc_n_ = 0;
            CK(cudaMalloc(&async_acc_, n * sizeof(float4)));
            CK(cudaMallocHost((void**)&async_pinned_, n * sizeof(float4)));
            async_acc_n_ = n;
        }
        CK(cudaMemset(async_acc_, 0, n * sizeof(float4)));
        async_w_ = w; async_h_ = h; async_depth_ = std::max(1, max_depth);
    }
    {
        std::lock_guard<std::mutex> sl(snap_mu_);
        snap_.clear();
        snap_samples_ = 0;
    }
    async_reset_ = false;
    async_run_ = true;
    async_thread_ = std::thread([this] { async_worker(); });
    return LUCID_OK;
}

int Engine::async_reset(int w, int h, int max_depth) {
    if (!async_run_) return LUCID_OK;
    if ((size_t)w * h > async_acc_n_ || w <= 0 || h <= 0)
        return fail(LUCID_ERR_INVALID, "async reset: a larger resolution needs stop + start");
    {
        GpuLock gl(*this);
        async_w_ = w; async_h_ = h; async_depth_ = std::max(1, max_depth);
    }
    async_reset_ = true;
    return LUCID_OK;
}

int Engine::async_stop() {
    async_run_ = false;
    if (async_thread_.joinable()) async_thread_.join();
    return LUCID_OK;
}

int Engine::async_poll(int* samples, float* out, size_t cap_floats) {
    std::lock_guard<std::mutex> sl(snap_mu_);
    *samples = snap_samples_;
    if (snap_samples_ == 0) return LUCID_OK;
    if (!out || cap_floats < snap_.size()) return fail(LUCID_ERR_INVALID, "async poll: output buffer too small");
    std::copy(snap_.begin(), snap_.end(), out);
    return LUCID_OK;
}

void Engine::async_worker() {
    cudaSetDevice(device_);
    long long n = 0;
    int w = 0, h = 0, depth = 8;
    while (async_run_) {
        bool wipe = async_reset_.exchange(false);
        // std::mutex is not fair: back off while an API call waits for the
        // GPU, or a set_camera / reset from the UI thread could wait for
        // minutes behind the worker's back-to-back iterations
        while (gpu_waiters_.load() > 0 && async_run_) std::this_thread::sleep_for(std::chrono::microseconds(100));
        {
            std::lock_guard<std::mutex> gl(gpu_mu_);
            if (wipe || w != async_w_ || h != async_h_) {
                w = async_w_; h = async_h_;
                cudaMemsetAsync(async_acc_, 0, (size_t)w * h * sizeof(float4), S(stream_));
                n = 0;
            }
            depth = async_depth_;
            LucidRenderParams p{0, 0, w, h, w, h, 1, (int)n, depth, 0};
            int rc = render_impl(p, nullptr, nullptr, nullptr, async_acc_, true);
            if (rc != LUCID_OK) {
                async_err_ = err_;
            } else {
                ++n;
                if (n <= 8 ? ((n & (n - 1)) == 0) : (n % 16 == 0)) {
                    size_t np = (size_t)w * h;
                    cudaMemcpyAsync(async_pinned_, async_acc_, np * sizeof(float4), cudaMemcpyDeviceToHost, S(stream_));
                    cudaStreamSynchronize(S(stream_));
                    // average, camera sensitivity (EV 0 -> 1), clamp >= 0, alpha 1, Y flip
                    std::vector<float> img(np * 4);
                    const float inv = (float)n;
                    for (int y = 0; y < h; ++y)
                        for (int x = 0; x < w; ++x) {
                            const float* a = async_pinned_ + 4 * ((size_t)y * w + x);
                            float* o = img.data() + 4 * ((size_t)(h - 1 - y) * w + x);
                            for (int c = 0; c < 3; ++c) {
                                float v = (a[c] / inv) * 1.0f;
                                o[c] = (v < 0.0f) ? 0.0f : v;
                            }
                            o[3] = 1.0f;
                        }
                    std::lock_guard<std::mutex> sl(snap_mu_);
                    snap_.swap(img);
                    snap_samples_ = (int)n;
                    async_revision_.fetch_add(1);
                }
            }
        }
        if (async_err_.size()) {
            std::this_thread::sleep_for(std::chrono::milliseconds(2));   // the reference backs off 2 ms
            async_err_.clear();
        }
    }
}

// ---------------------------------------------------------------- no-allocation render
// Some callers cannot allocate device memory when they render: a host whose
// device memory is owned by another allocator (a framework's caching pool
// that hands out every byte), or a latency-critical thread such as a
// viewport draw callback that must not call cudaMalloc/cudaFree because
// those calls can synchronise the whole device.  lucid_cuda_render_noalloc
// serves them with the same kernels as lucid_cuda_render_device, but its
// working memory (path state, queues, counters, film) lives in the
// fixed-size device array below, which every GPU that loads this library
// holds until the process exits.  The scene itself was allocated earlier by
// lucid_cuda_load_scene_json.
constexpr int kNoAllocPaths = 65536;              // paths per wave
constexpr int kNoAllocPixels = 65536;             // tile pixels (e.g. 256 x 256)
constexpr int kNoAllocMaxDepth = 64;
constexpr size_t kNoAllocAlign = 256;
constexpr size_t na_round(size_t b) { return (b + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }
constexpr size_t kNaRng = na_round(sizeof(ulonglong2) * kNoAllocPaths);
constexpr size_t kNaF4 = na_round(sizeof(float4) * kNoAllocPaths);
constexpr size_t kNaF2 = na_round(sizeof(float2) * kNoAllocPaths);
constexpr size_t kNaQ = na_round(sizeof(int) * kNoAllocPaths);
constexpr size_t kNaCnt = na_round(sizeof(int) * kCountersPerDepth * (kNoAllocMaxDepth + 1));
constexpr size_t kNaErr = na_round(sizeof(int) * 4);
constexpr size_t kNaFilm = na_round(sizeof(float4) * kNoAllocPixels);
constexpr size_t kNoAllocBytes = kNaRng + 8 * kNaF4 + kNaF2 + 3 * kNaQ + kNaCnt + kNaErr + kNaFilm;   // ~12 MB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
// Device address of g_noalloc_scratch per device, looked up once with that
// device current (a host-side reference to the array is not a device
// address).
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[64] = {};
// Grid sizes (blocks) of the four wave kernels per device and integrator,
// from the occupancy queries made on that device's first call.
int g_noalloc_grid[64][5][4] = {};
}  // namespace

int Engine::render_noalloc(const LucidRenderParams& p, float* d_out) {
    GpuLock gl(*this);
    reset_cancel();
    if (!d_out) return fail(LUCID_ERR_INVALID, "output pointer is null");
    if (p.tile_w <= 0 || p.tile_h <= 0 || p.full_w <= 0 || p.full_h <= 0)
        return fail(LUCID_ERR_INVALID, "tile and image sizes must be positive");
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    long long np = (long long)p.tile_w * p.tile_h;
    if (np > kNoAllocPixels)
        return fail(LUCID_ERR_INVALID, "render_noalloc: tile of " + std::to_string(np) + " pixels exceeds the " +
                                           std::to_string(kNoAllocPixels) + "-pixel limit of its fixed scratch");
    if (p.max_depth < 1 || p.max_depth > kNoAllocMaxDepth)
        return fail(LUCID_ERR_INVALID, "render_noalloc: max_depth must be in [1, " + std::to_string(kNoAllocMaxDepth) + "]");
    if (p.samples <= 0) return fail(LUCID_ERR_INVALID, "samples must be >= 1");
    if (device_ < 0 || device_ >= 64) return fail(LUCID_ERR_INVALID, "device index out of range");
    if (algo_ < 0 || algo_ > 4) return fail(LUCID_ERR_INVALID, "unknown integrator");
    // Diagnostics and path guiding keep per-render buffers that this entry
    // point cannot allocate; rendering without them would give a different
    // image than lucid_cuda_render_device, so refuse instead.
    if (diag_enabled_)
        return fail(LUCID_ERR_INVALID, "render_noalloc: path diagnostics are enabled; they need allocated record "
                                       "buffers (disable them or use lucid_cuda_render_device)");
    if (guide_ && guide_->on && algo_ == ALGO_MIS)
        return fail(LUCID_ERR_INVALID, "render_noalloc: path guiding is on; it needs allocated training and "
                                       "inference buffers (turn it off or use lucid_cuda_render_device)");
    CK(cudaSetDevice(device_));
    const ShadeKernel shade = shade_kernel(algo_);
    unsigned char* base;
    int grid[4];
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[device_]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return fail(LUCID_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
            g_noalloc_addr[device_] = (unsigned char*)ptr;
        }
        base = g_noalloc_addr[device_];
        int* g = g_noalloc_grid[device_][algo_];
        if (g[0] == 0) {
            int occ[4] = {1, 1, 1, 1};
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_trace_primary_t<false>, 128, 0);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_trace_lb<9>, 128, 0);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], shade, 128, 0);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[3], k_shadow_lb<9>, 128, 0);
            for (int k = 0; k < 4; ++k) g[k] = num_sms_ * std::max(1, occ[k]);
        }
        for (int k = 0; k < 4; ++k) grid[k] = g[k];
    }
    PathView v{};
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char* q = base + off; off += bytes; return (void*)q; };
    v.rng = (ulonglong2*)take(kNaRng);
    v.ray_o = (float4*)take(kNaF4); v.ray_d = (float4*)take(kNaF4); v.thr = (float4*)take(kNaF4);
    v.rad = (float4*)take(kNaF4); v.hit = (float4*)take(kNaF4); v.sh_o = (float4*)take(kNaF4);
    v.sh_d = (float4*)take(kNaF4); v.sh_c = (float4*)take(kNaF4);
    v.lhit = (float2*)take(kNaF2);
    int* q0 = (int*)take(kNaQ);
    int* q1 = (int*)take(kNaQ);
    v.qs = (int*)take(kNaQ);
    v.counters = (int*)take(kNaCnt);
    v.errors = (int*)take(kNaErr);
    float4* film = (float4*)take(kNaFilm);
    v.q0 = q0; v.q1 = q1;
    v.rec_prim = nullptr; v.rec_cnt = nullptr; v.rec_hash = nullptr;

    cudaStream_t st = S(stream_);
    // the array keeps the previous call's contents: clear what starts at zero
    CK(cudaMemsetAsync(film, 0, sizeof(float4) * np, st));
    CK(cudaMemsetAsync(v.errors, 0, sizeof(int) * 4, st));
    FrameParams f{};
    for (int k = 0; k < 3; ++k) { f.pos[k] = cam_.pos[k]; f.fwd[k] = cam_.forward[k]; f.right[k] = cam_.right[k]; f.up[k] = cam_.up[k]; }
    f.aspect = (float)p.full_w / (float)p.full_h;
    f.scale = std::tan(cam_.fov * 0.5f);
    f.tile_x = p.tile_x; f.tile_y = p.tile_y; f.tile_w = p.tile_w; f.tile_h = p.tile_h;
    f.full_w = p.full_w; f.full_h = p.full_h;
    f.samples = p.samples; f.sample_offset = p.sample_offset; f.max_depth = p.max_depth; f.algo = algo_;
    f.npix = (int)np;
    f.records = 0;
    const int g_trace0 = grid[0], g_trace = grid[1], g_shade = grid[2], g_shadow = grid[3];
    const int spw = (int)std::max<long long>(1, std::min<long long>(p.samples, kNoAllocPaths / np));
    int status = LUCID_OK;
    for (int s0 = 0; s0 < p.samples; s0 += spw) {
        if (is_cancelled()) { status = LUCID_ERR_CANCELLED; break; }
        int this_spw = std::min(spw, p.samples - s0);
        f.s0 = s0;
        f.n_wave = (int)(this_spw * np);
        CK(cudaMemsetAsync(v.counters, 0, sizeof(int) * kCountersPerDepth * (p.max_depth + 1), st));
        for (int depth = 0; depth < p.max_depth; ++depth) {
            int* cnt = v.counters + kCountersPerDepth * depth;
            int* cnt_next = v.counters + kCountersPerDepth * (depth + 1);
            PathView pv = v;
            int* qin = (depth & 1) ? q1 : q0;
            int* qout = (depth & 1) ? q0 : q1;
            pv.q0 = qin;
            if (depth == 0) k_trace_primary_for(ds_->view, f.pos)<<<g_trace0, 128, 0, st>>>(ds_->view, f, pv, cnt, 0, -1);
            else k_trace_lb<9><<<g_trace, 128, 0, st>>>(ds_->view, pv, cnt, 0, 0, -1);
            shade<<<g_shade, 128, 0, st>>>(ds_->view, f, pv, cnt, cnt_next, depth == 0, qin, qout);
            k_shadow_lb<9><<<g_shadow, 128, 0, st>>>(ds_->view, pv, cnt, 0);
        }
        k_film<<<(f.npix + 255) / 256, 256, 0, st>>>(f.npix, this_spw, v.rad, film);
        CK(cudaGetLastError());
        // no wait here: stream order keeps the next wave behind this film sum
    }
    k_output<<<(f.npix + 255) / 256, 256, 0, st>>>(p.tile_w, p.tile_h, film, (float4*)d_out);
    int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, v.errors, sizeof(herr), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr[0] != 0) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    if (status == LUCID_ERR_CANCELLED) return fail(LUCID_ERR_CANCELLED, "render cancelled");
    return LUCID_OK;
}

int Engine::render_debug(int tx, int ty, int tw, int th, int fw, int fh, const char* mode, float* out_host) {
    GpuLock gl(*this);
    reset_cancel();
    if (tw <= 0 || th <= 0 || fw <= 0 || fh <= 0) return fail(LUCID_ERR_INVALID, "tile and image sizes must be positive");
    size_t np = (size_t)tw * th;
    std::fill(out_host, out_host + np * 4, 0.0f);
    if (!scene_loaded_ || !camera_set_) return fail(LUCID_ERR_NO_SCENE, "scene or camera not set");
    std::string m = mode ? mode : "";
    int md;
    if (m == "normal") md = 0;
    else if (m == "albedo") md = 1;
    else if (m == "emission") md = 2;
    else {
        // unknown mode: magenta, as render_debug does (pybind_renderer.hpp:420-422)
        for (size_t i = 0; i < np; ++i) { out_host[4 * i] = 1.0f; out_host[4 * i + 1] = 0.0f; out_host[4 * i + 2] = 1.0f; out_host[4 * i + 3] = 1.0f; }
        return LUCID_OK;
    }
    CK(cudaSetDevice(device_));
    cudaStream_t st = S(stream_);
    PathPool& P = *pool_;
    if (P.film_n < np) { CK(P.film.alloc(np)); CK(P.out.alloc(np)); P.film_n = np; }
    if (!P.errors.p) CK(P.errors.alloc(4));
    CK(cudaMemsetAsync(P.errors.p, 0, 4 * sizeof(int), st));
    FrameParams f{};
    for (int k = 0; k < 3; ++k) { f.pos[k] = cam_.pos[k]; f.fwd[k] = cam_.forward[k]; f.right[k] = cam_.right[k]; f.up[k] = cam_.up[k]; }
    f.aspect = (float)fw / (float)fh;
    f.scale = std::tan(cam_.fov * 0.5f);
    f.tile_x = tx; f.tile_y = ty; f.tile_w = tw; f.tile_h = th; f.full_w = fw; f.full_h = fh; f.npix = (int)np;
    k_debug<<<((int)np + 255) / 256, 256, 0, st>>>(ds_->view, f, md, P.out.p, P.errors.p);
    CK(cudaGetLastError());
    int herr[4];
    CK(cudaMemcpyAsync(herr, P.errors.p, sizeof(herr), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out_host, P.out.p, np * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr[0]) return fail(LUCID_ERR_OVERFLOW, "BVH traversal stack overflow");
    return LUCID_OK;
}

}  // namespace lucid
