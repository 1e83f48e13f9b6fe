// lucid_guide.cu — training of the path-guiding network (fused forward,
// backward and weight gradients on the tensor cores; Adam on FP32 masters).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "lucid_guide.cuh"
#include "lucid_guide_host.h"

namespace lucid {

static_assert(kGuideParams == kGParams && kGuideInputs == kGIn && kGuideOutputs == kGOut, "guide layout");
static inline __nv_bfloat16* WQ(void* p) { return static_cast<__nv_bfloat16*>(p); }

// ---- training tile -----------------------------------------------------------------
struct TrainTile {
    GuideTile t;
    __nv_bfloat16 dout[16 * kLdH];   // dL/d(raw outputs), 48 used
    __nv_bfloat16 da[16 * kLdH], db[16 * kLdH];
};
constexpr int kTrainWarps = 3;
constexpr size_t kTrainSmem = sizeof(GuideSmemW) + kTrainWarps * sizeof(TrainTile) + kGParams * sizeof(float);

// grad[MOUT][KIN] += D^T H over the tile's 16 rows (D: 16 x MOUT, H: 16 x KIN).
template <int MOUT, int KIN, int LDD, int LDH>
LD void tile_wgrad(const __nv_bfloat16* D, const __nv_bfloat16* H, float* grad) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll 1
    for (int mb = 0; mb < MOUT / 16; ++mb) {
        const int m0 = mb * 16 + g;
        unsigned a[4];
        a[0] = pair2(D + (2 * q) * LDD + m0, D + (2 * q + 1) * LDD + m0);
        a[1] = pair2(D + (2 * q) * LDD + m0 + 8, D + (2 * q + 1) * LDD + m0 + 8);
        a[2] = pair2(D + (2 * q + 8) * LDD + m0, D + (2 * q + 9) * LDD + m0);
        a[3] = pair2(D + (2 * q + 8) * LDD + m0 + 8, D + (2 * q + 9) * LDD + m0 + 8);
#pragma unroll 2
        for (int nb = 0; nb < KIN / 8; ++nb) {
            const int n0 = nb * 8 + g;
            unsigned b[2];
            b[0] = pair2(H + (2 * q) * LDH + n0, H + (2 * q + 1) * LDH + n0);
            b[1] = pair2(H + (2 * q + 8) * LDH + n0, H + (2 * q + 9) * LDH + n0);
            float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            mma16816(acc, a, b);
            const int c = nb * 8 + 2 * q;
            atomicAdd(&grad[m0 * KIN + c], acc[0]);
            atomicAdd(&grad[m0 * KIN + c + 1], acc[1]);
            atomicAdd(&grad[(m0 + 8) * KIN + c], acc[2]);
            atomicAdd(&grad[(m0 + 8) * KIN + c + 1], acc[3]);
        }
    }
}

// out[16 x KIN] = (D[16 x MOUT] W[MOUT][KIN]) * (H > 0), as BF16 (ld kLdH);
// the column sums go to gbias (the bias gradient of the layer below).
template <int MOUT, int KIN, int LDD, int LDW>
LD void tile_backprop(const __nv_bfloat16* D, const __nv_bfloat16* W, const __nv_bfloat16* H, __nv_bfloat16* out,
                      float* gbias) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    float acc[KIN / 8][4];
#pragma unroll
    for (int nb = 0; nb < KIN / 8; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.0f;
#pragma unroll
    for (int kb = 0; kb < MOUT / 16; ++kb) {
        unsigned a[4];
        a[0] = ld_pair(D + g * LDD + kb * 16 + 2 * q);
        a[1] = ld_pair(D + (g + 8) * LDD + kb * 16 + 2 * q);
        a[2] = ld_pair(D + g * LDD + kb * 16 + 2 * q + 8);
        a[3] = ld_pair(D + (g + 8) * LDD + kb * 16 + 2 * q + 8);
        const int k0 = kb * 16 + 2 * q;
#pragma unroll
        for (int nb = 0; nb < KIN / 8; ++nb) {
            const int n0 = nb * 8 + g;
            unsigned b[2];
            b[0] = pair2(W + k0 * LDW + n0, W + (k0 + 1) * LDW + n0);
            b[1] = pair2(W + (k0 + 8) * LDW + n0, W + (k0 + 9) * LDW + n0);
            mma16816(acc[nb], a, b);
        }
    }
#pragma unroll
    for (int nb = 0; nb < KIN / 8; ++nb) {
        const int c = nb * 8 + 2 * q;
        float v[4];
        v[0] = __bfloat162float(H[g * kLdH + c]) > 0.0f ? acc[nb][0] : 0.0f;
        v[1] = __bfloat162float(H[g * kLdH + c + 1]) > 0.0f ? acc[nb][1] : 0.0f;
        v[2] = __bfloat162float(H[(g + 8) * kLdH + c]) > 0.0f ? acc[nb][2] : 0.0f;
        v[3] = __bfloat162float(H[(g + 8) * kLdH + c + 1]) > 0.0f ? acc[nb][3] : 0.0f;
        *reinterpret_cast<unsigned*>(out + g * kLdH + c) = pack_bf16(v[0], v[1]);
        *reinterpret_cast<unsigned*>(out + (g + 8) * kLdH + c) = pack_bf16(v[2], v[3]);
        atomicAdd(&gbias[c], v[0] + v[2]);
        atomicAdd(&gbias[c + 1], v[1] + v[3]);
    }
}

// dL/d(raw) of L = -c log q(wi) for one row (kGOut values, padding zero).
LD void mixture_grad(const float* raw, V3 wi, float c, float* d) {
    for (int i = 0; i < kGOut; ++i) d[i] = 0.0f;
    if (!(c > 0.0f)) return;
    GuideMix gm;
    guide_mix_from_raw(raw, gm);
    float p[kGLobes], qsum = 0.0f;
    for (int k = 0; k < kGLobes; ++k) { p[k] = vmf_pdf(gm.k[k], gm.mu[k], wi); qsum += gm.w[k] * p[k]; }
    if (!(qsum > 1e-30f)) return;
    for (int k = 0; k < kGLobes; ++k) {
        float gam = gm.w[k] * p[k] / qsum;
        d[k] = c * (gm.w[k] - gam);
        float r = raw[kGLobes + k];
        float kap = gm.k[k];
        if (kap < kGKappaMax) {
            float e = __expf(-2.0f * kap);
            float mw = dot(gm.mu[k], wi);
            float dlogp = 1.0f / kap - 2.0f * e / (1.0f - e) + (mw - 1.0f);
            d[kGLobes + k] = -c * gam * dlogp * sigmoidf(r);
        }
        V3 m = v3(raw[16 + 3 * k], raw[17 + 3 * k], raw[18 + 3 * k]);
        float l = len(m);
        if (l > 1e-6f) {
            float mw = dot(gm.mu[k], wi);
            V3 gdir = (wi - gm.mu[k] * mw) * (-c * gam * kap / l);
            d[16 + 3 * k] = gdir.x; d[17 + 3 * k] = gdir.y; d[18 + 3 * k] = gdir.z;
        }
    }
}

// Encodes one record's inputs into row `r` of the tile (lanes 0..15).
LD void encode_row(__nv_bfloat16* x, int r, const GuideRec& rec) {
    __nv_bfloat16* row = x + r * kLdIn;
    guide_encode(v3(rec.p[0], rec.p[1], rec.p[2]), v3(rec.n[0], rec.n[1], rec.n[2]),
                 v3(rec.wo[0], rec.wo[1], rec.wo[2]), [&](int i, float v) { row[i] = __float2bfloat16(v); });
}

__global__ void k_guide_coeff_sum(const GuideRec* recs, int n, float* sum) {
    float s = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GuideRec& r = recs[i];
        float F = 0.2126f * r.L[0] + 0.7152f * r.L[1] + 0.0722f * r.L[2];
        if (F > 0.0f && r.pdf > 0.0f && isfinite(F)) s += F / r.pdf;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

// Fused forward + backward over tiles of 16 records; weight gradients are
// summed in shared memory and added to `grad` once per block.  The loss is
// sum_s c_s (-log q(wi_s)) with c_s = (F_s / pdf_s) / sum_t F_t / pdf_t.
__global__ void __launch_bounds__(32 * kTrainWarps) k_guide_train(const GuideRec* recs, int n,
                                                                 const __nv_bfloat16* wq, const float* master,
                                                                 const float* csum, float* grad) {
    extern __shared__ __align__(16) unsigned char smem[];
    GuideSmemW& W = *reinterpret_cast<GuideSmemW*>(smem);
    TrainTile* tiles = reinterpret_cast<TrainTile*>(smem + sizeof(GuideSmemW));
    float* sg = reinterpret_cast<float*>(smem + sizeof(GuideSmemW) + kTrainWarps * sizeof(TrainTile));
    guide_load_weights(W, wq, master);
    for (int i = threadIdx.x; i < kGParams; i += blockDim.x) sg[i] = 0.0f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainTile& T = tiles[warp];
    const float inv_sum = *csum > 0.0f ? 1.0f / *csum : 0.0f;
    const int ntiles = (n + 15) / 16;
    for (int tile = blockIdx.x * kTrainWarps + warp; tile < ntiles; tile += gridDim.x * kTrainWarps) {
        const int r = tile * 16 + lane;
        GuideRec rec{};
        bool valid = lane < 16 && r < n;
        if (valid) rec = recs[r];
        if (lane < 16) {
            if (valid) encode_row(T.t.x, lane, rec);
            else for (int i = 0; i < kGIn; ++i) T.t.x[lane * kLdIn + i] = __float2bfloat16(0.0f);
        }
        __syncwarp();
        guide_forward_tile(W, T.t);
        if (lane < 16) {
            float F = 0.2126f * rec.L[0] + 0.7152f * rec.L[1] + 0.0722f * rec.L[2];
            float c = (valid && F > 0.0f && rec.pdf > 0.0f && isfinite(F)) ? F / rec.pdf * inv_sum : 0.0f;
            float d[kGOut];
            mixture_grad(T.t.raw + lane * kGOut, v3(rec.wi[0], rec.wi[1], rec.wi[2]), c, d);
            for (int i = 0; i < kGOut; i += 2)
                *reinterpret_cast<unsigned*>(T.dout + lane * kLdH + i) = pack_bf16(d[i], d[i + 1]);
            for (int i = 0; i < kGOut; ++i)
                if (d[i] != 0.0f) atomicAdd(&sg[kGB4 + i], d[i]);
        }
        __syncwarp();
        tile_wgrad<kGOut, kGHid, kLdH, kLdH>(T.dout, T.t.h3, sg + kGW4);
        tile_backprop<kGOut, kGHid, kLdH, kLdH>(T.dout, W.w4, T.t.h3, T.da, sg + kGB3);
        __syncwarp();
        tile_wgrad<kGHid, kGHid, kLdH, kLdH>(T.da, T.t.h2, sg + kGW3);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.da, W.w3, T.t.h2, T.db, sg + kGB2);
        __syncwarp();
        tile_wgrad<kGHid, kGHid, kLdH, kLdH>(T.db, T.t.h1, sg + kGW2);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.db, W.w2, T.t.h1, T.da, sg + kGB1);
        __syncwarp();
        tile_wgrad<kGHid, kGIn, kLdH, kLdIn>(T.da, T.t.x, sg + kGW1);
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kGParams; i += blockDim.x)
        if (sg[i] != 0.0f) atomicAdd(&grad[i], sg[i]);
}

__global__ void k_guide_adam(float* master, float* m, float* v, float* grad, __nv_bfloat16* wq, int n, float lr,
                             float b1, float b2, float eps, float bc1, float bc2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float g = grad[i];
    if (!isfinite(g)) g = 0.0f;
    float mi = b1 * m[i] + (1.0f - b1) * g;
    float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float w = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    master[i] = w;
    wq[i] = __float2bfloat16(w);
    grad[i] = 0.0f;
}

__global__ void k_guide_quantise(const float* master, __nv_bfloat16* wq, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wq[i] = __float2bfloat16(master[i]);
}

// Raw outputs for given input rows (n x kGIn floats): one warp per 16 rows.
__global__ void __launch_bounds__(128) k_guide_forward_rows(const float* in, int n, const __nv_bfloat16* wq,
                                                            const float* master, float* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    GuideSmemW& W = *reinterpret_cast<GuideSmemW*>(smem);
    GuideTile* tiles = reinterpret_cast<GuideTile*>(smem + sizeof(GuideSmemW));
    guide_load_weights(W, wq, master);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    GuideTile& T = tiles[warp];
    const int ntiles = (n + 15) / 16;
    for (int tile = blockIdx.x * 4 + warp; tile < ntiles; tile += gridDim.x * 4) {
        for (int e = lane; e < 16 * kGIn; e += 32) {
            int r = e / kGIn, c = e % kGIn;
            int row = tile * 16 + r;
            T.x[r * kLdIn + c] = __float2bfloat16(row < n ? in[(size_t)row * kGIn + c] : 0.0f);
        }
        __syncwarp();
        guide_forward_tile(W, T);
        for (int e = lane; e < 16 * kGOut; e += 32) {
            int r = e / kGOut, row = tile * 16 + r;
            if (row < n) out[(size_t)row * kGOut + e % kGOut] = T.raw[e];
        }
        __syncwarp();
    }
}

__global__ void k_guide_encode_rows(const float* p01, const float* nrm, const float* wo, int n, float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* row = out + (size_t)i * kGIn;
    guide_encode(v3(p01[3 * i], p01[3 * i + 1], p01[3 * i + 2]), v3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]),
                 v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), [&](int k, float v) { row[k] = v; });
}

// ---- host --------------------------------------------------------------------------
#define GCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) { err_ = std::string(#call) + ": " + cudaGetErrorString(e_);     \
                                 return e_ == cudaErrorMemoryAllocation ? -2 : -6; }            \
    } while (0)

GuideNet::~GuideNet() { release(); }

void GuideNet::release() {
    for (void* p : {(void*)master_, (void*)m_, (void*)v_, (void*)grad_, (void*)wq_, (void*)csum_})
        if (p) cudaFree(p);
    master_ = m_ = v_ = grad_ = csum_ = nullptr;
    wq_ = nullptr;
}

int GuideNet::init(int seed, cudaStream_t st) {
    release();
    GCK(cudaMalloc(&master_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&m_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&v_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&grad_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&csum_, sizeof(float)));
    GCK(cudaMalloc(&wq_, kGParams * sizeof(__nv_bfloat16)));
    std::vector<float> w(kGParams, 0.0f);
    std::mt19937 rng((unsigned)seed);
    auto fill = [&](int off, int out, int in, float gain) {
        float a = gain * std::sqrt(6.0f / (float)(in + out));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < out * in; ++i) w[off + i] = u(rng);
    };
    fill(kGW1, kGHid, kGInUsed, 1.0f);
    for (int o = 0; o < kGHid; ++o)
        for (int i = kGInUsed; i < kGIn; ++i) w[kGW1 + o * kGIn + i] = 0.0f;   // padding inputs
    fill(kGW2, kGHid, kGHid, 1.0f);
    fill(kGW3, kGHid, kGHid, 1.0f);
    fill(kGW4, kGOut, kGHid, 0.1f);
    for (int o = 40; o < kGOut; ++o)
        for (int i = 0; i < kGHid; ++i) w[kGW4 + o * kGHid + i] = 0.0f;     // padding outputs
    return set_params(w.data(), st);
}

int GuideNet::set_params(const float* w, cudaStream_t st) {
    GCK(cudaMemcpyAsync(master_, w, kGParams * sizeof(float), cudaMemcpyHostToDevice, st));
    GCK(cudaMemsetAsync(m_, 0, kGParams * sizeof(float), st));
    GCK(cudaMemsetAsync(v_, 0, kGParams * sizeof(float), st));
    GCK(cudaMemsetAsync(grad_, 0, kGParams * sizeof(float), st));
    k_guide_quantise<<<(kGParams + 255) / 256, 256, 0, st>>>(master_, WQ(wq_), kGParams);
    GCK(cudaGetLastError());
    step_ = 0;
    return 0;
}

int GuideNet::get_params(float* w, cudaStream_t st) {
    GCK(cudaMemcpyAsync(w, master_, kGParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    GCK(cudaStreamSynchronize(st));
    return 0;
}

int GuideNet::gradient(const GuideRec* recs, int n, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        GCK(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
        attr = true;
    }
    GCK(cudaMemsetAsync(csum_, 0, sizeof(float), st));
    if (n <= 0) return 0;
    k_guide_coeff_sum<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(recs, n, csum_);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = std::max(1, std::min(sms, (n + 16 * kTrainWarps - 1) / (16 * kTrainWarps)));
    k_guide_train<<<blocks, 32 * kTrainWarps, kTrainSmem, st>>>(recs, n, WQ(wq_), master_, csum_, grad_);
    GCK(cudaGetLastError());
    return 0;
}

int GuideNet::adam(cudaStream_t st, float lr) {
    ++step_;
    const float b1 = 0.9f, b2 = 0.999f;
    float bc1 = 1.0f - std::pow(b1, (float)step_), bc2 = 1.0f - std::pow(b2, (float)step_);
    k_guide_adam<<<(kGParams + 255) / 256, 256, 0, st>>>(master_, m_, v_, grad_, WQ(wq_), kGParams, lr, b1, b2,
                                                       1e-8f, bc1, bc2);
    GCK(cudaGetLastError());
    return 0;
}

int GuideNet::train_step(const GuideRec* recs, int n, cudaStream_t st, float lr) {
    int rc = gradient(recs, n, st);
    if (rc != 0) return rc;
    return adam(st, lr);
}

int GuideNet::forward_rows(const float* d_in, int n, float* d_out, cudaStream_t st) {
    const size_t smem = sizeof(GuideSmemW) + 4 * sizeof(GuideTile);
    static bool attr = false;
    if (!attr) {
        GCK(cudaFuncSetAttribute(k_guide_forward_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    int blocks = std::max(1, std::min(148, (n + 63) / 64));
    k_guide_forward_rows<<<blocks, 128, smem, st>>>(d_in, n, WQ(wq_), master_, d_out);
    GCK(cudaGetLastError());
    return 0;
}

int GuideNet::encode_rows(const float* p01, const float* nrm, const float* wo, int n, float* out, cudaStream_t st) {
    k_guide_encode_rows<<<(n + 127) / 128, 128, 0, st>>>(p01, nrm, wo, n, out);
    GCK(cudaGetLastError());
    return 0;
}

}  // namespace lucid
