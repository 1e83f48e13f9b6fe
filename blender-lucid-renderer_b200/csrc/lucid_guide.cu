// lucid_guide.cu — training of the path-guiding network (forward/backward
// pass and split-K weight-gradient GEMMs on the tensor cores; Adam on FP32
// masters).
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

// The loss of a batch is sum_s c_s (-log q(wi_s)) with
// c_s = (F_s / pdf_s) / sum_t F_t / pdf_t.

// ---- training in two passes ---------------------------------------------------
// Pass 1 (k_guide_fb): per warp tile of 16 records, forward, mixture
// gradient and backpropagation of the gradients through the layers; the
// layer inputs (x, h1..h3) and output gradients (d4..d1) go to global memory
// as BF16 and the bias gradients are summed per block.  Pass 2
// (k_guide_wgrad): each weight gradient dW = D^T H as a split-K GEMM over the
// records, accumulated in registers over a slice of records and added to the
// gradient once per block.
constexpr int kFbWarps = 7;
constexpr size_t kFbSmem = sizeof(GuideSmemW) + kFbWarps * sizeof(TrainTile) + 256 * sizeof(float);
// per-record offsets (BF16 elements) in the pass-1 workspace
constexpr int kWsX = 0, kWsH1 = kGIn, kWsH2 = kWsH1 + kGHid, kWsH3 = kWsH2 + kGHid, kWsD4 = kWsH3 + kGHid,
              kWsD3 = kWsD4 + kGOut, kWsD2 = kWsD3 + kGHid, kWsD1 = kWsD2 + kGHid, kWsRow = kWsD1 + kGHid;

// Copies a 16-row tile (ld `ld` in shared memory) to rows r0.. of a global
// matrix of `cols` columns inside the record workspace (row stride kWsRow).
LD void tile_store(const __nv_bfloat16* src, int ld, int cols, __nv_bfloat16* dst, int r0, int n) {
    const int lane = threadIdx.x & 31;
    for (int e = lane; e < 16 * (cols / 2); e += 32) {
        int r = e / (cols / 2), c = 2 * (e % (cols / 2));
        if (r0 + r < n)
            *reinterpret_cast<unsigned*>(dst + (size_t)(r0 + r) * kWsRow + c) =
                *reinterpret_cast<const unsigned*>(src + r * ld + c);
    }
}

// Backpropagation without the weight gradient (tile_backprop's data part).
__global__ void __launch_bounds__(32 * kFbWarps) k_guide_fb(const GuideRec* recs, int n, const __nv_bfloat16* wq,
                                                           const float* master, const float* csum,
                                                           __nv_bfloat16* ws, float* grad) {
    extern __shared__ __align__(16) unsigned char smem[];
    GuideSmemW& W = *reinterpret_cast<GuideSmemW*>(smem);
    TrainTile* tiles = reinterpret_cast<TrainTile*>(smem + sizeof(GuideSmemW));
    float* sb = reinterpret_cast<float*>(smem + sizeof(GuideSmemW) + kFbWarps * sizeof(TrainTile));
    guide_load_weights(W, wq, master);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sb[i] = 0.0f;
    __syncthreads();
    // bias gradients in sb: b1 [0, 64), b2 [64, 128), b3 [128, 192), b4 [192, 240)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainTile& T = tiles[warp];
    const float inv_sum = *csum > 0.0f ? 1.0f / *csum : 0.0f;
    const int ntiles = (n + 15) / 16;
    for (int tile = blockIdx.x * kFbWarps + warp; tile < ntiles; tile += gridDim.x * kFbWarps) {
        const int r0 = tile * 16, r = r0 + lane;
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
                if (d[i] != 0.0f) atomicAdd(&sb[192 + i], d[i]);
        }
        __syncwarp();
        tile_backprop<kGOut, kGHid, kLdH, kLdH>(T.dout, W.w4, T.t.h3, T.da, sb + 128);
        __syncwarp();
        tile_store(T.t.x, kLdIn, kGIn, ws + kWsX, r0, n);
        tile_store(T.t.h1, kLdH, kGHid, ws + kWsH1, r0, n);
        tile_store(T.t.h2, kLdH, kGHid, ws + kWsH2, r0, n);
        tile_store(T.t.h3, kLdH, kGHid, ws + kWsH3, r0, n);
        tile_store(T.dout, kLdH, kGOut, ws + kWsD4, r0, n);
        tile_store(T.da, kLdH, kGHid, ws + kWsD3, r0, n);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.da, W.w3, T.t.h2, T.db, sb + 64);
        __syncwarp();
        tile_store(T.db, kLdH, kGHid, ws + kWsD2, r0, n);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.db, W.w2, T.t.h1, T.da, sb);
        __syncwarp();
        tile_store(T.da, kLdH, kGHid, ws + kWsD1, r0, n);
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kGHid; i += blockDim.x) {
        if (sb[i] != 0.0f) atomicAdd(&grad[kGB1 + i], sb[i]);
        if (sb[64 + i] != 0.0f) atomicAdd(&grad[kGB2 + i], sb[64 + i]);
        if (sb[128 + i] != 0.0f) atomicAdd(&grad[kGB3 + i], sb[128 + i]);
    }
    for (int i = threadIdx.x; i < kGOut; i += blockDim.x)
        if (sb[192 + i] != 0.0f) atomicAdd(&grad[kGB4 + i], sb[192 + i]);
}

// grad[O][I] += sum over this block's records of D[s][o] H[s][i] (8 warps;
// the (16 x 8) output fragments are split over the warps and accumulated in
// registers over 32-record chunks staged in shared memory).
constexpr int kWgChunk = 32, kWgSlice = 2048;
template <int O, int I>
__global__ void __launch_bounds__(256) k_guide_wgrad(const __nv_bfloat16* ws, int doff, int hoff, int n, float* grad) {
    constexpr int LDD = O + 8, LDH = I + 8, NB = I / 8, FR = (O / 16) * NB, FPW = (FR + 7) / 8;
    __shared__ __align__(16) __nv_bfloat16 Ds[kWgChunk * LDD];
    __shared__ __align__(16) __nv_bfloat16 Hs[kWgChunk * LDH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    float acc[FPW][4];
#pragma unroll
    for (int j = 0; j < FPW; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    const int k0 = blockIdx.x * kWgSlice, k1 = min(n, k0 + kWgSlice);
    for (int c0 = k0; c0 < k1; c0 += kWgChunk) {
        __syncthreads();
        for (int e = threadIdx.x; e < kWgChunk * (O / 2); e += blockDim.x) {
            int r = e / (O / 2), c = 2 * (e % (O / 2));
            unsigned v = 0;
            if (c0 + r < k1) v = *reinterpret_cast<const unsigned*>(ws + (size_t)(c0 + r) * kWsRow + doff + c);
            *reinterpret_cast<unsigned*>(Ds + r * LDD + c) = v;
        }
        for (int e = threadIdx.x; e < kWgChunk * (I / 2); e += blockDim.x) {
            int r = e / (I / 2), c = 2 * (e % (I / 2));
            unsigned v = 0;
            if (c0 + r < k1) v = *reinterpret_cast<const unsigned*>(ws + (size_t)(c0 + r) * kWsRow + hoff + c);
            *reinterpret_cast<unsigned*>(Hs + r * LDH + c) = v;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < FPW; ++j) {
            const int f = warp + 8 * j;
            if (f < FR) {
                const int m0 = (f / NB) * 16 + g, n0 = (f % NB) * 8 + g;
#pragma unroll
                for (int ks = 0; ks < kWgChunk; ks += 16) {
                    unsigned a[4], b[2];
                    const __nv_bfloat16* D = Ds + ks * LDD;
                    const __nv_bfloat16* H = Hs + ks * LDH;
                    a[0] = pair2(D + (2 * q) * LDD + m0, D + (2 * q + 1) * LDD + m0);
                    a[1] = pair2(D + (2 * q) * LDD + m0 + 8, D + (2 * q + 1) * LDD + m0 + 8);
                    a[2] = pair2(D + (2 * q + 8) * LDD + m0, D + (2 * q + 9) * LDD + m0);
                    a[3] = pair2(D + (2 * q + 8) * LDD + m0 + 8, D + (2 * q + 9) * LDD + m0 + 8);
                    b[0] = pair2(H + (2 * q) * LDH + n0, H + (2 * q + 1) * LDH + n0);
                    b[1] = pair2(H + (2 * q + 8) * LDH + n0, H + (2 * q + 9) * LDH + n0);
                    mma16816(acc[j], a, b);
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < FPW; ++j) {
        const int f = warp + 8 * j;
        if (f < FR) {
            const int m0 = (f / NB) * 16 + g, c = (f % NB) * 8 + 2 * q;
            atomicAdd(&grad[m0 * I + c], acc[j][0]);
            atomicAdd(&grad[m0 * I + c + 1], acc[j][1]);
            atomicAdd(&grad[(m0 + 8) * I + c], acc[j][2]);
            atomicAdd(&grad[(m0 + 8) * I + c + 1], acc[j][3]);
        }
    }
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
    for (void* p : {(void*)master_, (void*)m_, (void*)v_, (void*)grad_, (void*)wq_, (void*)csum_, ws_})
        if (p) cudaFree(p);
    master_ = m_ = v_ = grad_ = csum_ = nullptr;
    wq_ = ws_ = nullptr;
    ws_n_ = 0;
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
    GCK(cudaMemsetAsync(csum_, 0, sizeof(float), st));
    if (n <= 0) return 0;
    k_guide_coeff_sum<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(recs, n, csum_);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    static bool attr_fb = false;
    if (!attr_fb) {
        GCK(cudaFuncSetAttribute(k_guide_fb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFbSmem));
        attr_fb = true;
    }
    if (ws_n_ < n) {
        if (ws_) cudaFree(ws_);
        ws_ = nullptr;
        GCK(cudaMalloc(&ws_, (size_t)n * kWsRow * sizeof(__nv_bfloat16)));
        ws_n_ = n;
    }
    __nv_bfloat16* ws = WQ(ws_);
    int blocks = std::max(1, std::min(sms, (n + 16 * kFbWarps - 1) / (16 * kFbWarps)));
    k_guide_fb<<<blocks, 32 * kFbWarps, kFbSmem, st>>>(recs, n, WQ(wq_), master_, csum_, ws, grad_);
    const int slices = (n + kWgSlice - 1) / kWgSlice;
    k_guide_wgrad<kGHid, kGIn><<<slices, 256, 0, st>>>(ws, kWsD1, kWsX, n, grad_ + kGW1);
    k_guide_wgrad<kGHid, kGHid><<<slices, 256, 0, st>>>(ws, kWsD2, kWsH1, n, grad_ + kGW2);
    k_guide_wgrad<kGHid, kGHid><<<slices, 256, 0, st>>>(ws, kWsD3, kWsH2, n, grad_ + kGW3);
    k_guide_wgrad<kGOut, kGHid><<<slices, 256, 0, st>>>(ws, kWsD4, kWsH3, n, grad_ + kGW4);
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
