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
// One warp's 16 records (12.5 KB): the input rows are reused, once they are
// stored, for the FP32 raw outputs, dL/d(raw) and one gradient buffer; the
// other gradient buffer reuses h3 once backpropagation has passed it.
struct TrainTile {
    __nv_bfloat16 x[16 * kLdIn];
    __nv_bfloat16 h1[16 * kLdH], h2[16 * kLdH], h3[16 * kLdH];
    LD float* raw() { return reinterpret_cast<float*>(x); }              // bytes [0, 3072)
    LD __nv_bfloat16* dout() { return x + 16 * kGOut * 2; }               // bytes [3072, 5376)
    LD __nv_bfloat16* da() { return x; }                                  // bytes [0, 2304)
    LD __nv_bfloat16* db() { return h3; }
};
static_assert(16 * kGOut * 4 + 16 * kLdH * 2 <= 16 * kLdIn * 2, "raw outputs and dL/d(raw) fit the input rows");

// out[16 x KIN] = (D[16 x MOUT] W[MOUT][KIN]) * (H > 0), as BF16 (ld kLdH).
template <int MOUT, int KIN, int LDD, int LDW>
LD void tile_backprop(const __nv_bfloat16* D, const __nv_bfloat16* W, const __nv_bfloat16* H, __nv_bfloat16* out) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    float acc[KIN / 8][4];
#pragma unroll
    for (int nb = 0; nb < KIN / 8; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.0f;
    // B[k][n] = W[k][n]: transposed loads of (k0, n0), (k0 + 8, n0),
    // (k0, n0 + 8), (k0 + 8, n0 + 8)
    const unsigned d_base = smem_u32(D + ldsm_a_offset(LDD)), w_base = smem_u32(W + ldsm_a_offset(LDW));
#pragma unroll
    for (int kb = 0; kb < MOUT / 16; ++kb) {
        unsigned a[4];
        ldsm_x4(d_base + 32u * kb, a);
#pragma unroll
        for (int nb = 0; nb < KIN / 8; nb += 2) {
            unsigned b[4];
            ldsm_x4_trans(w_base + 2u * (unsigned)(kb * 16 * LDW + nb * 8), b);
            mma16816(acc[nb], a, b);
            mma16816(acc[nb + 1], a, b + 2);
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
    }
}

// dL/d(raw) of L = -c log q(wi) for one row, split over two lanes (xor 16)
// that run the same instructions: half h handles lobes 4h..4h+3 and half 1
// also the zero padding.  st(i, value) receives every output once.
template <class Store>
LD void mixture_grad_half(const float* raw, V3 wi, float c, int half, Store&& st) {
    GuideMix gm;
    guide_mix_from_raw(raw, gm);
    const int k0 = half * (kGLobes / 2);
    // this half's lobes, picked with constant indices (no local-memory arrays)
    float w[kGLobes / 2], kp[kGLobes / 2], p[kGLobes / 2], own = 0.0f;
    V3 mu[kGLobes / 2];
#pragma unroll
    for (int j = 0; j < kGLobes / 2; ++j) {
        w[j] = half ? gm.w[kGLobes / 2 + j] : gm.w[j];
        kp[j] = half ? gm.k[kGLobes / 2 + j] : gm.k[j];
        mu[j] = half ? gm.mu[kGLobes / 2 + j] : gm.mu[j];
        p[j] = vmf_pdf(kp[j], mu[j], wi);
        own += w[j] * p[j];
    }
    const float other = __shfl_xor_sync(0xffffffffu, own, 16);
    const float qsum = half ? other + own : own + other;
    const bool live = c > 0.0f && qsum > 1e-30f;
#pragma unroll
    for (int j = 0; j < kGLobes / 2; ++j) {
        const int k = k0 + j;
        float dl = 0.0f, dk = 0.0f;
        V3 gdir = v3(0.0f, 0.0f, 0.0f);
        if (live) {
            const float gam = w[j] * p[j] / qsum;
            dl = c * (w[j] - gam);
            const float kap = kp[j], mw = dot(mu[j], wi);
            if (kap < kGKappaMax) {
                float e = __expf(-2.0f * kap);
                float dlogp = 1.0f / kap - 2.0f * e / (1.0f - e) + (mw - 1.0f);
                dk = -c * gam * dlogp * sigmoidf(raw[kGLobes + k]);
            }
            const float l = len(v3(raw[16 + 3 * k], raw[17 + 3 * k], raw[18 + 3 * k]));
            if (l > 1e-6f) gdir = (wi - mu[j] * mw) * (-c * gam * kap / l);
        }
        st(k, dl);
        st(kGLobes + k, dk);
        st(16 + 3 * k, gdir.x); st(17 + 3 * k, gdir.y); st(18 + 3 * k, gdir.z);
    }
    if (half)
        for (int i = 40; i < kGOut; ++i) st(i, 0.0f);
}

// Encodes one record's inputs into row `r` of the tile, half of the
// features per lane (lanes r and r + 16).
LD void encode_row(__nv_bfloat16* x, int r, int half, const GuideRec& rec) {
    __nv_bfloat16* row = x + r * kLdIn;
    guide_encode_half(v3(rec.p[0], rec.p[1], rec.p[2]), v3(rec.n[0], rec.n[1], rec.n[2]),
                      v3(rec.wo[0], rec.wo[1], rec.wo[2]), half, [&](int i, float v) { row[i] = __float2bfloat16(v); });
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
// gradient and backpropagation through the layers; the layer inputs
// (x, h1..h3) and the gradients of the layer outputs (d4..d1) go to a
// per-record BF16 workspace row.  Pass 2 (k_guide_wgrad): every weight and
// bias gradient, dW = D^T H and db = D^T 1, as one split-K GEMM over the
// records: each block streams chunks of workspace rows into shared memory
// with bulk async copies (double-buffered) and keeps its share of the
// gradient in registers; the per-block partial gradients are summed by
// k_guide_reduce in block order.
constexpr int kFbWarps = 14;
constexpr size_t kFbSmem = sizeof(GuideSmemW) + kFbWarps * sizeof(TrainTile);
// per-record offsets (BF16 elements) in a workspace row; every block starts
// on a 16-byte boundary and the row (616 elements, 1232 bytes) is padded so
// that eight consecutive rows fall in different shared-memory banks
constexpr int kWsX = 0, kWsH1 = kGIn, kWsH2 = kWsH1 + kGHid, kWsH3 = kWsH2 + kGHid, kWsD4 = kWsH3 + kGHid,
              kWsD3 = kWsD4 + kGOut, kWsD2 = kWsD3 + kGHid, kWsD1 = kWsD2 + kGHid, kWsRow = kWsD1 + kGHid + 8;
static_assert(kWsRow * 2 % 16 == 0 && kWsH1 % 8 == 0 && kWsD4 % 8 == 0 && kWsD1 % 8 == 0, "workspace alignment");

// Copies a 16-row tile (ld `ld` in shared memory) to rows r0.. of the
// workspace column block at `dst` (16-byte vectors).
LD void tile_store(const __nv_bfloat16* src, int ld, int cols, __nv_bfloat16* dst, int r0, int n) {
    const int lane = threadIdx.x & 31, vec = cols / 8;
    for (int e = lane; e < 16 * vec; e += 32) {
        int r = e / vec, c = 8 * (e % vec);
        if (r0 + r < n)
            *reinterpret_cast<uint4*>(dst + (size_t)(r0 + r) * kWsRow + c) =
                *reinterpret_cast<const uint4*>(src + r * ld + c);
    }
}

__global__ void __launch_bounds__(32 * kFbWarps) k_guide_fb(const GuideRec* recs, int n, const __nv_bfloat16* wq,
                                                           const float* master, const float* csum,
                                                           __nv_bfloat16* ws) {
    extern __shared__ __align__(16) unsigned char smem[];
    GuideSmemW& W = *reinterpret_cast<GuideSmemW*>(smem);
    TrainTile* tiles = reinterpret_cast<TrainTile*>(smem + sizeof(GuideSmemW));
    guide_load_weights(W, wq, master);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TrainTile& T = tiles[warp];
    const float inv_sum = *csum > 0.0f ? 1.0f / *csum : 0.0f;
    const int ntiles = (n + 15) / 16;
    for (int tile = blockIdx.x * kFbWarps + warp; tile < ntiles; tile += gridDim.x * kFbWarps) {
        const int r0 = tile * 16, row = lane & 15, r = r0 + row, half = lane >> 4;
        GuideRec rec{};
        const bool valid = r < n;
        if (valid) rec = recs[r];
        if (valid) encode_row(T.x, row, half, rec);
        else
            for (int i = half * 88; i < half * 88 + 88; ++i) T.x[row * kLdIn + i] = __float2bfloat16(0.0f);
        __syncwarp();
        tile_layer<kGIn, kGHid, kLdIn, kLdIn, true>(T.x, W.w1, W.b1, T.h1, nullptr);
        __syncwarp();
        tile_store(T.x, kLdIn, kGIn, ws + kWsX, r0, n);
        tile_layer<kGHid, kGHid, kLdH, kLdH, true>(T.h1, W.w2, W.b2, T.h2, nullptr);
        __syncwarp();
        tile_layer<kGHid, kGHid, kLdH, kLdH, true>(T.h2, W.w3, W.b3, T.h3, nullptr);
        __syncwarp();
        tile_layer<kGHid, kGOut, kLdH, kLdH, false>(T.h3, W.w4, W.b4, nullptr, T.raw());
        __syncwarp();
        {
            float F = 0.2126f * rec.L[0] + 0.7152f * rec.L[1] + 0.0722f * rec.L[2];
            float c = (valid && F > 0.0f && rec.pdf > 0.0f && isfinite(F)) ? F / rec.pdf * inv_sum : 0.0f;
            __nv_bfloat16* drow = T.dout() + row * kLdH;
            mixture_grad_half(T.raw() + row * kGOut, v3(rec.wi[0], rec.wi[1], rec.wi[2]), c, half,
                              [&](int i, float v) { drow[i] = __float2bfloat16(v); });
        }
        __syncwarp();
        tile_backprop<kGOut, kGHid, kLdH, kLdH>(T.dout(), W.w4, T.h3, T.da());
        __syncwarp();
        tile_store(T.h1, kLdH, kGHid, ws + kWsH1, r0, n);
        tile_store(T.h2, kLdH, kGHid, ws + kWsH2, r0, n);
        tile_store(T.h3, kLdH, kGHid, ws + kWsH3, r0, n);
        tile_store(T.dout(), kLdH, kGOut, ws + kWsD4, r0, n);
        tile_store(T.da(), kLdH, kGHid, ws + kWsD3, r0, n);
        __syncwarp();
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.da(), W.w3, T.h2, T.db());
        __syncwarp();
        tile_store(T.db(), kLdH, kGHid, ws + kWsD2, r0, n);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.db(), W.w2, T.h1, T.da());
        __syncwarp();
        tile_store(T.da(), kLdH, kGHid, ws + kWsD1, r0, n);
        __syncwarp();
    }
}

// Pass 2 work units: a 16 x 16 block of one weight gradient (two m16n8
// fragments) or a 16-row block of one bias gradient (one fragment against a
// column of ones).  Units 0..87 are the weight blocks (W1 44, W2 16, W3 16,
// W4 12), units 88..102 the bias blocks (b1 4, b2 4, b3 4, b4 3).
constexpr int kWgRows = 64, kWgWarps = 16, kWgUnits = 103, kWgMaxUnits = (kWgUnits + kWgWarps - 1) / kWgWarps;
constexpr size_t kWgChunkBytes = (size_t)kWgRows * kWsRow * 2;
constexpr size_t kWgSmem = 2 * kWgChunkBytes;
constexpr long long kWgSpin = 1ll << 24;   // bound on the polls of one chunk's arrival

struct WgUnit {
    int a_off, b_off;   // workspace column of the A block (D^T) and B block (H^T); b_off < 0: bias
    int goff, cols;     // gradient offset of the block's first element and the row length
};
LD WgUnit wg_unit(int u) {
    // per layer: D column, H column, weight offset, bias offset, outputs, inputs
    const int dcol[4] = {kWsD1, kWsD2, kWsD3, kWsD4}, hcol[4] = {kWsX, kWsH1, kWsH2, kWsH3};
    const int wofs[4] = {kGW1, kGW2, kGW3, kGW4}, bofs[4] = {kGB1, kGB2, kGB3, kGB4};
    const int outs[4] = {kGHid, kGHid, kGHid, kGOut}, ins[4] = {kGIn, kGHid, kGHid, kGHid};
    WgUnit w{};
    if (u < 88) {
        int l = 0;
        while (u >= (outs[l] / 16) * (ins[l] / 16)) { u -= (outs[l] / 16) * (ins[l] / 16); ++l; }
        const int pb = ins[l] / 16, m0 = (u / pb) * 16, n0 = (u % pb) * 16;
        w.a_off = dcol[l] + m0; w.b_off = hcol[l] + n0;
        w.goff = wofs[l] + m0 * ins[l] + n0; w.cols = ins[l];
    } else {
        u -= 88;
        int l = 0;
        while (u >= outs[l] / 16) { u -= outs[l] / 16; ++l; }
        w.a_off = dcol[l] + u * 16; w.b_off = -1;
        w.goff = bofs[l] + u * 16; w.cols = 1;
    }
    return w;
}

LD void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
LD void bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
// Polls the barrier's phase `parity` at most kWgSpin times; false if it
// never completed.
LD bool mbar_wait(unsigned bar, unsigned parity) {
    for (long long i = 0; i < kWgSpin; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(32 * kWgWarps, 1) k_guide_wgrad(const __nv_bfloat16* ws, int chunks, float* part,
                                                                  int* flag) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const unsigned buf0 = smem_u32(smem), bar0 = smem_u32(&bars[0]);
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();
    // this warp's units
    const int u_lo = warp * kWgUnits / kWgWarps, u_hi = (warp + 1) * kWgUnits / kWgWarps;
    int a_off[kWgMaxUnits], b_off[kWgMaxUnits];
#pragma unroll
    for (int j = 0; j < kWgMaxUnits; ++j) {
        WgUnit w = wg_unit(min(u_lo + j, kWgUnits - 1));
        a_off[j] = w.a_off; b_off[j] = w.b_off;
    }
    float acc[kWgMaxUnits][8];
#pragma unroll
    for (int j = 0; j < kWgMaxUnits; ++j)
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[j][i] = 0.0f;
    // ldmatrix row addresses: A = D^T blocks (matrices k0|m0, k0|m0+8,
    // k0+8|m0, k0+8|m0+8), B = H^T blocks (k0|n0, k0+8|n0, k0|n0+8, k0+8|n0+8)
    const int mi = lane >> 3, ri = lane & 7;
    const int a_lane = (ri + ((mi >> 1) << 3)) * kWsRow + ((mi & 1) << 3);
    const int b_lane = (ri + ((mi & 1) << 3)) * kWsRow + ((mi >> 1) << 3);
    const unsigned ones = pack_bf16(1.0f, 1.0f);
    bool ok = true;
    if (threadIdx.x == 0 && (int)blockIdx.x < chunks)
        bulk_load(buf0, ws + (size_t)blockIdx.x * kWgRows * kWsRow, (unsigned)kWgChunkBytes, bar0);
    int it = 0;
    for (int c = blockIdx.x; c < chunks; c += gridDim.x, ++it) {
        const int b = it & 1;
        const int nxt = c + gridDim.x;
        if (threadIdx.x == 0 && nxt < chunks)
            bulk_load(buf0 + (unsigned)((b ^ 1) * kWgChunkBytes), ws + (size_t)nxt * kWgRows * kWsRow,
                      (unsigned)kWgChunkBytes, bar0 + 8 * (b ^ 1));
        ok = mbar_wait(bar0 + 8 * b, (it >> 1) & 1);
        if (!__syncthreads_and(ok)) break;
        const unsigned base = buf0 + (unsigned)(b * kWgChunkBytes);
#pragma unroll
        for (int ks = 0; ks < kWgRows; ks += 16) {
            const unsigned kb = base + 2u * (unsigned)(ks * kWsRow);
            int a_cur = -1;
            unsigned a[4] = {0, 0, 0, 0};
#pragma unroll
            for (int j = 0; j < kWgMaxUnits; ++j) {
                if (u_lo + j < u_hi) {
                    if (a_off[j] != a_cur) {
                        ldsm_x4_trans(kb + 2u * (unsigned)(a_lane + a_off[j]), a);
                        a_cur = a_off[j];
                    }
                    if (b_off[j] >= 0) {
                        unsigned bb[4];
                        ldsm_x4_trans(kb + 2u * (unsigned)(b_lane + b_off[j]), bb);
                        mma16816(acc[j], a, bb);
                        mma16816(acc[j] + 4, a, bb + 2);
                    } else {
                        const unsigned bo[2] = {ones, ones};
                        mma16816(acc[j], a, bo);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!ok) {
        // give the copies still in flight (this chunk's, the prefetched
        // one's) a bounded time to land before the shared memory goes away
        if (threadIdx.x == 0) {
            atomicExch(flag, 1);
            const int c = blockIdx.x + it * gridDim.x;
            mbar_wait(bar0 + 8 * (it & 1), (it >> 1) & 1);
            if (c + (int)gridDim.x < chunks) mbar_wait(bar0 + 8 * ((it + 1) & 1), ((it + 1) >> 1) & 1);
        }
        return;
    }
    float* dst = part + (size_t)blockIdx.x * kGParams;
#pragma unroll
    for (int j = 0; j < kWgMaxUnits; ++j) {
        if (u_lo + j < u_hi) {
            const WgUnit w = wg_unit(u_lo + j);
            if (w.b_off >= 0) {
                float* o = dst + w.goff;
                o[g * w.cols + 2 * q] = acc[j][0];
                o[g * w.cols + 2 * q + 1] = acc[j][1];
                o[(g + 8) * w.cols + 2 * q] = acc[j][2];
                o[(g + 8) * w.cols + 2 * q + 1] = acc[j][3];
                o[g * w.cols + 8 + 2 * q] = acc[j][4];
                o[g * w.cols + 8 + 2 * q + 1] = acc[j][5];
                o[(g + 8) * w.cols + 8 + 2 * q] = acc[j][6];
                o[(g + 8) * w.cols + 8 + 2 * q + 1] = acc[j][7];
            } else if (q == 0) {
                dst[w.goff + g] = acc[j][0];
                dst[w.goff + g + 8] = acc[j][2];
            }
        }
    }
}

// grad[i] += sum over blocks of part[block][i], in block order.
__global__ void k_guide_reduce(const float* part, int blocks, float* grad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGParams; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < blocks; ++b) s += part[(size_t)b * kGParams + i];
        grad[i] += s;
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
    for (void* p : {(void*)master_, (void*)m_, (void*)v_, (void*)grad_, (void*)wq_, (void*)csum_, ws_, (void*)part_,
                    (void*)flag_})
        if (p) cudaFree(p);
    master_ = m_ = v_ = grad_ = csum_ = part_ = nullptr;
    wq_ = ws_ = nullptr;
    flag_ = nullptr;
    ws_rows_ = part_blocks_ = 0;
}

int GuideNet::init(int seed, cudaStream_t st) {
    release();
    GCK(cudaMalloc(&master_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&m_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&v_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&grad_, kGParams * sizeof(float)));
    GCK(cudaMalloc(&csum_, sizeof(float)));
    GCK(cudaMalloc(&flag_, sizeof(int)));
    GCK(cudaMemsetAsync(flag_, 0, sizeof(int), st));
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
    static bool attr = false;
    if (!attr) {
        GCK(cudaFuncSetAttribute(k_guide_fb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFbSmem));
        GCK(cudaFuncSetAttribute(k_guide_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgSmem));
        attr = true;
    }
    // workspace rows for whole chunks; rows past n stay zero
    const int chunks = (n + kWgRows - 1) / kWgRows, rows = chunks * kWgRows;
    const int wblocks = std::min(chunks, sms);
    if (ws_rows_ < rows || part_blocks_ < wblocks) {
        if (ws_) cudaFree(ws_);
        if (part_) cudaFree(part_);
        ws_ = nullptr;
        part_ = nullptr;
        ws_rows_ = part_blocks_ = 0;
        GCK(cudaMalloc(&ws_, (size_t)rows * kWsRow * sizeof(__nv_bfloat16)));
        GCK(cudaMalloc(&part_, (size_t)sms * kGParams * sizeof(float)));
        ws_rows_ = rows;
        part_blocks_ = sms;
    }
    __nv_bfloat16* ws = WQ(ws_);
    if (rows > n) GCK(cudaMemsetAsync(ws + (size_t)n * kWsRow, 0, (size_t)(rows - n) * kWsRow * sizeof(__nv_bfloat16), st));
    int blocks = std::max(1, std::min(sms, (n + 16 * kFbWarps - 1) / (16 * kFbWarps)));
    k_guide_fb<<<blocks, 32 * kFbWarps, kFbSmem, st>>>(recs, n, WQ(wq_), master_, csum_, ws);
    k_guide_wgrad<<<wblocks, 32 * kWgWarps, kWgSmem, st>>>(ws, chunks, part_, flag_);
    k_guide_reduce<<<(kGParams + 255) / 256, 256, 0, st>>>(part_, wblocks, grad_);
    GCK(cudaGetLastError());
    return 0;
}

int GuideNet::failed(cudaStream_t st) {
    int h = 0;
    GCK(cudaMemcpyAsync(&h, flag_, sizeof(int), cudaMemcpyDeviceToHost, st));
    GCK(cudaStreamSynchronize(st));
    if (h) {
        err_ = "guide training: a bounded wait for a workspace copy gave up";
        return -3;
    }
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
