// lucid_guide.cu — training of the path-guiding network (forward/backward
// pass, then every weight gradient as tcgen05 GEMMs over the records with
// TMA-fed shared memory and TMEM accumulators; Adam on FP32 masters).
#include <cuda.h>
#include <cudaTypedefs.h>
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
// (x, h1..h3) and the gradients of the layer outputs (d4..d1) go to a BF16
// workspace stored feature-major (one row of records per feature).  Pass 2
// (k_guide_wgrad_tc): every weight and bias gradient, dW = D^T H and
// db = D^T 1, as two tcgen05 GEMMs contracting over the records: TMA streams
// 64-record chunks of the feature rows into swizzled shared memory, one
// thread issues the MMAs into TMEM accumulators, and each block writes its
// partial gradient; k_guide_reduce_tc sums the partials in block order.
constexpr int kFbWarps = 14;
constexpr size_t kFbSmem = sizeof(GuideSmemW) + kFbWarps * sizeof(TrainTile);
// Feature rows of the workspace, in the order the GEMMs read them:
//   A_a = [d1 | d4] (112 rows)   B_a = [x | h3] (240 rows)
//   A_b = [d2 | d3] (128 rows)   B_b = [h1 | h2] (128 rows)
// GEMM a: rows 0..63 of A_a against rows 0..175 of B_a give dW1, rows 64..111
// against rows 176..239 give dW4; GEMM b: d2 x h1 = dW2, d3 x h2 = dW3 (the
// off-diagonal blocks are computed and discarded).  A ones row after each B
// block gives the bias gradients in the same accumulators.
constexpr int kTD1 = 0, kTD4 = kTD1 + kGHid, kTX = kTD4 + kGOut, kTH3 = kTX + kGIn, kTD2 = kTH3 + kGHid,
              kTD3 = kTD2 + kGHid, kTH1 = kTD3 + kGHid, kTH2 = kTH1 + kGHid, kTFeat = kTH2 + kGHid;
static_assert(kTD4 + kGOut == kTX && kTX - kTD1 == 112 && kTD2 - kTX == 240 && kTFeat == 608, "workspace rows");

// Copies a 16-record tile (row r = record r0 + r, ld `ld` in shared memory,
// ld and cols even) into feature rows f0.. of the feature-major workspace
// (rcap records per row).  Each lane takes two features of 8 records: eight
// 32-bit reads of feature pairs, regrouped by byte permutes into one 16-byte
// vector per feature.
LD void tile_store_t(const __nv_bfloat16* src, int ld, int cols, __nv_bfloat16* ws, int f0, int r0, int n, int rcap) {
    const int lane = threadIdx.x & 31;
    for (int e = lane; e < cols; e += 32) {   // cols / 2 feature pairs x 2 record halves
        const int f = 2 * (e >> 1), h = e & 1, rb = r0 + 8 * h;
        const unsigned* s32 = reinterpret_cast<const unsigned*>(src + 8 * h * ld + f);
        unsigned w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) w[k] = s32[k * (ld >> 1)];
        __nv_bfloat16* d0 = ws + (size_t)(f0 + f) * rcap + rb;
        __nv_bfloat16* d1 = d0 + rcap;
        if (rb + 8 <= n) {
            *reinterpret_cast<uint4*>(d0) = make_uint4(__byte_perm(w[0], w[1], 0x5410), __byte_perm(w[2], w[3], 0x5410),
                                                       __byte_perm(w[4], w[5], 0x5410), __byte_perm(w[6], w[7], 0x5410));
            *reinterpret_cast<uint4*>(d1) = make_uint4(__byte_perm(w[0], w[1], 0x7632), __byte_perm(w[2], w[3], 0x7632),
                                                       __byte_perm(w[4], w[5], 0x7632), __byte_perm(w[6], w[7], 0x7632));
        } else {
            for (int k = 0; k < 8 && rb + k < n; ++k) {
                d0[k] = src[(8 * h + k) * ld + f];
                d1[k] = src[(8 * h + k) * ld + f + 1];
            }
        }
    }
}

__global__ void __launch_bounds__(32 * kFbWarps) k_guide_fb(const GuideRec* recs, int n, const __nv_bfloat16* wq,
                                                           const float* master, const float* csum,
                                                           __nv_bfloat16* ws, int rcap) {
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
        tile_store_t(T.x, kLdIn, kGIn, ws, kTX, r0, n, rcap);
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
        tile_store_t(T.h1, kLdH, kGHid, ws, kTH1, r0, n, rcap);
        tile_store_t(T.h2, kLdH, kGHid, ws, kTH2, r0, n, rcap);
        tile_store_t(T.h3, kLdH, kGHid, ws, kTH3, r0, n, rcap);
        tile_store_t(T.dout(), kLdH, kGOut, ws, kTD4, r0, n, rcap);
        tile_store_t(T.da(), kLdH, kGHid, ws, kTD3, r0, n, rcap);
        __syncwarp();
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.da(), W.w3, T.h2, T.db());
        __syncwarp();
        tile_store_t(T.db(), kLdH, kGHid, ws, kTD2, r0, n, rcap);
        tile_backprop<kGHid, kGHid, kLdH, kLdH>(T.db(), W.w2, T.h1, T.da());
        __syncwarp();
        tile_store_t(T.da(), kLdH, kGHid, ws, kTD1, r0, n, rcap);
        __syncwarp();
    }
}

// ---- pass 2: tcgen05 weight-gradient GEMMs ----------------------------------------
// Each stage holds 64 records of every operand block, K-major with the
// 128-byte swizzle TMA writes (one 128-byte row per feature, 8-row groups
// 1024 bytes apart).  Rows past a block's TMA box are written once at
// start: zeros, and a row of ones at B_a row 240 and B_b row 128.
constexpr int kTcK = 64;                                     // records per stage
constexpr int kTcNa = 256, kTcNb = 144;                      // GEMM N (B rows incl. ones row + zeros)
constexpr unsigned kTcAa = 0, kTcBa = kTcAa + 128 * 128, kTcAb = kTcBa + kTcNa * 128, kTcBb = kTcAb + 128 * 128,
                   kTcStage = kTcBb + kTcNb * 128;           // 83,968 bytes
constexpr unsigned kTcTx = (112 + 240 + 128 + 128) * 128;     // TMA bytes per stage
constexpr size_t kTcSmem = 2 * (size_t)kTcStage + 1024;      // two stages + alignment
constexpr int kTcSlots = 128 * (kTcNa + kTcNb);              // partial floats per block
constexpr unsigned kTcCols = 512;                            // TMEM columns allocated
static_assert(kTcStage % 1024 == 0 && kTcBa % 1024 == 0 && kTcAb % 1024 == 0 && kTcBb % 1024 == 0, "1024-B stages");
constexpr long long kWgSpin = 1ll << 24;   // bound on the polls of one barrier phase

LD void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
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
LD void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}
// Shared-memory matrix descriptor (sm100): start address, leading offset
// 16 B (unused by swizzled K-major layouts), 8-row groups 1024 B apart,
// descriptor version 1, 128-byte swizzle.
LD unsigned long long tc_desc(unsigned saddr) {
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}
// Instruction descriptor, kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr unsigned tc_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(m >> 4) << 24);
}
LD void tc_mma(unsigned d_tmem, unsigned long long a, unsigned long long b, unsigned idesc, unsigned acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}
// The barrier's arrival once every tcgen05.mma this thread issued so far has
// completed.
LD void tc_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
LD void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
LD void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// 32 lanes x 16 consecutive columns of FP32 from TMEM (this warp's lanes).
LD void tmem_ld16(unsigned taddr, float* v) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15},"
        " [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// One block per SM (its shared memory and 512 TMEM columns leave room for no
// second one).  Warp 0 lane 0 feeds the stages by TMA, warp 1 lane 0 issues
// the MMAs; all four warps then move the accumulators (TMEM lanes = GEMM
// rows) to this block's partial, column-major so the stores coalesce.
__global__ void __launch_bounds__(128, 1)
    k_guide_wgrad_tc(const __grid_constant__ CUtensorMap m112, const __grid_constant__ CUtensorMap m240,
                     const __grid_constant__ CUtensorMap m128, int chunks, float* part, int* flag) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bars[5];   // full[2], empty[2], done
    __shared__ unsigned tmem_base_s;
    __shared__ int abort_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const unsigned full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[2]), done = smem_u32(&bars[4]);
    const int iters = chunks > (int)blockIdx.x ? (chunks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;

    // constant rows of both stages: zeros, and the ones rows of the B blocks
    unsigned char* gbase = smem_raw + (base - smem_u32(smem_raw));
    for (int s = 0; s < 2; ++s) {
        unsigned char* st = gbase + s * kTcStage;
        for (int e = threadIdx.x; e < 3 * 16 * 8; e += blockDim.x) {   // 3 blocks x 16 rows x 8 vectors
            const int blk = e / 128, row = (e / 8) % 16, vec = e % 8;
            const unsigned off = blk == 0 ? kTcAa + (112 + row) * 128 : blk == 1 ? kTcBa + (240 + row) * 128
                                                                                : kTcBb + (128 + row) * 128;
            const unsigned one = row == 0 && blk > 0 ? 0x3F803F80u : 0u;   // BF16 1.0 pairs
            *reinterpret_cast<uint4*>(st + off + vec * 16) = make_uint4(one, one, one, one);
        }
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < 5; ++i) mbar_init(full0 + 8 * i, 1);
        abort_s = 0;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // the MMAs read the rows written above
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     ::"r"(smem_u32(&tmem_base_s)), "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_base_s;

    if (warp == 0 && lane == 0) {
        // producer
        for (int it = 0; it < iters; ++it) {
            const int s = it & 1;
            if (it >= 2 && !mbar_wait(empty0 + 8 * s, ((it >> 1) - 1) & 1)) { abort_s = 1; break; }
            if (*(volatile int*)&abort_s) break;
            const int x = (blockIdx.x + it * gridDim.x) * kTcK;
            const unsigned sb = base + s * kTcStage, fb = full0 + 8 * s;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(kTcTx) : "memory");
            tma_load_2d(sb + kTcAa, &m112, x, kTD1, fb);
            tma_load_2d(sb + kTcBa, &m240, x, kTX, fb);
            tma_load_2d(sb + kTcAb, &m128, x, kTD2, fb);
            tma_load_2d(sb + kTcBb, &m128, x, kTH1, fb);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: D_a = A_a B_a^T in TMEM columns [0, 256), D_b in [256, 400)
        const unsigned ida = tc_idesc(128, kTcNa), idb = tc_idesc(128, kTcNb);
        for (int it = 0; it < iters; ++it) {
            const int s = it & 1;
            if (!mbar_wait(full0 + 8 * s, (it >> 1) & 1)) { abort_s = 1; break; }
            tc_fence_after();
            const unsigned sb = base + s * kTcStage;
            const unsigned long long da = tc_desc(sb + kTcAa), db = tc_desc(sb + kTcBa), dc = tc_desc(sb + kTcAb),
                                     dd = tc_desc(sb + kTcBb);
#pragma unroll
            for (int k = 0; k < kTcK / 16; ++k) {   // 16 records (32 bytes) per MMA
                const unsigned acc = (it > 0 || k > 0) ? 1u : 0u;
                tc_mma(tmem, da + 2 * k, db + 2 * k, ida, acc);
                tc_mma(tmem + kTcNa, dc + 2 * k, dd + 2 * k, idb, acc);
            }
            tc_commit(empty0 + 8 * s);
        }
        tc_commit(done);
    }
    __syncwarp();
    // epilogue: every thread waits for the last MMAs (bounded)
    const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0) && !*(volatile int*)&abort_s);
    tc_fence_after();
    if (ok && iters > 0) {
        float* dst = part + (size_t)blockIdx.x * kTcSlots + warp * 32 + lane;
        const unsigned lane_base = tmem + ((unsigned)(warp * 32) << 16);
        for (int c0 = 0; c0 < kTcNa + kTcNb; c0 += 16) {
            float v[16];
            tmem_ld16(lane_base + (unsigned)c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) dst[(size_t)(c0 + i) * 128] = v[i];
        }
    } else if (threadIdx.x == 0) {
        atomicExch(flag, 1);
    }
    if (!ok && threadIdx.x == 0) {
        // give the loads still in flight a bounded time to land before the
        // shared memory goes away
        for (int s = 0; s < 2; ++s) mbar_wait(full0 + 8 * s, 0), mbar_wait(full0 + 8 * s, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTcCols));
    }
}

// Slot of parameter i in a block's partial: D_a(row, col) at col * 128 + row
// (cols 0..255), D_b(row, col) at 128 * 256 + col * 128 + row.
LD int tc_slot(int i) {
    constexpr int Db = 128 * kTcNa;
    if (i < kGB1) return (i % kGIn) * 128 + i / kGIn;                                     // W1: D_a(o, x)
    if (i < kGW2) return 240 * 128 + (i - kGB1);                                          // b1: D_a(o, ones)
    if (i < kGB2) { const int j = i - kGW2; return Db + (j % kGHid) * 128 + j / kGHid; }  // W2: D_b(o, h1)
    if (i < kGW3) return Db + 128 * 128 + (i - kGB2);                                     // b2: D_b(o, ones)
    if (i < kGB3) { const int j = i - kGW3; return Db + (64 + j % kGHid) * 128 + 64 + j / kGHid; }   // W3
    if (i < kGW4) return Db + 128 * 128 + 64 + (i - kGB3);                                // b3
    if (i < kGB4) { const int j = i - kGW4; return (kGIn + j % kGHid) * 128 + 64 + j / kGHid; }      // W4
    return 240 * 128 + 64 + (i - kGB4);                                                    // b4
}

// grad[i] += sum over blocks of the block partials, in block order.
__global__ void k_guide_reduce_tc(const float* part, int blocks, float* grad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGParams; i += gridDim.x * blockDim.x) {
        const int slot = tc_slot(i);
        float s = 0.0f;
        for (int b = 0; b < blocks; ++b) s += part[(size_t)b * kTcSlots + slot];
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

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 2-D map over the feature-major workspace: n records (x, innermost) by
// kTFeat feature rows (y), rows rcap records apart; boxes of 64 records by
// `rows` features, 128-byte swizzle; records past n read as zeros.
static bool workspace_map(CUtensorMap* m, void* ws, int n, int rcap, int rows) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)kTFeat};
    cuuint64_t strides[1] = {(cuuint64_t)rcap * sizeof(__nv_bfloat16)};
    cuuint32_t box[2] = {(cuuint32_t)kTcK, (cuuint32_t)rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ws, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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
        GCK(cudaFuncSetAttribute(k_guide_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
        attr = true;
    }
    // feature rows of whole 64-record chunks (the GEMM reads records past n
    // as zeros through the tensor map)
    const int chunks = (n + kTcK - 1) / kTcK, rcap_need = chunks * kTcK;
    const int wblocks = std::min(chunks, sms);
    if (ws_rows_ < rcap_need || part_blocks_ < sms) {
        if (ws_) cudaFree(ws_);
        if (part_) cudaFree(part_);
        ws_ = nullptr;
        part_ = nullptr;
        ws_rows_ = part_blocks_ = 0;
        GCK(cudaMalloc(&ws_, (size_t)kTFeat * rcap_need * sizeof(__nv_bfloat16)));
        GCK(cudaMalloc(&part_, (size_t)sms * kTcSlots * sizeof(float)));
        ws_rows_ = rcap_need;
        part_blocks_ = sms;
    }
    const int rcap = ws_rows_;
    CUtensorMap m112, m240, m128;
    if (!workspace_map(&m112, ws_, n, rcap, 112) || !workspace_map(&m240, ws_, n, rcap, 240) ||
        !workspace_map(&m128, ws_, n, rcap, 128)) {
        err_ = "guide training: cuTensorMapEncodeTiled failed for the workspace";
        return -6;
    }
    int blocks = std::max(1, std::min(sms, (n + 16 * kFbWarps - 1) / (16 * kFbWarps)));
    k_guide_fb<<<blocks, 32 * kFbWarps, kFbSmem, st>>>(recs, n, WQ(wq_), master_, csum_, WQ(ws_), rcap);
    k_guide_wgrad_tc<<<wblocks, 128, kTcSmem, st>>>(m112, m240, m128, chunks, part_, flag_);
    k_guide_reduce_tc<<<(kGParams + 255) / 256, 256, 0, st>>>(part_, wblocks, grad_);
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
