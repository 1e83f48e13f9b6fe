// lucid_guide.cuh — the neural path-guiding distribution (device side).
//
// No reference counterpart.  A small MLP maps an encoded surface point
// (position: 16 sin/cos frequencies per axis over the scene box; normal;
// outgoing direction: one-blob over (cos theta, phi), 32 bins each) through
// three 64-wide ReLU layers to an 8-lobe von Mises-Fisher mixture (softmax
// weights, softplus concentrations, normalised mean directions).  Weights and
// activations are BF16 with FP32 accumulation on the tensor cores
// (mma.sync m16n8k16: the layers are 64 wide, far below one tcgen05 tile);
// the optimiser keeps FP32 master weights.  Guided vertices sample the BSDF
// or the mixture with probability 1/2 each and weight the sample by the
// balance heuristic (one-sample MIS), so the estimator stays unbiased.
#pragma once

#include <cuda_bf16.h>

#include "lucid_device.cuh"

namespace lucid {

constexpr int kGIn = 176;        // 96 position + 3 normal + 64 direction (+13 zero padding)
constexpr int kGInUsed = 163;
constexpr int kGHid = 64;
constexpr int kGOut = 48;        // 8 logits, 8 concentrations, 8 x 3 mean directions (+8 padding)
constexpr int kGLobes = 8;
constexpr int kGFreq = 16;
constexpr int kGBins = 32;
// parameter layout (FP32 master and BF16 copies): W1[64][176] b1[64]
// W2[64][64] b2[64] W3[64][64] b3[64] W4[48][64] b4[48]
constexpr int kGW1 = 0, kGB1 = kGW1 + kGHid * kGIn, kGW2 = kGB1 + kGHid, kGB2 = kGW2 + kGHid * kGHid,
              kGW3 = kGB2 + kGHid, kGB3 = kGW3 + kGHid * kGHid, kGW4 = kGB3 + kGHid, kGB4 = kGW4 + kGOut * kGHid,
              kGParams = kGB4 + kGOut;
constexpr float kGKappaMin = 0.05f, kGKappaMax = 2000.0f;

// Mixture parameters of one vertex (40 floats): weights, concentrations,
// mean directions.
struct GuideMix {
    float w[kGLobes], k[kGLobes];
    V3 mu[kGLobes];
};

// ---- encoding --------------------------------------------------------------
// Writes the kGIn input features; p01 is the position in [0,1]^3 of the
// scene box.  The frequencies are pi * 2^j, j = 0..15.
LD float one_blob(float x, int b) {
    float c = ((float)b + 0.5f) * (1.0f / kGBins);
    float d = (x - c) * (float)kGBins;
    return __expf(-0.5f * d * d);
}
// sin and cos of pi t: t reduced exactly to r = t - 2 rint(t / 2) in
// [-1, 1], then the hardware approximations on [-pi, pi] (absolute error
// below 1e-6, far under the BF16 rounding the features go through).
LD void sincospi_fast(float t, float* s, float* c) {
    const float r = t - 2.0f * rintf(0.5f * t);
    __sincosf(kPI * r, s, c);
}
// Features [0, 96): the position frequencies.
template <class Store>
LD void guide_encode_position(V3 p01, Store&& st) {
    const float pc[3] = {p01.x, p01.y, p01.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float x = pc[a];
        for (int j = 0; j < kGFreq; ++j) {
            float s, c;
            sincospi_fast(x * (float)(1 << j), &s, &c);
            st(a * 2 * kGFreq + 2 * j, s);
            st(a * 2 * kGFreq + 2 * j + 1, c);
        }
    }
}
// Features [96, kGIn): normal, one-blob outgoing direction, zero padding.
template <class Store>
LD void guide_encode_direction(V3 n, V3 wo, Store&& st) {
    st(96, n.x); st(97, n.y); st(98, n.z);
    float u = sclamp(0.5f * (wo.z + 1.0f), 0.0f, 1.0f);
    float v = atan2f(wo.y, wo.x) * (0.5f * kINV_PI) + 0.5f;
    for (int b = 0; b < kGBins; ++b) {
        st(99 + b, one_blob(u, b));
        st(99 + kGBins + b, one_blob(v, b));
    }
    for (int i = kGInUsed; i < kGIn; ++i) st(i, 0.0f);
}
template <class Store>
LD void guide_encode(V3 p01, V3 n, V3 wo, Store&& st) {
    guide_encode_position(p01, st);
    guide_encode_direction(n, wo, st);
}
// The same features split over two lanes that run the same instructions:
// half 0 writes frequencies 0..7, the normal and the cos-theta one-blob;
// half 1 frequencies 8..15, the phi one-blob and the padding.
template <class Store>
LD void guide_encode_half(V3 p01, V3 n, V3 wo, int half, Store&& st) {
    const float pc[3] = {p01.x, p01.y, p01.z};
    const int j0 = half * (kGFreq / 2);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll 2
        for (int j = j0; j < j0 + kGFreq / 2; ++j) {
            float s, c;
            sincospi_fast(pc[a] * (float)(1 << j), &s, &c);
            st(a * 2 * kGFreq + 2 * j, s);
            st(a * 2 * kGFreq + 2 * j + 1, c);
        }
    }
    float x;
    if (half == 0) {
        st(96, n.x); st(97, n.y); st(98, n.z);
        x = sclamp(0.5f * (wo.z + 1.0f), 0.0f, 1.0f);
    } else {
        x = atan2f(wo.y, wo.x) * (0.5f * kINV_PI) + 0.5f;
        for (int i = kGInUsed; i < kGIn; ++i) st(i, 0.0f);
    }
    const int base = 99 + half * kGBins;
#pragma unroll 4
    for (int b = 0; b < kGBins; ++b) st(base + b, one_blob(x, b));
}

// ---- vMF mixture ----------------------------------------------------------------
LD float softplusf(float x) { return x > 20.0f ? x : log1pf(__expf(x)); }
LD float sigmoidf(float x) { return 1.0f / (1.0f + __expf(-x)); }

// Raw network outputs (kGOut floats) -> mixture parameters.
LD void guide_mix_from_raw(const float* raw, GuideMix& g) {
    float mx = raw[0];
    for (int i = 1; i < kGLobes; ++i) mx = fmaxf(mx, raw[i]);
    float sum = 0.0f;
    for (int i = 0; i < kGLobes; ++i) { g.w[i] = __expf(raw[i] - mx); sum += g.w[i]; }
    for (int i = 0; i < kGLobes; ++i) {
        g.w[i] /= sum;
        g.k[i] = fminf(softplusf(raw[kGLobes + i]) + kGKappaMin, kGKappaMax);
        V3 m = v3(raw[16 + 3 * i], raw[17 + 3 * i], raw[18 + 3 * i]);
        float l = len(m);
        g.mu[i] = l > 1e-6f ? m / l : v3(0.0f, 0.0f, 1.0f);
    }
}

// vMF density kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.w - 1)).
LD float vmf_pdf(float kappa, V3 mu, V3 w) {
    float norm = kappa / (kTWO_PI * (1.0f - __expf(-2.0f * kappa)));
    return norm * __expf(kappa * (dot(mu, w) - 1.0f));
}
LD float guide_pdf(const GuideMix& g, V3 w) {
    float p = 0.0f;
    for (int i = 0; i < kGLobes; ++i) p += g.w[i] * vmf_pdf(g.k[i], g.mu[i], w);
    return p;
}
// Lobe chosen by u0, direction by (u1, u2) (inversion of the vMF's cosine
// marginal, the numerically stable form of Jakob, "Numerically stable
// sampling of the von Mises Fisher distribution on S2", 2012).
LD V3 guide_sample(const GuideMix& g, float u0, float u1, float u2) {
    int lobe = kGLobes - 1;
    float c = 0.0f;
    for (int i = 0; i < kGLobes; ++i) {
        c += g.w[i];
        if (u0 < c) { lobe = i; break; }
    }
    float kappa = g.k[lobe];
    float w = 1.0f + logf(u1 + (1.0f - u1) * __expf(-2.0f * kappa)) / kappa;
    w = sclamp(w, -1.0f, 1.0f);
    float r = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float s, cs;
    sincospif(2.0f * u2, &s, &cs);
    V3 t, b;
    onb(g.mu[lobe], t, b);
    return make_dir_or(t * (r * cs) + b * (r * s) + g.mu[lobe] * w, g.mu[lobe]);
}

// ---- compact mixture (inference output, read by shading) ------------------------
// 40 floats per vertex: per lobe l a float4 (kappa mu, log(w norm) - kappa),
// so that the mixture density is sum_l exp(A_l.xyz . wi + A_l.w), then the
// cumulative lobe weights.  Lanes h = 0, 1 of a row write lobes 4h..4h+3
// (float4s h*4.. and the cumulative weights 4h..4h+3).
constexpr int kGMixFloats = 40;
LD void guide_compact_half(const float* raw, int half, float4* out) {
    float mx = raw[0];
    for (int i = 1; i < kGLobes; ++i) mx = fmaxf(mx, raw[i]);
    float e[kGLobes], sum = 0.0f;
#pragma unroll
    for (int i = 0; i < kGLobes; ++i) { e[i] = __expf(raw[i] - mx); sum += e[i]; }
    const float inv = 1.0f / sum, lsum = __logf(sum);
    float cw[kGLobes], c = 0.0f;
#pragma unroll
    for (int i = 0; i < kGLobes; ++i) { c += e[i] * inv; cw[i] = c; }
#pragma unroll
    for (int j = 0; j < kGLobes / 2; ++j) {
        const int l = half * (kGLobes / 2) + j;
        const float x = raw[kGLobes + l];
        const float sp = x > 20.0f ? x : __logf(1.0f + __expf(x));
        const float kappa = fminf(sp + kGKappaMin, kGKappaMax);
        const V3 m = v3(raw[16 + 3 * l], raw[17 + 3 * l], raw[18 + 3 * l]);
        const float l2 = dot(m, m);
        const V3 mu = l2 > 1e-12f ? m * rsqrtf(l2) : v3(0.0f, 0.0f, 1.0f);
        // log(w) + log(kappa / (2 pi (1 - e^{-2 kappa}))) - kappa
        const float lw = raw[l] - mx - lsum;
        const float ln = __logf(kappa) - __logf(kTWO_PI * (1.0f - __expf(-2.0f * kappa)));
        out[j] = make_float4(kappa * mu.x, kappa * mu.y, kappa * mu.z, lw + ln - kappa);
    }
    out[4] = half ? make_float4(cw[4], cw[5], cw[6], cw[7]) : make_float4(cw[0], cw[1], cw[2], cw[3]);
}
LD float guide_pdf_c(const float* gm, V3 wi) {
    const float4* A = reinterpret_cast<const float4*>(gm);
    float p = 0.0f;
#pragma unroll
    for (int l = 0; l < kGLobes; ++l) {
        const float4 a = A[l];
        p += __expf(a.x * wi.x + a.y * wi.y + a.z * wi.z + a.w);
    }
    return p;
}
// Lobe by u0 from the cumulative weights, then the vMF inversion of
// guide_sample on that lobe.
LD V3 guide_sample_c(const float* gm, float u0, float u1, float u2) {
    const float4* A = reinterpret_cast<const float4*>(gm);
    const float4 c0 = A[8], c1 = A[9];
    const float cw[kGLobes] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    int lobe = kGLobes - 1;
#pragma unroll
    for (int i = kGLobes - 2; i >= 0; --i)
        if (u0 < cw[i]) lobe = i;
    const float4 a = A[lobe];
    const float kappa = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    const V3 mu = kappa > 0.0f ? v3(a.x, a.y, a.z) / kappa : v3(0.0f, 0.0f, 1.0f);
    float w = 1.0f + logf(u1 + (1.0f - u1) * __expf(-2.0f * kappa)) / kappa;
    w = sclamp(w, -1.0f, 1.0f);
    float r = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    float s, cs;
    sincospif(2.0f * u2, &s, &cs);
    V3 t, b;
    onb(mu, t, b);
    return make_dir_or(t * (r * cs) + b * (r * s) + mu * w, mu);
}

// ---- tensor-core tiles ---------------------------------------------------------
// mma.sync.m16n8k16 BF16 -> FP32.  Fragment ownership (PTX ISA, "Matrix
// fragments for mma.m16n8k16"): with g = lane / 4 and q = lane % 4,
// A (16x16, row major): regs 0,1 = A[g][2q..2q+1], A[g+8][2q..2q+1];
// regs 2,3 = A[g][2q+8..], A[g+8][2q+8..].  B (16x8, "col"): reg 0 =
// B[2q..2q+1][g], reg 1 = B[2q+8..2q+9][g].  C/D (16x8): c0,c1 = D[g][2q..],
// c2,c3 = D[g+8][2q..].
LD unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned*>(&v);
}
LD void mma16816(float* d, const unsigned* a, const unsigned* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---- shared-memory images ------------------------------------------------------
// Rows padded by 8 BF16 so that the eight fragment rows of a warp fall in
// different banks (184 and 72 elements = 92 and 36 words per row).
constexpr int kLdIn = kGIn + 8;
constexpr int kLdH = kGHid + 8;
struct GuideSmemW {
    __nv_bfloat16 w1[kGHid * kLdIn];
    __nv_bfloat16 w2[kGHid * kLdH];
    __nv_bfloat16 w3[kGHid * kLdH];
    __nv_bfloat16 w4[kGOut * kLdH];
    float b1[kGHid], b2[kGHid], b3[kGHid], b4[kGOut];
};
// One warp's 16-row tile: inputs, the three hidden activations, raw outputs.
struct GuideTile {
    __nv_bfloat16 x[16 * kLdIn];
    __nv_bfloat16 h1[16 * kLdH], h2[16 * kLdH], h3[16 * kLdH];
    float raw[16 * kGOut];
};

// Copies the BF16 weights (dense [out][in]) and the FP32 biases into the
// padded shared image (all threads of the block).
LD void guide_load_weights(GuideSmemW& s, const __nv_bfloat16* wq, const float* master) {
    for (int i = threadIdx.x; i < kGHid * kGIn; i += blockDim.x) s.w1[(i / kGIn) * kLdIn + i % kGIn] = wq[kGW1 + i];
    for (int i = threadIdx.x; i < kGHid * kGHid; i += blockDim.x) {
        s.w2[(i / kGHid) * kLdH + i % kGHid] = wq[kGW2 + i];
        s.w3[(i / kGHid) * kLdH + i % kGHid] = wq[kGW3 + i];
    }
    for (int i = threadIdx.x; i < kGOut * kGHid; i += blockDim.x) s.w4[(i / kGHid) * kLdH + i % kGHid] = wq[kGW4 + i];
    for (int i = threadIdx.x; i < kGHid; i += blockDim.x) {
        s.b1[i] = master[kGB1 + i]; s.b2[i] = master[kGB2 + i]; s.b3[i] = master[kGB3 + i];
    }
    for (int i = threadIdx.x; i < kGOut; i += blockDim.x) s.b4[i] = master[kGB4 + i];
}

LD unsigned ld_pair(const __nv_bfloat16* p) { return *reinterpret_cast<const unsigned*>(p); }
LD unsigned pair2(const __nv_bfloat16* a, const __nv_bfloat16* b) {
    __nv_bfloat162 v;
    v.x = *a;
    v.y = *b;
    return *reinterpret_cast<unsigned*>(&v);
}

// ldmatrix: four 8x8 BF16 matrices, one 16-byte row address per lane
// (lanes 8j..8j+7 address the rows of matrix j); register j of a lane holds
// the two elements of matrix j at row lane/4, columns 2(lane%4) and +1 (the
// transposed variant: rows 2(lane%4) and +1 of column lane/4).
LD unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
LD void ldsm_x4(unsigned addr, unsigned* r) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
LD void ldsm_x4_trans(unsigned addr, unsigned* r) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
// Lane row addresses (element offsets) for a 16x16 row-major A block:
// matrices (r0, k0), (r0 + 8, k0), (r0, k0 + 8), (r0 + 8, k0 + 8) = a0..a3.
LD int ldsm_a_offset(int ld) {
    const int lane = threadIdx.x & 31, j = lane >> 3, r = lane & 7;
    return (r + ((j & 1) << 3)) * ld + ((j >> 1) << 3);
}
// ... and for the B fragments of two n-blocks of W stored [N][K]: matrices
// (n0, k0), (n0, k0 + 8), (n0 + 8, k0), (n0 + 8, k0 + 8) = (b0, b1) of n0,
// then of n0 + 8.
LD int ldsm_b_offset(int ld) {
    const int lane = threadIdx.x & 31, j = lane >> 3, r = lane & 7;
    return (r + ((j >> 1) << 3)) * ld + ((j & 1) << 3);
}

// out[16 x N] = act(A[16 x K] W^T + b), W stored [N][K]: one warp.  With
// RELU the result is stored as BF16 (ld kLdH); otherwise as FP32 (ld N).
template <int K, int N, int LDA, int LDW, bool RELU>
LD void tile_layer(const __nv_bfloat16* A, const __nv_bfloat16* W, const float* bias, __nv_bfloat16* outh,
                   float* outf) {
    static_assert(N % 16 == 0 && K % 16 == 0, "tile shape");
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    float acc[N / 8][4];
#pragma unroll
    for (int nb = 0; nb < N / 8; ++nb) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.0f;
    const unsigned a_base = smem_u32(A + ldsm_a_offset(LDA)), w_base = smem_u32(W + ldsm_b_offset(LDW));
#pragma unroll
    for (int kb = 0; kb < K / 16; ++kb) {
        unsigned a[4];
        ldsm_x4(a_base + 32u * kb, a);
#pragma unroll
        for (int nb = 0; nb < N / 8; nb += 2) {
            unsigned b[4];
            ldsm_x4(w_base + 2u * (unsigned)(nb * 8 * LDW + kb * 16), b);
            mma16816(acc[nb], a, b);
            mma16816(acc[nb + 1], a, b + 2);
        }
    }
#pragma unroll
    for (int nb = 0; nb < N / 8; ++nb) {
        const int c = nb * 8 + 2 * q;
        float v0 = acc[nb][0] + bias[c], v1 = acc[nb][1] + bias[c + 1];
        float v2 = acc[nb][2] + bias[c], v3 = acc[nb][3] + bias[c + 1];
        if (RELU) {
            *reinterpret_cast<unsigned*>(outh + g * kLdH + c) = pack_bf16(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
            *reinterpret_cast<unsigned*>(outh + (g + 8) * kLdH + c) = pack_bf16(fmaxf(v2, 0.0f), fmaxf(v3, 0.0f));
        } else {
            outf[g * N + c] = v0; outf[g * N + c + 1] = v1;
            outf[(g + 8) * N + c] = v2; outf[(g + 8) * N + c + 1] = v3;
        }
    }
}

// The whole network on one warp's tile (inputs already in t.x).
LD void guide_forward_tile(const GuideSmemW& w, GuideTile& t) {
    tile_layer<kGIn, kGHid, kLdIn, kLdIn, true>(t.x, w.w1, w.b1, t.h1, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGHid, kLdH, kLdH, true>(t.h1, w.w2, w.b2, t.h2, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGHid, kLdH, kLdH, true>(t.h2, w.w3, w.b3, t.h3, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGOut, kLdH, kLdH, false>(t.h3, w.w4, w.b4, nullptr, t.raw);
    __syncwarp();
}

// Inference tile: the layers alternate between two activation buffers and
// the raw outputs overwrite the inputs (10.25 KB per warp).
struct GuideLeanTile {
    __nv_bfloat16 x[16 * kLdIn];   // inputs, then the FP32 raw outputs (16 x kGOut)
    __nv_bfloat16 ha[16 * kLdH], hb[16 * kLdH];
    LD float* raw() { return reinterpret_cast<float*>(x); }
};
static_assert(sizeof(float) * 16 * kGOut <= sizeof(__nv_bfloat16) * 16 * kLdIn, "raw outputs fit the input rows");
LD void guide_forward_lean(const GuideSmemW& w, GuideLeanTile& t) {
    tile_layer<kGIn, kGHid, kLdIn, kLdIn, true>(t.x, w.w1, w.b1, t.ha, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGHid, kLdH, kLdH, true>(t.ha, w.w2, w.b2, t.hb, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGHid, kLdH, kLdH, true>(t.hb, w.w3, w.b3, t.ha, nullptr);
    __syncwarp();
    tile_layer<kGHid, kGOut, kLdH, kLdH, false>(t.ha, w.w4, w.b4, nullptr, t.raw());
    __syncwarp();
}

}  // namespace lucid
