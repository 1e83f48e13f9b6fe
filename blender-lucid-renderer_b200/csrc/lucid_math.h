// lucid_math.h — deterministic FP32 transcendental functions shared by the
// host (C++) and the device (CUDA) so that a path traced on the GPU and the
// same path traced on the CPU follow bit-identical float sequences.
//
// The reference renderer calls libm's std::sin / std::cos / std::exp /
// std::log / std::pow in its hot path (bsdf/ggx.hpp:154-155,194-195,
// bsdf/fresnel.hpp:33,41, light/light.hpp:202,285-286, volume/phase.hpp:67-68,
// volume/transmittance.hpp:127,208,262).  libm and CUDA's math library do not
// round identically, so the renderer uses these project-written versions on
// both sides instead.  Every function is built only from IEEE-754 operations
// that are correctly rounded on both targets (+, -, *, /, sqrt, fmaf) plus
// integer bit manipulation, evaluated in a fixed order, so the results agree
// bit for bit between gcc (-ffp-contract=off) and nvcc (-fmad=false).
//
// Methods (from the mathematics, not from any vendor library):
//   sin/cos : Cody–Waite argument reduction by pi/2 with a three-part split
//             constant, then the Taylor series of sin (to r^11) and cos (to
//             r^12) on |r| <= pi/4, evaluated by Horner's rule with fmaf.
//   exp     : x = k ln2 + r (two-part ln2), Taylor series of e^r to r^7,
//             scaled by 2^k built from the exponent field.
//   log     : x = m 2^e with m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
//             log m = 2 atanh(s) = 2s + 2s(z/3 + z^2/5 + ...), z = s^2.
//   pow5    : x^5 as (x*x)*(x*x)*x.
// Accuracy (checked by tests against libm in float64): <= 2 ulp on the
// argument ranges the renderer uses.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define LM_HD __host__ __device__ __forceinline__
#else
#define LM_HD inline
#include <math.h>
#endif

namespace lucid_math {

LM_HD float lm_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

LM_HD uint32_t lm_f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

LM_HD float lm_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

// Round to nearest integer (ties away from zero is not needed: any fixed rule
// works as long as both sides use it).  floor(x + 0.5) on the small magnitudes
// used here; the result only selects the reduction quadrant.
LM_HD float lm_round_half_up(float x) {
#if defined(__CUDA_ARCH__)
    return floorf(__fadd_rn(x, 0.5f));
#else
    return floorf(x + 0.5f);
#endif
}

// 2^n for n in [-126, 127] as an exact float.
LM_HD float lm_exp2i(int n) { return lm_u2f((uint32_t)(n + 127) << 23); }

// ---- sin / cos ---------------------------------------------------------------
// pi/2 split into three floats whose sum carries ~72 bits.
#define LM_PIO2_HI  1.5707963705062866211e+00f   /* float(pi/2)             */
#define LM_PIO2_MID -4.3711388286737928865e-08f  /* float(pi/2 - HI)        */
#define LM_PIO2_LO  -1.7151245100058819e-15f  /* float(pi/2 - HI - MID)  */
#define LM_2_OVER_PI 6.366197466850281e-01f

// Taylor coefficients 1/n! (rounded to float).
#define LM_S3  -1.6666667163372039795e-01f  /* -1/3!  */
#define LM_S5   8.3333337679505348206e-03f  /*  1/5!  */
#define LM_S7  -1.9841270113829523325e-04f  /* -1/7!  */
#define LM_S9   2.7557318844628753e-06f  /*  1/9!  */
#define LM_S11 -2.5052107943679403e-08f  /* -1/11! */
#define LM_C2  -5.0000000000000000000e-01f  /* -1/2!  */
#define LM_C4   4.1666667908430099487e-02f  /*  1/4!  */
#define LM_C6  -1.3888889225199818611e-03f  /* -1/6!  */
#define LM_C8   2.4801587642286904156e-05f  /*  1/8!  */
#define LM_C10 -2.755731998149713e-07f  /* -1/10! */
#define LM_C12  2.0876755879584152e-09f  /*  1/12! */

LM_HD float lm_sin_poly(float r) {
    float z = r * r;
    float p = lm_fma(z, LM_S11, LM_S9);
    p = lm_fma(z, p, LM_S7);
    p = lm_fma(z, p, LM_S5);
    p = lm_fma(z, p, LM_S3);
    return lm_fma(r * z, p, r);
}

LM_HD float lm_cos_poly(float r) {
    float z = r * r;
    float p = lm_fma(z, LM_C12, LM_C10);
    p = lm_fma(z, p, LM_C8);
    p = lm_fma(z, p, LM_C6);
    p = lm_fma(z, p, LM_C4);
    p = lm_fma(z, p, LM_C2);
    return lm_fma(z, p, 1.0f);
}

// Reduce x to r in [-pi/4, pi/4] and quadrant q (0..3).  Valid for |x| < 2^15.
LM_HD float lm_reduce_pio2(float x, int* q) {
    float k = lm_round_half_up(x * LM_2_OVER_PI);
    float r = lm_fma(-k, LM_PIO2_HI, x);
    r = lm_fma(-k, LM_PIO2_MID, r);
    r = lm_fma(-k, LM_PIO2_LO, r);
    *q = ((int)k) & 3;
    return r;
}

LM_HD float lm_sinf(float x) {
    int q;
    float r = lm_reduce_pio2(x, &q);
    float s = lm_sin_poly(r), c = lm_cos_poly(r);
    switch (q) {
        case 0: return s;
        case 1: return c;
        case 2: return -s;
        default: return -c;
    }
}

LM_HD float lm_cosf(float x) {
    int q;
    float r = lm_reduce_pio2(x, &q);
    float s = lm_sin_poly(r), c = lm_cos_poly(r);
    switch (q) {
        case 0: return c;
        case 1: return -s;
        case 2: return -c;
        default: return s;
    }
}

// ---- exp ---------------------------------------------------------------------
#define LM_LOG2E   1.4426950216293334961e+00f
#define LM_LN2_HI  6.931471824645996e-01f      /* float(ln2)                     */
#define LM_LN2_LO  -1.9046542121259336e-09f    /* float(ln2 - LN2_HI)            */
#define LM_E2 5.0000000000000000000e-01f
#define LM_E3 1.6666667163372039795e-01f
#define LM_E4 4.1666667908430099487e-02f
#define LM_E5 8.3333337679505348206e-03f
#define LM_E6 1.3888889225199818611e-03f
#define LM_E7 1.9841270113829523325e-04f

LM_HD float lm_expf(float x) {
    if (x != x) return x;                       // NaN
    if (x > 88.72283935546875f) return lm_u2f(0x7f800000u);   // +inf
    if (x < -103.97208404541015625f) return 0.0f;
    float k = lm_round_half_up(x * LM_LOG2E);
    float r = lm_fma(-k, LM_LN2_HI, x);
    r = lm_fma(-k, LM_LN2_LO, r);
    float p = lm_fma(r, LM_E7, LM_E6);
    p = lm_fma(r, p, LM_E5);
    p = lm_fma(r, p, LM_E4);
    p = lm_fma(r, p, LM_E3);
    p = lm_fma(r, p, LM_E2);
    p = lm_fma(r, p, 1.0f);
    p = lm_fma(r, p, 1.0f);
    int n = (int)k;
    // Two exact scalings keep 2^n representable for n in [-150, 128].
    int n1 = n / 2;
    int n2 = n - n1;
    return (p * lm_exp2i(n1)) * lm_exp2i(n2);
}

// ---- log ---------------------------------------------------------------------
#define LM_SQRT2 1.4142135381698608398e+00f
#define LM_L1 6.6666668653488159180e-01f   /* 2/3  */
#define LM_L2 4.0000000596046447754e-01f   /* 2/5  */
#define LM_L3 2.8571429848670959473e-01f   /* 2/7  */
#define LM_L4 2.2222222387790679932e-01f   /* 2/9  */
#define LM_L5 1.8181818723678588867e-01f   /* 2/11 */
#define LM_L6 1.5384615957736968994e-01f   /* 2/13 */

LM_HD float lm_logf(float x) {
    if (x != x) return x;
    if (x <= 0.0f) return x == 0.0f ? -lm_u2f(0x7f800000u) : lm_u2f(0x7fc00000u);
    if (lm_f2u(x) == 0x7f800000u) return x;
    int e = 0;
    if (x < 1.17549435e-38f) {                  // subnormal: scale by 2^24
        x = x * 16777216.0f;
        e = -24;
    }
    uint32_t u = lm_f2u(x);
    e += (int)((u >> 23) & 0xffu) - 127;
    float m = lm_u2f((u & 0x007fffffu) | 0x3f800000u);   // [1, 2)
    if (m > LM_SQRT2) { m = m * 0.5f; e += 1; }
    float f = m - 1.0f;
    float s = f / (2.0f + f);
    float z = s * s;
    float p = lm_fma(z, LM_L6, LM_L5);
    p = lm_fma(z, p, LM_L4);
    p = lm_fma(z, p, LM_L3);
    p = lm_fma(z, p, LM_L2);
    p = lm_fma(z, p, LM_L1);
    // log(m) = 2s + s*z*p  with f = 2s + s*f - ... rearranged as f - s*(f - z*p)
    float logm = lm_fma(s, lm_fma(z, p, -f), f);
    float fe = (float)e;
    return lm_fma(fe, LM_LN2_HI, lm_fma(fe, LM_LN2_LO, logm));
}

LM_HD float lm_pow5(float x) {
    float x2 = x * x;
    return (x2 * x2) * x;
}

}  // namespace lucid_math
