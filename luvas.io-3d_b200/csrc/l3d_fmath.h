/*
 * Deterministic scalar math shared by the CUDA kernels and by host code.
 *
 * PatchMatch is chaotic: a one-ulp difference in a bilateral weight or a random normal flips an
 * argmin and the flip propagates through the red/black sweeps.  Bit-exact agreement between the
 * GPU path and a CPU restatement therefore needs every transcendental to be computed by the same
 * sequence of correctly rounded IEEE operations on both sides.  This header provides them:
 *
 *   l3d_expf      exp(x) by Cody & Waite argument reduction (x = k ln2 + r, |r| <= ln2/2,
 *                 ln2 split as 355/512 - 2.121944400546905828e-4, the split published in
 *                 Cody & Waite, "Software Manual for the Elementary Functions", 1980) and a
 *                 degree-7 Taylor polynomial of exp(r) in Horner form.  Error < 2 ulp.
 *   l3d_sincosf   sin and cos for |a| < 2^15 by reduction modulo pi/2 with a two-part pi/2
 *                 (its f32 rounding plus the f32 rounding of the remainder) and Taylor
 *                 polynomials of degree 9 (sin) and 10 (cos) on |r| <= pi/4.  Error < 2 ulp
 *                 for the argument range used here ([0, 2 pi)).
 *   l3d_f32_to_f16 / l3d_f16_to_f32
 *                 IEEE binary16 conversions, round to nearest even (the WGSL pack2x16float
 *                 contract), written with integer operations only.
 *   l3d_pcg       the PCG-style 32-bit hash used as counter-based RNG
 *                 (frontend/src/app/vision/mvs/patchmatch.wgsl.ts:56-60).
 *
 * Every fused multiply-add is written explicitly (fmaf); the code that includes this header is
 * compiled without implicit contraction (nvcc --fmad=false, g++ -ffp-contract=off) so that a*b+c
 * written without fmaf rounds twice on both sides.  Division and sqrtf are the IEEE correctly
 * rounded operations on both sides (nvcc default -prec-div=true -prec-sqrt=true, SSE on x86-64).
 */
#ifndef L3D_FMATH_H
#define L3D_FMATH_H

#include <stdint.h>
#include <math.h>
#include <string.h>

#ifdef __CUDACC__
#define L3D_HD __host__ __device__ __forceinline__
#else
#define L3D_HD static inline
#endif

L3D_HD uint32_t l3d_f2u(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

L3D_HD float l3d_u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

/* 2^k as a float for -126 <= k <= 127. */
L3D_HD float l3d_pow2i(int k) { return l3d_u2f((uint32_t)(k + 127) << 23); }

L3D_HD float l3d_expf(float x) {
    if (!(x == x)) return x;                       /* NaN */
    if (x > 88.7228394f) return l3d_u2f(0x7f800000u); /* +inf */
    if (x < -103.972084f) return 0.0f;             /* below half the smallest subnormal */
    const float log2e = 1.44269502f;               /* f32(1 / ln 2) */
    const float c1 = 0.693359375f;                 /* 355 / 512: exact, 9 significant bits */
    const float c2 = -2.12194440e-4f;              /* ln 2 - 355/512 */
    float k = rintf(x * log2e);
    float r = fmaf(k, -c1, x);
    r = fmaf(k, -c2, r);
    /* exp(r) = sum r^n / n!, n = 0..7 */
    float p = 1.98412701e-4f;                      /* 1/5040 */
    p = fmaf(p, r, 1.38888892e-3f);                /* 1/720 */
    p = fmaf(p, r, 8.33333377e-3f);                /* 1/120 */
    p = fmaf(p, r, 4.16666679e-2f);                /* 1/24 */
    p = fmaf(p, r, 1.66666672e-1f);                /* 1/6 */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    if (ki < -125) {                               /* subnormal result: scale in two steps */
        p = p * l3d_pow2i(ki + 64);                /* exact: ki + 64 >= -86 stays normal */
        return p * 5.42101086e-20f;                /* 2^-64: the one rounding */
    }
    if (ki > 127) return (p * 2.0f) * l3d_pow2i(ki - 1);
    return p * l3d_pow2i(ki);
}

/* sin(a) and cos(a); intended for |a| < 2^15 (the PatchMatch angles lie in [0, 2 pi)). */
L3D_HD void l3d_sincosf(float a, float* s, float* c) {
    const float two_over_pi = 0.636619747f;        /* f32(2 / pi) */
    const float pio2_hi = 1.57079637f;             /* f32(pi / 2) */
    const float pio2_lo = -4.37113883e-8f;         /* f32(pi / 2 - pio2_hi) */
    float k = rintf(a * two_over_pi);
    float r = fmaf(k, -pio2_hi, a);
    r = fmaf(k, -pio2_lo, r);
    float r2 = r * r;
    /* sin r = r + r^3 (-1/6 + r^2 (1/120 + r^2 (-1/5040 + r^2 / 362880))) */
    float ps = 2.75573188e-6f;                     /* 1/362880 */
    ps = fmaf(ps, r2, -1.98412701e-4f);            /* -1/5040 */
    ps = fmaf(ps, r2, 8.33333377e-3f);             /* 1/120 */
    ps = fmaf(ps, r2, -1.66666672e-1f);            /* -1/6 */
    float sr = fmaf(ps * r2, r, r);
    /* cos r = 1 + r^2 (-1/2 + r^2 (1/24 + r^2 (-1/720 + r^2 (1/40320 - r^2 / 3628800)))) */
    float pc = -2.75573188e-7f;                    /* -1/3628800 */
    pc = fmaf(pc, r2, 2.48015876e-5f);             /* 1/40320 */
    pc = fmaf(pc, r2, -1.38888892e-3f);            /* -1/720 */
    pc = fmaf(pc, r2, 4.16666679e-2f);             /* 1/24 */
    pc = fmaf(pc, r2, -0.5f);
    float cr = fmaf(pc, r2, 1.0f);
    int q = ((int)k) & 3;
    float so, co;
    if (q == 0) { so = sr; co = cr; }
    else if (q == 1) { so = cr; co = -sr; }
    else if (q == 2) { so = -sr; co = -cr; }
    else { so = -cr; co = sr; }
    *s = so;
    *c = co;
}

/* f32 -> IEEE binary16 bits, round to nearest even; overflow gives +-inf, NaN stays NaN. */
L3D_HD uint32_t l3d_f32_to_f16(float f) {
    uint32_t x = l3d_f2u(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u);
    if (ax >= 0x477ff000u) return sign | 0x7c00u;  /* rounds to >= 65520: overflow */
    if (ax < 0x38800000u) {                        /* below 2^-14: subnormal half or zero */
        if (ax < 0x33000000u) return sign;         /* < 2^-25: rounds to zero (ties included) */
        uint32_t e = ax >> 23;                     /* 102 .. 112 */
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        uint32_t shift = 126u - e;                 /* value = m * 2^(e-150); half ulp = 2^-24 */
        uint32_t h = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (h & 1u))) h += 1u;
        return sign | h;
    }
    uint32_t h = ((ax >> 13) - (112u << 10));      /* rebias exponent 127 -> 15 */
    uint32_t rem = ax & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;
    return sign | h;
}

/* IEEE binary16 bits -> f32 (exact). */
L3D_HD float l3d_f16_to_f32(uint32_t h) {
    uint32_t sign = (h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 31u;
    uint32_t m = h & 1023u;
    if (e == 0) {
        /* subnormal: m * 2^-24, exact in f32 */
        float v = (float)m * 5.96046448e-8f;
        return sign ? -v : v;
    }
    if (e == 31) return l3d_u2f(sign | 0x7f800000u | (m << 13));
    return l3d_u2f(sign | ((e + 112u) << 23) | (m << 13));
}

/* Counter-based hash used as RNG (patchmatch.wgsl.ts:56-60). */
L3D_HD uint32_t l3d_pcg(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

/* random() of patchmatch.wgsl.ts:62-65: advances the state, returns (rng >> 8) / 2^24. */
L3D_HD float l3d_random(uint32_t* rng) {
    *rng = l3d_pcg(*rng);
    return (float)(*rng >> 8u) * 5.96046448e-8f;  /* exact: 2^-24 */
}

#endif
