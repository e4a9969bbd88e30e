// Ewald real-space helpers shared by the pair and exclusion kernels.
#pragma once

// Approximate reciprocal square root and quotient of the special-function unit, flushing
// subnormal inputs to zero (the pair kernels only see normal operands: r^2 >= ~1e-2 for pairs
// that count, a denominator >= 1), which spares the subnormal rescaling of the non-flushing forms.
__device__ __forceinline__ float sb_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sb_fdiv(float a, float b) {
    float y;
    asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
    return y;
}

// G(z) = [erf(x) - 2x e^{-x^2}/sqrt(pi)] / x^3 with x = sqrt(z) = beta*r.
// Coulomb part of the pair force scalar:   qq * (1/r^3 - beta^3 G(beta^2 r^2))
// exclusion-correction force scalar:       qq * beta^3 G(beta^2 r^2)
// Rational (5,4) fit on z in [0, 9] (fit_ewald_rational.py): max |error| 3.3e-8 in FP64,
// 1.1e-7 in FP32 Horner evaluation; the denominator has no zero for z >= 0. Beyond z = 9
// (beta*r > 3) the exact expression is used.
__device__ __forceinline__ float sb_ewald_G(float z) {
    if (z <= 9.0f) {
        float p = -1.034988821e-06f;
        p = fmaf(p, z, 5.361237187e-05f);
        p = fmaf(p, z, -1.155735711e-03f);
        p = fmaf(p, z, 1.953816643e-02f);
        p = fmaf(p, z, -8.191096247e-02f);
        p = fmaf(p, z, 7.522527569e-01f);
        float q = 7.681388070e-04f;
        q = fmaf(q, z, 1.258269309e-02f);
        q = fmaf(q, z, 1.063599183e-01f);
        q = fmaf(q, z, 4.911114809e-01f);
        q = fmaf(q, z, 1.0f);
        return __fdividef(p, q);
    }
    float x = sqrtf(z);
    return (erff(x) - 1.1283791670955126f * x * expf(-z)) / (z * x);
}

// The numerator coefficients of G, in Horner order (highest degree first).
#define SB_EWALD_P5 -1.034988821e-06
#define SB_EWALD_P4 5.361237187e-05
#define SB_EWALD_P3 -1.155735711e-03
#define SB_EWALD_P2 1.953816643e-02
#define SB_EWALD_P1 -8.191096247e-02
#define SB_EWALD_P0 7.522527569e-01

// beta^3 G(z) by the rational alone, no branch: valid for z <= 9. The pair kernel uses it when
// (beta rc)^2 <= 8.9 (an Ewald tolerance of 1e-5 gives beta rc near 2.8), where in-cutoff pairs
// never leave the fitted range and out-of-range values only reach pairs that are discarded.
__device__ __forceinline__ float sb_ewald_G_rational(float z, const float* gp) {
    float p = gp[0];
    p = fmaf(p, z, gp[1]);
    p = fmaf(p, z, gp[2]);
    p = fmaf(p, z, gp[3]);
    p = fmaf(p, z, gp[4]);
    p = fmaf(p, z, gp[5]);
    float q = 7.681388070e-04f;
    q = fmaf(q, z, 1.258269309e-02f);
    q = fmaf(q, z, 1.063599183e-01f);
    q = fmaf(q, z, 4.911114809e-01f);
    q = fmaf(q, z, 1.0f);
    return sb_fdiv(p, q);
}

// beta^3 G(z) with the numerator coefficients pre-multiplied by beta^3 (gp[0] = beta^3 P5 ...
// gp[5] = beta^3 P0, filled on the host), one multiply fewer per pair.
__device__ __forceinline__ float sb_ewald_G_scaled(float z, const float* gp) {
    if (z <= 9.0f) {
        float p = gp[0];
        p = fmaf(p, z, gp[1]);
        p = fmaf(p, z, gp[2]);
        p = fmaf(p, z, gp[3]);
        p = fmaf(p, z, gp[4]);
        p = fmaf(p, z, gp[5]);
        float q = 7.681388070e-04f;
        q = fmaf(q, z, 1.258269309e-02f);
        q = fmaf(q, z, 1.063599183e-01f);
        q = fmaf(q, z, 4.911114809e-01f);
        q = fmaf(q, z, 1.0f);
        return __fdividef(p, q);
    }
    // beta^3 = gp[5] / P0
    return (gp[5] * (float)(1.0 / SB_EWALD_P0)) * sb_ewald_G(z);
}
