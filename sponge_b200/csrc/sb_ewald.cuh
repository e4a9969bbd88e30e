// Ewald real-space helpers shared by the pair and exclusion kernels.
#pragma once

// G(z) = [erf(x) - 2x e^{-x^2}/sqrt(pi)] / x^3 with x = sqrt(z) = beta*r.
// Coulomb part of the pair force scalar:   qq * (1/r^3 - beta^3 G(beta^2 r^2))
// exclusion-correction force scalar:       qq * beta^3 G(beta^2 r^2)
// Rational (5,5) fit on z in [0, 12] (fit_ewald_rational.py): max |error| 1.5e-8 in FP64,
// ~1.1e-7 in FP32 Horner evaluation. Beyond z = 12 (beta*r > 3.46) the exact expression is used.
__device__ __forceinline__ float sb_ewald_G(float z) {
    if (z <= 12.0f) {
        float p = -4.234642899e-07f;
        p = fmaf(p, z, 3.557744695e-05f);
        p = fmaf(p, z, -2.489903094e-05f);
        p = fmaf(p, z, 1.708683818e-02f);
        p = fmaf(p, z, -2.884509870e-02f);
        p = fmaf(p, z, 7.522527883e-01f);
        float q = 1.255407394e-04f;
        q = fmaf(q, z, 2.169710712e-03f);
        q = fmaf(q, z, 2.242775561e-02f);
        q = fmaf(q, z, 1.454184461e-01f);
        q = fmaf(q, z, 5.616555609e-01f);
        q = fmaf(q, z, 1.0f);
        return __fdividef(p, q);
    }
    float x = sqrtf(z);
    return (erff(x) - 1.1283791670955126f * x * expf(-z)) / (z * x);
}
