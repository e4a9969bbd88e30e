// 4th-order cardinal B-spline stencil of smooth PME (PME_force.cu:8-14, :367-421).
//
// Grid coordinate u = uint * K / 2^32 taken from an exact 64-bit product: base = floor(u),
// fr = u - base. Grid point (base - k) mod K carries weight w_k(fr), k = 0..3.
#pragma once

#include <stdint.h>

__device__ __forceinline__ void sb_grid_coord(uint32_t u, int K, int& base, float& fr) {
    const unsigned long long p = (unsigned long long)u * (unsigned)K;
    base = (int)(p >> 32);
    fr = (float)(uint32_t)(p & 0xffffffffull) * 2.3283064365386963e-10f;
}

// weights w_k(f)
__device__ __forceinline__ void sb_bspline4(float f, float w[4]) {
    const float f2 = f * f, f3 = f2 * f;
    w[0] = f3 * (1.0f / 6.0f);
    w[1] = -0.5f * f3 + 0.5f * f2 + 0.5f * f + (1.0f / 6.0f);
    w[2] = 0.5f * f3 - f2 + (2.0f / 3.0f);
    w[3] = -f3 * (1.0f / 6.0f) + 0.5f * f2 - 0.5f * f + (1.0f / 6.0f);
}

// first derivatives dw_k/df
__device__ __forceinline__ void sb_bspline4d(float f, float d[4]) {
    const float f2 = f * f;
    d[0] = 0.5f * f2;
    d[1] = -1.5f * f2 + f + 0.5f;
    d[2] = 1.5f * f2 - 2.0f * f;
    d[3] = -0.5f * f2 + f - 0.5f;
}

// second derivatives d2w_k/df2 (they sum to zero for every f)
__device__ __forceinline__ void sb_bspline4dd(float f, float h[4]) {
    h[0] = f;
    h[1] = 1.0f - 3.0f * f;
    h[2] = 3.0f * f - 2.0f;
    h[3] = 1.0f - f;
}
