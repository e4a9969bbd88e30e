// Adjoint of the nonbonded energy and forces for force-field fitting.
//
// For a loss L(E, F) of the nonbonded potential energy E (LJ + long-range correction + Ewald
// direct + exclusion correction + self + reciprocal, as the forward modules compute it) and
// the forces F = -dE/dx, the caller supplies gE = dL/dE and gF = dL/dF. This file computes
//     dL/dp = gE dE/dp + sum_i gF_i . dF_i/dp
// for p = positions, per-atom charges and the LJ pair tables A12, B6 (the forms the LJ module
// stores, Lennard_Jones_force.cu:1092-1098), i.e. the Jacobian-vector product of the force
// field with the loss cotangents. Per-type sigma/epsilon gradients follow from the table
// gradients by the mixing rule, on the caller's side.
//
// Pair terms. For a pair (i, j) with d = x_i - x_j, r = |d|, potential U(r) and the force
// factor f = -U'(r)/r (F_i = f d), with w = gF_i - gF_j:
//     dL/dx_i = f (w - gE d) + (f'(r)/r) (w.d) d,      dL/dx_j = -dL/dx_i
// and for every parameter c that U is linear in (qq for Coulomb, A12 and B6 for LJ), with
// per-unit potential u_c and force factor a_c:  dL/dc = gE u_c + a_c (w.d).
// The pair pass walks the cluster pair list of the forward force kernel; the exclusion pass
// walks the exclusion CSR in FP64.
//
// Reciprocal space. With Q = sum_i q_i W_i (the spread charge grid), theta = G * Q (the
// convolved grid the forward gather reads, E_rec = 1/2 <Q, theta>), and P = sum_i q_i
// gF_i . grad W_i (the force cotangent spread with the spline gradients), Psi = G * P:
//     dL/dx_j = gE q_j grad phi_j - q_j (Hess phi_j gF_j + grad psi_j)
//     dL/dq_j = gE phi_j - gF_j . grad phi_j - psi_j
// where phi_j, psi_j interpolate theta and Psi at atom j. The charge grid is recomputed
// rather than stored; P is spread into the same int64 fixed-point grid after scaling the
// cotangents by 1 / max|gF| (the result is scaled back in the gather), so both convolutions
// run through the forward's FFT and Green's-function table.

#include <math.h>

#include <vector>

#include "sb_bspline.cuh"
#include "sb_internal.cuh"

struct sb_adjoint {
    int n = 0;
    int nt = 0;
    int K[3] = {0, 0, 0};
    size_t G = 0;
    float* d_theta_q = nullptr;  // [G] convolved charge grid
    float4* d_gfs = nullptr;     // [slot_cap] force cotangents in slot order
    int slot_cap = 0;
    double* d_cnt = nullptr;     // [nt] atoms per LJ type
    float* d_scale = nullptr;    // [1] max |gF|
    double* d_qsum = nullptr;    // [1] sum of charges
};

#define SB_ADJ_WARPS 4
#define SB_ADJ_TAB_MAX 48  // LJ types up to which the table gradient is staged in shared memory

struct AdjPairParams {
    float sx, sy, sz;  // fixed-point to A
    float rc2;
    float beta, beta2, two_beta_sqrtpi;
    int nt;
    int ent_cap;
    int tab_smem;
};

__global__ void k_adj_prep(int n, const float* __restrict__ gF, const float* __restrict__ q,
                           float* __restrict__ scale, double* __restrict__ qsum) {
    __shared__ float sm[1024];
    __shared__ double sq[1024];
    float m = 0.f;
    double s = 0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) m = fmaxf(m, fabsf(gF[i]));
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += (double)q[i];
    sm[threadIdx.x] = m;
    sq[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sm[threadIdx.x] = fmaxf(sm[threadIdx.x], sm[threadIdx.x + o]);
            sq[threadIdx.x] += sq[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scale[0] = sm[0];
        qsum[0] = sq[0];
    }
}

__global__ void k_adj_pack(const int* __restrict__ meta, const int* __restrict__ slot_atom,
                           const float* __restrict__ gF, float4* __restrict__ gfs) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= meta[3]) return;
    const int a = slot_atom[s];
    gfs[s] = a >= 0 ? make_float4(gF[3 * a], gF[3 * a + 1], gF[3 * a + 2], 0.f)
                    : make_float4(0.f, 0.f, 0.f, 0.f);
}

// warp per cluster over the forward's cluster pair list (entries j | imask << 24)
__global__ void __launch_bounds__(32 * SB_ADJ_WARPS) k_adj_pair(
    AdjPairParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const float4* __restrict__ gfs,
    const float2* __restrict__ AB, const int* __restrict__ slot_atom, float gE,
    double* __restrict__ gx, double* __restrict__ gq, double* __restrict__ gtab) {
    extern __shared__ float s_tab[];  // [2][nt][nt] when P.tab_smem
    __shared__ uint4 s_x[SB_ADJ_WARPS][SB_CLUSTER];
    __shared__ float4 s_g[SB_ADJ_WARPS][SB_CLUSTER];
    __shared__ int s_t[SB_ADJ_WARPS][SB_CLUSTER];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nt2 = P.nt * P.nt;
    if (P.tab_smem) {
        for (int t = threadIdx.x; t < 2 * nt2; t += blockDim.x) s_tab[t] = 0.f;
        __syncthreads();
    }
    const int nclu = meta[0];
    for (int c = blockIdx.x * SB_ADJ_WARPS + warp; c < nclu; c += gridDim.x * SB_ADJ_WARPS) {
        const int base = c * SB_CLUSTER;
        if (lane < SB_CLUSTER) {
            s_x[warp][lane] = xq[base + lane];
            s_g[warp][lane] = gfs[base + lane];
            s_t[warp][lane] = stype[base + lane];
        }
        __syncwarp();
        float gi[SB_CLUSTER][4];
#pragma unroll
        for (int k = 0; k < SB_CLUSTER; k++) gi[k][0] = gi[k][1] = gi[k][2] = gi[k][3] = 0.f;
        const uint32_t* __restrict__ ents = cl_ent + (size_t)c * P.ent_cap;
        const int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, P.ent_cap);
        for (int t = lane; t < cnt; t += 32) {
            const uint32_t v = ents[t];
            const int j = (int)(v & 0xffffffu);
            const uint32_t mask = v >> 24;
            const uint4 xj = xq[j];
            const float4 gj = gfs[j];
            const int tj = stype[j];
            const float qj = __uint_as_float(xj.w);
            float aj0 = 0.f, aj1 = 0.f, aj2 = 0.f, aj3 = 0.f;
#pragma unroll
            for (int k = 0; k < SB_CLUSTER; k++) {
                if (!((mask >> k) & 1u)) continue;
                const uint4 xi = s_x[warp][k];
                const float dx = __int2float_rn((int)(xi.x - xj.x)) * P.sx;
                const float dy = __int2float_rn((int)(xi.y - xj.y)) * P.sy;
                const float dz = __int2float_rn((int)(xi.z - xj.z)) * P.sz;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                if (!(r2 < P.rc2)) continue;
                const float4 g_i = s_g[warp][k];
                const int ti = s_t[warp][k];
                const float qi = __uint_as_float(xi.w);
                const float wx = g_i.x - gj.x, wy = g_i.y - gj.y, wz = g_i.z - gj.z;
                const float wd = fmaf(wx, dx, fmaf(wy, dy, wz * dz));
                const float ri2 = 1.0f / r2;
                const float r = sqrtf(r2);
                const float ri = r * ri2;
                // LJ: u_A = r^-12/12, a_A = r^-14, b_A = -14 r^-16; u_B = -r^-6/6, a_B = -r^-8,
                // b_B = 8 r^-10
                const float ri6 = ri2 * ri2 * ri2;
                const float uA = ri6 * ri6 * (1.0f / 12.0f), uB = ri6 * (-1.0f / 6.0f);
                const float aA = ri6 * ri6 * ri2, aB = -ri6 * ri2;
                const float bA = -14.0f * aA * ri2, bB = -8.0f * aB * ri2;
                const float2 ab = AB[ti * P.nt + tj];
                // Ewald direct: u = erfc(br)/r, a = (u + g)/r^2, b = -(3a + 2 beta^2 g)/r^2,
                // g = 2 beta/sqrt(pi) exp(-beta^2 r^2)
                const float br = P.beta * r;
                const float g = P.two_beta_sqrtpi * expf(-br * br);
                const float uc = erfcf(br) * ri;
                const float ac = (uc + g) * ri2;
                const float bc = -(3.0f * ac + 2.0f * P.beta2 * g) * ri2;
                const float qq = qi * qj;
                const float f = ab.x * aA + ab.y * aB + qq * ac;
                const float fb = ab.x * bA + ab.y * bB + qq * bc;
                const float s2 = fb * wd;
                const float px = f * (wx - gE * dx) + s2 * dx;
                const float py = f * (wy - gE * dy) + s2 * dy;
                const float pz = f * (wz - gE * dz) + s2 * dz;
                const float hq = gE * uc + ac * wd;
                gi[k][0] += px;
                gi[k][1] += py;
                gi[k][2] += pz;
                gi[k][3] += qj * hq;
                aj0 -= px;
                aj1 -= py;
                aj2 -= pz;
                aj3 += qi * hq;
                const float dA = gE * uA + aA * wd, dB = gE * uB + aB * wd;
                const int tix = ti * P.nt + tj;
                if (P.tab_smem) {
                    atomicAdd(&s_tab[tix], dA);
                    atomicAdd(&s_tab[nt2 + tix], dB);
                } else {
                    atomicAdd(&gtab[tix], (double)dA);
                    atomicAdd(&gtab[nt2 + tix], (double)dB);
                }
            }
            const int a = slot_atom[j];
            if (a >= 0 && (aj0 != 0.f || aj1 != 0.f || aj2 != 0.f || aj3 != 0.f)) {
                atomicAdd(&gx[3 * a], (double)aj0);
                atomicAdd(&gx[3 * a + 1], (double)aj1);
                atomicAdd(&gx[3 * a + 2], (double)aj2);
                atomicAdd(&gq[a], (double)aj3);
            }
        }
#pragma unroll
        for (int k = 0; k < SB_CLUSTER; k++) {
#pragma unroll
            for (int m = 0; m < 4; m++) {
                float v = gi[k][m];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                gi[k][m] = v;
            }
            if (lane == k) {
                const int a = slot_atom[base + k];
                if (a >= 0) {
                    atomicAdd(&gx[3 * a], (double)gi[k][0]);
                    atomicAdd(&gx[3 * a + 1], (double)gi[k][1]);
                    atomicAdd(&gx[3 * a + 2], (double)gi[k][2]);
                    atomicAdd(&gq[a], (double)gi[k][3]);
                }
            }
        }
        __syncwarp();
    }
    if (P.tab_smem) {
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * nt2; t += blockDim.x)
            if (s_tab[t] != 0.f) atomicAdd(&gtab[t], (double)s_tab[t]);
    }
}

// exclusion correction pairs in FP64: U = -qq erf(beta r)/r (PME_force.cu:620-695)
__global__ void k_adj_excluded(int n, const uint32_t* __restrict__ uc, double sx, double sy,
                               double sz, const float* __restrict__ q, double beta,
                               const int* __restrict__ es, const int* __restrict__ el,
                               const int* __restrict__ en, const float* __restrict__ gF,
                               double gE, double* __restrict__ gx, double* __restrict__ gq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cnt = en[i];
    if (cnt <= 0) return;
    const int s0 = es[i];
    const double qi = q[i];
    const double gix = gF[3 * i], giy = gF[3 * i + 1], giz = gF[3 * i + 2];
    const double tbs = 2.0 * beta / sqrt(M_PI);
    double ax = 0, ay = 0, az = 0, aq = 0;
    for (int k = s0; k < s0 + cnt; k++) {
        const int j = el[k];
        const double dx = (double)(int)(uc[3 * i] - uc[3 * j]) * sx;
        const double dy = (double)(int)(uc[3 * i + 1] - uc[3 * j + 1]) * sy;
        const double dz = (double)(int)(uc[3 * i + 2] - uc[3 * j + 2]) * sz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double r = sqrt(r2);
        const double qj = q[j];
        const double qq = qi * qj;
        const double er = erf(beta * r);
        const double g = tbs * exp(-beta * beta * r2);
        const double u = -er / r;
        const double a = (g * r - er) / (r2 * r);
        const double b = -(3.0 * a + 2.0 * beta * beta * g) / r2;
        const double wx = gix - gF[3 * j], wy = giy - gF[3 * j + 1], wz = giz - gF[3 * j + 2];
        const double wd = wx * dx + wy * dy + wz * dz;
        const double f = qq * a, fb = qq * b;
        const double px = f * (wx - gE * dx) + fb * wd * dx;
        const double py = f * (wy - gE * dy) + fb * wd * dy;
        const double pz = f * (wz - gE * dz) + fb * wd * dz;
        const double hq = gE * u + a * wd;
        ax += px;
        ay += py;
        az += pz;
        aq += qj * hq;
        atomicAdd(&gx[3 * j], -px);
        atomicAdd(&gx[3 * j + 1], -py);
        atomicAdd(&gx[3 * j + 2], -pz);
        atomicAdd(&gq[j], qi * hq);
    }
    atomicAdd(&gx[3 * i], ax);
    atomicAdd(&gx[3 * i + 1], ay);
    atomicAdd(&gx[3 * i + 2], az);
    atomicAdd(&gq[i], aq);
}

// charge spread (as the forward's fixed-point spread): 4 threads per atom, thread = x offset
__global__ void k_adj_spread_q(int n, const uint32_t* __restrict__ uc, const float* __restrict__ q,
                               int K0, int K1, int K2, long long* __restrict__ gfix) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt >> 2, kx = gt & 3;
    if (i >= n) return;
    int b0, b1, b2;
    float f0, f1, f2;
    sb_grid_coord(uc[3 * i], K0, b0, f0);
    sb_grid_coord(uc[3 * i + 1], K1, b1, f1);
    sb_grid_coord(uc[3 * i + 2], K2, b2, f2);
    float wx[4], wy[4], wz[4];
    sb_bspline4(f0, wx);
    sb_bspline4(f1, wy);
    sb_bspline4(f2, wz);
    const float qw = q[i] * wx[kx];
    int gx = b0 - kx;
    if (gx < 0) gx += K0;
#pragma unroll
    for (int ky = 0; ky < 4; ky++) {
        int gy = b1 - ky;
        if (gy < 0) gy += K1;
        const size_t row = ((size_t)gx * K1 + gy) * K2;
#pragma unroll
        for (int kz = 0; kz < 4; kz++) {
            int gz = b2 - kz;
            if (gz < 0) gz += K2;
            const long long f = __float2ll_rn(qw * wy[ky] * wz[kz] * SB_GRID_SCALE);
            if (f) sb_red_add(&gfix[row + gz], f);
        }
    }
}

// P / max|gF|: q_i (gF_i / s) . grad W_i spread into the fixed-point grid
__global__ void k_adj_spread_p(int n, const uint32_t* __restrict__ uc, const float* __restrict__ q,
                               const float* __restrict__ gF, const float* __restrict__ scale,
                               int K0, int K1, int K2, float ix, float iy, float iz,
                               long long* __restrict__ gfix) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gt >> 2, kx = gt & 3;
    if (i >= n) return;
    const float s = scale[0];
    if (!(s > 0.f)) return;
    const float inv = 1.0f / s;
    const float qi = q[i];
    const float gxs = qi * gF[3 * i] * inv * ix;
    const float gys = qi * gF[3 * i + 1] * inv * iy;
    const float gzs = qi * gF[3 * i + 2] * inv * iz;
    int b0, b1, b2;
    float f0, f1, f2;
    sb_grid_coord(uc[3 * i], K0, b0, f0);
    sb_grid_coord(uc[3 * i + 1], K1, b1, f1);
    sb_grid_coord(uc[3 * i + 2], K2, b2, f2);
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    sb_bspline4(f0, wx);
    sb_bspline4(f1, wy);
    sb_bspline4(f2, wz);
    sb_bspline4d(f0, dx);
    sb_bspline4d(f1, dy);
    sb_bspline4d(f2, dz);
    int gx = b0 - kx;
    if (gx < 0) gx += K0;
    const float cx = gxs * dx[kx], cw = wx[kx];
#pragma unroll
    for (int ky = 0; ky < 4; ky++) {
        int gy = b1 - ky;
        if (gy < 0) gy += K1;
        const size_t row = ((size_t)gx * K1 + gy) * K2;
        const float a = cx * wy[ky] + gys * cw * dy[ky];
        const float b = gzs * cw * wy[ky];
#pragma unroll
        for (int kz = 0; kz < 4; kz++) {
            int gz = b2 - kz;
            if (gz < 0) gz += K2;
            const float v = a * wz[kz] + b * dz[kz];
            const long long f = __float2ll_rn(v * SB_GRID_SCALE);
            if (f) sb_red_add(&gfix[row + gz], f);
        }
    }
}

// reciprocal-space and self-energy terms; one thread per atom (runs after the pair passes)
__global__ void k_adj_gather(int n, const uint32_t* __restrict__ uc, const float* __restrict__ q,
                             const float* __restrict__ gF, const float* __restrict__ theta,
                             const float* __restrict__ psi_grid, const float* __restrict__ scale,
                             const double* __restrict__ qsum, int K0, int K1, int K2, float ix,
                             float iy, float iz, double gE, double self_q, double neutral2,
                             double* __restrict__ gx, double* __restrict__ gq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b0, b1, b2;
    float f0, f1, f2;
    sb_grid_coord(uc[3 * i], K0, b0, f0);
    sb_grid_coord(uc[3 * i + 1], K1, b1, f1);
    sb_grid_coord(uc[3 * i + 2], K2, b2, f2);
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4], hx[4], hy[4], hz[4];
    sb_bspline4(f0, wx);
    sb_bspline4(f1, wy);
    sb_bspline4(f2, wz);
    sb_bspline4d(f0, dx);
    sb_bspline4d(f1, dy);
    sb_bspline4d(f2, dz);
    sb_bspline4dd(f0, hx);
    sb_bspline4dd(f1, hy);
    sb_bspline4dd(f2, hz);
    int gz[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int g = b2 - k;
        gz[k] = g < 0 ? g + K2 : g;
    }
    float phi = 0.f, px = 0.f, py = 0.f, pz = 0.f;
    float hxx = 0.f, hyy = 0.f, hzz = 0.f, hxy = 0.f, hxz = 0.f, hyz = 0.f;
    float ps = 0.f, sxg = 0.f, syg = 0.f, szg = 0.f;
#pragma unroll
    for (int kx = 0; kx < 4; kx++) {
        int gxi = b0 - kx;
        if (gxi < 0) gxi += K0;
#pragma unroll
        for (int ky = 0; ky < 4; ky++) {
            int gyi = b1 - ky;
            if (gyi < 0) gyi += K1;
            const size_t row = ((size_t)gxi * K1 + gyi) * K2;
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, t0 = 0.f, t1 = 0.f;
#pragma unroll
            for (int kz = 0; kz < 4; kz++) {
                const float th = theta[row + gz[kz]];
                const float pg = psi_grid[row + gz[kz]];
                s0 = fmaf(th, wz[kz], s0);
                s1 = fmaf(th, dz[kz], s1);
                s2 = fmaf(th, hz[kz], s2);
                t0 = fmaf(pg, wz[kz], t0);
                t1 = fmaf(pg, dz[kz], t1);
            }
            const float ww = wx[kx] * wy[ky], dw = dx[kx] * wy[ky], wd = wx[kx] * dy[ky];
            phi = fmaf(ww, s0, phi);
            px = fmaf(dw, s0, px);
            py = fmaf(wd, s0, py);
            pz = fmaf(ww, s1, pz);
            hxx = fmaf(hx[kx] * wy[ky], s0, hxx);
            hyy = fmaf(wx[kx] * hy[ky], s0, hyy);
            hzz = fmaf(ww, s2, hzz);
            hxy = fmaf(dx[kx] * dy[ky], s0, hxy);
            hxz = fmaf(dw, s1, hxz);
            hyz = fmaf(wd, s1, hyz);
            ps = fmaf(ww, t0, ps);
            sxg = fmaf(dw, t0, sxg);
            syg = fmaf(wd, t0, syg);
            szg = fmaf(ww, t1, szg);
        }
    }
    const double s = scale[0] > 0.f ? (double)scale[0] : 0.0;
    const double qi = q[i];
    const double Gx = gF[3 * i], Gy = gF[3 * i + 1], Gz = gF[3 * i + 2];
    const double ex = (double)px * ix, ey = (double)py * iy, ez = (double)pz * iz;
    const double Hxx = (double)hxx * ix * ix, Hyy = (double)hyy * iy * iy,
                 Hzz = (double)hzz * iz * iz;
    const double Hxy = (double)hxy * ix * iy, Hxz = (double)hxz * ix * iz,
                 Hyz = (double)hyz * iy * iz;
    const double psi = s * ps;
    const double qx = s * sxg * ix, qy = s * syg * iy, qz = s * szg * iz;
    gx[3 * i] += gE * qi * ex - qi * (Hxx * Gx + Hxy * Gy + Hxz * Gz + qx);
    gx[3 * i + 1] += gE * qi * ey - qi * (Hxy * Gx + Hyy * Gy + Hyz * Gz + qy);
    gx[3 * i + 2] += gE * qi * ez - qi * (Hxz * Gx + Hyz * Gy + Hzz * Gz + qz);
    gq[i] += gE * (double)phi - (Gx * ex + Gy * ey + Gz * ez) - psi +
             gE * (self_q * qi + neutral2 * qsum[0]);
}

// long-range correction E = factor / V, factor = kappa sum_ab cnt_a cnt_b B6_ab
__global__ void k_adj_lrc(int nt, const double* __restrict__ cnt, double coef,
                          double* __restrict__ gtab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt * nt) return;
    const int a = t / nt, b = t - a * nt;
    gtab[nt * nt + t] += coef * cnt[a] * cnt[b];
}

// ---------------------------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------------------------

// parameter update for fitting: new lower-triangular A12/B6 tables into the LJ module's device
// tables (lower-triangular and full square) and its FP64 long-range correction factor
extern "C" int sb_lj_set_tables(sb_lennard_jones* lj, const float* h_A, const float* h_B) {
    if (!lj || !h_A || !h_B) {
        sb_set_error("sb_lj_set_tables: null argument");
        return SB_ERR_ARG;
    }
    const int nt = lj->ntypes, n = lj->n;
    const int np = nt * (nt + 1) / 2;
    std::vector<float2> ab((size_t)nt * nt);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            const int M = a > b ? a : b, m = a > b ? b : a;
            const int k = M * (M + 1) / 2 + m;
            ab[(size_t)a * nt + b] = make_float2(h_A[k], h_B[k]);
        }
    std::vector<int> types(n);
    SB_CHECK_CUDA(cudaMemcpy(types.data(), lj->d_type, sizeof(int) * n, cudaMemcpyDeviceToHost));
    std::vector<double> cnt(nt, 0.0);
    for (int t : types) cnt[t] += 1.0;
    double sumB = 0;
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) sumB += cnt[a] * cnt[b] * (double)ab[(size_t)a * nt + b].y;
    const double rc = lj->cutoff;
    SB_CHECK_CUDA(cudaMemcpy(lj->d_A, h_A, sizeof(float) * np, cudaMemcpyHostToDevice));
    SB_CHECK_CUDA(cudaMemcpy(lj->d_B, h_B, sizeof(float) * np, cudaMemcpyHostToDevice));
    SB_CHECK_CUDA(cudaMemcpy(lj->d_AB, ab.data(), sizeof(float2) * nt * nt,
                             cudaMemcpyHostToDevice));
    lj->long_range_factor = sumB * (-2.0 / 3.0 * M_PI / (rc * rc * rc) / 6.0);
    return SB_OK;
}

extern "C" int sb_adjoint_destroy(sb_adjoint* adj) {
    if (!adj) return SB_OK;
    cudaDeviceSynchronize();
    void* ps[] = {adj->d_theta_q, adj->d_gfs, adj->d_cnt, adj->d_scale, adj->d_qsum};
    for (void* p : ps) sb_free(p);
    delete adj;
    return SB_OK;
}

extern "C" int sb_adjoint_create(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                                 sb_adjoint** out) {
    if (!nl || !lj || !pme || !out) {
        sb_set_error("sb_adjoint_create: null argument");
        return SB_ERR_ARG;
    }
    if (nl->form != SB_FORM_FIXED || lj->form != SB_FORM_FIXED || pme->form != SB_FORM_FIXED) {
        sb_set_error("sb_adjoint_create: the adjoint needs the fixed-point form of all modules");
        return SB_ERR_ARG;
    }
    if (lj->n != nl->n || pme->n != nl->n) {
        sb_set_error("sb_adjoint_create: modules disagree on the atom count");
        return SB_ERR_ARG;
    }
    sb_adjoint* a = new sb_adjoint();
    a->n = nl->n;
    a->nt = lj->ntypes;
    for (int d = 0; d < 3; d++) a->K[d] = pme->K[d];
    a->G = pme->G;
    a->slot_cap = nl->slot_cap;
    int st = SB_OK;
    if ((st = sb_malloc((void**)&a->d_theta_q, sizeof(float) * a->G, "adjoint grid")) ||
        (st = sb_malloc((void**)&a->d_gfs, sizeof(float4) * a->slot_cap, "adjoint cotangents")) ||
        (st = sb_malloc((void**)&a->d_cnt, sizeof(double) * a->nt, "adjoint type counts")) ||
        (st = sb_malloc((void**)&a->d_scale, sizeof(float), "adjoint scale")) ||
        (st = sb_malloc((void**)&a->d_qsum, sizeof(double), "adjoint charge sum"))) {
        sb_adjoint_destroy(a);
        return st;
    }
    std::vector<int> types(a->n);
    std::vector<double> cnt(a->nt, 0.0);
    cudaError_t e = cudaMemcpy(types.data(), lj->d_type, sizeof(int) * a->n,
                               cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
        for (int t : types) cnt[t] += 1.0;
        e = cudaMemcpy(a->d_cnt, cnt.data(), sizeof(double) * a->nt, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        sb_set_error("sb_adjoint_create: %s", cudaGetErrorString(e));
        sb_adjoint_destroy(a);
        return SB_ERR_CUDA;
    }
    *out = a;
    return SB_OK;
}

extern "C" int sb_adjoint_backward(sb_adjoint* adj, sb_neighbor_list* nl, sb_lennard_jones* lj,
                                   sb_pme* pme, const uint32_t* d_uint_crd, const float* d_charge,
                                   const int* es, const int* el, const int* en,
                                   double grad_energy, const float* d_grad_frc,
                                   double* d_grad_crd, double* d_grad_charge,
                                   double* d_grad_lj, void* stream) {
    if (!adj || !nl || !lj || !pme || !d_uint_crd || !d_charge || !d_grad_frc || !d_grad_crd ||
        !d_grad_charge || !d_grad_lj) {
        sb_set_error("sb_adjoint_backward: null argument");
        return SB_ERR_ARG;
    }
    if (nl->n != adj->n || lj->n != adj->n || pme->n != adj->n || lj->ntypes != adj->nt ||
        nl->slot_cap != adj->slot_cap || pme->G != adj->G) {
        sb_set_error("sb_adjoint_backward: modules do not match the adjoint context");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    const int n = adj->n, nt = adj->nt;
    SB_CHECK_CUDA(cudaMemsetAsync(d_grad_crd, 0, sizeof(double) * 3 * n, s));
    SB_CHECK_CUDA(cudaMemsetAsync(d_grad_charge, 0, sizeof(double) * n, s));
    SB_CHECK_CUDA(cudaMemsetAsync(d_grad_lj, 0, sizeof(double) * 2 * nt * nt, s));
    k_adj_prep<<<1, 1024, 0, s>>>(n, d_grad_frc, d_charge, adj->d_scale, adj->d_qsum);
    SB_CHECK_LAUNCH();

    // pair terms over the cluster list
    SB_TRY(sb_nl_pack(nl, d_uint_crd, d_charge, lj->d_type, s));
    k_adj_pack<<<(nl->slot_cap + 255) / 256, 256, 0, s>>>(nl->meta, nl->slot_atom, d_grad_frc,
                                                          adj->d_gfs);
    SB_CHECK_LAUNCH();
    AdjPairParams P;
    P.sx = nl->box[0] * (1.0f / 4294967296.0f);
    P.sy = nl->box[1] * (1.0f / 4294967296.0f);
    P.sz = nl->box[2] * (1.0f / 4294967296.0f);
    P.rc2 = lj->cutoff * lj->cutoff;
    P.beta = pme->beta;
    P.beta2 = pme->beta * pme->beta;
    P.two_beta_sqrtpi = (float)(2.0 * pme->beta / sqrt(M_PI));
    P.nt = nt;
    P.ent_cap = nl->ent_cap;
    P.tab_smem = nt <= SB_ADJ_TAB_MAX;
    const size_t smem = P.tab_smem ? sizeof(float) * 2 * nt * nt : 0;
    const int want = (nl->clu_cap + SB_ADJ_WARPS - 1) / SB_ADJ_WARPS;
    const int blocks = want < 148 * 16 ? want : 148 * 16;
    k_adj_pair<<<blocks, 32 * SB_ADJ_WARPS, smem, s>>>(
        P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, adj->d_gfs, lj->d_AB,
        nl->slot_atom, (float)grad_energy, d_grad_crd, d_grad_charge, d_grad_lj);
    SB_CHECK_LAUNCH();
    if (es && el && en) {
        k_adj_excluded<<<(n + 127) / 128, 128, 0, s>>>(
            n, d_uint_crd, (double)pme->box[0] / 4294967296.0, (double)pme->box[1] / 4294967296.0,
            (double)pme->box[2] / 4294967296.0, d_charge, (double)pme->beta, es, el, en,
            d_grad_frc, grad_energy, d_grad_crd, d_grad_charge);
        SB_CHECK_LAUNCH();
    }

    // reciprocal space: theta = G * Q (recomputed), Psi = G * P
    const int K0 = adj->K[0], K1 = adj->K[1], K2 = adj->K[2];
    const float ix = (float)K0 / pme->box[0], iy = (float)K1 / pme->box[1],
                iz = (float)K2 / pme->box[2];
    int nparts = 0;
    k_adj_spread_q<<<(4 * n + 255) / 256, 256, 0, s>>>(n, d_uint_crd, d_charge, K0, K1, K2,
                                                       pme->d_qfix);
    SB_CHECK_LAUNCH();
    SB_TRY(sb_fft_plane_forward(&pme->plan, pme->d_qfix, pme->d_spec, s));
    SB_TRY(sb_fft_x_convolve(&pme->plan, pme->d_spec, pme->d_bc, pme->d_epart, 0, s, &nparts));
    SB_TRY(sb_fft_plane_inverse(&pme->plan, pme->d_spec, adj->d_theta_q, s));
    k_adj_spread_p<<<(4 * n + 255) / 256, 256, 0, s>>>(n, d_uint_crd, d_charge, d_grad_frc,
                                                       adj->d_scale, K0, K1, K2, ix, iy, iz,
                                                       pme->d_qfix);
    SB_CHECK_LAUNCH();
    SB_TRY(sb_fft_plane_forward(&pme->plan, pme->d_qfix, pme->d_spec, s));
    SB_TRY(sb_fft_x_convolve(&pme->plan, pme->d_spec, pme->d_bc, pme->d_epart, 0, s, &nparts));
    SB_TRY(sb_fft_plane_inverse(&pme->plan, pme->d_spec, pme->d_theta, s));
    // self energy -beta/sqrt(pi) sum q^2 + neutral (sum q)^2
    const double self_q = -2.0 * (double)pme->beta / sqrt(M_PI);
    const double neutral2 = 2.0 * pme->neutralizing_factor;
    k_adj_gather<<<(n + 127) / 128, 128, 0, s>>>(n, d_uint_crd, d_charge, d_grad_frc,
                                                 adj->d_theta_q, pme->d_theta, adj->d_scale,
                                                 adj->d_qsum, K0, K1, K2, ix, iy, iz,
                                                 grad_energy, self_q, neutral2, d_grad_crd,
                                                 d_grad_charge);
    SB_CHECK_LAUNCH();

    // long-range correction: factor = -(2 pi / 3) / rc^3 / 6 sum cnt_a cnt_b B6_ab, E = factor/V
    const double V = (double)lj->box[0] * lj->box[1] * lj->box[2];
    const double rc = lj->cutoff;
    const double coef = grad_energy * (-2.0 / 3.0 * M_PI / (rc * rc * rc) / 6.0) / V;
    k_adj_lrc<<<(nt * nt + 255) / 256, 256, 0, s>>>(nt, adj->d_cnt, coef, d_grad_lj);
    SB_CHECK_LAUNCH();
    return SB_OK;
}
