// PME reciprocal space and the Ewald exclusion correction — replaces Particle_Mesh_Ewald
// (SPONGE/PME_force/PME_force.cu).
//
// Grid convention (PME_force.cu:367-421): u = uint * K / 2^32, base = floor(u), fr = u - base;
// grid point (base - k) mod K receives weight w_k(fr), k = 0..3, with the 4th-order cardinal
// B-spline polynomials of PME_force.cu:8-14. Here base and fr come from an exact 64-bit
// integer product instead of the reference's FP32 product, so the stencil never flips at a
// rounding boundary.
//
// Chosen form: spread with int64 fixed-point atomics (order independent), the hand-written
// FFT + convolution of sb_fft.cu, gather with one thread per atom (one writer per atom).
// Plain form: float atomicAdd spread into a float grid, cuFFT R2C/C2R with a separate BC
// multiply, same gather.
// Energies (PME_force.cu:753-771) are reduced in FP64 in fixed order.

#include <cufft.h>
#include <stdio.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "sb_ewald.cuh"
#include "sb_internal.cuh"


__device__ __forceinline__ void grid_coord(uint32_t u, int K, int& base, float& fr) {
    const unsigned long long p = (unsigned long long)u * (unsigned)K;
    base = (int)(p >> 32);
    fr = (float)(uint32_t)(p & 0xffffffffull) * 2.3283064365386963e-10f;
}

__device__ __forceinline__ void bspline4(float f, float w[4]) {
    const float f2 = f * f, f3 = f2 * f;
    w[0] = f3 * (1.0f / 6.0f);
    w[1] = -0.5f * f3 + 0.5f * f2 + 0.5f * f + (1.0f / 6.0f);
    w[2] = 0.5f * f3 - f2 + (2.0f / 3.0f);
    w[3] = -f3 * (1.0f / 6.0f) + 0.5f * f2 - 0.5f * f + (1.0f / 6.0f);
}

__device__ __forceinline__ void bspline4d(float f, float d[4]) {
    const float f2 = f * f;
    d[0] = 0.5f * f2;
    d[1] = -1.5f * f2 + f + 0.5f;
    d[2] = 1.5f * f2 - 2.0f * f;
    d[3] = -0.5f * f2 + f - 0.5f;
}

// 4 threads per atom, one per z offset: the four lanes of an atom update adjacent words of one
// z row at each (x, y) offset. Grid-stride, so that the fused step can run it on a small grid
// beside the pair kernel.
template <bool FIXED>
__device__ __forceinline__ void spread_one(int gt, const uint32_t* __restrict__ uc,
                                           const float* __restrict__ q, int K0, int K1, int K2,
                                           long long* __restrict__ gfix, float* __restrict__ gf) {
    const int i = gt >> 2, kz = gt & 3;
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(uc[3 * i], K0, b0, f0);
    grid_coord(uc[3 * i + 1], K1, b1, f1);
    grid_coord(uc[3 * i + 2], K2, b2, f2);
    float wx[4], wy[4], wz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    const float qi = q[i];
    int gz = b2 - kz;
    if (gz < 0) gz += K2;
    const float wzk = kz == 0 ? wz[0] : kz == 1 ? wz[1] : kz == 2 ? wz[2] : wz[3];
#pragma unroll
    for (int kx = 0; kx < 4; kx++) {
        int gx = b0 - kx;
        if (gx < 0) gx += K0;
        const float qw = qi * wx[kx];
#pragma unroll
        for (int ky = 0; ky < 4; ky++) {
            int gy = b1 - ky;
            if (gy < 0) gy += K1;
            const size_t at = ((size_t)gx * K1 + gy) * K2 + gz;
            const float v = qw * wy[ky] * wzk;
            if (FIXED) {
                const long long f = __float2ll_rn(v * SB_GRID_SCALE);
                if (f) sb_red_add(&gfix[at], f);
            } else {
                atomicAdd(&gf[at], v);
            }
        }
    }
}

template <bool FIXED>
__global__ void k_spread(int n, const uint32_t* __restrict__ uc, const float* __restrict__ q,
                         int K0, int K1, int K2, long long* __restrict__ gfix,
                         float* __restrict__ gf) {
    for (int gt = blockIdx.x * blockDim.x + threadIdx.x; gt < 4 * n;
         gt += gridDim.x * blockDim.x)
        spread_one<FIXED>(gt, uc, q, K0, K1, K2, gfix, gf);
}

// force interpolation (PME_Final, PME_force.cu:485-550); one thread per atom, one writer
__global__ void k_gather(int n, const uint32_t* __restrict__ uc, const float* __restrict__ q,
                         const float* __restrict__ theta, int K0, int K1, int K2, float ix,
                         float iy, float iz, float* __restrict__ frc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(uc[3 * i], K0, b0, f0);
    grid_coord(uc[3 * i + 1], K1, b1, f1);
    grid_coord(uc[3 * i + 2], K2, b2, f2);
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    bspline4d(f0, dx);
    bspline4d(f1, dy);
    bspline4d(f2, dz);
    int gz[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int g = b2 - k;
        gz[k] = g < 0 ? g + K2 : g;
    }
    float Fx = 0.f, Fy = 0.f, Fz = 0.f;
#pragma unroll
    for (int kx = 0; kx < 4; kx++) {
        int gx = b0 - kx;
        if (gx < 0) gx += K0;
#pragma unroll
        for (int ky = 0; ky < 4; ky++) {
            int gy = b1 - ky;
            if (gy < 0) gy += K1;
            const float* row = theta + ((size_t)gx * K1 + gy) * K2;
            float sw = 0.f, sd = 0.f;
#pragma unroll
            for (int kz = 0; kz < 4; kz++) {
                const float t = row[gz[kz]];
                sw = fmaf(t, wz[kz], sw);
                sd = fmaf(t, dz[kz], sd);
            }
            Fx = fmaf(dx[kx] * wy[ky], sw, Fx);
            Fy = fmaf(wx[kx] * dy[ky], sw, Fy);
            Fz = fmaf(wx[kx] * wy[ky], sd, Fz);
        }
    }
    const float s = -q[i];
    frc[3 * i] += s * Fx * ix;
    frc[3 * i + 1] += s * Fy * iy;
    frc[3 * i + 2] += s * Fz * iz;
}

// plain form: FQ *= BC on the cuFFT half spectrum (PME_BCFQ, PME_force.cu:473-483)
__global__ void k_bcfq(size_t nh, float2* __restrict__ fq, const float* __restrict__ bc) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nh) {
        const float g = bc[i];
        float2 v = fq[i];
        fq[i] = make_float2(v.x * g, v.y * g);
    }
}

// plain form energy: 1/2 sum Q * theta over the real grid (PME_Energy_Product, :553-566)
__global__ void k_grid_dot(size_t G, const float* __restrict__ a, const float* __restrict__ b,
                           double* __restrict__ part) {
    __shared__ double red[256];
    double s = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < G;
         i += (size_t)gridDim.x * blockDim.x)
        s += (double)a[i] * (double)b[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = 0.5 * red[0];
}

// exclusion correction (PME_Excluded_Force_With_Atom_Energy_Correction, PME_force.cu:620-695)
template <bool FIXED>
__global__ void k_excluded(int n, const uint32_t* __restrict__ uc, float sx, float sy, float sz,
                           const float* __restrict__ q, float beta, float beta2, float beta3,
                           const int* __restrict__ es, const int* __restrict__ el,
                           const int* __restrict__ en, long long* __restrict__ fix,
                           float* __restrict__ frc, float* __restrict__ ene) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cnt = en[i];
    if (cnt <= 0) return;
    const int s0 = es[i];
    const uint32_t ux = uc[3 * i], uy = uc[3 * i + 1], uz = uc[3 * i + 2];
    const float qi = q[i];
    float fx = 0.f, fy = 0.f, fz = 0.f, e = 0.f;
    for (int k = s0; k < s0 + cnt; k++) {
        const int j = el[k];
        const float dx = __int2float_rn((int)(uc[3 * j] - ux)) * sx;
        const float dy = __int2float_rn((int)(uc[3 * j + 1] - uy)) * sy;
        const float dz = __int2float_rn((int)(uc[3 * j + 2] - uz)) * sz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float r = sqrtf(r2);
        const float qq = qi * q[j];
        float fs;
        if (FIXED) {
            fs = qq * beta3 * sb_ewald_G(beta2 * r2);
        } else {
            const float br = beta * r;
            float t = br * 1.1283791670218446f * expf(-br * br) + erfcf(br);
            fs = -qq * (t - 1.0f) / r2 / r;
        }
        const float tx = fs * dx, ty = fs * dy, tz = fs * dz;
        fx += tx;
        fy += ty;
        fz += tz;
        e -= qq * erff(beta * r) / r;
        if (FIXED) {
            sb_red_add(&fix[3 * j], __float2ll_rn(-tx * SB_FORCE_SCALE));
            sb_red_add(&fix[3 * j + 1], __float2ll_rn(-ty * SB_FORCE_SCALE));
            sb_red_add(&fix[3 * j + 2], __float2ll_rn(-tz * SB_FORCE_SCALE));
        } else {
            atomicAdd(&frc[3 * j], -tx);
            atomicAdd(&frc[3 * j + 1], -ty);
            atomicAdd(&frc[3 * j + 2], -tz);
        }
    }
    if (FIXED) {
        sb_red_add(&fix[3 * i], __float2ll_rn(fx * SB_FORCE_SCALE));
        sb_red_add(&fix[3 * i + 1], __float2ll_rn(fy * SB_FORCE_SCALE));
        sb_red_add(&fix[3 * i + 2], __float2ll_rn(fz * SB_FORCE_SCALE));
    } else {
        atomicAdd(&frc[3 * i], fx);
        atomicAdd(&frc[3 * i + 1], fy);
        atomicAdd(&frc[3 * i + 2], fz);
    }
    if (ene) atomicAdd(&ene[i], e);
}

__global__ void k_fix_to_frc(int n, long long* __restrict__ fix, float* __restrict__ frc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    const long long v = fix[t];
    if (v) {
        fix[t] = 0;
        frc[t] += (float)((double)v * SB_FORCE_UNSCALE);
    }
}

__global__ void k_zero_f(int n, float* p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.f;
}

// FP64 fixed-order block reduction helper
__device__ double block_sum(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// ered: [0] reciprocal, [1] self (+neutralising), [2] direct, [3] correction
__global__ void __launch_bounds__(1024) k_pme_energy_finish(
    int n, const float* __restrict__ q, const double* __restrict__ epart, int nparts,
    const float* __restrict__ direct, const float* __restrict__ corr, double beta,
    double neutral, double* __restrict__ ered, int need_virial, int need_energy,
    float* __restrict__ d_virial, float* __restrict__ d_potential) {
    __shared__ double red[1024];
    double a = 0, b = 0, c = 0, d = 0, e = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double qi = q[i];
        a += qi * qi;
        b += qi;
        if (direct) c += direct[i];
        if (corr) d += corr[i];
    }
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) e += epart[p];
    const double s2 = block_sum(a, red);
    const double s1 = block_sum(b, red);
    const double sd = block_sum(c, red);
    const double sc = block_sum(d, red);
    const double er = block_sum(e, red);
    if (threadIdx.x == 0) {
        const double self = -beta / sqrt(M_PI) * s2 + neutral * s1 * s1;
        ered[0] = er;
        ered[1] = self;
        ered[2] = sd;
        ered[3] = sc;
        if (need_energy && d_potential) d_potential[0] += (float)(sc + self + er);
        if (need_virial && d_virial) d_virial[0] += (float)(sd + sc + self + er);
    }
}

// ---------------------------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------------------------
static int check_2357(int number) {
    const int primes[4] = {2, 3, 5, 7};
    for (int p : primes) {
        while (number > 0) {
            if (number == 1) return 1;
            int t = number / p;
            if (t * p != number) break;
            number = t;
        }
    }
    return number == 1;
}

// Get_Fft_Patameter (SPONGE/common.cu:513-534)
static int fft_size(float length) {
    int t = ((int)ceil(length + 3.0f)) >> 2 << 2;
    if (t >= 60 && t <= 68) t = 64;
    else if (t >= 120 && t <= 136) t = 128;
    else if (t >= 240 && t <= 272) t = 256;
    else if (t >= 480 && t <= 544) t = 512;
    else if (t >= 960 && t <= 1088) t = 1024;
    while (!check_2357(t)) t += 4;
    return t;
}

// Get_Beta (PME_force.cu:71-100) with the same float/double mix
static float get_beta(float cutoff, float tolerance) {
    float beta = 0, low, high, tempf;
    int ilow, ihigh;
    high = 1.0f;
    ihigh = 1;
    while (1) {
        float hc = high * cutoff;
        tempf = (float)(erfc((double)hc) / (double)cutoff);
        if (tempf <= tolerance) break;
        high *= 2;
        ihigh++;
    }
    ihigh += 50;
    low = 0.0f;
    for (ilow = 1; ilow < ihigh; ilow++) {
        beta = (low + high) / 2;
        float bc = beta * cutoff;
        tempf = (float)(erfc((double)bc) / (double)cutoff);
        if (tempf >= tolerance)
            low = beta;
        else
            high = beta;
    }
    return beta;
}

// FP64 B-spline moduli and Green's function table on the half spectrum (PME_force.cu:45-67,
// :253-286): BC = B1 B2 B3 exp(-pi^2 m^2 / beta^2) / (pi m^2 V), BC(0) = 0
static int build_bc(sb_pme* p) {
    const int K0 = p->K[0], K1 = p->K[1], K2 = p->K[2], H = K2 / 2 + 1;
    std::vector<double> B[3];
    for (int d = 0; d < 3; d++) {
        B[d].resize(p->K[d]);
        for (int k = 0; k < p->K[d]; k++) {
            double re = 0, im = 0;
            const double M4[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
            for (int j = 0; j < 3; j++) {
                double a = 2 * M_PI * j * (double)k / p->K[d];
                re += M4[j] * cos(a);
                im += M4[j] * sin(a);
            }
            B[d][k] = 1.0 / (re * re + im * im);
        }
    }
    const double Lx = p->box[0], Ly = p->box[1], Lz = p->box[2];
    const double V = Lx * Ly * Lz;
    const double beta = p->beta;
    std::vector<float> bc((size_t)K0 * K1 * H);
    for (int x = 0; x < K0; x++) {
        const int mx = x > K0 / 2 ? K0 - x : x;
        for (int y = 0; y < K1; y++) {
            const int my = y > K1 / 2 ? K1 - y : y;
            for (int z = 0; z < H; z++) {
                const int mz = z;
                double v = 0;
                if (x + y + z != 0) {
                    const double m2 = mx * mx / (Lx * Lx) + my * my / (Ly * Ly) + mz * mz / (Lz * Lz);
                    v = B[0][x] * B[1][y] * B[2][z] * exp(-M_PI * M_PI * m2 / (beta * beta)) /
                        (M_PI * m2 * V);
                }
                bc[((size_t)x * K1 + y) * H + z] = (float)v;
            }
        }
    }
    SB_CHECK_CUDA(cudaMemcpy(p->d_bc, bc.data(), sizeof(float) * bc.size(), cudaMemcpyHostToDevice));
    p->neutralizing_factor = -0.5 * M_PI / (beta * beta * V);
    return SB_OK;
}

extern "C" int sb_pme_create(int atom_numbers, const float box_length[3], float cutoff,
                             float tolerance, int fftx, int ffty, int fftz, int form,
                             sb_pme** out) {
    if (!out || atom_numbers <= 0 || !box_length || cutoff <= 0) {
        sb_set_error("sb_pme_create: invalid argument");
        return SB_ERR_ARG;
    }
    sb_pme* p = new sb_pme();
    p->n = atom_numbers;
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            sms > 0)
            p->num_sms = sms;
    }
    p->form = form;
    for (int d = 0; d < 3; d++) p->box[d] = box_length[d];
    p->cutoff = cutoff;
    p->tolerance = tolerance > 0 ? tolerance : 1e-5f;
    p->K[0] = fftx > 0 ? fftx : fft_size(box_length[0]);
    p->K[1] = ffty > 0 ? ffty : fft_size(box_length[1]);
    p->K[2] = fftz > 0 ? fftz : fft_size(box_length[2]);
    p->beta = get_beta(cutoff, p->tolerance);
    p->G = (size_t)p->K[0] * p->K[1] * p->K[2];
    p->Gh = (size_t)p->K[0] * p->K[1] * (p->K[2] / 2 + 1);
    int st = SB_OK;
    auto fail = [&](int s) {
        sb_pme_destroy(p);
        return s;
    };
    if (form == SB_FORM_FIXED) {
        if ((st = sb_fft_plan_create(&p->plan, p->K))) return fail(st);
        if ((st = sb_malloc((void**)&p->d_qfix, sizeof(long long) * p->G, "PME grid"))) return fail(st);
        cudaMemset(p->d_qfix, 0, sizeof(long long) * p->G);
        p->nparts = sb_fft_xconv_parts(&p->plan);
    } else {
        if ((st = sb_malloc((void**)&p->d_qf, sizeof(float) * p->G, "PME grid"))) return fail(st);
        cufftHandle a, b;
        if (cufftPlan3d(&a, p->K[0], p->K[1], p->K[2], CUFFT_R2C) != CUFFT_SUCCESS ||
            cufftPlan3d(&b, p->K[0], p->K[1], p->K[2], CUFFT_C2R) != CUFFT_SUCCESS) {
            sb_set_error("sb_pme_create: cuFFT plan creation failed");
            return fail(SB_ERR_CUDA);
        }
        p->cufft_r2c = (void*)(intptr_t)a;
        p->cufft_c2r = (void*)(intptr_t)b;
        p->cufft_ok = 1;
        p->nparts = 1184;
    }
    if ((st = sb_malloc((void**)&p->d_spec, sizeof(float2) * p->Gh, "PME spectrum")) ||
        (st = sb_malloc((void**)&p->d_theta, sizeof(float) * p->G, "PME potential grid")) ||
        (st = sb_malloc((void**)&p->d_bc, sizeof(float) * p->Gh, "PME BC")) ||
        (st = sb_malloc((void**)&p->d_epart, sizeof(double) * std::max(p->nparts, 1), "PME parts")) ||
        (st = sb_malloc((void**)&p->d_ered, sizeof(double) * 8, "PME energies")) ||
        (st = sb_malloc((void**)&p->d_direct_atom_energy, sizeof(float) * atom_numbers, "direct E")) ||
        (st = sb_malloc((void**)&p->d_correction_atom_energy, sizeof(float) * atom_numbers, "corr E")) ||
        (st = sb_malloc((void**)&p->d_fix, sizeof(long long) * 3 * atom_numbers, "excl fix")))
        return fail(st);
    cudaMemset(p->d_fix, 0, sizeof(long long) * 3 * atom_numbers);
    cudaMemset(p->d_direct_atom_energy, 0, sizeof(float) * atom_numbers);
    cudaMemset(p->d_correction_atom_energy, 0, sizeof(float) * atom_numbers);
    cudaMemset(p->d_ered, 0, sizeof(double) * 8);
    if ((st = build_bc(p))) return fail(st);
    if (form == SB_FORM_FIXED) {
        // kernel shapes of the FFT passes, picked by timing on this grid
        if ((st = sb_fft_plan_tune(&p->plan, p->d_spec, p->d_bc, 0)))
            return fail(st);
        cudaMemset(p->d_spec, 0, sizeof(float2) * p->Gh);
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (cudaStreamCreateWithPriority(&p->side, cudaStreamNonBlocking, hi) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) != cudaSuccess) {
            sb_set_error("sb_pme_create: stream/event creation failed");
            return fail(SB_ERR_CUDA);
        }
    }
    *out = p;
    return SB_OK;
}

extern "C" int sb_pme_set_fft_variant(sb_pme* p, int variant) {
    if (!p) {
        sb_set_error("sb_pme_set_fft_variant: null handle");
        return SB_ERR_ARG;
    }
    if (variant != SB_FFT_AUTO && variant != SB_FFT_GENERIC && variant != SB_FFT_LINES) {
        sb_set_error("sb_pme_set_fft_variant: variant %d is not AUTO, GENERIC or LINES", variant);
        return SB_ERR_ARG;
    }
    if (p->form != SB_FORM_FIXED) return SB_OK;  // the plain form runs the library FFT
    SB_CHECK_CUDA(cudaDeviceSynchronize());
    p->plan.variant = variant;
    SB_TRY(sb_fft_plan_tune(&p->plan, p->d_spec, p->d_bc, 0));
    SB_CHECK_CUDA(cudaMemset(p->d_spec, 0, sizeof(float2) * p->Gh));
    SB_CHECK_CUDA(cudaDeviceSynchronize());
    return SB_OK;
}

extern "C" int sb_pme_destroy(sb_pme* p) {
    if (!p) return SB_OK;
    cudaDeviceSynchronize();
    sb_fft_plan_destroy(&p->plan);
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    if (p->side) cudaStreamDestroy(p->side);
    if (p->cufft_ok) {
        cufftDestroy((cufftHandle)(intptr_t)p->cufft_r2c);
        cufftDestroy((cufftHandle)(intptr_t)p->cufft_c2r);
    }
    void* ps[] = {p->d_qfix, p->d_qf, p->d_spec, p->d_theta, p->d_bc, p->d_epart, p->d_ered,
                  p->d_direct_atom_energy, p->d_correction_atom_energy, p->d_fix,
                  p->energy_scratch};
    for (void* x : ps) sb_free(x);
    delete p;
    return SB_OK;
}

extern "C" int sb_pme_info(sb_pme* p, float* h_beta, int* h_fft3) {
    if (!p) {
        sb_set_error("sb_pme_info: null handle");
        return SB_ERR_ARG;
    }
    if (h_beta) *h_beta = p->beta;
    if (h_fft3)
        for (int d = 0; d < 3; d++) h_fft3[d] = p->K[d];
    return SB_OK;
}

extern "C" int sb_pme_atom_energy_arrays(sb_pme* p, float** d_direct, float** d_corr) {
    if (!p) {
        sb_set_error("sb_pme_atom_energy_arrays: null handle");
        return SB_ERR_ARG;
    }
    if (d_direct) *d_direct = p->d_direct_atom_energy;
    if (d_corr) *d_corr = p->d_correction_atom_energy;
    return SB_OK;
}

static int excluded_force(sb_pme* p, const uint32_t* uc, const float scaler[3], const float* q,
                          const int* es, const int* el, const int* en, float* frc, float* ene,
                          cudaStream_t s) {
    const int n = p->n, tb = 128;
    const float b = p->beta;
    if (p->form == SB_FORM_FIXED) {
        k_excluded<true><<<(n + tb - 1) / tb, tb, 0, s>>>(n, uc, scaler[0], scaler[1], scaler[2],
                                                          q, b, b * b, b * b * b, es, el, en,
                                                          p->d_fix, frc, ene);
        SB_CHECK_LAUNCH();
        k_fix_to_frc<<<(3 * n + 255) / 256, 256, 0, s>>>(n, p->d_fix, frc);
        SB_CHECK_LAUNCH();
    } else {
        k_excluded<false><<<(n + tb - 1) / tb, tb, 0, s>>>(n, uc, scaler[0], scaler[1],
                                                           scaler[2], q, b, b * b, b * b * b, es,
                                                           el, en, p->d_fix, frc, ene);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_pme_excluded_force(sb_pme* p, const uint32_t* d_uint_crd, const float scaler[3],
                                     const float* d_charge, const int* es, const int* el,
                                     const int* en, float* d_frc, float* d_atom_energy,
                                     void* stream) {
    if (!p || !d_uint_crd || !scaler || !d_charge || !d_frc) {
        sb_set_error("sb_pme_excluded_force: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    // Reset_List(d_correction_atom_energy) precedes the kernel as in PME_force.cu:701
    k_zero_f<<<(p->n + 1023) / 1024, 1024, 0, s>>>(p->n, p->d_correction_atom_energy);
    SB_CHECK_LAUNCH();
    if (!es || !el || !en) return SB_OK;
    return excluded_force(p, d_uint_crd, scaler, d_charge, es, el, en, d_frc, d_atom_energy, s);
}

// returns a status; *nparts_out receives the number of reciprocal-energy partials written
static int reciprocal(sb_pme* p, const uint32_t* uc, const float* q, float* frc, int want_e,
                      cudaStream_t s, int* nparts_out) {
    const int n = p->n;
    const int K0 = p->K[0], K1 = p->K[1], K2 = p->K[2];
    int nparts = 0;
    if (p->form == SB_FORM_FIXED) {
        k_spread<true><<<(4 * n + 255) / 256, 256, 0, s>>>(n, uc, q, K0, K1, K2, p->d_qfix, nullptr);
        SB_CHECK_LAUNCH();
        SB_TRY(sb_fft_plane_forward(&p->plan, p->d_qfix, p->d_spec, s));
        SB_TRY(sb_fft_x_convolve(&p->plan, p->d_spec, p->d_bc, p->d_epart, want_e, s, &nparts));
        SB_TRY(sb_fft_plane_inverse(&p->plan, p->d_spec, p->d_theta, s));
    } else {
        SB_CHECK_CUDA(cudaMemsetAsync(p->d_qf, 0, sizeof(float) * p->G, s));
        k_spread<false><<<(4 * n + 255) / 256, 256, 0, s>>>(n, uc, q, K0, K1, K2, nullptr, p->d_qf);
        SB_CHECK_LAUNCH();
        cufftHandle a = (cufftHandle)(intptr_t)p->cufft_r2c, b = (cufftHandle)(intptr_t)p->cufft_c2r;
        if (cufftSetStream(a, s) != CUFFT_SUCCESS || cufftSetStream(b, s) != CUFFT_SUCCESS ||
            cufftExecR2C(a, p->d_qf, (cufftComplex*)p->d_spec) != CUFFT_SUCCESS) {
            sb_set_error("cuFFT R2C failed");
            return SB_ERR_CUDA;
        }
        k_bcfq<<<(unsigned)((p->Gh + 1023) / 1024), 1024, 0, s>>>(p->Gh, p->d_spec, p->d_bc);
        SB_CHECK_LAUNCH();
        if (cufftExecC2R(b, (cufftComplex*)p->d_spec, p->d_theta) != CUFFT_SUCCESS) {
            sb_set_error("cuFFT C2R failed");
            return SB_ERR_CUDA;
        }
        if (want_e) {
            nparts = p->nparts;
            k_grid_dot<<<nparts, 256, 0, s>>>(p->G, p->d_qf, p->d_theta, p->d_epart);
            SB_CHECK_LAUNCH();
        }
    }
    k_gather<<<(n + 127) / 128, 128, 0, s>>>(n, uc, q, p->d_theta, K0, K1, K2,
                                             (float)K0 / p->box[0], (float)K1 / p->box[1],
                                             (float)K2 / p->box[2], frc);
    SB_CHECK_LAUNCH();
    *nparts_out = nparts;
    return SB_OK;
}

extern "C" int sb_pme_reciprocal_force(sb_pme* p, const uint32_t* d_uint_crd,
                                       const float* d_charge, float* d_frc, int need_virial,
                                       int need_energy, float* d_virial, float* d_potential,
                                       void* stream) {
    if (!p || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_pme_reciprocal_force: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const int want = (need_virial > 0 || need_energy > 0);
    int nparts = 0;
    SB_TRY(reciprocal(p, d_uint_crd, d_charge, d_frc, want, s, &nparts));
    if (want) {
        k_pme_energy_finish<<<1, 1024, 0, s>>>(p->n, d_charge, p->d_epart, nparts,
                                               p->d_direct_atom_energy,
                                               p->d_correction_atom_energy, (double)p->beta,
                                               p->neutralizing_factor, p->d_ered, need_virial > 0,
                                               need_energy > 0, d_virial, d_potential);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_pme_bc_table(sb_pme* p, const float** d_bc) {
    if (!p || !d_bc) {
        sb_set_error("sb_pme_bc_table: null argument");
        return SB_ERR_ARG;
    }
    *d_bc = p->d_bc;
    return SB_OK;
}

extern "C" int sb_pme_update_box(sb_pme* p, const float box_length[3]) {
    if (!p || !box_length) {
        sb_set_error("sb_pme_update_box: null argument");
        return SB_ERR_ARG;
    }
    for (int d = 0; d < 3; d++) p->box[d] = box_length[d];
    return build_bc(p);
}

// direct-space Coulomb energy over the list (PME_Direct_Atom_Energy, PME_force.cu:570-617)
__global__ void k_direct_energy_list(int n, const void* __restrict__ agv,
                                     const uint32_t* __restrict__ uc, const float* __restrict__ q,
                                     float sx, float sy, float sz, float beta, float rc2,
                                     float* __restrict__ out) {
    struct AG {
        int atom_numbers;
        int* atom_serial;
    };
    const AG* ag = (const AG*)agv;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const AG g = ag[i];
    float e = 0.f;
    for (int t = 0; t < g.atom_numbers; t++) {
        const int j = g.atom_serial[t];
        const float dx = __int2float_rn((int)(uc[3 * j] - uc[3 * i])) * sx;
        const float dy = __int2float_rn((int)(uc[3 * j + 1] - uc[3 * i + 1])) * sy;
        const float dz = __int2float_rn((int)(uc[3 * j + 2] - uc[3 * i + 2])) * sz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (r2 < rc2) {
            const float r = sqrtf(r2);
            e += q[i] * q[j] * erfcf(beta * r) / r;
        }
    }
    out[i] = e;
}

extern "C" int sb_pme_get_energy(sb_pme* p, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                                 const float* d_charge, const float scaler[3], const int* es,
                                 const int* el, const int* en, int which_part, float* h_energy,
                                 double* h_parts, void* stream) {
    if (!p || !d_uint_crd || !d_charge || !scaler) {
        sb_set_error("sb_pme_get_energy: null argument");
        return SB_ERR_ARG;
    }
    if (which_part < 0 || which_part > 4) {
        sb_set_error("sb_pme_get_energy: energy part %d is not allowed", which_part);
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const int n = p->n;
    const int all = which_part == SB_PME_TOTAL;
    const int want_rec = all || which_part == SB_PME_RECIPROCAL;
    const int want_dir = all || which_part == SB_PME_DIRECT;
    const int want_cor = all || which_part == SB_PME_CORRECTION;
    if (want_dir) {
        if (!nl) {
            sb_set_error("sb_pme_get_energy: the DIRECT part needs the neighbor list");
            return SB_ERR_ARG;
        }
        if (nl->n != n) {
            sb_set_error("sb_pme_get_energy: the neighbor list holds %d atoms, the PME module %d",
                         nl->n, n);
            return SB_ERR_ARG;
        }
    }
    int nparts = 0;
    if ((want_rec || want_cor) && !p->energy_scratch) {
        // the reciprocal and exclusion passes produce forces that the energy query discards:
        // they go to an array of the module, allocated on the first query and kept
        SB_TRY(sb_malloc((void**)&p->energy_scratch, sizeof(float) * 3 * n, "energy scratch"));
    }
    if (want_rec || want_cor)
        SB_CHECK_CUDA(cudaMemsetAsync(p->energy_scratch, 0, sizeof(float) * 3 * n, s));
    if (want_rec) SB_TRY(reciprocal(p, d_uint_crd, d_charge, p->energy_scratch, 1, s, &nparts));
    float* direct = nullptr;
    float* corr = nullptr;
    if (want_dir) {
        SB_TRY(sb_nl_build_atom_group(nl, s));
        k_direct_energy_list<<<(n + 127) / 128, 128, 0, s>>>(n, nl->ag, d_uint_crd, d_charge,
                                                             scaler[0], scaler[1], scaler[2],
                                                             p->beta, p->cutoff * p->cutoff,
                                                             p->d_direct_atom_energy);
        SB_CHECK_LAUNCH();
        direct = p->d_direct_atom_energy;
    }
    if (want_cor) {
        k_zero_f<<<(n + 1023) / 1024, 1024, 0, s>>>(n, p->d_correction_atom_energy);
        SB_CHECK_LAUNCH();
        if (es && el && en)
            SB_TRY(excluded_force(p, d_uint_crd, scaler, d_charge, es, el, en, p->energy_scratch,
                                  p->d_correction_atom_energy, s));
        corr = p->d_correction_atom_energy;
    }
    k_pme_energy_finish<<<1, 1024, 0, s>>>(n, d_charge, p->d_epart, nparts, direct, corr,
                                           (double)p->beta, p->neutralizing_factor, p->d_ered, 0,
                                           0, nullptr, nullptr);
    cudaError_t e = cudaGetLastError();
    double parts[4] = {0, 0, 0, 0};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(parts, p->d_ered, sizeof(double) * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        sb_set_error("sb_pme_get_energy: %s", cudaGetErrorString(e));
        return SB_ERR_CUDA;
    }
    const double rec = parts[0], self = parts[1], dir = parts[2], cor = parts[3];
    const double tot = rec + self + dir + cor;
    double v = tot;
    switch (which_part) {
        case SB_PME_DIRECT: v = dir; break;
        case SB_PME_RECIPROCAL: v = rec; break;
        case SB_PME_CORRECTION: v = cor; break;
        case SB_PME_SELF: v = self; break;
        default: break;
    }
    if (h_energy) *h_energy = (float)v;
    if (h_parts) {
        h_parts[0] = tot;
        h_parts[1] = dir;
        h_parts[2] = rec;
        h_parts[3] = cor;
        h_parts[4] = self;
    }
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// fused fixed-form step: reciprocal kernels adding into the neighbor list's fixed-point force
// buffer (x, y, z planes of slot_cap int64 each)
// ---------------------------------------------------------------------------------------------


int sb_pme_zero_atom_energy(sb_pme* p, float* d_atom_energy, cudaStream_t s) {
    if (d_atom_energy) {
        k_zero_f<<<(p->n + 1023) / 1024, 1024, 0, s>>>(p->n, d_atom_energy);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

// reciprocal gather of atom i (atom order, from the fixed-point coordinates and charges) into its
// slot's fixed-point accumulator, followed by the atom's exclusion correction; reads nothing the
// pair kernel's packing produces, so it can run beside it
__device__ __forceinline__ void gather_atom_one(int i, const uint32_t* __restrict__ uc,
                                                const float* __restrict__ qa,
                                                const float* __restrict__ theta, int K0, int K1,
                                                int K2, float ix, float iy, float iz,
                                                long long* __restrict__ fix, int slot_cap,
                                                const SbExclPass& X) {
    const float q = qa[i];
    if (q == 0.f) return;  // an uncharged atom has zero reciprocal force and exclusion terms
    const uint32_t ux = uc[3 * i], uy = uc[3 * i + 1], uz = uc[3 * i + 2];
    const int sl = X.atom_slot[i];
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(ux, K0, b0, f0);
    grid_coord(uy, K1, b1, f1);
    grid_coord(uz, K2, b2, f2);
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    bspline4d(f0, dx);
    bspline4d(f1, dy);
    bspline4d(f2, dz);
    int gz[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int g = b2 - k;
        gz[k] = g < 0 ? g + K2 : g;
    }
    float Fx = 0.f, Fy = 0.f, Fz = 0.f;
#pragma unroll
    for (int kx = 0; kx < 4; kx++) {
        int gx = b0 - kx;
        if (gx < 0) gx += K0;
#pragma unroll
        for (int ky = 0; ky < 4; ky++) {
            int gy = b1 - ky;
            if (gy < 0) gy += K1;
            const float* row = theta + ((size_t)gx * K1 + gy) * K2;
            float sw = 0.f, sd = 0.f;
#pragma unroll
            for (int kz = 0; kz < 4; kz++) {
                const float t = row[gz[kz]];
                sw = fmaf(t, wz[kz], sw);
                sd = fmaf(t, dz[kz], sd);
            }
            Fx = fmaf(dx[kx] * wy[ky], sw, Fx);
            Fy = fmaf(wx[kx] * dy[ky], sw, Fy);
            Fz = fmaf(wx[kx] * wy[ky], sd, Fz);
        }
    }
    const float sq = -q;
    long long fx = __float2ll_rn(sq * Fx * ix * SB_FORCE_SCALE);
    long long fy = __float2ll_rn(sq * Fy * iy * SB_FORCE_SCALE);
    long long fz = __float2ll_rn(sq * Fz * iz * SB_FORCE_SCALE);
    const int cnt = X.en ? X.en[i] : 0;
    if (cnt > 0) {
        const int s0 = X.es[i];
        float ex = 0.f, ey = 0.f, ez = 0.f, e = 0.f;
        for (int k = s0; k < s0 + cnt; k++) {
            const int j = X.el[k];
            const int sj = X.atom_slot[j];
            const float ddx = __int2float_rn((int)(uc[3 * j] - ux)) * X.sx;
            const float ddy = __int2float_rn((int)(uc[3 * j + 1] - uy)) * X.sy;
            const float ddz = __int2float_rn((int)(uc[3 * j + 2] - uz)) * X.sz;
            const float r2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
            const float qq = q * qa[j];
            const float fs = qq * X.beta3 * sb_ewald_G(X.beta2 * r2);
            const float tx = fs * ddx, ty = fs * ddy, tz = fs * ddz;
            ex += tx;
            ey += ty;
            ez += tz;
            if (X.ene) {
                const float r = sqrtf(r2);
                e -= qq * erff(X.beta * r) / r;
            }
            sb_red_add(&fix[sj], __float2ll_rn(-tx * SB_FORCE_SCALE));
            sb_red_add(&fix[slot_cap + sj], __float2ll_rn(-ty * SB_FORCE_SCALE));
            sb_red_add(&fix[2 * slot_cap + sj], __float2ll_rn(-tz * SB_FORCE_SCALE));
        }
        fx += __float2ll_rn(ex * SB_FORCE_SCALE);
        fy += __float2ll_rn(ey * SB_FORCE_SCALE);
        fz += __float2ll_rn(ez * SB_FORCE_SCALE);
        if (X.ene) atomicAdd(&X.ene[i], e);
    }
    sb_red_add(&fix[sl], fx);
    sb_red_add(&fix[slot_cap + sl], fy);
    sb_red_add(&fix[2 * slot_cap + sl], fz);
}

// thread per atom (grid-stride; a grid of fewer blocks, as for the spread, was slower here: the
// gather ends the side chain)
__global__ void k_gather_atom(int n, const uint32_t* __restrict__ uc, const float* __restrict__ qa,
                              const float* __restrict__ theta, int K0, int K1, int K2, float ix,
                              float iy, float iz, long long* __restrict__ fix, int slot_cap,
                              SbExclPass X) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        gather_atom_one(i, uc, qa, theta, K0, K1, K2, ix, iy, iz, fix, slot_cap, X);
}

int sb_pme_fused_grid_atoms(sb_pme* p, sb_neighbor_list* nl, int want_energy, cudaStream_t s,
                            const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                            const int* el, const int* en, float* d_excl_energy) {
    const int K0 = p->K[0], K1 = p->K[1], K2 = p->K[2], n = p->n;
    // a small grid (4 blocks per SM) looping over the atoms: the spread then holds few SM
    // resources beside the pair kernel (137.4 -> 134.1 us per step on the 96k-atom box)
    k_spread<true><<<std::min((4 * n + 255) / 256, 4 * p->num_sms), 256, 0, s>>>(
        n, d_uint_crd, d_charge, K0, K1, K2, p->d_qfix, nullptr);
    SB_CHECK_LAUNCH();
    SB_TRY(sb_fft_plane_forward(&p->plan, p->d_qfix, p->d_spec, s));
    SB_TRY(sb_fft_x_convolve(&p->plan, p->d_spec, p->d_bc, p->d_epart, want_energy, s,
                             &p->rec_nparts));
    SB_TRY(sb_fft_plane_inverse(&p->plan, p->d_spec, p->d_theta, s));
    const float b = p->beta;
    const bool excl = es && el && en;
    const SbExclPass X{nl->slot_atom, nl->atom_slot, excl ? es : nullptr, excl ? el : nullptr,
                       excl ? en : nullptr, (1.0f / 4294967296.0f) * p->box[0],
                       (1.0f / 4294967296.0f) * p->box[1], (1.0f / 4294967296.0f) * p->box[2],
                       b, b * b, b * b * b, d_excl_energy};
    k_gather_atom<<<(n + 127) / 128, 128, 0, s>>>(
        n, d_uint_crd, d_charge, p->d_theta, K0, K1, K2, (float)K0 / p->box[0],
        (float)K1 / p->box[1], (float)K2 / p->box[2], nl->fix, nl->slot_cap, X);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

int sb_pme_fused_finish(sb_pme* p, sb_neighbor_list* nl, float* d_frc, const float* d_charge,
                        int need_virial, int need_energy, float* d_virial, float* d_potential,
                        cudaStream_t s) {
    SB_TRY(sb_nl_finalize_forces(nl, d_frc, s));
    if (need_virial > 0 || need_energy > 0) {
        k_pme_energy_finish<<<1, 1024, 0, s>>>(p->n, d_charge, p->d_epart, p->rec_nparts,
                                               p->d_direct_atom_energy,
                                               p->d_correction_atom_energy, (double)p->beta,
                                               p->neutralizing_factor, p->d_ered, need_virial > 0,
                                               need_energy > 0, d_virial, d_potential);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

int sb_pme_fused_reciprocal(sb_pme* p, sb_neighbor_list* nl, float* d_frc,
                            const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                            const int* el, const int* en, int need_virial, int need_energy,
                            float* d_virial, float* d_potential, cudaStream_t s) {
    SB_TRY(sb_pme_fused_grid_atoms(p, nl, need_virial > 0 || need_energy > 0, s, d_uint_crd,
                                   d_charge, es, el, en, nullptr));
    return sb_pme_fused_finish(p, nl, d_frc, d_charge, need_virial, need_energy, d_virial,
                               d_potential, s);
}

// ---------------------------------------------------------------------------------------------
// TI cross terms of PME (TI_core.cu:670-730): for charges changing by dq per unit lambda,
// d E_rec / d lambda = sum_i dq_i phi_i with phi the SPME potential of the current charges (the
// reference spreads dq onto a second grid and dots it with the convolved grid; the same number),
// and the exclusion-correction derivative at fixed geometry. Accumulated as 2^32 fixed point.
// ---------------------------------------------------------------------------------------------
#define SB_TI_SCALE 4294967296.0f
#define SB_TI_UNSCALE (1.0 / 4294967296.0)

__device__ __forceinline__ float phi_at(uint32_t ux, uint32_t uy, uint32_t uz,
                                        const float* __restrict__ theta, int K0, int K1, int K2) {
    int b0, b1, b2;
    float f0, f1, f2;
    grid_coord(ux, K0, b0, f0);
    grid_coord(uy, K1, b1, f1);
    grid_coord(uz, K2, b2, f2);
    float wx[4], wy[4], wz[4];
    bspline4(f0, wx);
    bspline4(f1, wy);
    bspline4(f2, wz);
    float phi = 0.f;
#pragma unroll
    for (int kx = 0; kx < 4; kx++) {
        int gx = b0 - kx;
        if (gx < 0) gx += K0;
#pragma unroll
        for (int ky = 0; ky < 4; ky++) {
            int gy = b1 - ky;
            if (gy < 0) gy += K1;
            const float* row = theta + ((size_t)gx * K1 + gy) * K2;
            float sw = 0.f;
#pragma unroll
            for (int kz = 0; kz < 4; kz++) {
                int gz = b2 - kz;
                if (gz < 0) gz += K2;
                sw = fmaf(row[gz], wz[kz], sw);
            }
            phi = fmaf(wx[kx] * wy[ky], sw, phi);
        }
    }
    return phi;
}

__device__ __forceinline__ void ti_red(long long* p, float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) {
        const long long q = __float2ll_rn(v * SB_TI_SCALE);
        if (q) atomicAdd((unsigned long long*)p, (unsigned long long)q);
    }
}

// dq phi of packed slot s (a slot of an uncharged-change atom or an empty slot gives 0)
__device__ __forceinline__ float ti_rec_slot(int s, const uint4* __restrict__ xq,
                                             const float* __restrict__ slot_dq,
                                             const float* __restrict__ theta, int K0, int K1,
                                             int K2) {
    const float d = slot_dq[s];
    if (d == 0.f) return 0.f;
    const uint4 u = xq[s];
    return d * phi_at(u.x, u.y, u.z, theta, K0, K1, K2);
}

// sum dq phi over atoms in original order (n) or over packed slots (xq != null, n = slots)
__global__ void k_ti_rec(int n, const int* __restrict__ meta, const uint32_t* __restrict__ uc,
                         const uint4* __restrict__ xq, const float* __restrict__ dq,
                         const float* __restrict__ theta, int K0, int K1, int K2,
                         long long* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lim = meta ? meta[3] : n;
    float v = 0.f;
    if (i < lim) {
        if (xq) {
            v = ti_rec_slot(i, xq, dq, theta, K0, K1, K2);
        } else {
            const float d = dq[i];
            if (d != 0.f)
                v = d * phi_at(uc[3 * i], uc[3 * i + 1], uc[3 * i + 2], theta, K0, K1, K2);
        }
    }
    ti_red(acc, v);
}

// d/dlambda of atom i's exclusion corrections -qq erf(beta r)/r at fixed geometry
__device__ __forceinline__ float ti_corr_atom(int i, const uint32_t* __restrict__ uc, float sx,
                                              float sy, float sz, const float* __restrict__ q,
                                              const float* __restrict__ dq, float beta,
                                              const int* __restrict__ es,
                                              const int* __restrict__ el,
                                              const int* __restrict__ en) {
    float v = 0.f;
    const int cnt = en[i], s0 = es[i];
    const float qi = q[i], dqi = dq[i];
    for (int k = s0; k < s0 + cnt; k++) {
        const int j = el[k];
        const float dqq = qi * dq[j] + dqi * q[j];
        if (dqq == 0.f) continue;
        const float dx = __int2float_rn((int)(uc[3 * j] - uc[3 * i])) * sx;
        const float dy = __int2float_rn((int)(uc[3 * j + 1] - uc[3 * i + 1])) * sy;
        const float dz = __int2float_rn((int)(uc[3 * j + 2] - uc[3 * i + 2])) * sz;
        const float r = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        v -= dqq * erff(beta * r) / r;
    }
    return v;
}

__global__ void k_ti_corr(int n, const uint32_t* __restrict__ uc, float sx, float sy, float sz,
                          const float* __restrict__ q, const float* __restrict__ dq, float beta,
                          const int* __restrict__ es, const int* __restrict__ el,
                          const int* __restrict__ en, long long* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float v = i < n ? ti_corr_atom(i, uc, sx, sy, sz, q, dq, beta, es, el, en) : 0.f;
    ti_red(acc, v);
}

__global__ void k_ti_zero(long long* a, int n) {
    if ((int)threadIdx.x < n) a[threadIdx.x] = 0;
}

__global__ void __launch_bounds__(1024) k_ti_finish(int n, const float* __restrict__ q,
                                                    const float* __restrict__ dq,
                                                    const long long* __restrict__ acc,
                                                    double self_coef, double neutral2,
                                                    double* __restrict__ out) {
    __shared__ double r1[1024], r2[1024], r3[1024];
    double a = 0, b = 0, c = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += (double)q[i] * dq[i];
        b += q[i];
        c += dq[i];
    }
    r1[threadIdx.x] = a;
    r2[threadIdx.x] = b;
    r3[threadIdx.x] = c;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            r1[threadIdx.x] += r1[threadIdx.x + o];
            r2[threadIdx.x] += r2[threadIdx.x + o];
            r3[threadIdx.x] += r3[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = (double)acc[0] * SB_TI_UNSCALE;
        out[1] = self_coef * r1[0] + neutral2 * r2[0] * r3[0];
        out[2] = (double)acc[1] * SB_TI_UNSCALE;
    }
}

// fused FEP step: reciprocal and exclusion cross terms after sb_pme_fused_reciprocal left the
// convolved grid in d_theta; adds into acc[0] (reciprocal) and acc[1] (correction)
int sb_pme_ti_terms_slot(sb_pme* p, sb_neighbor_list* nl, const float* slot_dq,
                         const uint32_t* uc, const float* q, const float* dq, const int* es,
                         const int* el, const int* en, long long* acc, cudaStream_t s) {
    k_ti_rec<<<(nl->slot_cap + 255) / 256, 256, 0, s>>>(nl->slot_cap, nl->meta, nullptr, nl->xq,
                                                        slot_dq, p->d_theta, p->K[0], p->K[1],
                                                        p->K[2], acc);
    SB_CHECK_LAUNCH();
    if (es && el && en) {
        const float sx = (1.0f / 4294967296.0f) * p->box[0], sy = (1.0f / 4294967296.0f) * p->box[1],
                    sz = (1.0f / 4294967296.0f) * p->box[2];
        k_ti_corr<<<(p->n + 255) / 256, 256, 0, s>>>(p->n, uc, sx, sy, sz, q, dq, p->beta, es, el,
                                                     en, acc + 1);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_pme_ti_cross(sb_pme* p, const uint32_t* d_uint_crd, const float* d_charge,
                               const float* d_dq, const int* es, const int* el, const int* en,
                               double* h_parts, void* stream) {
    if (!p || !d_uint_crd || !d_charge || !d_dq || !h_parts) {
        sb_set_error("sb_pme_ti_cross: null argument");
        return SB_ERR_ARG;
    }
    if (p->form != SB_FORM_FIXED) {
        sb_set_error("sb_pme_ti_cross: needs the fixed-point form");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const int n = p->n;
    // two int64 accumulators in the FP64 energy slots 4 and 5; the results go to slots 0..2
    long long* acc = (long long*)(p->d_ered + 4);
    k_ti_zero<<<1, 32, 0, s>>>(acc, 2);
    SB_CHECK_LAUNCH();
    // theta of the current charges (recomputed, as TI_CORE does)
    k_spread<true><<<(4 * n + 255) / 256, 256, 0, s>>>(n, d_uint_crd, d_charge, p->K[0], p->K[1],
                                                      p->K[2], p->d_qfix, nullptr);
    SB_CHECK_LAUNCH();
    int nparts = 0;
    SB_TRY(sb_fft_plane_forward(&p->plan, p->d_qfix, p->d_spec, s));
    SB_TRY(sb_fft_x_convolve(&p->plan, p->d_spec, p->d_bc, p->d_epart, 0, s, &nparts));
    SB_TRY(sb_fft_plane_inverse(&p->plan, p->d_spec, p->d_theta, s));
    k_ti_rec<<<(n + 255) / 256, 256, 0, s>>>(n, nullptr, d_uint_crd, nullptr, d_dq, p->d_theta,
                                             p->K[0], p->K[1], p->K[2], acc);
    SB_CHECK_LAUNCH();
    if (es && el && en) {
        const float sx = (1.0f / 4294967296.0f) * p->box[0], sy = (1.0f / 4294967296.0f) * p->box[1],
                    sz = (1.0f / 4294967296.0f) * p->box[2];
        k_ti_corr<<<(n + 255) / 256, 256, 0, s>>>(n, d_uint_crd, sx, sy, sz, d_charge, d_dq,
                                                  p->beta, es, el, en, acc + 1);
        SB_CHECK_LAUNCH();
    }
    k_ti_finish<<<1, 1024, 0, s>>>(n, d_charge, d_dq, acc, -2.0 * (double)p->beta / sqrt(M_PI),
                                   2.0 * p->neutralizing_factor, p->d_ered);
    SB_CHECK_LAUNCH();
    double h[3];
    SB_CHECK_CUDA(cudaMemcpyAsync(h, p->d_ered, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 3; k++) h_parts[k] = h[k];
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free energy query
//
// sb_pme_get_energy needs a 3N-float force array to run the reciprocal and exclusion passes
// (their forces are thrown away; only the energies are kept) and obtains it with cudaMalloc /
// cudaFree on every call. Some callers cannot do that: a host program whose device memory is
// fully handed to its own pool allocator, or a driver loop that must not pay for cudaFree, which
// waits for the whole device. sb_pme_get_energy_noalloc takes that array from a fixed block of
// device memory of this library instead (it exists on a device once the library's device code
// is loaded there: at the latest in sb_pme_create).
// ---------------------------------------------------------------------------------------------
#define SB_NOALLOC_MAX_ATOMS 131072  // 3 x 131072 floats = 1.5 MiB, held by every GPU that loads
                                     // the library until the process exits
#define SB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) float g_noalloc_frc[3 * SB_NOALLOC_MAX_ATOMS];

// Host code may not hand g_noalloc_frc itself to a kernel (on the host it only names a stand-in
// object); its device address is looked up once per device, with that device current, and kept
// for the life of the process. A kept address is stale after cudaDeviceReset (or anything else
// that destroys the device's primary context); the header says callers must not call the entry
// point after that.
static float* g_noalloc_frc_addr[SB_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(float** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        sb_set_error("sb_pme_get_energy_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
        return SB_ERR_CUDA;
    }
    if (dev < 0 || dev >= SB_NOALLOC_MAX_DEVICES) {
        sb_set_error("sb_pme_get_energy_noalloc: device %d is beyond the %d devices supported", dev,
                     SB_NOALLOC_MAX_DEVICES);
        return SB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_frc_addr[dev]) {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_noalloc_frc);
        if (e != cudaSuccess || !addr) {
            sb_set_error("sb_pme_get_energy_noalloc: cudaGetSymbolAddress failed: %s",
                         cudaGetErrorString(e));
            return SB_ERR_CUDA;
        }
        g_noalloc_frc_addr[dev] = (float*)addr;
    }
    *out = g_noalloc_frc_addr[dev];
    return SB_OK;
}

extern "C" int sb_pme_get_energy_noalloc(sb_pme* p, sb_neighbor_list* nl,
                                         const uint32_t* d_uint_crd, const float* d_charge,
                                         const float scaler[3], const int* es, const int* el,
                                         const int* en, int which_part, float* h_energy,
                                         double* h_parts, void* stream) {
    if (!p || !d_uint_crd || !d_charge || !scaler) {
        sb_set_error("sb_pme_get_energy_noalloc: null argument");
        return SB_ERR_ARG;
    }
    if (which_part < 0 || which_part > 4) {
        sb_set_error("sb_pme_get_energy_noalloc: energy part %d is not allowed", which_part);
        return SB_ERR_ARG;
    }
    const int n = p->n;
    if (n > SB_NOALLOC_MAX_ATOMS) {
        sb_set_error("sb_pme_get_energy_noalloc: %d atoms exceed the maximum of %d; use "
                     "sb_pme_get_energy", n, SB_NOALLOC_MAX_ATOMS);
        return SB_ERR_ARG;
    }
    const int all = which_part == SB_PME_TOTAL;
    const int want_rec = all || which_part == SB_PME_RECIPROCAL;
    const int want_dir = all || which_part == SB_PME_DIRECT;
    const int want_cor = all || which_part == SB_PME_CORRECTION;
    if (want_dir) {
        if (!nl) {
            sb_set_error("sb_pme_get_energy_noalloc: the DIRECT part needs the neighbor list");
            return SB_ERR_ARG;
        }
        if (nl->n != n) {
            sb_set_error("sb_pme_get_energy_noalloc: the neighbor list holds %d atoms, the PME "
                         "module %d", nl->n, n);
            return SB_ERR_ARG;
        }
        if (!nl->ag) {
            // the list's ATOM_GROUP export is allocated on its first use
            sb_set_error("sb_pme_get_energy_noalloc: the DIRECT part reads the list's ATOM_GROUP "
                         "export, which allocates on first use; call sb_nl_atom_group once first");
            return SB_ERR_STATE;
        }
    }
    float* scratch = nullptr;
    SB_TRY(noalloc_scratch(&scratch));
    cudaStream_t s = sb_stream(stream);
    // the thrown-away forces accumulate here: clear the part this call uses
    if (want_rec || want_cor)
        SB_CHECK_CUDA(cudaMemsetAsync(scratch, 0, sizeof(float) * 3 * n, s));
    int nparts = 0;
    if (want_rec) SB_TRY(reciprocal(p, d_uint_crd, d_charge, scratch, 1, s, &nparts));
    float* direct = nullptr;
    float* corr = nullptr;
    if (want_dir) {
        SB_TRY(sb_nl_build_atom_group(nl, s));
        k_direct_energy_list<<<(n + 127) / 128, 128, 0, s>>>(n, nl->ag, d_uint_crd, d_charge,
                                                             scaler[0], scaler[1], scaler[2],
                                                             p->beta, p->cutoff * p->cutoff,
                                                             p->d_direct_atom_energy);
        SB_CHECK_LAUNCH();
        direct = p->d_direct_atom_energy;
    }
    if (want_cor) {
        k_zero_f<<<(n + 1023) / 1024, 1024, 0, s>>>(n, p->d_correction_atom_energy);
        SB_CHECK_LAUNCH();
        if (es && el && en)
            SB_TRY(excluded_force(p, d_uint_crd, scaler, d_charge, es, el, en, scratch,
                                  p->d_correction_atom_energy, s));
        corr = p->d_correction_atom_energy;
    }
    k_pme_energy_finish<<<1, 1024, 0, s>>>(n, d_charge, p->d_epart, nparts, direct, corr,
                                           (double)p->beta, p->neutralizing_factor, p->d_ered, 0,
                                           0, nullptr, nullptr);
    SB_CHECK_LAUNCH();
    double parts[4] = {0, 0, 0, 0};
    SB_CHECK_CUDA(cudaMemcpyAsync(parts, p->d_ered, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    const double rec = parts[0], self = parts[1], dir = parts[2], cor = parts[3];
    const double tot = rec + self + dir + cor;
    double v = tot;
    switch (which_part) {
        case SB_PME_DIRECT: v = dir; break;
        case SB_PME_RECIPROCAL: v = rec; break;
        case SB_PME_CORRECTION: v = cor; break;
        case SB_PME_SELF: v = self; break;
        default: break;
    }
    if (h_energy) *h_energy = (float)v;
    if (h_parts) {
        h_parts[0] = tot;
        h_parts[1] = dir;
        h_parts[2] = rec;
        h_parts[3] = cor;
        h_parts[4] = self;
    }
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched reciprocal chain of many FEP boxes (sb_fep_batch_*): every launch covers all boxes,
// block b working for box tab[b].x on its block tab[b].y (blocks never straddle boxes, so a warp
// belongs to one box). Each thread does what the same thread of the box's own launches does and
// the sums are fixed point or keep their warps, so every box gets the bits of its single steps.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS)
    k_spread_batch(const SbFepBox* __restrict__ B, const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const SbFepBox& b = B[t.x];
    const int gt = t.y * SB_FEP_BATCH_THREADS + threadIdx.x;
    if (gt < 4 * b.n) spread_one<true>(gt, b.uc, b.q, b.K0, b.K1, b.K2, b.qfix, nullptr);
}

// reciprocal gather with the exclusion correction, and (dH) the exclusion cross term of
// dU/dlambda summed per warp as k_ti_corr does
template <bool DH>
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS, 4)
    k_gather_batch(const SbFepBox* __restrict__ B, const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const SbFepBox& b = B[t.x];
    const int i = t.y * SB_FEP_BATCH_THREADS + threadIdx.x;
    if (DH && b.X.es) {
        const float v = i < b.n ? ti_corr_atom(i, b.uc, b.X.sx, b.X.sy, b.X.sz, b.q, b.dq,
                                               b.X.beta, b.X.es, b.X.el, b.X.en)
                                : 0.f;
        ti_red(b.hfix + 3, v);
    }
    if (i < b.n)
        gather_atom_one(i, b.uc, b.q, b.theta, b.K0, b.K1, b.K2, b.ix, b.iy, b.iz, b.fix,
                        b.slot_cap, b.X);
}

// fixed-point forces to the boxes' float arrays, and (dH) the reciprocal cross term over slots
template <bool DH>
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS)
    k_slots_batch(const SbFepBox* __restrict__ B, const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const SbFepBox& b = B[t.x];
    const int s = t.y * SB_FEP_BATCH_THREADS + threadIdx.x;
    // the slot's data are loaded beside the slot count (the blocks cover the allocation)
    const bool in = s < b.slot_cap;
    const int a = in ? b.slot_atom[s] : -1;
    long long fx = 0, fy = 0, fz = 0;
    if (in) {
        fx = b.fix[s];
        fy = b.fix[b.slot_cap + s];
        fz = b.fix[2 * b.slot_cap + s];
    }
    const float d = DH && in ? b.slot_dq[s] : 0.f;
    const int lim = b.meta[3];
    if (s == 0) sb_retire_prune(b.meta);
    if (DH) {
        float v = 0.f;
        if (s < lim && d != 0.f) {
            const uint4 u = b.xq[s];
            v = d * phi_at(u.x, u.y, u.z, b.theta, b.K0, b.K1, b.K2);
        }
        ti_red(b.hfix + 2, v);
    }
    if (s < lim) sb_finalize_slot(s, a, fx, fy, fz, b.fix, b.slot_cap, b.frc);
}

int sb_pme_batch_spread(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, cudaStream_t s) {
    k_spread_batch<<<nblocks, SB_FEP_BATCH_THREADS, 0, s>>>(d_boxes, d_tab);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

int sb_pme_batch_gather(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, int dh,
                        cudaStream_t s) {
    if (dh)
        k_gather_batch<true><<<nblocks, SB_FEP_BATCH_THREADS, 0, s>>>(d_boxes, d_tab);
    else
        k_gather_batch<false><<<nblocks, SB_FEP_BATCH_THREADS, 0, s>>>(d_boxes, d_tab);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

int sb_pme_batch_slots(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, int dh,
                       cudaStream_t s) {
    if (dh)
        k_slots_batch<true><<<nblocks, SB_FEP_BATCH_THREADS, 0, s>>>(d_boxes, d_tab);
    else
        k_slots_batch<false><<<nblocks, SB_FEP_BATCH_THREADS, 0, s>>>(d_boxes, d_tab);
    SB_CHECK_LAUNCH();
    return SB_OK;
}
