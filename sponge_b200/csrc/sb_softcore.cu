// Soft-core LJ + Ewald direct space for FEP/TI — replaces LJ_SOFT_CORE
// (SPONGE/Lennard_Jones_force/LJ_soft_core.cu) — and the FEP force step with dU/dlambda.
//
// Two end states A and B. A pair is soft-cored when its atoms' perturbation masks differ or
// when exactly one end state has LJ between them (LJ_soft_core.cu:243-297); then
//   r_A^6 = r^6 + alpha lambda^p sigma_A^6,   r_B^6 = r^6 + alpha (1-lambda)^p sigma_B^6,
//   E = (1-l) [A_A/12 r_A^-12 - B_A/6 r_A^-6 + qq erfc(b r_A)/r_A] + l [same, B state, r_B],
// sigma^6 = max(A/(2B), sigma_min^6), or sigma^6 when either coefficient vanishes. Other pairs
// use the tables mixed linearly in lambda at the plain distance. qq is the product of the charges
// at lambda (the caller's charge array). dH/dlambda is the exact lambda derivative of that
// energy at fixed geometry, including the charge change dq = q_B - q_A.
//
// Chosen form: the cluster list of the neighbor list (warp per 8-atom cluster, one lane per
// entry), forces and dH/dlambda accumulated as 64-bit fixed point. Plain form: the per-atom
// ATOM_GROUP list with float atomics (the reference's structure).

#include <math.h>

#include <vector>

#include "sb_ewald.cuh"
#include "sb_internal.cuh"

#define SB_DHDL_SCALE 4294967296.0f      // 2^32 fixed-point units per kcal/mol
#define SB_DHDL_UNSCALE (1.0 / 4294967296.0)
#define SB_EV_ENERGY_SC 1
#define SB_EV_VIRIAL_SC 2

struct sb_softcore {
    int n = 0;
    int ntA = 0, ntB = 0;
    int form = SB_FORM_FIXED;
    float cutoff = 10.f;
    float box[3];
    float lambda = 0.f, alpha = 0.5f, p = 1.f, sigma = 3.f, sigma_min = 0.f;
    std::vector<float> hA12a, hB6a, hA12b, hB6b;  // lower-triangular tables (x12, x6)
    std::vector<int> htA, htB;
    double lrc_factor = 0, lrc_ti = 0;             // x kappa; energy = factor / V
    float2* d_ABa = nullptr;   // [ntA^2] {A12, B6} of state A
    float2* d_ABb = nullptr;   // [ntB^2] of state B
    float* d_Aa = nullptr;     // lower-triangular copies for the plain form
    float* d_Ba = nullptr;
    float* d_Ab = nullptr;
    float* d_Bb = nullptr;
    int* d_typeA = nullptr;
    int* d_typeB = nullptr;
    int* d_mask = nullptr;
    float* d_dq = nullptr;
    int slot_cap = 0;
    int* d_slot_ext = nullptr;     // [slot_cap] typeB | mask << 16
    float* d_slot_dq = nullptr;    // [slot_cap]
    long long* d_hfix = nullptr;   // [4] fixed-point dH/dlambda: LJ, direct, reciprocal, correction
    double* d_red = nullptr;       // [8] FP64 scratch
    float* d_scratch_frc = nullptr;  // [3N] plain-form dH/dlambda pass (forces discarded)
    // split form of the fused FEP step (split != 0): the pairs of two unperturbed atoms go
    // through the packed LJ + Ewald kernel with the A-state table (for them the soft-core
    // energy is the A-state energy and adds nothing to dH/dlambda), the pairs with a perturbed
    // atom through a soft-core pass over the perturbed atoms
    int npert = 0;
    int split = 0;
    int* d_pert = nullptr;         // [npert] perturbed atoms, ascending
    int* d_tu = nullptr;           // [N] A type, or the ghost type ntA for a perturbed atom
    float2* d_ABu = nullptr;       // [(ntA+1)^2] A-state square table, zero ghost row/column
    double* d_sums = nullptr;      // [3] sums of q dq, q, dq of the last FEP step
    int2* d_ppairs = nullptr;      // [pcap] pairs with a perturbed atom found by the step
    int* d_pcount = nullptr;       // their count
    int pcap = 0;
};

// pairs with a perturbed atom held per perturbed atom (more raise SB_STATUS_LIST_OVERFLOW)
#define SB_SC_PAIRS_PER_ATOM 2048

// at most this many perturbed atoms (and at most one in eight atoms) for the split form: its
// soft-core pass tests every atom against every perturbed atom
#define SB_SC_SPLIT_MAX 512

struct ScParams {
    float sx, sy, sz, rc2;
    float beta, beta2, tsp_beta;  // 2 beta / sqrt(pi)
    float l, l_;                  // lambda, 1 - lambda
    float cA, cB;                 // alpha lambda^p, alpha (1-lambda)^p
    float dcA, dcB;               // their lambda derivatives
    float s6, s6min;
    float gp[6];
    int wide;
    int ntA, ntB;
    int slot_cap, ent_cap;
};

// force factor fs (force on i = fs (r_j - r_i)) of one pair inside the cutoff, with the optional
// energy, LJ virial and dH/dlambda contributions
template <bool EV, bool DH>
__device__ __forceinline__ float sc_pair(const ScParams& P, float r2, float qq, float dqq,
                                         bool soft, float2 a, float2 b, float& e_lj, float& e_c,
                                         float& v_lj, float& h_lj, float& h_c) {
    if (!soft) {
        const float ri = rsqrtf(r2);
        const float ri2 = ri * ri, ri6 = ri2 * ri2 * ri2;
        const float Am = P.l_ * a.x + P.l * b.x, Bm = P.l_ * a.y + P.l * b.y;
        const float flj = (Bm - Am * ri6) * (ri6 * ri2);
        const float bg = P.wide ? sb_ewald_G_scaled(P.beta2 * r2, P.gp)
                                : sb_ewald_G_rational(P.beta2 * r2, P.gp);
        const float fc = qq * (ri * ri2 - bg);
        if (EV || DH) {
            const float ec = (EV || dqq != 0.f) ? erfcf(P.beta * r2 * ri) * ri : 0.f;
            if (EV) {
                e_lj += (0.083333333f * Am * ri6 - 0.166666667f * Bm) * ri6;
                e_c += qq * ec;
                v_lj -= flj * r2;
            }
            if (DH) {
                h_lj += (0.083333333f * (b.x - a.x) * ri6 - 0.166666667f * (b.y - a.y)) * ri6;
                h_c += dqq * ec;
            }
        }
        return flj - fc;
    }
    const float r4 = r2 * r2, r6 = r4 * r2;
    const float sgA = (a.x < 1e-6f || a.y < 1e-6f) ? P.s6 : fmaxf(0.5f * a.x / a.y, P.s6min);
    const float sgB = (b.x < 1e-6f || b.y < 1e-6f) ? P.s6 : fmaxf(0.5f * b.x / b.y, P.s6min);
    const float sA = 1.0f / (r6 + P.cA * sgA), sB = 1.0f / (r6 + P.cB * sgB);
    const float flj = r4 * (P.l_ * (a.y - a.x * sA) * sA * sA + P.l * (b.y - b.x * sB) * sB * sB);
    const float rAi = powf(sA, 1.0f / 6.0f), rBi = powf(sB, 1.0f / 6.0f);  // 1/r_A, 1/r_B
    const float gA = P.tsp_beta * expf(-P.beta2 / (rAi * rAi));
    const float gB = P.tsp_beta * expf(-P.beta2 / (rBi * rBi));
    const float phA = erfcf(P.beta / rAi) * rAi, phB = erfcf(P.beta / rBi) * rBi;
    const float fc = qq * r4 * (P.l_ * (gA + phA) * sA + P.l * (gB + phB) * sB);
    const float EA = (0.083333333f * a.x * sA - 0.166666667f * a.y) * sA;
    const float EB = (0.083333333f * b.x * sB - 0.166666667f * b.y) * sB;
    if (EV) {
        e_lj += P.l_ * EA + P.l * EB;
        e_c += qq * (P.l_ * phA + P.l * phB);
        v_lj -= flj * r2;
    }
    if (DH) {
        const float dEA = (0.166666667f * a.x * sA - 0.166666667f * a.y) * (-sA * sA * P.dcA * sgA);
        const float dEB = (0.166666667f * b.x * sB - 0.166666667f * b.y) * (-sB * sB * P.dcB * sgB);
        h_lj += EB - EA + P.l_ * dEA + P.l * dEB;
        const float dphA = -(gA + phA) * sA * 0.166666667f * P.dcA * sgA;
        const float dphB = -(gB + phB) * sB * 0.166666667f * P.dcB * sgB;
        h_c += qq * (phB - phA + P.l_ * dphA + P.l * dphB) + dqq * (P.l_ * phA + P.l * phB);
    }
    return flj - fc;
}

__device__ __forceinline__ bool sc_is_soft(int mi, int mj, float2 a, float2 b) {
    return mi != mj || (b.x > 1e-6f && a.x < 1e-6f) || (b.x < 1e-6f && a.x > 1e-6f);
}

__device__ __forceinline__ void red_fix_sc(long long* p, float v, float scale) {
    const long long q = __float2ll_rn(v * scale);
    if (q) sb_red_add(p, q);
}

// per-slot B type, mask and charge change
__device__ __forceinline__ void sc_pack_slot(int s, const int* __restrict__ slot_atom,
                                             const int* __restrict__ typeB,
                                             const int* __restrict__ mask,
                                             const float* __restrict__ dq, int* __restrict__ ext,
                                             float* __restrict__ sdq) {
    const int a = slot_atom[s];
    ext[s] = a >= 0 ? (typeB[a] | (mask[a] << 16)) : 0;
    sdq[s] = a >= 0 ? dq[a] : 0.f;
}

__global__ void k_sc_pack(const int* __restrict__ meta, const int* __restrict__ slot_atom,
                          const int* __restrict__ typeB, const int* __restrict__ mask,
                          const float* __restrict__ dq, int* __restrict__ ext,
                          float* __restrict__ sdq) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < meta[3]) sc_pack_slot(s, slot_atom, typeB, mask, dq, ext, sdq);
}

// chosen form: warp per cluster, one lane per list entry, the 8 cluster atoms in registers;
// block `blk` of 4 warps takes clusters 4 blk .. 4 blk + 3
template <int EV, bool DH>
__device__ __forceinline__ void pair_sc_block(
    const ScParams& P, int blk, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const int* __restrict__ sext, const float* __restrict__ sdq,
    const float2* __restrict__ ABa, const float2* __restrict__ ABb,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    long long* __restrict__ hfix, float* __restrict__ atom_energy,
    float* __restrict__ atom_virial, float* __restrict__ atom_direct) {
    extern __shared__ float2 sAB[];  // [ntA^2] A tables, then [ntB^2] B tables
    __shared__ int s_ta[4][SB_CLUSTER], s_tb[4][SB_CLUSTER], s_m[4][SB_CLUSTER];
    __shared__ float s_dq[4][SB_CLUSTER];
    const int na = P.ntA * P.ntA, nb = P.ntB * P.ntB;
    for (int t = threadIdx.x; t < na; t += blockDim.x) sAB[t] = ABa[t];
    for (int t = threadIdx.x; t < nb; t += blockDim.x) sAB[na + t] = ABb[t];
    __syncthreads();
    const float2* sA = sAB;
    const float2* sB = sAB + na;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blk * 4 + w;
    if (c >= meta[0]) return;
    const int base = c * SB_CLUSTER;
    const uint4 my = lane < SB_CLUSTER ? xq[base + lane] : make_uint4(0, 0, 0, 0);
    if (lane < SB_CLUSTER) {
        const int ex = sext[base + lane];
        s_ta[w][lane] = stype[base + lane] * P.ntA;
        s_tb[w][lane] = (ex & 0xffff) * P.ntB;
        s_m[w][lane] = ex >> 16;
        s_dq[w][lane] = sdq[base + lane];
    }
    __syncwarp();
    const bool exact = (cl_count[c] & SB_CL_EXACT) != 0;
    float xi[SB_CLUSTER], yi[SB_CLUSTER], zi[SB_CLUSTER], qi[SB_CLUSTER];
    uint32_t ux[SB_CLUSTER], uy[SB_CLUSTER], uz[SB_CLUSTER];
    float fxi[SB_CLUSTER], fyi[SB_CLUSTER], fzi[SB_CLUSTER];
    float el[SB_CLUSTER], ec[SB_CLUSTER], ev[SB_CLUSTER];
#pragma unroll
    for (int k = 0; k < SB_CLUSTER; k++) {
        ux[k] = __shfl_sync(0xffffffffu, my.x, k);
        uy[k] = __shfl_sync(0xffffffffu, my.y, k);
        uz[k] = __shfl_sync(0xffffffffu, my.z, k);
        qi[k] = __uint_as_float(__shfl_sync(0xffffffffu, my.w, k));
        xi[k] = __int2float_rn((int)(ux[k] - ux[0])) * P.sx;
        yi[k] = __int2float_rn((int)(uy[k] - uy[0])) * P.sy;
        zi[k] = __int2float_rn((int)(uz[k] - uz[0])) * P.sz;
        fxi[k] = fyi[k] = fzi[k] = 0.f;
        el[k] = ec[k] = ev[k] = 0.f;
    }
    float h_lj = 0.f, h_c = 0.f;
    const int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, P.ent_cap);
    const uint32_t* ents = cl_ent + (size_t)c * P.ent_cap;
    for (int e = lane; e < cnt; e += 32) {
        const uint32_t v = ents[e];
        const int j = (int)(v & 0xffffffu);
        const uint32_t m = v >> 24;
        const uint4 xj = xq[j];
        const int tja = stype[j];
        const int exj = sext[j];
        const int tjb = exj & 0xffff, mj = exj >> 16;
        const float qj = __uint_as_float(xj.w), dqj = sdq[j];
        const float xjr = __int2float_rn((int)(xj.x - ux[0])) * P.sx;
        const float yjr = __int2float_rn((int)(xj.y - uy[0])) * P.sy;
        const float zjr = __int2float_rn((int)(xj.z - uz[0])) * P.sz;
        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
#pragma unroll
        for (int k = 0; k < SB_CLUSTER; k++) {
            if (!((m >> k) & 1u)) continue;
            float dx, dy, dz;
            if (exact) {
                dx = __int2float_rn((int)(xj.x - ux[k])) * P.sx;
                dy = __int2float_rn((int)(xj.y - uy[k])) * P.sy;
                dz = __int2float_rn((int)(xj.z - uz[k])) * P.sz;
            } else {
                dx = xjr - xi[k];
                dy = yjr - yi[k];
                dz = zjr - zi[k];
            }
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (!(r2 < P.rc2)) continue;
            const float2 a = sA[s_ta[w][k] + tja];
            const float2 b = sB[s_tb[w][k] + tjb];
            const bool soft = sc_is_soft(s_m[w][k], mj, a, b);
            const float qq = qi[k] * qj;
            const float dqq = dqj * qi[k] + qj * s_dq[w][k];
            float e1 = 0.f, e2 = 0.f, v1 = 0.f;
            const float fs = sc_pair<EV != 0, DH>(P, r2, qq, dqq, soft, a, b, e1, e2, v1, h_lj, h_c);
            fxi[k] = fmaf(fs, dx, fxi[k]);
            fyi[k] = fmaf(fs, dy, fyi[k]);
            fzi[k] = fmaf(fs, dz, fzi[k]);
            fjx = fmaf(-fs, dx, fjx);
            fjy = fmaf(-fs, dy, fjy);
            fjz = fmaf(-fs, dz, fjz);
            if (EV) {
                el[k] += e1;
                ec[k] += e2;
                ev[k] += v1;
            }
        }
        red_fix_sc(&fix[j], fjx, SB_FORCE_SCALE);
        red_fix_sc(&fix[P.slot_cap + j], fjy, SB_FORCE_SCALE);
        red_fix_sc(&fix[2 * P.slot_cap + j], fjz, SB_FORCE_SCALE);
    }
#pragma unroll
    for (int k = 0; k < SB_CLUSTER; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            fxi[k] += __shfl_xor_sync(0xffffffffu, fxi[k], o);
            fyi[k] += __shfl_xor_sync(0xffffffffu, fyi[k], o);
            fzi[k] += __shfl_xor_sync(0xffffffffu, fzi[k], o);
            if (EV) {
                el[k] += __shfl_xor_sync(0xffffffffu, el[k], o);
                ec[k] += __shfl_xor_sync(0xffffffffu, ec[k], o);
                ev[k] += __shfl_xor_sync(0xffffffffu, ev[k], o);
            }
        }
        if (lane == k) {
            const int s = base + k;
            const int a = slot_atom[s];
            if (a >= 0) {
                red_fix_sc(&fix[s], fxi[k], SB_FORCE_SCALE);
                red_fix_sc(&fix[P.slot_cap + s], fyi[k], SB_FORCE_SCALE);
                red_fix_sc(&fix[2 * P.slot_cap + s], fzi[k], SB_FORCE_SCALE);
                if (EV & SB_EV_ENERGY_SC) atom_energy[a] += el[k] + ec[k];
                if (EV & SB_EV_VIRIAL_SC) {
                    atom_virial[a] += ev[k];
                    atom_direct[a] = ec[k];
                }
            }
        }
    }
    if (DH) {
        for (int o = 16; o > 0; o >>= 1) {
            h_lj += __shfl_xor_sync(0xffffffffu, h_lj, o);
            h_c += __shfl_xor_sync(0xffffffffu, h_c, o);
        }
        if (lane == 0) {
            red_fix_sc(&hfix[0], h_lj, SB_DHDL_SCALE);
            red_fix_sc(&hfix[1], h_c, SB_DHDL_SCALE);
        }
    }
}

template <int EV, bool DH>
__global__ void __launch_bounds__(128) k_pair_sc(
    ScParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const int* __restrict__ sext, const float* __restrict__ sdq,
    const float2* __restrict__ ABa, const float2* __restrict__ ABb,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    long long* __restrict__ hfix, float* __restrict__ atom_energy,
    float* __restrict__ atom_virial, float* __restrict__ atom_direct) {
    pair_sc_block<EV, DH>(P, blockIdx.x, meta, cl_count, cl_ent, xq, stype, sext, sdq, ABa, ABb,
                          slot_atom, fix, hfix, atom_energy, atom_virial, atom_direct);
}

// plain form: warp per atom over the ATOM_GROUP half list, float atomics (the reference's
// LJ_Soft_Core_Force_With_Direct_CF_CUDA structure, LJ_soft_core.cu:159-317)
struct ScAtomGroup {
    int atom_numbers;
    int* atom_serial;
};

__device__ __forceinline__ int sc_tri(int a, int b) {
    const int M = max(a, b), m = min(a, b);
    return (M * (M + 1) >> 1) + m;
}

template <int EV, bool DH>
__global__ void __launch_bounds__(256) k_pair_sc_plain(
    ScParams P, int n, const ScAtomGroup* __restrict__ nl, const uint32_t* __restrict__ uc,
    const float* __restrict__ q, const float* __restrict__ dq, const int* __restrict__ ta,
    const int* __restrict__ tb, const int* __restrict__ mask, const float* __restrict__ Aa,
    const float* __restrict__ Ba, const float* __restrict__ Ab, const float* __restrict__ Bb,
    float* __restrict__ frc, float* __restrict__ hsum, float* __restrict__ atom_energy,
    float* __restrict__ atom_virial, float* __restrict__ atom_direct) {
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n) return;
    const ScAtomGroup g = nl[i];
    const uint32_t ux = uc[3 * i], uy = uc[3 * i + 1], uz = uc[3 * i + 2];
    const float qi = q[i], dqi = dq[i];
    const int tai = ta[i], tbi = tb[i], mi = mask[i];
    float fx = 0.f, fy = 0.f, fz = 0.f, e1 = 0.f, e2 = 0.f, v1 = 0.f, h1 = 0.f, h2 = 0.f;
    for (int t = threadIdx.x; t < g.atom_numbers; t += blockDim.x) {
        const int j = g.atom_serial[t];
        const float dx = (float)(int)(uc[3 * j] - ux) * P.sx;
        const float dy = (float)(int)(uc[3 * j + 1] - uy) * P.sy;
        const float dz = (float)(int)(uc[3 * j + 2] - uz) * P.sz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (!(r2 < P.rc2)) continue;
        const int ka = sc_tri(tai, ta[j]), kb = sc_tri(tbi, tb[j]);
        const float2 a = make_float2(Aa[ka], Ba[ka]);
        const float2 b = make_float2(Ab[kb], Bb[kb]);
        const bool soft = sc_is_soft(mi, mask[j], a, b);
        const float qj = q[j];
        const float fs = sc_pair<EV != 0, DH>(P, r2, qi * qj, dq[j] * qi + qj * dqi, soft, a, b,
                                              e1, e2, v1, h1, h2);
        const float tx = fs * dx, ty = fs * dy, tz = fs * dz;
        fx += tx;
        fy += ty;
        fz += tz;
        atomicAdd(&frc[3 * j], -tx);
        atomicAdd(&frc[3 * j + 1], -ty);
        atomicAdd(&frc[3 * j + 2], -tz);
    }
    for (int o = 16; o > 0; o >>= 1) {
        fx += __shfl_down_sync(0xffffffffu, fx, o);
        fy += __shfl_down_sync(0xffffffffu, fy, o);
        fz += __shfl_down_sync(0xffffffffu, fz, o);
        if (EV) {
            e1 += __shfl_down_sync(0xffffffffu, e1, o);
            e2 += __shfl_down_sync(0xffffffffu, e2, o);
            v1 += __shfl_down_sync(0xffffffffu, v1, o);
        }
        if (DH) {
            h1 += __shfl_down_sync(0xffffffffu, h1, o);
            h2 += __shfl_down_sync(0xffffffffu, h2, o);
        }
    }
    if (threadIdx.x == 0) {
        atomicAdd(&frc[3 * i], fx);
        atomicAdd(&frc[3 * i + 1], fy);
        atomicAdd(&frc[3 * i + 2], fz);
        if (EV & SB_EV_ENERGY_SC) atom_energy[i] += e1 + e2;
        if (EV & SB_EV_VIRIAL_SC) {
            atom_virial[i] += v1;
            atom_direct[i] = e2;
        }
        if (DH) {
            atomicAdd(&hsum[0], h1);
            atomicAdd(&hsum[1], h2);
        }
    }
}

__global__ void k_sc_zero(long long* __restrict__ h, int n) {
    const int t = threadIdx.x;
    if (t < n) h[t] = 0;
}

// FP64 sums of q dq, q and dq over the box (one block of 1024 threads, fixed order) -> out[0..2]
__device__ __forceinline__ void fep_self_sums(int n, const float* __restrict__ q,
                                              const float* __restrict__ dq,
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
        out[0] = r1[0];
        out[1] = r2[0];
        out[2] = r3[0];
    }
}

// dU/dlambda: hfix [LJ, direct, reciprocal, correction] (fixed point) + the self term from the
// sums of fep_self_sums + the long-range term -> out (FP64); optionally the parts[7]
__device__ __forceinline__ void fep_combine(const long long* __restrict__ hfix,
                                            const double* __restrict__ sums, double self_coef,
                                            double neutral2, double lrc, double* __restrict__ out,
                                            double* __restrict__ parts) {
    const double lj = (double)hfix[0] * SB_DHDL_UNSCALE, dir = (double)hfix[1] * SB_DHDL_UNSCALE;
    const double rec = (double)hfix[2] * SB_DHDL_UNSCALE, cor = (double)hfix[3] * SB_DHDL_UNSCALE;
    const double self = self_coef * sums[0] + neutral2 * sums[1] * sums[2];
    if (out) out[0] = lj + dir + rec + cor + self + lrc;
    if (parts) {
        parts[0] = lj;
        parts[1] = dir;
        parts[2] = rec;
        parts[3] = self;
        parts[4] = cor;
        parts[5] = lrc;
        parts[6] = lj + dir + rec + cor + self + lrc;
    }
}

__global__ void __launch_bounds__(1024) k_fep_self(int n, const float* __restrict__ q,
                                                   const float* __restrict__ dq,
                                                   double* __restrict__ sums) {
    fep_self_sums(n, q, dq, sums);
}

__global__ void k_fep_combine(const long long* __restrict__ hfix, const double* __restrict__ sums,
                              double self_coef, double neutral2, double lrc,
                              double* __restrict__ out) {
    if (threadIdx.x == 0) fep_combine(hfix, sums, self_coef, neutral2, lrc, out, nullptr);
}

// ---------------------------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------------------------
static void sc_lrc(sb_softcore* sc) {
    // dispersion factor mixed linearly in lambda over atom-pair types (LJ_soft_core.cu:85-156)
    const int nt2 = sc->ntA > sc->ntB ? sc->ntA : sc->ntB;
    (void)nt2;
    std::vector<double> cnt((size_t)sc->ntA * sc->ntB, 0.0);
    for (int i = 0; i < sc->n; i++) cnt[(size_t)sc->htA[i] * sc->ntB + sc->htB[i]] += 1.0;
    double sa = 0, sb = 0;
    for (int a1 = 0; a1 < sc->ntA; a1++)
        for (int b1 = 0; b1 < sc->ntB; b1++) {
            const double c1 = cnt[(size_t)a1 * sc->ntB + b1];
            if (c1 == 0) continue;
            for (int a2 = 0; a2 < sc->ntA; a2++)
                for (int b2 = 0; b2 < sc->ntB; b2++) {
                    const double c2 = cnt[(size_t)a2 * sc->ntB + b2];
                    if (c2 == 0) continue;
                    const int ka = a1 > a2 ? a1 * (a1 + 1) / 2 + a2 : a2 * (a2 + 1) / 2 + a1;
                    const int kb = b1 > b2 ? b1 * (b1 + 1) / 2 + b2 : b2 * (b2 + 1) / 2 + b1;
                    sa += c1 * c2 * (double)sc->hB6a[ka];
                    sb += c1 * c2 * (double)sc->hB6b[kb];
                }
        }
    const double rc = sc->cutoff;
    const double kappa = -2.0 / 3.0 * M_PI / (rc * rc * rc) / 6.0;
    sc->lrc_factor = kappa * ((1.0 - sc->lambda) * sa + sc->lambda * sb);
    sc->lrc_ti = kappa * (sb - sa);
}

static ScParams sc_params(const sb_softcore* sc, const sb_neighbor_list* nl, float beta) {
    ScParams P;
    P.sx = (1.0f / 4294967296.0f) * nl->box[0];
    P.sy = (1.0f / 4294967296.0f) * nl->box[1];
    P.sz = (1.0f / 4294967296.0f) * nl->box[2];
    P.rc2 = sc->cutoff * sc->cutoff;
    P.beta = beta;
    P.beta2 = beta * beta;
    P.tsp_beta = (float)(2.0 * beta / sqrt(M_PI));
    P.l = sc->lambda;
    P.l_ = 1.0f - sc->lambda;
    const double l = sc->lambda, l_ = 1.0 - l, a = sc->alpha, p = sc->p;
    P.cA = (float)(a * pow(l, p));
    P.cB = (float)(a * pow(l_, p));
    P.dcA = (float)(a * p * pow(l, p - 1.0));
    P.dcB = (float)(-a * p * pow(l_, p - 1.0));
    P.s6 = (float)pow((double)sc->sigma, 6.0);
    P.s6min = (float)pow((double)sc->sigma_min, 6.0);
    const double b3 = (double)beta * beta * beta;
    const double pc[6] = {SB_EWALD_P5, SB_EWALD_P4, SB_EWALD_P3, SB_EWALD_P2, SB_EWALD_P1,
                          SB_EWALD_P0};
    for (int k = 0; k < 6; k++) P.gp[k] = (float)(b3 * pc[k]);
    const double brc = (double)beta * sc->cutoff;
    P.wide = brc * brc > 8.9;
    P.ntA = sc->ntA;
    P.ntB = sc->ntB;
    P.slot_cap = nl->slot_cap;
    P.ent_cap = nl->ent_cap;
    return P;
}

extern "C" int sb_sc_destroy(sb_softcore* sc) {
    if (!sc) return SB_OK;
    cudaDeviceSynchronize();
    void* ps[] = {sc->d_ABa, sc->d_ABb, sc->d_Aa, sc->d_Ba, sc->d_Ab, sc->d_Bb, sc->d_typeA,
                  sc->d_typeB, sc->d_mask, sc->d_dq, sc->d_slot_ext, sc->d_slot_dq, sc->d_hfix,
                  sc->d_red, sc->d_scratch_frc, sc->d_pert, sc->d_tu, sc->d_ABu,
                  sc->d_ppairs, sc->d_pcount, sc->d_sums};
    for (void* x : ps) sb_free(x);
    delete sc;
    return SB_OK;
}

static std::vector<float2> square_table(int nt, const float* A, const float* B) {
    std::vector<float2> t((size_t)nt * nt);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            const int M = a > b ? a : b, m = a > b ? b : a;
            const int k = M * (M + 1) / 2 + m;
            t[(size_t)a * nt + b] = make_float2(A[k], B[k]);
        }
    return t;
}

// The perturbed atoms of the split form: every atom with a mask or a charge change, and every
// atom whose (A type, B type) pair is not interchangeable with the other unperturbed atoms' (the
// A table between two unperturbed atoms must equal the B table between them, coefficient for
// coefficient, so that the lambda-mixed pair is the A-state pair); the rest are unperturbed.
static int sc_split_setup(sb_softcore* sc, const int* hmask, const float* hdq) {
    const int n = sc->n, ntA = sc->ntA, ntB = sc->ntB;
    std::vector<char> pert(n);
    for (int i = 0; i < n; i++) pert[i] = hmask[i] != 0 || hdq[i] != 0.f;
    auto tri = [](int a, int b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
    for (bool changed = true; changed;) {
        changed = false;
        std::vector<char> seen((size_t)ntA * ntB, 0);
        std::vector<int> combos;
        for (int i = 0; i < n; i++) {
            const int c = sc->htA[i] * ntB + sc->htB[i];
            if (!pert[i] && !seen[c]) seen[c] = 1, combos.push_back(c);
        }
        std::vector<char> bad((size_t)ntA * ntB, 0);
        for (int c1 : combos)
            for (int c2 : combos) {
                const int ka = tri(c1 / ntB, c2 / ntB), kb = tri(c1 % ntB, c2 % ntB);
                if (sc->hA12a[ka] != sc->hA12b[kb] || sc->hB6a[ka] != sc->hB6b[kb]) bad[c1] = 1;
            }
        for (int i = 0; i < n; i++)
            if (!pert[i] && bad[sc->htA[i] * ntB + sc->htB[i]]) pert[i] = 1, changed = true;
    }
    std::vector<int> plist;
    for (int i = 0; i < n; i++)
        if (pert[i]) plist.push_back(i);
    sc->npert = (int)plist.size();
    sc->split = sc->npert > 0 && sc->npert <= SB_SC_SPLIT_MAX && 8 * (long long)sc->npert <= n;
    if (!sc->split) return SB_OK;
    std::vector<int> tu(n);
    for (int i = 0; i < n; i++) tu[i] = pert[i] ? ntA : sc->htA[i];
    const int nu = ntA + 1;
    std::vector<float2> abu((size_t)nu * nu, make_float2(0.f, 0.f));
    for (int a = 0; a < ntA; a++)
        for (int b = 0; b < ntA; b++) {
            const int k = tri(a, b);
            abu[(size_t)a * nu + b] = make_float2(sc->hA12a[k], sc->hB6a[k]);
        }
    SB_TRY(sb_malloc((void**)&sc->d_pert, sizeof(int) * plist.size(), "perturbed atoms"));
    SB_TRY(sb_malloc((void**)&sc->d_tu, sizeof(int) * n, "split types"));
    SB_TRY(sb_malloc((void**)&sc->d_ABu, sizeof(float2) * abu.size(), "split table"));
    sc->pcap = sc->npert * std::min(n, SB_SC_PAIRS_PER_ATOM);
    SB_TRY(sb_malloc((void**)&sc->d_ppairs, sizeof(int2) * sc->pcap, "perturbed pairs"));
    SB_TRY(sb_malloc((void**)&sc->d_pcount, sizeof(int), "perturbed pair count"));
    SB_CHECK_CUDA(cudaMemset(sc->d_pcount, 0, sizeof(int)));
    SB_CHECK_CUDA(cudaMemcpy(sc->d_pert, plist.data(), sizeof(int) * plist.size(),
                             cudaMemcpyHostToDevice));
    SB_CHECK_CUDA(cudaMemcpy(sc->d_tu, tu.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    SB_CHECK_CUDA(cudaMemcpy(sc->d_ABu, abu.data(), sizeof(float2) * abu.size(),
                             cudaMemcpyHostToDevice));
    return SB_OK;
}

extern "C" int sb_sc_create(int n, int ntA, const float* hAA, const float* hAB, int ntB,
                            const float* hBA, const float* hBB, const int* htA, const int* htB,
                            const int* hmask, const float* hdq, float cutoff,
                            const float box_length[3], float lambda, float alpha, float p,
                            float sigma, float sigma_min, int form, sb_softcore** out) {
    if (!out || n <= 0 || ntA <= 0 || ntB <= 0 || !hAA || !hAB || !hBA || !hBB || !htA ||
        !htB || !hmask || !hdq || !box_length || cutoff <= 0 || ntB > 0xffff) {
        sb_set_error("sb_sc_create: invalid argument");
        return SB_ERR_ARG;
    }
    for (int i = 0; i < n; i++)
        if (htA[i] < 0 || htA[i] >= ntA || htB[i] < 0 || htB[i] >= ntB || hmask[i] < 0 ||
            hmask[i] > 0x7fff) {
            sb_set_error("sb_sc_create: atom %d has types (%d, %d) or mask %d out of range", i,
                         htA[i], htB[i], hmask[i]);
            return SB_ERR_ARG;
        }
    if ((size_t)(ntA * ntA + ntB * ntB) * sizeof(float2) > 96 * 1024) {
        sb_set_error("sb_sc_create: LJ type tables too large for shared memory");
        return SB_ERR_ARG;
    }
    sb_softcore* sc = new sb_softcore();
    sc->n = n;
    sc->ntA = ntA;
    sc->ntB = ntB;
    sc->form = form;
    sc->cutoff = cutoff;
    for (int d = 0; d < 3; d++) sc->box[d] = box_length[d];
    sc->lambda = lambda;
    sc->alpha = alpha;
    sc->p = p;
    sc->sigma = sigma;
    sc->sigma_min = sigma_min;
    const int npa = ntA * (ntA + 1) / 2, npb = ntB * (ntB + 1) / 2;
    sc->hA12a.assign(hAA, hAA + npa);
    sc->hB6a.assign(hAB, hAB + npa);
    sc->hA12b.assign(hBA, hBA + npb);
    sc->hB6b.assign(hBB, hBB + npb);
    sc->htA.assign(htA, htA + n);
    sc->htB.assign(htB, htB + n);
    const std::vector<float2> ta = square_table(ntA, hAA, hAB), tb = square_table(ntB, hBA, hBB);
    int st = SB_OK;
    if ((st = sb_malloc((void**)&sc->d_ABa, sizeof(float2) * ta.size(), "soft-core A table")) ||
        (st = sb_malloc((void**)&sc->d_ABb, sizeof(float2) * tb.size(), "soft-core B table")) ||
        (st = sb_malloc((void**)&sc->d_Aa, sizeof(float) * npa, "soft-core AA")) ||
        (st = sb_malloc((void**)&sc->d_Ba, sizeof(float) * npa, "soft-core AB")) ||
        (st = sb_malloc((void**)&sc->d_Ab, sizeof(float) * npb, "soft-core BA")) ||
        (st = sb_malloc((void**)&sc->d_Bb, sizeof(float) * npb, "soft-core BB")) ||
        (st = sb_malloc((void**)&sc->d_typeA, sizeof(int) * n, "soft-core type A")) ||
        (st = sb_malloc((void**)&sc->d_typeB, sizeof(int) * n, "soft-core type B")) ||
        (st = sb_malloc((void**)&sc->d_mask, sizeof(int) * n, "soft-core mask")) ||
        (st = sb_malloc((void**)&sc->d_dq, sizeof(float) * n, "soft-core dq")) ||
        (st = sb_malloc((void**)&sc->d_hfix, sizeof(long long) * 4, "dH/dlambda")) ||
        (st = sb_malloc((void**)&sc->d_red, sizeof(double) * 8, "soft-core reduce")) ||
        (st = sb_malloc((void**)&sc->d_sums, sizeof(double) * 3, "FEP self sums"))) {
        sb_sc_destroy(sc);
        return st;
    }
    cudaMemcpy(sc->d_ABa, ta.data(), sizeof(float2) * ta.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_ABb, tb.data(), sizeof(float2) * tb.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_Aa, hAA, sizeof(float) * npa, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_Ba, hAB, sizeof(float) * npa, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_Ab, hBA, sizeof(float) * npb, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_Bb, hBB, sizeof(float) * npb, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_typeA, htA, sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_typeB, htB, sizeof(int) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(sc->d_mask, hmask, sizeof(int) * n, cudaMemcpyHostToDevice);
    const cudaError_t e = cudaMemcpy(sc->d_dq, hdq, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        sb_set_error("sb_sc_create: %s", cudaGetErrorString(e));
        sb_sc_destroy(sc);
        return SB_ERR_CUDA;
    }
    sc_lrc(sc);
    if ((st = sc_split_setup(sc, hmask, hdq))) {
        sb_sc_destroy(sc);
        return st;
    }
    *out = sc;
    return SB_OK;
}

extern "C" int sb_sc_split_form(const sb_softcore* sc, int* h_split, int* h_n_perturbed) {
    if (!sc || !h_split || !h_n_perturbed) {
        sb_set_error("sb_sc_split_form: null argument");
        return SB_ERR_ARG;
    }
    *h_split = sc->split;
    *h_n_perturbed = sc->npert;
    return SB_OK;
}

extern "C" int sb_sc_set_lambda(sb_softcore* sc, float lambda) {
    if (!sc || !(lambda >= 0.f && lambda <= 1.f)) {
        sb_set_error("sb_sc_set_lambda: lambda must lie in [0, 1]");
        return SB_ERR_ARG;
    }
    sc->lambda = lambda;
    sc_lrc(sc);
    return SB_OK;
}

// per-slot extras sized for the list (re-created when a list with more slots comes along)
static int sc_slots_alloc(sb_softcore* sc, const sb_neighbor_list* nl) {
    if (sc->slot_cap < nl->slot_cap) {
        sb_free(sc->d_slot_ext);
        sb_free(sc->d_slot_dq);
        sc->d_slot_ext = nullptr;
        sc->d_slot_dq = nullptr;
        sc->slot_cap = 0;
        SB_TRY(sb_malloc((void**)&sc->d_slot_ext, sizeof(int) * nl->slot_cap, "soft-core slots"));
        SB_TRY(sb_malloc((void**)&sc->d_slot_dq, sizeof(float) * nl->slot_cap, "soft-core slots"));
        sc->slot_cap = nl->slot_cap;
    }
    return SB_OK;
}

static int sc_slots(sb_softcore* sc, sb_neighbor_list* nl, cudaStream_t s) {
    SB_TRY(sc_slots_alloc(sc, nl));
    k_sc_pack<<<(nl->slot_cap + 255) / 256, 256, 0, s>>>(nl->meta, nl->slot_atom, sc->d_typeB,
                                                         sc->d_mask, sc->d_dq, sc->d_slot_ext,
                                                         sc->d_slot_dq);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

// fixed form: pack + soft-core pair kernel into the list's fixed-point force buffer
static int sc_pair_fixed(sb_softcore* sc, sb_neighbor_list* nl, float beta, int ev, bool dh,
                         float* ae, float* av, float* ad, cudaStream_t s) {
    const ScParams P = sc_params(sc, nl, beta);
    const size_t smem = sizeof(float2) * (size_t)(sc->ntA * sc->ntA + sc->ntB * sc->ntB);
    const int blocks = (nl->clu_cap + 3) / 4;
#define SB_LAUNCH_SC(EVV, DHV)                                                                   \
    do {                                                                                         \
        if (smem > 40 * 1024)                                                                    \
            cudaFuncSetAttribute(k_pair_sc<EVV, DHV>,                                            \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);        \
        k_pair_sc<EVV, DHV><<<blocks, 128, smem, s>>>(                                           \
            P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, sc->d_slot_ext,            \
            sc->d_slot_dq, sc->d_ABa, sc->d_ABb, nl->slot_atom, nl->fix, sc->d_hfix, ae, av, ad); \
    } while (0)
    if (dh) {
        switch (ev) {
            case 0: SB_LAUNCH_SC(0, true); break;
            case 1: SB_LAUNCH_SC(1, true); break;
            case 2: SB_LAUNCH_SC(2, true); break;
            default: SB_LAUNCH_SC(3, true); break;
        }
    } else {
        switch (ev) {
            case 0: SB_LAUNCH_SC(0, false); break;
            case 1: SB_LAUNCH_SC(1, false); break;
            case 2: SB_LAUNCH_SC(2, false); break;
            default: SB_LAUNCH_SC(3, false); break;
        }
    }
#undef SB_LAUNCH_SC
    SB_CHECK_LAUNCH();
    return SB_OK;
}

static int sc_launch_fixed(sb_softcore* sc, sb_neighbor_list* nl, const uint32_t* uc,
                           const float* q, float beta, int ev, bool dh, float* ae, float* av,
                           float* ad, cudaStream_t s) {
    SB_TRY(sb_nl_pack(nl, uc, q, sc->d_typeA, s));
    SB_TRY(sc_slots(sc, nl, s));
    return sc_pair_fixed(sc, nl, beta, ev, dh, ae, av, ad, s);
}

// plain form: ATOM_GROUP walk with float atomics; dH/dlambda into d_red (float pair [0..1])
static int sc_launch_plain(sb_softcore* sc, sb_neighbor_list* nl, const uint32_t* uc,
                           const float* q, float* frc, float beta, int ev, bool dh, float* ae,
                           float* av, float* ad, cudaStream_t s) {
    SB_TRY(sb_nl_build_atom_group(nl, s));
    const ScParams P = sc_params(sc, nl, beta);
    const dim3 blk(32, 8);
    const int grid = (sc->n + 7) / 8;
    float* hsum = (float*)sc->d_red;
#define SB_LAUNCH_SCP(EVV, DHV)                                                                  \
    k_pair_sc_plain<EVV, DHV><<<grid, blk, 0, s>>>(                                             \
        P, sc->n, (const ScAtomGroup*)nl->ag, uc, q, sc->d_dq, sc->d_typeA, sc->d_typeB,        \
        sc->d_mask, sc->d_Aa, sc->d_Ba, sc->d_Ab, sc->d_Bb, frc, hsum, ae, av, ad)
    if (dh) {
        switch (ev) {
            case 0: SB_LAUNCH_SCP(0, true); break;
            case 1: SB_LAUNCH_SCP(1, true); break;
            case 2: SB_LAUNCH_SCP(2, true); break;
            default: SB_LAUNCH_SCP(3, true); break;
        }
    } else {
        switch (ev) {
            case 0: SB_LAUNCH_SCP(0, false); break;
            case 1: SB_LAUNCH_SCP(1, false); break;
            case 2: SB_LAUNCH_SCP(2, false); break;
            default: SB_LAUNCH_SCP(3, false); break;
        }
    }
#undef SB_LAUNCH_SCP
    SB_CHECK_LAUNCH();
    return SB_OK;
}

__global__ void k_sc_zero_f(int n, float* p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.f;
}

extern "C" int sb_sc_pme_direct_force(sb_softcore* sc, sb_neighbor_list* nl, int atom_numbers,
                                      const uint32_t* d_uint_crd, const float* d_charge,
                                      float* d_frc, float pme_beta, int need_atom_energy,
                                      float* d_atom_energy, int need_virial,
                                      float* d_atom_lj_virial, float* d_atom_direct_pme_energy,
                                      void* stream) {
    if (!sc || !nl || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_sc_pme_direct_force: null argument");
        return SB_ERR_ARG;
    }
    if (atom_numbers != sc->n || nl->n != sc->n) {
        sb_set_error("sb_sc_pme_direct_force: atom count %d does not match the modules (%d, %d)",
                     atom_numbers, sc->n, nl->n);
        return SB_ERR_ARG;
    }
    if ((need_atom_energy > 0 && !d_atom_energy) ||
        (need_virial > 0 && (!d_atom_lj_virial || !d_atom_direct_pme_energy))) {
        sb_set_error("sb_sc_pme_direct_force: energy/virial output missing");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    const int ev = (need_atom_energy > 0 ? SB_EV_ENERGY_SC : 0) |
                   (need_virial > 0 ? SB_EV_VIRIAL_SC : 0);
    if (sc->form == SB_FORM_PLAIN)
        return sc_launch_plain(sc, nl, d_uint_crd, d_charge, d_frc, pme_beta, ev, false,
                               d_atom_energy, d_atom_lj_virial, d_atom_direct_pme_energy, s);
    SB_TRY(sc_launch_fixed(sc, nl, d_uint_crd, d_charge, pme_beta, ev, false, d_atom_energy,
                           d_atom_lj_virial, d_atom_direct_pme_energy, s));
    return sb_nl_finalize_forces(nl, d_frc, s);
}

__global__ void k_sc_device_add(float* p, float v) { p[0] += v; }

extern "C" int sb_sc_long_range_correction(sb_softcore* sc, int need_pressure, float* d_virial,
                                           int need_potential, float* d_potential,
                                           void* stream) {
    if (!sc) {
        sb_set_error("sb_sc_long_range_correction: null handle");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const double V = (double)sc->box[0] * sc->box[1] * sc->box[2];
    if (need_pressure > 0) {
        if (!d_virial) {
            sb_set_error("sb_sc_long_range_correction: d_virial is NULL");
            return SB_ERR_ARG;
        }
        k_sc_device_add<<<1, 1, 0, s>>>(d_virial, (float)(sc->lrc_factor * 6.0 / V));
        SB_CHECK_LAUNCH();
    }
    if (need_potential > 0) {
        if (!d_potential) {
            sb_set_error("sb_sc_long_range_correction: d_potential is NULL");
            return SB_ERR_ARG;
        }
        k_sc_device_add<<<1, 1, 0, s>>>(d_potential, (float)(sc->lrc_factor / V));
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

__global__ void k_sc_hsum(const float* __restrict__ hf, const long long* __restrict__ hfix,
                          int plain, double* __restrict__ out) {
    if (threadIdx.x == 0) {
        out[0] = plain ? (double)hf[0] : (double)hfix[0] * SB_DHDL_UNSCALE;
        out[1] = plain ? (double)hf[1] : (double)hfix[1] * SB_DHDL_UNSCALE;
    }
}

extern "C" int sb_sc_dh_dlambda(sb_softcore* sc, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                                const float* d_charge, float pme_beta, double* h_dhdl,
                                void* stream) {
    if (!sc || !nl || !d_uint_crd || !d_charge || !h_dhdl) {
        sb_set_error("sb_sc_dh_dlambda: null argument");
        return SB_ERR_ARG;
    }
    if (nl->n != sc->n) {
        sb_set_error("sb_sc_dh_dlambda: the list has %d atoms, the module %d", nl->n, sc->n);
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    const int plain = sc->form == SB_FORM_PLAIN;
    if (plain) {
        if (!sc->d_scratch_frc)
            SB_TRY(sb_malloc((void**)&sc->d_scratch_frc, sizeof(float) * 3 * sc->n, "dH scratch"));
        SB_CHECK_CUDA(cudaMemsetAsync(sc->d_red, 0, sizeof(double) * 8, s));
        SB_TRY(sc_launch_plain(sc, nl, d_uint_crd, d_charge, sc->d_scratch_frc, pme_beta, 0, true,
                               nullptr, nullptr, nullptr, s));
    } else {
        k_sc_zero<<<1, 32, 0, s>>>(sc->d_hfix, 4);
        SB_CHECK_LAUNCH();
        SB_TRY(sc_launch_fixed(sc, nl, d_uint_crd, d_charge, pme_beta, 0, true, nullptr, nullptr,
                               nullptr, s));
        // the pass also accumulated forces: discard them
        SB_CHECK_CUDA(cudaMemsetAsync(nl->fix, 0, sizeof(long long) * 3 * nl->slot_cap, s));
    }
    k_sc_hsum<<<1, 32, 0, s>>>((const float*)sc->d_red, sc->d_hfix, plain, sc->d_red + 4);
    SB_CHECK_LAUNCH();
    double h[2];
    SB_CHECK_CUDA(cudaMemcpyAsync(h, sc->d_red + 4, sizeof(h), cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    const double V = (double)sc->box[0] * sc->box[1] * sc->box[2];
    h_dhdl[0] = h[0];
    h_dhdl[1] = h[1];
    h_dhdl[2] = sc->lrc_ti / V;
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// The fused FEP step of one box (sb_fep_step) and of many boxes (sb_fep_batch_*). Both run the
// same device code on a descriptor of the box (SbFepBox): the pack (slot-order coordinates,
// charges and types, the soft-core slot extras, dH/dlambda accumulators cleared), the pair
// stage, the reciprocal chain, the finalize and the dU/dlambda finish. In the split form the
// pair stage is the packed LJ + Ewald kernel over the unperturbed pairs (the perturbed atoms
// packed as an uncharged ghost type) plus the soft-core pass over the perturbed atoms; without
// it, the soft-core cluster kernel over all pairs.
// ---------------------------------------------------------------------------------------------
// slot s (< slot_cap) of a box; its atom a and prune snapshot o are loaded by the caller, beside
// the slot count
__device__ __forceinline__ void fep_pack_one(int s, int a, uint4 o, const SbFepBox& b) {
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    int t = 0;
    if (a >= 0) {
        v.x = b.uc[3 * a];
        v.y = b.uc[3 * a + 1];
        v.z = b.uc[3 * a + 2];
        t = b.split ? b.tu[a] : b.typeA[a];
        v.w = (b.split && t == b.ghost) ? 0u : __float_as_uint(b.q[a]);
        if (b.xq_prune) {
            const float dx = __int2float_rn((int)(v.x - o.x)) * b.usx;
            const float dy = __int2float_rn((int)(v.y - o.y)) * b.usy;
            const float dz = __int2float_rn((int)(v.z - o.z)) * b.usz;
            if (dx * dx + dy * dy + dz * dz > b.move2) b.meta[6] = 1;
        }
    }
    b.xq[s] = v;
    b.stype[s] = t;
    b.slot_ext[s] = a >= 0 ? (b.typeB[a] | (b.mask[a] << 16)) : 0;
    b.slot_dq[s] = a >= 0 ? b.dq[a] : 0.f;
}

__device__ __forceinline__ void fep_pack_slot(int s, const SbFepBox& b) {
    if (s >= b.slot_cap) return;
    const int a = b.slot_atom[s];
    const uint4 o = b.xq_prune ? b.xq_prune[s] : make_uint4(0u, 0u, 0u, 0u);
    if (s < b.meta[3]) fep_pack_one(s, a, o, b);
}

__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS) k_fep_pack(SbFepBox b, int dh) {
    const int s = blockIdx.x * SB_FEP_BATCH_THREADS + threadIdx.x;
    if (dh && blockIdx.x == 0 && threadIdx.x < 4) b.hfix[threadIdx.x] = 0;
    if (b.split && blockIdx.x == 0 && threadIdx.x == 4) b.pcount[0] = 0;
    fep_pack_slot(s, b);
}

// pair {a < b} is excluded iff b is in a's exclusion list (the list's rule)
__device__ __forceinline__ bool sc_excluded(int a, int b, const SbExclPass& X) {
    if (!X.es) return false;
    const int k0 = X.es[a], k1 = k0 + X.en[a];
    for (int k = k0; k < k1; k++)
        if (X.el[k] == b) return true;
    return false;
}

// Soft-core pass of the split form, in two launches. The search (block `blk` of 256 list
// slots, slot order being spatial): for each perturbed atom p (staged in shared memory, 256 at a
// time) every lane tests its slot's atom j and the hits (pairs inside the cut-off at the current
// coordinates, not excluded, a pair of two perturbed atoms taken once as p < j) are appended to
// the box's pair buffer, a warp's hits at once. The evaluation: one pair per thread, forces and
// dH/dlambda (LJ, direct: hfix[0..1]) converted to fixed point pair by pair, so the result does
// not depend on the order of the buffer.
#define SB_SC_PERT_CHUNK 256
#define SB_SC_EVAL_BLOCKS 32  // evaluation blocks per box (grid-stride over its pairs)
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// squared distance from x to the interval [lo, hi] on one periodic axis of length L, x and the
// interval being minimum images relative to the same point (so the pair vector is one of x's
// images shifted by -L, 0 or +L)
__device__ __forceinline__ float axis_gap2(float x, float lo, float hi, float L) {
    float g = 3.0e38f;
#pragma unroll
    for (int k = -1; k <= 1; k++) {
        const float y = x + (float)k * L;
        const float d = fmaxf(fmaxf(lo - y, y - hi), 0.f);
        g = fminf(g, d);
    }
    return g * g;
}

__device__ __forceinline__ void sc_pert_find(const ScParams& P, int blk, const SbFepBox& b) {
    constexpr int T = SB_FEP_BATCH_THREADS;
    __shared__ uint32_t s_u[3][SB_SC_PERT_CHUNK];
    __shared__ int s_idx[SB_SC_PERT_CHUNK];
    const int lane = threadIdx.x & 31;
    const int sj = blk * T + threadIdx.x;
    const int j = sj < b.meta[3] ? b.slot_atom[sj] : -1;
    const bool in = j >= 0;
    uint32_t ux = 0, uy = 0, uz = 0;
    bool pj = false;
    if (in) {
        const uint4 u = b.xq[sj];  // packed by this step
        ux = u.x;
        uy = u.y;
        uz = u.z;
        pj = b.tu[j] == b.ghost;
    }
    // the warp's bounding box, relative to its first atom (minimum images)
    const unsigned live = __ballot_sync(0xffffffffu, in);
    const int l0 = live ? __ffs(live) - 1 : 0;
    const uint32_t rx = __shfl_sync(0xffffffffu, ux, l0);
    const uint32_t ry = __shfl_sync(0xffffffffu, uy, l0);
    const uint32_t rz = __shfl_sync(0xffffffffu, uz, l0);
    const float ox = in ? __int2float_rn((int)(ux - rx)) * P.sx : 0.f;
    const float oy = in ? __int2float_rn((int)(uy - ry)) * P.sy : 0.f;
    const float oz = in ? __int2float_rn((int)(uz - rz)) * P.sz : 0.f;
    const float lox = warp_min(ox), hix = warp_max(ox);
    const float loy = warp_min(oy), hiy = warp_max(oy);
    const float loz = warp_min(oz), hiz = warp_max(oz);
    const float Lx = P.sx * 4294967296.0f, Ly = P.sy * 4294967296.0f, Lz = P.sz * 4294967296.0f;
    const float cut2 = 1.01f * P.rc2;  // margin over the rounding of the two distance forms
    for (int c0 = 0; c0 < b.npert; c0 += SB_SC_PERT_CHUNK) {
        const int nc = min(SB_SC_PERT_CHUNK, b.npert - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < nc; t += T) {
            const int p = b.pert[c0 + t];
            s_idx[t] = p;
            s_u[0][t] = b.uc[3 * p];
            s_u[1][t] = b.uc[3 * p + 1];
            s_u[2][t] = b.uc[3 * p + 2];
        }
        __syncthreads();
        if (!live) continue;
        for (int k0 = 0; k0 < nc; k0 += 32) {
            // lane l screens perturbed atom k0 + l against the warp's box
            bool near = false;
            if (k0 + lane < nc) {
                const int k = k0 + lane;
                const float px = __int2float_rn((int)(s_u[0][k] - rx)) * P.sx;
                const float py = __int2float_rn((int)(s_u[1][k] - ry)) * P.sy;
                const float pz = __int2float_rn((int)(s_u[2][k] - rz)) * P.sz;
                near = axis_gap2(px, lox, hix, Lx) + axis_gap2(py, loy, hiy, Ly) +
                           axis_gap2(pz, loz, hiz, Lz) <
                       cut2;
            }
            unsigned cand = __ballot_sync(0xffffffffu, near);
            while (cand) {
                const int k = k0 + __ffs(cand) - 1;
                cand &= cand - 1;
                const int p = s_idx[k];
                bool hit = false;
                if (in && p != j && !(pj && j < p)) {
                    const float dx = __int2float_rn((int)(ux - s_u[0][k])) * P.sx;
                    const float dy = __int2float_rn((int)(uy - s_u[1][k])) * P.sy;
                    const float dz = __int2float_rn((int)(uz - s_u[2][k])) * P.sz;
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    hit = r2 < P.rc2 && !sc_excluded(min(p, j), max(p, j), b.X);
                }
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (m) {
                    int base = 0;
                    if (lane == 0) base = atomicAdd(b.pcount, __popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    const int at = base + __popc(m & ((1u << lane) - 1u));
                    if (hit) {
                        if (at < b.pcap)
                            b.ppairs[at] = make_int2(c0 + k, sj);
                        else
                            atomicOr(&b.meta[1], SB_STATUS_LIST_OVERFLOW);
                    }
                }
            }
        }
    }
}

// thread e of the box's evaluation blocks takes pairs e, e + stride, ...
template <bool DH>
__device__ __forceinline__ void sc_pert_eval(const ScParams& P, int e0, int stride,
                                             const SbFepBox& b) {
    const int np = min(b.pcount[0], b.pcap);
    long long h_lj = 0, h_c = 0;
    for (int e = e0; e < np; e += stride) {
        const int2 pr = b.ppairs[e];
        const int p = b.pert[pr.x], sj = pr.y, j = b.slot_atom[sj];
        const uint4 uj = b.xq[sj];
        // d = r_j - r_p: the force on p is fs d, the force on j its opposite
        const float dx = __int2float_rn((int)(uj.x - b.uc[3 * p])) * P.sx;
        const float dy = __int2float_rn((int)(uj.y - b.uc[3 * p + 1])) * P.sy;
        const float dz = __int2float_rn((int)(uj.z - b.uc[3 * p + 2])) * P.sz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float2 a = b.ABa[b.typeA[p] * P.ntA + b.typeA[j]];
        const float2 c = b.ABb[b.typeB[p] * P.ntB + b.typeB[j]];
        const bool soft = sc_is_soft(b.mask[p], b.mask[j], a, c);
        const float qp = b.q[p], qj = b.q[j];
        float e1 = 0.f, e2 = 0.f, v1 = 0.f, hl = 0.f, hc = 0.f;
        const float fs = sc_pair<false, DH>(P, r2, qp * qj, b.dq[j] * qp + qj * b.dq[p], soft,
                                            a, c, e1, e2, v1, hl, hc);
        const float tx = fs * dx, ty = fs * dy, tz = fs * dz;
        const int sp = b.X.atom_slot[p];
        red_fix_sc(&b.fix[sp], tx, SB_FORCE_SCALE);
        red_fix_sc(&b.fix[b.slot_cap + sp], ty, SB_FORCE_SCALE);
        red_fix_sc(&b.fix[2 * b.slot_cap + sp], tz, SB_FORCE_SCALE);
        red_fix_sc(&b.fix[sj], -tx, SB_FORCE_SCALE);
        red_fix_sc(&b.fix[b.slot_cap + sj], -ty, SB_FORCE_SCALE);
        red_fix_sc(&b.fix[2 * b.slot_cap + sj], -tz, SB_FORCE_SCALE);
        if (DH) {
            h_lj += __float2ll_rn(hl * SB_DHDL_SCALE);
            h_c += __float2ll_rn(hc * SB_DHDL_SCALE);
        }
    }
    if (DH) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            h_lj += __shfl_xor_sync(0xffffffffu, h_lj, o);
            h_c += __shfl_xor_sync(0xffffffffu, h_c, o);
        }
        if ((threadIdx.x & 31) == 0) {
            if (h_lj) atomicAdd((unsigned long long*)&b.hfix[0], (unsigned long long)h_lj);
            if (h_c) atomicAdd((unsigned long long*)&b.hfix[1], (unsigned long long)h_c);
        }
    }
}

__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS) k_sc_pert_find(ScParams P, SbFepBox b) {
    sc_pert_find(P, blockIdx.x, b);
}

template <bool DH>
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS) k_sc_pert_eval(ScParams P, SbFepBox b) {
    sc_pert_eval<DH>(P, blockIdx.x * SB_FEP_BATCH_THREADS + threadIdx.x,
                     gridDim.x * SB_FEP_BATCH_THREADS, b);
}

static SbFepBox fep_box_desc(sb_neighbor_list* nl, sb_softcore* sc, sb_pme* p, const uint32_t* uc,
                             const float* q, const int* es, const int* el, const int* en,
                             float* frc, double* dudl) {
    SbFepBox d{};
    d.meta = nl->meta;
    d.cl_count = nl->cl_count;
    d.cl_ent = nl->cl_ent;
    d.xq = nl->xq;
    d.stype = nl->stype;
    d.slot_atom = nl->slot_atom;
    d.fix = nl->fix;
    const bool pr = nl->prune_buffer > 0.f;
    d.xq_prune = pr ? nl->xq_prune : nullptr;
    const float half = 0.5f * nl->prune_buffer;
    d.move2 = half * half;
    d.usx = (1.0f / 4294967296.0f) * nl->box[0];
    d.usy = (1.0f / 4294967296.0f) * nl->box[1];
    d.usz = (1.0f / 4294967296.0f) * nl->box[2];
    d.slot_cap = nl->slot_cap;
    d.typeA = sc->d_typeA;
    d.typeB = sc->d_typeB;
    d.mask = sc->d_mask;
    d.dq = sc->d_dq;
    d.slot_ext = sc->d_slot_ext;
    d.slot_dq = sc->d_slot_dq;
    d.ABa = sc->d_ABa;
    d.ABb = sc->d_ABb;
    d.hfix = sc->d_hfix;
    d.sums = sc->d_sums;
    d.split = sc->split && sb_pair_fep_packed(nl, sc->cutoff, p->beta);
    d.ghost = sc->ntA;
    d.tu = sc->d_tu;
    d.ABu = sc->d_ABu;
    d.pert = sc->d_pert;
    d.npert = sc->npert;
    d.ppairs = sc->d_ppairs;
    d.pcount = sc->d_pcount;
    d.pcap = sc->pcap;
    d.qfix = p->d_qfix;
    d.theta = p->d_theta;
    d.K0 = p->K[0];
    d.K1 = p->K[1];
    d.K2 = p->K[2];
    d.ix = (float)p->K[0] / p->box[0];
    d.iy = (float)p->K[1] / p->box[1];
    d.iz = (float)p->K[2] / p->box[2];
    const float be = p->beta;
    const bool excl = es && el && en;
    d.X = SbExclPass{nl->slot_atom, nl->atom_slot, excl ? es : nullptr, excl ? el : nullptr,
                     excl ? en : nullptr, (1.0f / 4294967296.0f) * p->box[0],
                     (1.0f / 4294967296.0f) * p->box[1], (1.0f / 4294967296.0f) * p->box[2],
                     be, be * be, be * be * be, nullptr};
    d.uc = uc;
    d.q = q;
    d.frc = frc;
    d.dudl = dudl;
    d.n = nl->n;
    d.self_coef = -2.0 * (double)be / sqrt(M_PI);
    d.neutral2 = 2.0 * p->neutralizing_factor;
    const double V = (double)sc->box[0] * sc->box[1] * sc->box[2];
    d.lrc = sc->lrc_ti / V;
    return d;
}

extern "C" int sb_fep_step(sb_neighbor_list* nl, sb_softcore* sc, sb_pme* pme,
                           const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                           const int* el, const int* en, float* d_frc, double* d_dudl,
                           void* stream) {
    if (!nl || !sc || !pme || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_fep_step: null argument");
        return SB_ERR_ARG;
    }
    if (nl->n != sc->n || pme->n != sc->n) {
        sb_set_error("sb_fep_step: modules disagree on the atom count");
        return SB_ERR_ARG;
    }
    if (nl->form != SB_FORM_FIXED || sc->form != SB_FORM_FIXED || pme->form != SB_FORM_FIXED) {
        sb_set_error("sb_fep_step: needs the fixed-point form of all modules");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    SB_TRY(sc_slots_alloc(sc, nl));
    cudaStream_t s = sb_stream(stream);
    const bool dh = d_dudl != nullptr;
    const SbFepBox d = fep_box_desc(nl, sc, pme, d_uint_crd, d_charge, es, el, en, d_frc, d_dudl);
    k_fep_pack<<<(nl->slot_cap + SB_FEP_BATCH_THREADS - 1) / SB_FEP_BATCH_THREADS,
                 SB_FEP_BATCH_THREADS, 0, s>>>(d, dh ? 1 : 0);
    SB_CHECK_LAUNCH();
    if (d.split) {
        SB_TRY(sb_pair_fep(nl, sc->d_ABu, sc->ntA + 1, sc->cutoff, pme->beta, s));
        const ScParams P = sc_params(sc, nl, pme->beta);
        const int blocks = (nl->slot_cap + SB_FEP_BATCH_THREADS - 1) / SB_FEP_BATCH_THREADS;
        k_sc_pert_find<<<blocks, SB_FEP_BATCH_THREADS, 0, s>>>(P, d);
        SB_CHECK_LAUNCH();
        if (dh)
            k_sc_pert_eval<true><<<SB_SC_EVAL_BLOCKS, SB_FEP_BATCH_THREADS, 0, s>>>(P, d);
        else
            k_sc_pert_eval<false><<<SB_SC_EVAL_BLOCKS, SB_FEP_BATCH_THREADS, 0, s>>>(P, d);
        SB_CHECK_LAUNCH();
    } else {
        SB_TRY(sc_pair_fixed(sc, nl, pme->beta, 0, dh, nullptr, nullptr, nullptr, s));
    }
    SB_TRY(sb_pme_fused_reciprocal(pme, nl, d_frc, d_uint_crd, d_charge, es, el, en, 0, 0,
                                   nullptr, nullptr, s));
    if (dh) {
        SB_TRY(sb_pme_ti_terms_slot(pme, nl, sc->d_slot_dq, d_uint_crd, d_charge, sc->d_dq, es,
                                    el, en, sc->d_hfix + 2, s));
        k_fep_self<<<1, 1024, 0, s>>>(sc->n, d_charge, sc->d_dq, sc->d_sums);
        SB_CHECK_LAUNCH();
        k_fep_combine<<<1, 32, 0, s>>>(sc->d_hfix, sc->d_sums, d.self_coef, d.neutral2, d.lrc,
                                       d_dudl);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched FEP step: the sb_fep_step of many boxes (windows) in one launch per stage. Each box
// keeps its own list, soft-core and PME modules; the batch gathers their device pointers and
// constants into descriptors (SbFepBox) and block tables (block -> box, block of that box), so
// that each stage's launch covers all boxes. The FFTs run one launch per stage per group of
// equal grid sizes. Every thread does what the same thread of the box's own sb_fep_step does,
// and all sums are fixed point or keep their warps: each box gets the bits of its own step.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS)
    k_fep_pack_batch(const SbFepBox* __restrict__ B, const int2* __restrict__ tab, int dh) {
    const int2 t = tab[blockIdx.x];
    const SbFepBox& b = B[t.x];
    const int s = t.y * SB_FEP_BATCH_THREADS + threadIdx.x;
    if (dh && t.y == 0 && threadIdx.x < 4) b.hfix[threadIdx.x] = 0;
    if (b.split && t.y == 0 && threadIdx.x == 4) b.pcount[0] = 0;
    fep_pack_slot(s, b);
}

// the ScParams fields that differ between the boxes of one launch
struct ScBoxVar {
    float sx, sy, sz, l, l_, cA, cB, dcA, dcB;
    int slot_cap, ent_cap;
};

// the boxes of one launch share C's other fields, which stay kernel parameters (constant-bank
// operands, as in the single-box kernels) while the box's own ones are loaded per block
__device__ __forceinline__ ScParams sc_box_params(const ScParams& C, const ScBoxVar& v) {
    ScParams P = C;
    P.sx = v.sx;
    P.sy = v.sy;
    P.sz = v.sz;
    P.l = v.l;
    P.l_ = v.l_;
    P.cA = v.cA;
    P.cB = v.cB;
    P.dcA = v.dcA;
    P.dcB = v.dcB;
    P.slot_cap = v.slot_cap;
    P.ent_cap = v.ent_cap;
    return P;
}

// soft-core cluster kernel over the boxes without the split form
template <bool DH>
__global__ void __launch_bounds__(128, 4) k_pair_sc_batch(ScParams C,
                                                          const ScBoxVar* __restrict__ V,
                                                          const SbFepBox* __restrict__ B,
                                                          const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const ScParams P = sc_box_params(C, V[t.x]);
    const SbFepBox& b = B[t.x];
    pair_sc_block<0, DH>(P, t.y, b.meta, b.cl_count, b.cl_ent, b.xq, b.stype, b.slot_ext,
                         b.slot_dq, b.ABa, b.ABb, b.slot_atom, b.fix, b.hfix, nullptr, nullptr,
                         nullptr);
}

// soft-core pass over the perturbed atoms of the split boxes: the search over their slot
// blocks, then the evaluation (SB_SC_EVAL_BLOCKS blocks per box)
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS) k_sc_pert_find_batch(
    ScParams C, const ScBoxVar* __restrict__ V, const SbFepBox* __restrict__ B,
    const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const ScParams P = sc_box_params(C, V[t.x]);
    sc_pert_find(P, t.y, B[t.x]);
}

template <bool DH>
__global__ void __launch_bounds__(SB_FEP_BATCH_THREADS) k_sc_pert_eval_batch(
    ScParams C, const ScBoxVar* __restrict__ V, const SbFepBox* __restrict__ B,
    const int2* __restrict__ tab) {
    const int2 t = tab[blockIdx.x];
    const ScParams P = sc_box_params(C, V[t.x]);
    sc_pert_eval<DH>(P, t.y * SB_FEP_BATCH_THREADS + threadIdx.x,
                     SB_SC_EVAL_BLOCKS * SB_FEP_BATCH_THREADS, B[t.x]);
}

static ScBoxVar sc_box_var(const ScParams& P) {
    return ScBoxVar{P.sx, P.sy, P.sz, P.l, P.l_, P.cA, P.cB, P.dcA, P.dcB, P.slot_cap,
                    P.ent_cap};
}

// the fields a launch takes from its first box
static bool sc_same_common(const ScParams& a, const ScParams& b) {
    if (a.rc2 != b.rc2 || a.beta != b.beta || a.beta2 != b.beta2 || a.tsp_beta != b.tsp_beta ||
        a.s6 != b.s6 || a.s6min != b.s6min || a.wide != b.wide || a.ntA != b.ntA ||
        a.ntB != b.ntB)
        return false;
    for (int k = 0; k < 6; k++)
        if (a.gp[k] != b.gp[k]) return false;
    return true;
}

// block per box: the self-term sums (they need only the charges, so they run beside the pair
// stage); then thread per box: dU/dlambda
__global__ void __launch_bounds__(1024) k_fep_self_batch(const SbFepBox* __restrict__ B) {
    const SbFepBox& b = B[blockIdx.x];
    fep_self_sums(b.n, b.q, b.dq, b.sums);
}

__global__ void k_fep_combine_batch(const SbFepBox* __restrict__ B, int nb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nb) {
        const SbFepBox& b = B[k];
        fep_combine(b.hfix, b.sums, b.self_coef, b.neutral2, b.lrc, b.dudl, nullptr);
    }
}

struct SbFftGroup {
    const SbFftPlan* plan;         // the plan of the group's first box (all share its sizes)
    std::vector<int> boxes;
    std::vector<SbFftBatchIo> io;  // what d_io holds
    SbFftBatchIo* d_io = nullptr;
    bool batched = false;          // false: the boxes' own plan calls, one after another
    int fused = 0;
};

struct sb_fep_batch {
    int nb = 0;
    int dh = 0;
    std::vector<sb_neighbor_list*> nls;
    std::vector<sb_softcore*> scs;
    std::vector<sb_pme*> pmes;
    std::vector<SbFepBox> hbox;   // what the descriptors were built from (staleness check)
    std::vector<ScParams> hP;
    std::vector<float> lam;
    std::vector<const void*> cl_ent_in;
    SbFepBox* d_box = nullptr;
    ScBoxVar* d_var = nullptr;
    int2* d_tab = nullptr;
    int off_slot = 0, n_slot = 0, off_spread = 0, n_spread = 0, off_atom = 0, n_atom = 0;
    // soft-core launches: boxes with equal common parameters (usually all); the cluster blocks
    // of their boxes without the split form and the atom blocks of their split boxes
    struct ScGroup {
        int first_box, off_pair, n_pair, off_pert, n_pert, off_eval, n_eval;
    };
    std::vector<ScGroup> sc_groups;
    SbX2Batch* x2 = nullptr;      // packed pair kernel over the split boxes
    size_t smem = 0;              // dynamic shared memory of the soft-core cluster launch
    std::vector<SbFftGroup> groups;
    // the reciprocal chain (spread, FFT groups, gather) runs beside the pair launches: on `rec`
    // (highest priority) with the FFT groups spread over `fft` streams, joined by events
    cudaStream_t rec = nullptr;
    cudaStream_t pert = nullptr;  // the soft-core passes, beside the packed pair kernel
    std::vector<cudaStream_t> fft;
    cudaEvent_t ev_start = nullptr, ev_packed = nullptr, ev_spread = nullptr, ev_rec = nullptr,
                ev_pert = nullptr;
    std::vector<cudaEvent_t> ev_fft;
};

#define SB_FEP_FFT_STREAMS 4

static void fep_batch_free(sb_fep_batch* b) {
    if (b->rec) cudaStreamSynchronize(b->rec);
    for (cudaStream_t f : b->fft) cudaStreamSynchronize(f);
    if (b->pert) cudaStreamSynchronize(b->pert);
    for (cudaStream_t f : b->fft) cudaStreamDestroy(f);
    if (b->rec) cudaStreamDestroy(b->rec);
    if (b->pert) cudaStreamDestroy(b->pert);
    for (cudaEvent_t e : {b->ev_start, b->ev_packed, b->ev_spread, b->ev_rec, b->ev_pert})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_fft) cudaEventDestroy(e);
    for (auto& g : b->groups) sb_free(g.d_io);
    sb_pair_batch_destroy(b->x2);
    sb_free(b->d_box);
    sb_free(b->d_var);
    sb_free(b->d_tab);
    delete b;
}

static void fep_tab_add(std::vector<int2>& tab, int box, int blocks) {
    for (int k = 0; k < blocks; k++) tab.push_back(make_int2(box, k));
}

extern "C" int sb_fep_batch_destroy(sb_fep_batch* b) {
    if (!b) return SB_OK;
    fep_batch_free(b);
    return SB_OK;
}

extern "C" int sb_fep_batch_create(int n_boxes, sb_neighbor_list* const* nls,
                                   sb_softcore* const* scs, sb_pme* const* pmes,
                                   const uint32_t* const* d_uint_crd,
                                   const float* const* d_charge,
                                   const int* const* d_excluded_list_start,
                                   const int* const* d_excluded_list,
                                   const int* const* d_excluded_numbers, float* const* d_frc,
                                   double* const* d_dudl, sb_fep_batch** out) {
    if (!out || n_boxes < 1 || !nls || !scs || !pmes || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_fep_batch_create: invalid argument");
        return SB_ERR_ARG;
    }
    *out = nullptr;
    for (int k = 0; k < n_boxes; k++) {
        sb_neighbor_list* nl = nls[k];
        sb_softcore* sc = scs[k];
        sb_pme* p = pmes[k];
        if (!nl || !sc || !p || !d_uint_crd[k] || !d_charge[k] || !d_frc[k]) {
            sb_set_error("sb_fep_batch_create: box %d has a null module or buffer", k);
            return SB_ERR_ARG;
        }
        if (nl->n != sc->n || p->n != sc->n) {
            sb_set_error("sb_fep_batch_create: box %d: modules disagree on the atom count", k);
            return SB_ERR_ARG;
        }
        if (nl->form != SB_FORM_FIXED || sc->form != SB_FORM_FIXED || p->form != SB_FORM_FIXED) {
            sb_set_error("sb_fep_batch_create: box %d: needs the fixed-point form of all modules",
                         k);
            return SB_ERR_ARG;
        }
        SB_TRY(sb_nl_ensure_built(nl));
    }
    sb_fep_batch* b = new sb_fep_batch();
    b->nb = n_boxes;
    b->dh = d_dudl != nullptr;
    for (int k = 0; k < n_boxes && b->dh; k++)
        if (!d_dudl[k]) {
            sb_set_error("sb_fep_batch_create: box %d has no dU/dlambda output", k);
            delete b;
            return SB_ERR_ARG;
        }
    std::vector<int2> tab;
    int st = SB_OK;
    for (int k = 0; k < n_boxes && !st; k++) {
        b->nls.push_back(nls[k]);
        b->scs.push_back(scs[k]);
        b->pmes.push_back(pmes[k]);
        st = sc_slots_alloc(scs[k], nls[k]);
        if (st) break;
        const int* es = d_excluded_list_start ? d_excluded_list_start[k] : nullptr;
        const int* el = d_excluded_list ? d_excluded_list[k] : nullptr;
        const int* en = d_excluded_numbers ? d_excluded_numbers[k] : nullptr;
        b->hbox.push_back(fep_box_desc(nls[k], scs[k], pmes[k], d_uint_crd[k], d_charge[k], es,
                                       el, en, d_frc[k], d_dudl ? d_dudl[k] : nullptr));
        b->hP.push_back(sc_params(scs[k], nls[k], pmes[k]->beta));
        b->lam.push_back(scs[k]->lambda);
        b->cl_ent_in.push_back(nls[k]->cl_ent_in);
        if (!b->hbox.back().split) {
            const size_t sm = sizeof(float2) * (size_t)(scs[k]->ntA * scs[k]->ntA +
                                                        scs[k]->ntB * scs[k]->ntB);
            b->smem = std::max(b->smem, sm);
        }
    }
    if (!st) {
        const int T = SB_FEP_BATCH_THREADS;
        b->off_slot = (int)tab.size();
        for (int k = 0; k < n_boxes; k++) fep_tab_add(tab, k, (nls[k]->slot_cap + T - 1) / T);
        b->n_slot = (int)tab.size() - b->off_slot;
        std::vector<char> done(n_boxes, 0);
        for (int k = 0; k < n_boxes; k++) {
            if (done[k]) continue;
            sb_fep_batch::ScGroup g{k, (int)tab.size(), 0, 0, 0, 0, 0};
            for (int j = k; j < n_boxes; j++)
                if (!done[j] && sc_same_common(b->hP[k], b->hP[j]) && !b->hbox[j].split)
                    fep_tab_add(tab, j, (nls[j]->clu_cap + 3) / 4);
            g.n_pair = (int)tab.size() - g.off_pair;
            g.off_pert = (int)tab.size();
            for (int j = k; j < n_boxes; j++)
                if (!done[j] && sc_same_common(b->hP[k], b->hP[j]) && b->hbox[j].split)
                    fep_tab_add(tab, j, (nls[j]->slot_cap + T - 1) / T);
            g.n_pert = (int)tab.size() - g.off_pert;
            g.off_eval = (int)tab.size();
            for (int j = k; j < n_boxes; j++)
                if (!done[j] && sc_same_common(b->hP[k], b->hP[j])) {
                    done[j] = 1;
                    if (b->hbox[j].split) fep_tab_add(tab, j, SB_SC_EVAL_BLOCKS);
                }
            g.n_eval = (int)tab.size() - g.off_eval;
            b->sc_groups.push_back(g);
        }
        b->off_spread = (int)tab.size();
        for (int k = 0; k < n_boxes; k++) fep_tab_add(tab, k, (4 * nls[k]->n + T - 1) / T);
        b->n_spread = (int)tab.size() - b->off_spread;
        b->off_atom = (int)tab.size();
        for (int k = 0; k < n_boxes; k++) fep_tab_add(tab, k, (nls[k]->n + T - 1) / T);
        b->n_atom = (int)tab.size() - b->off_atom;
        if (b->smem > 200 * 1024) {
            sb_set_error("sb_fep_batch_create: LJ tables too large for shared memory");
            st = SB_ERR_ARG;
        }
    }
    if (!st) {
        std::vector<int> ids, nts;
        std::vector<sb_neighbor_list*> xl;
        std::vector<const float2*> tabs;
        std::vector<float> cuts, betas;
        for (int k = 0; k < n_boxes; k++) {
            if (!b->hbox[k].split) continue;
            ids.push_back(k);
            xl.push_back(nls[k]);
            tabs.push_back(scs[k]->d_ABu);
            nts.push_back(scs[k]->ntA + 1);
            cuts.push_back(scs[k]->cutoff);
            betas.push_back(pmes[k]->beta);
        }
        if (!ids.empty())
            st = sb_pair_batch_create((int)ids.size(), ids.data(), xl.data(), tabs.data(),
                                      nts.data(), cuts.data(), betas.data(), &b->x2);
    }
    // grids of equal sizes and transform family share batched FFT launches
    for (int k = 0; k < n_boxes && !st; k++) {
        const SbFftPlan* pl = &pmes[k]->plan;
        SbFftGroup* g = nullptr;
        for (auto& h : b->groups) {
            const SbFftPlan* q = h.plan;
            if (h.batched && sb_fft_batchable(pl) && q->K[0] == pl->K[0] && q->K[1] == pl->K[1] &&
                q->K[2] == pl->K[2] && q->fused == pl->fused)
                g = &h;
        }
        if (!g) {
            b->groups.push_back(SbFftGroup());
            g = &b->groups.back();
            g->plan = pl;
            g->batched = sb_fft_batchable(pl);
            g->fused = pl->fused;
        }
        g->boxes.push_back(k);
    }
    for (auto& g : b->groups) {
        if (st || !g.batched) continue;
        for (int k : g.boxes) {
            sb_pme* p = pmes[k];
            g.io.push_back(SbFftBatchIo{p->d_qfix, p->d_spec, p->d_theta, p->d_bc, nullptr});
        }
        st = sb_malloc((void**)&g.d_io, sizeof(SbFftBatchIo) * g.io.size(),
                       "FEP batch FFT table");
        if (!st && cudaMemcpy(g.d_io, g.io.data(), sizeof(SbFftBatchIo) * g.io.size(),
                              cudaMemcpyHostToDevice) != cudaSuccess) {
            sb_set_error("sb_fep_batch_create: FFT table upload failed");
            st = SB_ERR_CUDA;
        }
    }
    std::vector<ScBoxVar> var;
    for (const ScParams& P : b->hP) var.push_back(sc_box_var(P));
    if (!st) st = sb_malloc((void**)&b->d_box, sizeof(SbFepBox) * n_boxes, "FEP batch boxes");
    if (!st) st = sb_malloc((void**)&b->d_var, sizeof(ScBoxVar) * n_boxes, "FEP batch params");
    if (!st) st = sb_malloc((void**)&b->d_tab, sizeof(int2) * tab.size(), "FEP batch tables");
    if (!st && (cudaMemcpy(b->d_box, b->hbox.data(), sizeof(SbFepBox) * n_boxes,
                           cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_var, var.data(), sizeof(ScBoxVar) * n_boxes,
                           cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_tab, tab.data(), sizeof(int2) * tab.size(),
                           cudaMemcpyHostToDevice) != cudaSuccess)) {
        sb_set_error("sb_fep_batch_create: descriptor upload failed");
        st = SB_ERR_CUDA;
    }
    if (!st) {
        int lo = 0, hi = 0;
        bool ok = cudaDeviceGetStreamPriorityRange(&lo, &hi) == cudaSuccess &&
                  cudaStreamCreateWithPriority(&b->rec, cudaStreamNonBlocking, hi) == cudaSuccess &&
                  cudaStreamCreateWithPriority(&b->pert, cudaStreamNonBlocking, hi) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_pert, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_packed, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_spread, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_rec, cudaEventDisableTiming) == cudaSuccess;
        const int nf = std::min((int)b->groups.size(), SB_FEP_FFT_STREAMS);
        for (int k = 0; k < nf && ok; k++) {
            cudaStream_t f = nullptr;
            cudaEvent_t e = nullptr;
            ok = cudaStreamCreateWithPriority(&f, cudaStreamNonBlocking, hi) == cudaSuccess;
            if (ok) b->fft.push_back(f);
            ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
            if (ok) b->ev_fft.push_back(e);
        }
        if (!ok) {
            sb_set_error("sb_fep_batch_create: stream or event creation failed");
            st = SB_ERR_CUDA;
        }
    }
    if (!st && b->smem > 40 * 1024) {
        const cudaError_t e1 = cudaFuncSetAttribute(
            k_pair_sc_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
        const cudaError_t e2 = cudaFuncSetAttribute(
            k_pair_sc_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            sb_set_error("sb_fep_batch_create: shared memory attribute refused");
            st = SB_ERR_CUDA;
        }
    }
    if (st) {
        fep_batch_free(b);
        return st;
    }
    *out = b;
    return SB_OK;
}

// the descriptors still describe the modules: same buffers, capacities, box, lambda, FFT
static int fep_batch_current(const sb_fep_batch* b) {
    for (int k = 0; k < b->nb; k++) {
        const sb_neighbor_list* nl = b->nls[k];
        const sb_softcore* sc = b->scs[k];
        const sb_pme* p = b->pmes[k];
        const SbFepBox& d = b->hbox[k];
        const bool pr = nl->prune_buffer > 0.f;
        const float half = 0.5f * nl->prune_buffer;
        if (!nl->built || nl->meta != d.meta || nl->cl_ent != d.cl_ent || nl->xq != d.xq ||
            nl->fix != d.fix || nl->slot_cap != d.slot_cap || nl->ent_cap != b->hP[k].ent_cap ||
            (pr ? nl->xq_prune : nullptr) != d.xq_prune || half * half != d.move2 ||
            nl->cl_ent_in != b->cl_ent_in[k] || (1.0f / 4294967296.0f) * nl->box[0] != d.usx ||
            (1.0f / 4294967296.0f) * nl->box[1] != d.usy ||
            (1.0f / 4294967296.0f) * nl->box[2] != d.usz || sc->d_slot_ext != d.slot_ext ||
            sc->d_slot_dq != d.slot_dq || sc->lambda != b->lam[k] || p->d_qfix != d.qfix ||
            p->d_theta != d.theta || (float)p->K[0] / p->box[0] != d.ix ||
            (float)p->K[1] / p->box[1] != d.iy || (float)p->K[2] / p->box[2] != d.iz ||
            p->beta != d.X.beta) {
            sb_set_error("sb_fep_batch_step: box %d changed (box, lambda, list capacity or "
                         "pruning) since sb_fep_batch_create; create the batch again", k);
            return SB_ERR_STATE;
        }
    }
    for (const auto& g : b->groups) {
        if (!g.batched) continue;
        for (size_t i = 0; i < g.boxes.size(); i++) {
            const sb_pme* p = b->pmes[g.boxes[i]];
            const SbFftBatchIo& io = g.io[i];
            if (!sb_fft_batchable(&p->plan) || p->plan.fused != g.fused ||
                p->d_spec != io.spec || p->d_bc != io.bc) {
                sb_set_error("sb_fep_batch_step: box %d changed its FFT since "
                             "sb_fep_batch_create; create the batch again", g.boxes[i]);
                return SB_ERR_STATE;
            }
        }
    }
    return SB_OK;
}

extern "C" int sb_fep_batch_step(sb_fep_batch* b, void* stream) {
    if (!b) {
        sb_set_error("sb_fep_batch_step: null handle");
        return SB_ERR_ARG;
    }
    SB_TRY(fep_batch_current(b));
    cudaStream_t s = sb_stream(stream);
    const int2* tab = b->d_tab;
    // reciprocal chain beside the pack and the pair launches: the spread reads the atom-order
    // coordinates and charges (and the grid the last forward FFT left zero), so it starts with
    // the pack; the gather, which adds to the dU/dlambda sums the pack zeroes, waits for it. Both
    // chains add to the fixed-point force planes (order-free integer sums); the finalize waits
    // for both.
    SB_CHECK_CUDA(cudaEventRecord(b->ev_start, s));
    SB_CHECK_CUDA(cudaStreamWaitEvent(b->rec, b->ev_start, 0));
    k_fep_pack_batch<<<b->n_slot, SB_FEP_BATCH_THREADS, 0, s>>>(b->d_box, tab + b->off_slot,
                                                               b->dh);
    SB_CHECK_LAUNCH();
    SB_CHECK_CUDA(cudaEventRecord(b->ev_packed, s));
    SB_TRY(sb_pme_batch_spread(b->d_box, tab + b->off_spread, b->n_spread, b->rec));
    SB_CHECK_CUDA(cudaEventRecord(b->ev_spread, b->rec));
    const int nf = (int)b->fft.size();
    for (int k = 0; k < nf; k++) SB_CHECK_CUDA(cudaStreamWaitEvent(b->fft[k], b->ev_spread, 0));
    for (size_t gi = 0; gi < b->groups.size(); gi++) {
        const SbFftGroup& g = b->groups[gi];
        cudaStream_t f = b->fft[gi % nf];
        if (g.batched) {
            const int n = (int)g.boxes.size();
            SB_TRY(sb_fft_batch_forward(g.plan, g.d_io, n, f));
            SB_TRY(sb_fft_batch_convolve(g.plan, g.d_io, n, 0, f));
            SB_TRY(sb_fft_batch_inverse(g.plan, g.d_io, n, f));
        } else {
            for (int k : g.boxes) {
                sb_pme* p = b->pmes[k];
                SB_TRY(sb_fft_plane_forward(&p->plan, p->d_qfix, p->d_spec, f));
                SB_TRY(sb_fft_x_convolve(&p->plan, p->d_spec, p->d_bc, p->d_epart, 0, f,
                                         &p->rec_nparts));
                SB_TRY(sb_fft_plane_inverse(&p->plan, p->d_spec, p->d_theta, f));
            }
        }
    }
    for (int k = 0; k < nf; k++) {
        SB_CHECK_CUDA(cudaEventRecord(b->ev_fft[k], b->fft[k]));
        SB_CHECK_CUDA(cudaStreamWaitEvent(b->rec, b->ev_fft[k], 0));
    }
    SB_CHECK_CUDA(cudaStreamWaitEvent(b->rec, b->ev_packed, 0));
    SB_TRY(sb_pme_batch_gather(b->d_box, tab + b->off_atom, b->n_atom, b->dh, b->rec));
    SB_CHECK_CUDA(cudaEventRecord(b->ev_rec, b->rec));
    SB_CHECK_CUDA(cudaStreamWaitEvent(b->pert, b->ev_packed, 0));
    for (const auto& g : b->sc_groups) {
        if (!g.n_pert) continue;
        const ScParams& C = b->hP[g.first_box];
        k_sc_pert_find_batch<<<g.n_pert, SB_FEP_BATCH_THREADS, 0, b->pert>>>(
            C, b->d_var, b->d_box, tab + g.off_pert);
        SB_CHECK_LAUNCH();
        if (b->dh)
            k_sc_pert_eval_batch<true><<<g.n_eval, SB_FEP_BATCH_THREADS, 0, b->pert>>>(
                C, b->d_var, b->d_box, tab + g.off_eval);
        else
            k_sc_pert_eval_batch<false><<<g.n_eval, SB_FEP_BATCH_THREADS, 0, b->pert>>>(
                C, b->d_var, b->d_box, tab + g.off_eval);
        SB_CHECK_LAUNCH();
    }
    if (b->dh) {
        k_fep_self_batch<<<b->nb, 1024, 0, b->pert>>>(b->d_box);
        SB_CHECK_LAUNCH();
    }
    SB_CHECK_CUDA(cudaEventRecord(b->ev_pert, b->pert));
    if (b->x2) SB_TRY(sb_pair_batch_launch(b->x2, s));
    for (const auto& g : b->sc_groups) {
        const ScParams& C = b->hP[g.first_box];
        if (g.n_pair) {
            if (b->dh)
                k_pair_sc_batch<true><<<g.n_pair, 128, b->smem, s>>>(C, b->d_var, b->d_box,
                                                                      tab + g.off_pair);
            else
                k_pair_sc_batch<false><<<g.n_pair, 128, b->smem, s>>>(C, b->d_var, b->d_box,
                                                                       tab + g.off_pair);
            SB_CHECK_LAUNCH();
        }
    }
    SB_CHECK_CUDA(cudaStreamWaitEvent(s, b->ev_pert, 0));
    SB_CHECK_CUDA(cudaStreamWaitEvent(s, b->ev_rec, 0));
    SB_TRY(sb_pme_batch_slots(b->d_box, tab + b->off_slot, b->n_slot, b->dh, s));
    if (b->dh) {
        k_fep_combine_batch<<<(b->nb + 127) / 128, 128, 0, s>>>(b->d_box, b->nb);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_fep_batch_launches(const sb_fep_batch* b) {
    if (!b) return -1;
    // pack, spread, gather, slots (+ self sums, combine), the pair launches
    int n = 4 + (b->dh ? 2 : 0) + (b->x2 ? sb_pair_batch_launches(b->x2) : 0);
    for (const auto& g : b->sc_groups) n += (g.n_pair ? 1 : 0) + (g.n_pert ? 2 : 0);
    for (const auto& g : b->groups) {
        if (g.batched)
            n += 3 + (g.plan->fused ? 0 : 2);
        else
            n += (int)g.boxes.size() * (g.plan->fused ? 3 : 5);
    }
    return n;
}
