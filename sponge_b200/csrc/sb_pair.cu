// LJ + PME direct-space pair force/energy/virial — replaces LENNARD_JONES_INFORMATION
// (SPONGE/Lennard_Jones_force/Lennard_Jones_force.cu).
//
// Chosen form (k_pair_fixed): one warp per 8-atom i-cluster. Each lane takes one list entry
// (a j atom plus an 8-bit mask of the i atoms it pairs with), loads j with one 128-bit load,
// and loops over the 8 i atoms held in registers. Positions are taken relative to the
// cluster's first atom: the fixed-point difference is exact, its float conversion is done once
// per j instead of once per pair, and close pairs keep full relative precision. The j force is
// complete after the 8-i loop and goes out as three 64-bit fixed-point atomics; the i forces
// stay in registers for the whole list and are reduced across the warp once. Fixed-point sums
// are order independent, so forces are bit-identical run to run.
//
// Pair math (Lennard_Jones_force.cu:83-139): for dr = r_j - r_i and r < rc,
//   F_i += [ (B6 - A12 r^-6) r^-8  -  qq (erfc(br) + 2br/sqrt(pi) e^{-b^2r^2}) r^-3 ] dr
// with the Coulomb bracket evaluated as qq (r^-3 - b^3 G(b^2 r^2)) (sb_ewald.cuh).
// Energies (:508-513): A12/12 r^-12 - B6/6 r^-6 + qq erfc(br)/r; LJ virial -(LJ scalar) r^2.
//
// Plain form (k_pair_plain): the reference's structure on the per-atom ATOM_GROUP list — one
// warp per atom i, lanes striding over its j list, float atomicAdd on every j, erfcf/expf.

#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sb_ewald.cuh"
#include "sb_internal.cuh"

struct SbAtomGroupP {
    int atom_numbers;
    int* atom_serial;
};

struct PairParams {
    float sx, sy, sz;
    float rc2, rc;
    float beta, beta2, beta3;
    float gp[6];  // beta^3 x numerator coefficients of the Ewald rational (sb_ewald.cuh)
    int wide;     // (beta rc)^2 > 12: in-cutoff pairs can leave the rational's fitted range
    int nt;
    int slot_cap;
    int ent_cap;
    // pruned list (packed kernel only): rb2 = (rc + prune buffer)^2, 0 without one
    float rb2;
    int* prune;                // meta + 6: [0] prune requested, [1] set by a pruning launch
    int* cl_count_in;
    uint32_t* cl_ent_in;
    uint32_t* cl_ent_tmp;
    uint4* xq_prune;
};

#define SB_EV_ENERGY 1
#define SB_EV_VIRIAL 2

__device__ __forceinline__ void red_fix(long long* p, float v) {
    long long q = __float2ll_rn(v * SB_FORCE_SCALE);
    if (q) atomicAdd((unsigned long long*)p, (unsigned long long)q);
}
// the same without the zero test: on the per-entry j forces of the pair kernels the test costs
// more issue slots than the atomics it saves (adding zero leaves the sum unchanged)
__device__ __forceinline__ void add_fix(long long* p, float v) {
    atomicAdd((unsigned long long*)p, (unsigned long long)__float2ll_rn(v * SB_FORCE_SCALE));
}

#include "sb_pair_fixed.cuh"
#include "sb_pair_compact.cuh"
#include "sb_pair_x2.cuh"

// dynamic shared memory of a packed-kernel block: the cluster's LJ table and the prune's counts
static size_t x2_smem(int ntypes) {
    return sizeof(float4) * 4 * (size_t)ntypes + sizeof(int) * SB_PAT_COUNTS;
}

// ---------------------------------------------------------------------------------------------
// plain form: reference structure (warp per atom, float atomics), Lennard_Jones_force.cu:47-158
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int lj_pair_index(int a, int b) {
    int M = max(a, b), m = min(a, b);
    return (M * (M + 1) >> 1) + m;
}

template <int EV>
__global__ void __launch_bounds__(1024) k_pair_plain(
    int n, const SbAtomGroupP* __restrict__ nl, const uint32_t* __restrict__ uc,
    const float* __restrict__ q, const int* __restrict__ type, const float* __restrict__ A,
    const float* __restrict__ B, float sx, float sy, float sz, float cutoff, float beta,
    float* __restrict__ frc, float* __restrict__ atom_energy, float* __restrict__ atom_virial,
    float* __restrict__ atom_direct) {
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n) return;
    const SbAtomGroupP g = nl[i];
    const uint32_t ux = uc[3 * i], uy = uc[3 * i + 1], uz = uc[3 * i + 2];
    const float qi = q[i];
    const int ti = type[i];
    float fx = 0.f, fy = 0.f, fz = 0.f, el = 0.f, ed = 0.f, vr = 0.f;
    for (int t = threadIdx.x; t < g.atom_numbers; t += blockDim.x) {
        const int j = g.atom_serial[t];
        const float dx = (float)(int)(uc[3 * j] - ux) * sx;
        const float dy = (float)(int)(uc[3 * j + 1] - uy) * sy;
        const float dz = (float)(int)(uc[3 * j + 2] - uz) * sz;
        const float r = norm3df(dx, dy, dz);
        if (r < cutoff) {
            const float ri = 1.0f / r;
            const float ri2 = ri * ri;
            const float ri4 = ri2 * ri2;
            const float ri6 = ri4 * ri2;
            const float ri8 = ri4 * ri4;
            const int k = lj_pair_index(ti, type[j]);
            const float a = A[k], b = B[k];
            float fs = (-a * ri6 + b) * ri8;
            const float br = beta * r;
            const float ec = erfcf(br);
            const float qq = qi * q[j];
            const float fc = qq * (br * 1.1283791670218446f * expf(-br * br) + ec) * ri2 * ri;
            if (EV & SB_EV_ENERGY) {
                ed += qq * ec * ri;
                el += (0.083333333f * a * ri6 - 0.166666666f * b) * ri6;
            }
            if (EV & SB_EV_VIRIAL) {
                vr -= fs * r * r;
                if (!(EV & SB_EV_ENERGY)) ed += qq * ec * ri;
            }
            fs -= fc;
            const float tx = fs * dx, ty = fs * dy, tz = fs * dz;
            fx += tx;
            fy += ty;
            fz += tz;
            atomicAdd(&frc[3 * j], -tx);
            atomicAdd(&frc[3 * j + 1], -ty);
            atomicAdd(&frc[3 * j + 2], -tz);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        fx += __shfl_down_sync(0xffffffffu, fx, o);
        fy += __shfl_down_sync(0xffffffffu, fy, o);
        fz += __shfl_down_sync(0xffffffffu, fz, o);
        if (EV) {
            el += __shfl_down_sync(0xffffffffu, el, o);
            ed += __shfl_down_sync(0xffffffffu, ed, o);
            vr += __shfl_down_sync(0xffffffffu, vr, o);
        }
    }
    if (threadIdx.x == 0) {
        atomicAdd(&frc[3 * i], fx);
        atomicAdd(&frc[3 * i + 1], fy);
        atomicAdd(&frc[3 * i + 2], fz);
        if (EV & SB_EV_ENERGY) atom_energy[i] += el + ed;
        if (EV & SB_EV_VIRIAL) {
            atom_virial[i] += vr;
            atom_direct[i] = ed;
        }
    }
}

// LJ energy only (LJ_Energy_CUDA, Lennard_Jones_force.cu:964-1025) over the cluster list
__global__ void __launch_bounds__(128) k_lj_energy_fixed(
    PairParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const float2* __restrict__ AB,
    const int* __restrict__ slot_atom, float* __restrict__ atom_energy) {
    const int lane = threadIdx.x & 31;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= meta[0]) return;
    const int base = c * SB_CLUSTER;
    const uint32_t* __restrict__ ents = cl_ent + (size_t)c * P.ent_cap;
    const int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, P.ent_cap);
    for (int k = 0; k < SB_CLUSTER; k++) {
        const uint4 xi = xq[base + k];
        const int ti = stype[base + k] * P.nt;
        float e = 0.f;
        for (int t = lane; t < cnt; t += 32) {
            const uint32_t v = ents[t];
            if (!((v >> (24 + k)) & 1u)) continue;
            const int j = (int)(v & 0xffffffu);
            const uint4 xj = xq[j];
            const float dx = __int2float_rn((int)(xj.x - xi.x)) * P.sx;
            const float dy = __int2float_rn((int)(xj.y - xi.y)) * P.sy;
            const float dz = __int2float_rn((int)(xj.z - xi.z)) * P.sz;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (r2 < P.rc2) {
                const float ri2 = 1.0f / r2;
                const float ri6 = ri2 * ri2 * ri2;
                const float2 ab = AB[ti + stype[j]];
                e += (0.083333333f * ab.x * ri6 - 0.166666667f * ab.y) * ri6;
            }
        }
        for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
        if (lane == 0) {
            const int a = slot_atom[base + k];
            if (a >= 0) atom_energy[a] += e;
        }
    }
}

__global__ void k_device_add(float* p, float v) { p[0] += v; }

__global__ void k_zero_f32(int n, float* p) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.f;
}

// ---------------------------------------------------------------------------------------------
// host API
// ---------------------------------------------------------------------------------------------
extern "C" int sb_lj_create(int atom_numbers, int atom_type_numbers, const float* h_A,
                            const float* h_B, const int* h_type, float cutoff,
                            const float box_length[3], int form, sb_lennard_jones** out) {
    if (!out || atom_numbers <= 0 || atom_type_numbers <= 0 || !h_A || !h_B || !h_type ||
        !box_length || cutoff <= 0) {
        sb_set_error("sb_lj_create: invalid argument");
        return SB_ERR_ARG;
    }
    const int nt = atom_type_numbers;
    for (int i = 0; i < atom_numbers; i++)
        if (h_type[i] < 0 || h_type[i] >= nt) {
            sb_set_error("sb_lj_create: atom %d has LJ type %d outside [0, %d)", i, h_type[i], nt);
            return SB_ERR_ARG;
        }
    sb_lennard_jones* lj = new sb_lennard_jones();
    lj->n = atom_numbers;
    lj->ntypes = nt;
    lj->form = form;
    lj->cutoff = cutoff;
    for (int d = 0; d < 3; d++) lj->box[d] = box_length[d];
    lj->volume = box_length[0] * box_length[1] * box_length[2];
    const int np = nt * (nt + 1) / 2;
    std::vector<float2> ab((size_t)nt * nt);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            int M = std::max(a, b), m = std::min(a, b);
            int k = M * (M + 1) / 2 + m;
            ab[(size_t)a * nt + b] = make_float2(h_A[k], h_B[k]);
        }
    // long-range correction factor, FP64 over type counts (Lennard_Jones_force.cu:1119-1130)
    std::vector<double> cnt(nt, 0.0);
    for (int i = 0; i < atom_numbers; i++) cnt[h_type[i]] += 1.0;
    double sumB = 0;
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) sumB += cnt[a] * cnt[b] * (double)ab[(size_t)a * nt + b].y;
    lj->long_range_factor = sumB * (-2.0 / 3.0 * M_PI / ((double)cutoff * cutoff * cutoff) / 6.0);
    int st = SB_OK;
    if ((st = sb_malloc((void**)&lj->d_A, sizeof(float) * np, "LJ_A")) ||
        (st = sb_malloc((void**)&lj->d_B, sizeof(float) * np, "LJ_B")) ||
        (st = sb_malloc((void**)&lj->d_AB, sizeof(float2) * nt * nt, "LJ_AB")) ||
        (st = sb_malloc((void**)&lj->d_type, sizeof(int) * atom_numbers, "LJ type")) ||
        (st = sb_malloc((void**)&lj->d_red, sizeof(double) * 8, "LJ reduce")) ||
        (st = sb_malloc((void**)&lj->d_energy_atom, sizeof(float) * atom_numbers, "LJ energy"))) {
        sb_lj_destroy(lj);
        return st;
    }
    cudaMemcpy(lj->d_A, h_A, sizeof(float) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_B, h_B, sizeof(float) * np, cudaMemcpyHostToDevice);
    cudaMemcpy(lj->d_AB, ab.data(), sizeof(float2) * nt * nt, cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(lj->d_type, h_type, sizeof(int) * atom_numbers,
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        sb_set_error("sb_lj_create: %s", cudaGetErrorString(e));
        sb_lj_destroy(lj);
        return SB_ERR_CUDA;
    }
    *out = lj;
    return SB_OK;
}

extern "C" int sb_lj_destroy(sb_lennard_jones* lj) {
    if (!lj) return SB_OK;
    sb_free(lj->d_A);
    sb_free(lj->d_B);
    sb_free(lj->d_AB);
    sb_free(lj->d_type);
    sb_free(lj->d_red);
    sb_free(lj->d_energy_atom);
    delete lj;
    return SB_OK;
}

static PairParams pair_params_of(const sb_neighbor_list* nl, int ntypes, float cutoff,
                                 float beta) {
    PairParams P;
    P.sx = (1.0f / 4294967296.0f) * nl->box[0];
    P.sy = (1.0f / 4294967296.0f) * nl->box[1];
    P.sz = (1.0f / 4294967296.0f) * nl->box[2];
    P.rc = cutoff;
    P.rc2 = cutoff * cutoff;
    P.beta = beta;
    P.beta2 = beta * beta;
    P.beta3 = beta * beta * beta;
    const double b3 = (double)beta * beta * beta;
    const double pc[6] = {SB_EWALD_P5, SB_EWALD_P4, SB_EWALD_P3,
                          SB_EWALD_P2, SB_EWALD_P1, SB_EWALD_P0};
    for (int k = 0; k < 6; k++) P.gp[k] = (float)(b3 * pc[k]);
    const double brc = (double)beta * cutoff;
    P.wide = brc * brc > 8.9;
    P.nt = ntypes;
    P.slot_cap = nl->slot_cap;
    P.ent_cap = nl->ent_cap;
    const bool pruned = nl->prune_buffer > 0.f && nl->cl_ent_in && nl->cl_ent_tmp;
    const float rb = cutoff + nl->prune_buffer;
    P.rb2 = pruned ? rb * rb : 0.f;
    P.prune = nl->meta + 6;
    P.cl_count_in = nl->cl_count_in;
    P.cl_ent_in = nl->cl_ent_in;
    P.cl_ent_tmp = nl->cl_ent_tmp;
    P.xq_prune = nl->xq_prune;
    return P;
}

static PairParams pair_params(const sb_lennard_jones* lj, const sb_neighbor_list* nl,
                              float beta) {
    return pair_params_of(nl, lj->ntypes, lj->cutoff, beta);
}

static int launch_pair_fixed(sb_lennard_jones* lj, sb_neighbor_list* nl, float beta, int ev,
                             float* ae, float* av, float* ad, cudaStream_t s) {
    PairParams P = pair_params(lj, nl, beta);
    const int warps = 1;  // one cluster per block (the launch bounds assume it)
    const int blocks = (nl->clu_cap + warps - 1) / warps;
    const size_t smem = sizeof(float2) * lj->ntypes * lj->ntypes;
    if (smem > 96 * 1024) {
        sb_set_error("LJ type table too large for shared memory (%d types)", lj->ntypes);
        return SB_ERR_ARG;
    }
#define SB_LAUNCH_PAIR(EVV, IPLV)                                                             \
    do {                                                                                      \
        if (smem > 48 * 1024)                                                                 \
            cudaFuncSetAttribute(k_pair_fixed<EVV, IPLV>,                                     \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
        k_pair_fixed<EVV, IPLV><<<blocks, 32 * warps, smem, s>>>(                             \
            P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, lj->d_AB,               \
            nl->slot_atom, nl->fix, ae, av, ad);                                              \
    } while (0)
#define SB_LAUNCH_COMPACT(EVV)                                                                \
    do {                                                                                      \
        if (smem + sizeof(CompactSmem<EVV>) > 48 * 1024)                                      \
            cudaFuncSetAttribute(k_pair_compact<EVV>,                                         \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
        k_pair_compact<EVV><<<(nl->clu_cap + SB_CP_WARPS - 1) / SB_CP_WARPS,                  \
                              32 * SB_CP_WARPS, smem, s>>>(                                   \
            P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, lj->d_AB,               \
            nl->slot_atom, nl->fix, ae, av, ad);                                              \
    } while (0)
#define SB_LAUNCH_X2(EVV)                                                                     \
    do {                                                                                      \
        if (x2_smem(lj->ntypes) > 48 * 1024)                                                  \
            cudaFuncSetAttribute(k_pair_x2<EVV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)x2_smem(lj->ntypes));                                   \
        k_pair_x2<EVV><<<x2_blocks, 32, x2_smem(lj->ntypes), s>>>(                            \
            P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, lj->d_AB,               \
            nl->slot_atom, nl->fix, ae, av, ad);                                              \
    } while (0)
    // packed kernel: one block per cluster (a grid of fewer blocks looping over the clusters
    // ran slower)
    const int x2_blocks = nl->clu_cap;
    if (lj->ipl == 2 && !P.wide) {
        switch (ev) {
            case 0: SB_LAUNCH_X2(0); break;
            case 1: SB_LAUNCH_X2(1); break;
            case 2: SB_LAUNCH_X2(2); break;
            default: SB_LAUNCH_X2(3); break;
        }
    } else if (lj->ipl == 1) {
        switch (ev) {
            case 0: SB_LAUNCH_COMPACT(0); break;
            case 1: SB_LAUNCH_COMPACT(1); break;
            case 2: SB_LAUNCH_COMPACT(2); break;
            default: SB_LAUNCH_COMPACT(3); break;
        }
    } else if (lj->ipl == 4) {
        switch (ev) {
            case 0: SB_LAUNCH_PAIR(0, 4); break;
            case 1: SB_LAUNCH_PAIR(1, 4); break;
            case 2: SB_LAUNCH_PAIR(2, 4); break;
            default: SB_LAUNCH_PAIR(3, 4); break;
        }
    } else {
        switch (ev) {
            case 0: SB_LAUNCH_PAIR(0, 8); break;
            case 1: SB_LAUNCH_PAIR(1, 8); break;
            case 2: SB_LAUNCH_PAIR(2, 8); break;
            default: SB_LAUNCH_PAIR(3, 8); break;
        }
    }
#undef SB_LAUNCH_PAIR
#undef SB_LAUNCH_COMPACT
    SB_CHECK_LAUNCH();
    return SB_OK;
}

static int launch_pair_plain(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* uc,
                             const float* q, float* frc, float beta, int ev, float* ae,
                             float* av, float* ad, cudaStream_t s) {
    SB_TRY(sb_nl_build_atom_group(nl, s));
    const float sx = (1.0f / 4294967296.0f) * nl->box[0];
    const float sy = (1.0f / 4294967296.0f) * nl->box[1];
    const float sz = (1.0f / 4294967296.0f) * nl->box[2];
    dim3 thr(32, 32);
    dim3 grid((lj->n + 31) / 32);
    const SbAtomGroupP* g = (const SbAtomGroupP*)nl->ag;
    switch (ev) {
        case 0:
            k_pair_plain<0><<<grid, thr, 0, s>>>(lj->n, g, uc, q, lj->d_type, lj->d_A, lj->d_B,
                                                 sx, sy, sz, lj->cutoff, beta, frc, ae, av, ad);
            break;
        case 1:
            k_pair_plain<1><<<grid, thr, 0, s>>>(lj->n, g, uc, q, lj->d_type, lj->d_A, lj->d_B,
                                                 sx, sy, sz, lj->cutoff, beta, frc, ae, av, ad);
            break;
        case 2:
            k_pair_plain<2><<<grid, thr, 0, s>>>(lj->n, g, uc, q, lj->d_type, lj->d_A, lj->d_B,
                                                 sx, sy, sz, lj->cutoff, beta, frc, ae, av, ad);
            break;
        default:
            k_pair_plain<3><<<grid, thr, 0, s>>>(lj->n, g, uc, q, lj->d_type, lj->d_A, lj->d_B,
                                                 sx, sy, sz, lj->cutoff, beta, frc, ae, av, ad);
            break;
    }
    SB_CHECK_LAUNCH();
    return SB_OK;
}

extern "C" int sb_lj_pme_direct_force(sb_lennard_jones* lj, sb_neighbor_list* nl,
                                      int atom_numbers, const uint32_t* d_uint_crd,
                                      const float* d_charge, float* d_frc, float pme_beta,
                                      int need_atom_energy, float* d_atom_energy,
                                      int need_virial, float* d_atom_lj_virial,
                                      float* d_atom_direct_pme_energy, void* stream) {
    if (!lj || !nl || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_lj_pme_direct_force: null argument");
        return SB_ERR_ARG;
    }
    if (atom_numbers != lj->n || nl->n != lj->n) {
        sb_set_error("sb_lj_pme_direct_force: atom count %d does not match the modules (%d, %d)",
                     atom_numbers, lj->n, nl->n);
        return SB_ERR_ARG;
    }
    if ((need_atom_energy > 0 && !d_atom_energy) ||
        (need_virial > 0 && (!d_atom_lj_virial || !d_atom_direct_pme_energy))) {
        sb_set_error("sb_lj_pme_direct_force: energy/virial output missing");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    const int ev = (need_atom_energy > 0 ? SB_EV_ENERGY : 0) | (need_virial > 0 ? SB_EV_VIRIAL : 0);
    if (lj->form == SB_FORM_PLAIN) {
        if (ev & SB_EV_VIRIAL) {
            int tb = 1024;
            k_zero_f32<<<(lj->n + tb - 1) / tb, tb, 0, s>>>(lj->n, d_atom_direct_pme_energy);
            SB_CHECK_LAUNCH();
        }
        return launch_pair_plain(lj, nl, d_uint_crd, d_charge, d_frc, pme_beta, ev,
                                 d_atom_energy, d_atom_lj_virial, d_atom_direct_pme_energy, s);
    }
    SB_TRY(sb_nl_pack(nl, d_uint_crd, d_charge, lj->d_type, s));
    SB_TRY(launch_pair_fixed(lj, nl, pme_beta, ev, d_atom_energy, d_atom_lj_virial,
                             d_atom_direct_pme_energy, s));
    SB_TRY(sb_nl_finalize_forces(nl, d_frc, s));
    return SB_OK;
}

// fused fixed-form step: pack + pair kernel into the list's slot-order fixed-point buffer, left
// there for the exclusion pass and the reciprocal gather to finish
int sb_lj_fused_pair(sb_lennard_jones* lj, sb_neighbor_list* nl, float pme_beta,
                     int need_atom_energy, float* d_atom_energy, int need_virial,
                     float* d_atom_lj_virial, float* d_atom_direct_pme_energy, cudaStream_t s) {
    if ((need_atom_energy > 0 && !d_atom_energy) ||
        (need_virial > 0 && (!d_atom_lj_virial || !d_atom_direct_pme_energy))) {
        sb_set_error("sb_nonbonded_step: energy/virial output missing");
        return SB_ERR_ARG;
    }
    const int ev = (need_atom_energy > 0 ? SB_EV_ENERGY : 0) | (need_virial > 0 ? SB_EV_VIRIAL : 0);
    return launch_pair_fixed(lj, nl, pme_beta, ev, d_atom_energy, d_atom_lj_virial,
                             d_atom_direct_pme_energy, s);
}

int sb_lj_fused_direct(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                       const float* d_charge, float pme_beta, int need_atom_energy,
                       float* d_atom_energy, int need_virial, float* d_atom_lj_virial,
                       float* d_atom_direct_pme_energy, cudaStream_t s) {
    SB_TRY(sb_nl_pack(nl, d_uint_crd, d_charge, lj->d_type, s));
    return sb_lj_fused_pair(lj, nl, pme_beta, need_atom_energy, d_atom_energy, need_virial,
                            d_atom_lj_virial, d_atom_direct_pme_energy, s);
}

extern "C" int sb_lj_long_range_correction(sb_lennard_jones* lj, int need_pressure,
                                           float* d_virial, int need_potential,
                                           float* d_potential, void* stream) {
    if (!lj) {
        sb_set_error("sb_lj_long_range_correction: null handle");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const double V = (double)lj->box[0] * lj->box[1] * lj->box[2];
    if (need_pressure > 0) {
        if (!d_virial) {
            sb_set_error("sb_lj_long_range_correction: d_virial is NULL");
            return SB_ERR_ARG;
        }
        k_device_add<<<1, 1, 0, s>>>(d_virial, (float)(lj->long_range_factor * 6.0 / V));
        SB_CHECK_LAUNCH();
    }
    if (need_potential > 0) {
        if (!d_potential) {
            sb_set_error("sb_lj_long_range_correction: d_potential is NULL");
            return SB_ERR_ARG;
        }
        k_device_add<<<1, 1, 0, s>>>(d_potential, (float)(lj->long_range_factor / V));
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_lj_get_energy(sb_lennard_jones* lj, sb_neighbor_list* nl,
                                const uint32_t* d_uint_crd, float* h_energy, void* stream) {
    if (!lj || !nl || !d_uint_crd) {
        sb_set_error("sb_lj_get_energy: null argument");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    int tb = 1024;
    k_zero_f32<<<(lj->n + tb - 1) / tb, tb, 0, s>>>(lj->n, lj->d_energy_atom);
    SB_CHECK_LAUNCH();
    // charges are irrelevant for the LJ energy; pack with the type table only
    SB_TRY(sb_nl_pack(nl, d_uint_crd, nullptr, lj->d_type, s));
    PairParams P = pair_params(lj, nl, 0.f);
    const int warps = 4;
    k_lj_energy_fixed<<<(nl->clu_cap + warps - 1) / warps, 32 * warps, 0, s>>>(
        P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, lj->d_AB, nl->slot_atom,
        lj->d_energy_atom);
    SB_CHECK_LAUNCH();
    SB_TRY(sb_reduce_sum_f32(lj->d_energy_atom, lj->n, lj->d_red, s));
    double e = 0;
    SB_CHECK_CUDA(cudaMemcpyAsync(&e, lj->d_red, sizeof(double), cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    const double V = (double)lj->box[0] * lj->box[1] * lj->box[2];
    e += lj->long_range_factor / V;
    if (h_energy) *h_energy = (float)e;
    return SB_OK;
}

extern "C" int sb_lj_update_volume(sb_lennard_jones* lj, const float box_length[3]) {
    if (!lj || !box_length) {
        sb_set_error("sb_lj_update_volume: null argument");
        return SB_ERR_ARG;
    }
    for (int d = 0; d < 3; d++) lj->box[d] = box_length[d];
    lj->volume = box_length[0] * box_length[1] * box_length[2];
    return SB_OK;
}

extern "C" int sb_lj_set_kernel_variant(sb_lennard_jones* lj, int atoms_per_lane) {
    if (!lj || (atoms_per_lane != 1 && atoms_per_lane != 2 && atoms_per_lane != 4 &&
                atoms_per_lane != 8)) {
        sb_set_error("sb_lj_set_kernel_variant: atoms_per_lane must be 1, 2, 4 or 8");
        return SB_ERR_ARG;
    }
    lj->ipl = atoms_per_lane;
    return SB_OK;
}

extern "C" int sb_lj_tune(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                          const float* d_charge, float pme_beta, int* h_chosen, void* stream) {
    if (!lj || !nl || !d_uint_crd || !d_charge) {
        sb_set_error("sb_lj_tune: null argument");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    if (lj->form != SB_FORM_FIXED) {
        if (h_chosen) *h_chosen = 0;
        return SB_OK;
    }
    cudaStream_t s = sb_stream(stream);
    SB_TRY(sb_nl_pack(nl, d_uint_crd, d_charge, lj->d_type, s));
    const int cand[4] = {1, 4, 8, 2};
    float best = 1e30f;
    int pick = lj->ipl;
    cudaEvent_t a, b;
    SB_CHECK_CUDA(cudaEventCreate(&a));
    SB_CHECK_CUDA(cudaEventCreate(&b));
    for (int c = 0; c < 4; c++) {
        lj->ipl = cand[c];
        SB_TRY(launch_pair_fixed(lj, nl, pme_beta, 0, nullptr, nullptr, nullptr, s));
        // a pruned list is built by the first packed launch; the timed ones walk it
        SB_TRY(sb_nl_retire_prune(nl, s));
        SB_CHECK_CUDA(cudaEventRecord(a, s));
        for (int r = 0; r < 3; r++)
            SB_TRY(launch_pair_fixed(lj, nl, pme_beta, 0, nullptr, nullptr, nullptr, s));
        SB_CHECK_CUDA(cudaEventRecord(b, s));
        SB_CHECK_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) {
            best = ms;
            pick = cand[c];
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    lj->ipl = pick;
    // the timing runs accumulated into the fixed-point buffers: clear them
    SB_CHECK_CUDA(cudaMemsetAsync(nl->fix, 0, sizeof(long long) * 3 * nl->slot_cap, s));
    if (h_chosen) *h_chosen = pick;
    return SB_OK;
}

extern "C" int sb_lj_long_range_factor(sb_lennard_jones* lj, float* h_factor) {
    if (!lj || !h_factor) {
        sb_set_error("sb_lj_long_range_factor: null argument");
        return SB_ERR_ARG;
    }
    *h_factor = (float)lj->long_range_factor;
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// FEP split form: the pairs of two unperturbed atoms of a soft-core box through the packed
// kernel (force only), with the box's A-state table extended by a zero ghost type that the
// FEP pack gives the perturbed atoms (their charges packed as 0), so that their pairs add
// exactly zero here and are left to the soft-core pass over the perturbed atoms.
// ---------------------------------------------------------------------------------------------
bool sb_pair_fep_packed(const sb_neighbor_list* nl, float cutoff, float beta) {
    return !pair_params_of(nl, 1, cutoff, beta).wide;
}

int sb_pair_fep(sb_neighbor_list* nl, const float2* d_AB, int ntypes, float cutoff, float beta,
                cudaStream_t s) {
    const PairParams P = pair_params_of(nl, ntypes, cutoff, beta);
    if (P.wide) {
        sb_set_error("sb_pair_fep: beta * cutoff beyond the packed kernel's Ewald fit");
        return SB_ERR_ARG;
    }
    if (x2_smem(ntypes) > 48 * 1024)
        cudaFuncSetAttribute(k_pair_x2<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)x2_smem(ntypes));
    k_pair_x2<0><<<nl->clu_cap, 32, x2_smem(ntypes), s>>>(
        P, nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype, d_AB, nl->slot_atom, nl->fix,
        nullptr, nullptr, nullptr);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

// the PairParams fields that differ between the boxes of one batched launch
struct X2BoxVar {
    float sx, sy, sz;
    int nt, slot_cap, ent_cap;
    float rb2;
    int* prune;
    int* cl_count_in;
    uint32_t* cl_ent_in;
    uint32_t* cl_ent_tmp;
    uint4* xq_prune;
};

// One one-warp block per cluster of any window. The windows' pointers and constants travel in
// the kernel parameters (a constant-bank block read with a block-uniform index; the fields that
// all windows of a launch share stay plain PairParams operands, as in k_pair_x2), and a block
// finds its window by a binary search over the windows' first blocks: a table entry and a
// descriptor in global memory, which each block waited for before its cluster's own loads, made
// the launch 2 % slower on fep48.
#define SB_X2_BATCH_MAX 96  // windows per launch
struct X2Box {
    const int* meta;
    const int* cl_count;
    const uint32_t* cl_ent;
    const uint4* xq;
    const int* stype;
    const float2* AB;
    const int* slot_atom;
    long long* fix;
    X2BoxVar v;
};
struct X2BatchParams {
    PairParams C;
    int nbox;
    int first[SB_X2_BATCH_MAX + 1];  // first block of each window; first[nbox] = grid size
    X2Box box[SB_X2_BATCH_MAX];
};

__global__ void __launch_bounds__(32, 24) k_pair_x2_batch(const __grid_constant__ X2BatchParams B) {
    extern __shared__ float4 ctab[];
    const int b = blockIdx.x;
    int lo = 0, hi = B.nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (B.first[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const X2Box& w = B.box[lo];
    const int c = b - B.first[lo];
    if (c >= w.meta[0]) return;
    PairParams P = B.C;
    P.sx = w.v.sx;
    P.sy = w.v.sy;
    P.sz = w.v.sz;
    P.nt = w.v.nt;
    P.slot_cap = w.v.slot_cap;
    P.ent_cap = w.v.ent_cap;
    P.rb2 = w.v.rb2;
    P.prune = w.v.prune;
    P.cl_count_in = w.v.cl_count_in;
    P.cl_ent_in = w.v.cl_ent_in;
    P.cl_ent_tmp = w.v.cl_ent_tmp;
    P.xq_prune = w.v.xq_prune;
    x2_cluster<0>(P, c, threadIdx.x & 31, ctab, w.cl_count, w.cl_ent, w.xq, w.stype, w.AB,
                  w.slot_atom, w.fix, nullptr, nullptr, nullptr);
}

struct SbX2Batch {
    std::vector<X2BatchParams> launches;  // windows with equal common fields, up to 96 a launch
    size_t smem = 0;
};

static bool x2_same_common(const PairParams& a, const PairParams& b) {
    if (a.rc2 != b.rc2 || a.rc != b.rc || a.beta != b.beta || a.beta2 != b.beta2 ||
        a.beta3 != b.beta3 || a.wide != b.wide)
        return false;
    for (int k = 0; k < 6; k++)
        if (a.gp[k] != b.gp[k]) return false;
    return true;
}

void sb_pair_batch_destroy(SbX2Batch* x) { delete x; }

int sb_pair_batch_create(int nb, const int* box_ids, sb_neighbor_list* const* nls,
                         const float2* const* tables, const int* ntypes, const float* cutoffs,
                         const float* betas, SbX2Batch** out) {
    *out = nullptr;
    std::vector<PairParams> P(nb);
    size_t smem = 0;
    for (int i = 0; i < nb; i++) {
        P[i] = pair_params_of(nls[i], ntypes[i], cutoffs[i], betas[i]);
        if (P[i].wide) {
            sb_set_error("sb_pair_batch_create: box %d beyond the packed kernel's Ewald fit",
                         box_ids[i]);
            return SB_ERR_ARG;
        }
        smem = std::max(smem, x2_smem(ntypes[i]));
    }
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_pair_x2_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess) {
        sb_set_error("sb_pair_batch_create: shared memory attribute refused");
        return SB_ERR_CUDA;
    }
    SbX2Batch* x = new SbX2Batch();
    x->smem = smem;
    std::vector<char> done(nb, 0);
    for (int i = 0; i < nb; i++) {
        if (done[i]) continue;
        X2BatchParams L;
        memset(&L, 0, sizeof(L));
        L.C = P[i];
        for (int j = i; j < nb; j++) {
            if (done[j] || !x2_same_common(P[i], P[j])) continue;
            done[j] = 1;
            if (L.nbox == SB_X2_BATCH_MAX) {
                x->launches.push_back(L);
                memset(&L.box, 0, sizeof(L.box));
                L.nbox = 0;
                L.first[0] = 0;
            }
            sb_neighbor_list* nl = nls[j];
            const PairParams& q = P[j];
            L.box[L.nbox] = X2Box{nl->meta, nl->cl_count, nl->cl_ent, nl->xq, nl->stype,
                                  tables[j], nl->slot_atom, nl->fix,
                                  X2BoxVar{q.sx, q.sy, q.sz, q.nt, q.slot_cap, q.ent_cap, q.rb2,
                                           q.prune, q.cl_count_in, q.cl_ent_in, q.cl_ent_tmp,
                                           q.xq_prune}};
            L.first[L.nbox + 1] = L.first[L.nbox] + nl->clu_cap;
            L.nbox++;
        }
        if (L.nbox) x->launches.push_back(L);
    }
    *out = x;
    return SB_OK;
}

int sb_pair_batch_launch(const SbX2Batch* x, cudaStream_t s) {
    for (const auto& L : x->launches) {
        k_pair_x2_batch<<<L.first[L.nbox], 32, x->smem, s>>>(L);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

int sb_pair_batch_launches(const SbX2Batch* x) { return (int)x->launches.size(); }
