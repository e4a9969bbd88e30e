// 1-4 nonbonded pairs (NON_BOND_14, SPONGE/nb14/nb14.cu) and virtual atoms
// (VIRTUAL_INFORMATION, SPONGE/virtual_atoms/virtual_atoms.cu) — the per-step kernels that sit
// next to the nonbonded path in Main_Calculate_Force (SPONGE/main.cu:195, :207) and
// Main_Iteration (:375).
//
// B200 design: both modules are short scatter passes whose reference form adds into the force
// array with float atomics (order-dependent bits). Here
//   * the 1-4 pass adds forces, per-atom energies and virials as 64-bit fixed point (the units
//     of the pair kernels) into module-owned buffers, and a finalize pass adds them to the
//     caller's float arrays and clears the buffers: same bits whatever the launch order;
//   * the virtual-atom force redistribution is a gather: each parent atom sums the shares of
//     its virtual atoms (one list per level, built on the host, in a fixed order) and the
//     virtual atoms are zeroed afterwards, level by level from the top (the reference's
//     reverse layer order, virtual_atoms.cu:513-530). No atomics, deterministic.

#include <algorithm>
#include <cmath>
#include <vector>

#include "sb_internal.cuh"

#define SB_NB14_TINY 1e-10f  // charges below this are clamped to it (nb14.cu:2, :77-82)

struct sb_nb14 {
    int n = 0;     // atoms
    int n14 = 0;   // pairs
    int* d_a = nullptr;
    int* d_b = nullptr;
    float* d_A = nullptr;   // per pair, x12 (LJ_A of the pair type times the LJ scale factor)
    float* d_B = nullptr;   // per pair, x6
    float* d_cf = nullptr;  // per pair Coulomb scale factor
    long long* d_fix = nullptr;   // [3n] force, [n] energy, [n] virial (2^-32 units)
    float* d_pair_e = nullptr;    // [n14] per-pair energies for the sums
    double* d_red = nullptr;
};

__device__ __forceinline__ float3 nb14_disp(const uint32_t* uc, int i, int j, float sx, float sy,
                                            float sz) {
    // Get_Periodic_Displacement(r_j, r_i) (common.cu:89-97): exact integer difference, wrap
    return make_float3((float)(int)(uc[3 * j] - uc[3 * i]) * sx,
                       (float)(int)(uc[3 * j + 1] - uc[3 * i + 1]) * sy,
                       (float)(int)(uc[3 * j + 2] - uc[3 * i + 2]) * sz);
}

__device__ __forceinline__ void nb14_add(long long* p, float v) {
    sb_red_add(p, __float2ll_rn(v * SB_FORCE_SCALE));
}

// Dihedral_14_LJ_CF_Force_With_Atom_Energy_And_Virial_Cuda (nb14.cu:92-170): force on the pair,
// energy and virial to the first atom
template <bool EV>
__global__ void k_nb14_force(int n14, int n, const uint32_t* __restrict__ uc,
                             const float* __restrict__ q, float sx, float sy, float sz,
                             const int* __restrict__ a14, const int* __restrict__ b14,
                             const float* __restrict__ A, const float* __restrict__ B,
                             const float* __restrict__ cf, long long* __restrict__ fix) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n14) return;
    const int i = a14[p], j = b14[p];
    const float3 dr = nb14_disp(uc, i, j, sx, sy, sz);
    const float dr2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
    const float dr_2 = 1.0f / dr2;
    const float dr_4 = dr_2 * dr_2;
    const float dr_8 = dr_4 * dr_4;
    const float dr_14 = dr_8 * dr_4 * dr_2;
    const float dr_1 = 1.0f / sqrtf(dr2);
    float qi = q[i], qj = q[j];
    if (fabsf(qi) < SB_NB14_TINY) qi = SB_NB14_TINY;
    if (fabsf(qj) < SB_NB14_TINY) qj = SB_NB14_TINY;
    const float fcf = -(cf[p] * dr_2 * dr_1) * qi * qj;
    const float fs = -A[p] * dr_14 + B[p] * dr_8 + fcf;
    const float fx = fs * dr.x, fy = fs * dr.y, fz = fs * dr.z;
    nb14_add(&fix[3 * j], -fx);
    nb14_add(&fix[3 * j + 1], -fy);
    nb14_add(&fix[3 * j + 2], -fz);
    nb14_add(&fix[3 * i], fx);
    nb14_add(&fix[3 * i + 1], fy);
    nb14_add(&fix[3 * i + 2], fz);
    if (EV) {
        const float e = cf[p] * dr_1 * qi * qj + 0.08333333f * A[p] * dr_4 * dr_8 -
                        0.1666666f * B[p] * dr_4 * dr_2;
        nb14_add(&fix[3 * n + i], e);
        nb14_add(&fix[4 * n + i], -(fx * dr.x + fy * dr.y + fz * dr.z));
    }
}

__global__ void k_nb14_finalize(int n, long long* __restrict__ fix, float* __restrict__ frc,
                                float* __restrict__ atom_energy, float* __restrict__ atom_virial) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long long v = fix[3 * a + d];
        if (v) {
            frc[3 * a + d] += (float)((double)v * SB_FORCE_UNSCALE);
            fix[3 * a + d] = 0;
        }
    }
    const long long e = fix[3 * n + a], w = fix[4 * n + a];
    if (e) {
        if (atom_energy) atom_energy[a] += (float)((double)e * SB_FORCE_UNSCALE);
        fix[3 * n + a] = 0;
    }
    if (w) {
        if (atom_virial) atom_virial[a] += (float)((double)w * SB_FORCE_UNSCALE);
        fix[4 * n + a] = 0;
    }
}

// Dihedral_14_LJ_Energy / Dihedral_14_CF_Energy (nb14.cu:5-91): per-pair energies
__global__ void k_nb14_energy(int n14, const uint32_t* __restrict__ uc,
                              const float* __restrict__ q, float sx, float sy, float sz,
                              const int* __restrict__ a14, const int* __restrict__ b14,
                              const float* __restrict__ A, const float* __restrict__ B,
                              const float* __restrict__ cf, int coulomb, float* __restrict__ ene) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n14) return;
    const int i = a14[p], j = b14[p];
    const float3 dr = nb14_disp(uc, i, j, sx, sy, sz);
    const float dr2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
    if (coulomb) {
        float qi = q[i], qj = q[j];
        if (fabsf(qi) < SB_NB14_TINY) qi = SB_NB14_TINY;
        if (fabsf(qj) < SB_NB14_TINY) qj = SB_NB14_TINY;
        ene[p] = cf[p] * qi * qj * (1.0f / sqrtf(dr2));
    } else {
        const float dr_2 = 1.0f / dr2;
        const float dr_6 = dr_2 * dr_2 * dr_2;
        const float dr_12 = dr_6 * dr_6;
        ene[p] = 0.08333333f * A[p] * dr_12 - 0.1666666f * B[p] * dr_6;
    }
}

extern "C" int sb_nb14_create(int atom_numbers, int nb14_numbers, const int* h_atom_a,
                              const int* h_atom_b, const float* h_A, const float* h_B,
                              const float* h_cf_scale, sb_nb14** out) {
    if (!out || atom_numbers <= 0 || nb14_numbers < 0 ||
        (nb14_numbers > 0 && (!h_atom_a || !h_atom_b || !h_A || !h_B || !h_cf_scale))) {
        sb_set_error("sb_nb14_create: invalid arguments");
        return SB_ERR_ARG;
    }
    for (int p = 0; p < nb14_numbers; p++)
        if (h_atom_a[p] < 0 || h_atom_a[p] >= atom_numbers || h_atom_b[p] < 0 ||
            h_atom_b[p] >= atom_numbers) {
            sb_set_error("sb_nb14_create: pair %d references atom outside [0, %d)", p,
                         atom_numbers);
            return SB_ERR_ARG;
        }
    sb_nb14* m = new sb_nb14();
    m->n = atom_numbers;
    m->n14 = nb14_numbers;
    const size_t np = std::max(1, nb14_numbers);
    int st = SB_OK;
    if ((st = sb_malloc((void**)&m->d_a, sizeof(int) * np, "nb14 a")) ||
        (st = sb_malloc((void**)&m->d_b, sizeof(int) * np, "nb14 b")) ||
        (st = sb_malloc((void**)&m->d_A, sizeof(float) * np, "nb14 A")) ||
        (st = sb_malloc((void**)&m->d_B, sizeof(float) * np, "nb14 B")) ||
        (st = sb_malloc((void**)&m->d_cf, sizeof(float) * np, "nb14 cf")) ||
        (st = sb_malloc((void**)&m->d_pair_e, sizeof(float) * np, "nb14 energies")) ||
        (st = sb_malloc((void**)&m->d_red, sizeof(double) * 2, "nb14 sums")) ||
        (st = sb_malloc((void**)&m->d_fix, sizeof(long long) * 5 * (size_t)atom_numbers,
                        "nb14 accumulators"))) {
        sb_nb14_destroy(m);
        return st;
    }
    if (nb14_numbers > 0) {
        cudaMemcpy(m->d_a, h_atom_a, sizeof(int) * nb14_numbers, cudaMemcpyHostToDevice);
        cudaMemcpy(m->d_b, h_atom_b, sizeof(int) * nb14_numbers, cudaMemcpyHostToDevice);
        cudaMemcpy(m->d_A, h_A, sizeof(float) * nb14_numbers, cudaMemcpyHostToDevice);
        cudaMemcpy(m->d_B, h_B, sizeof(float) * nb14_numbers, cudaMemcpyHostToDevice);
        cudaMemcpy(m->d_cf, h_cf_scale, sizeof(float) * nb14_numbers, cudaMemcpyHostToDevice);
    }
    cudaMemset(m->d_fix, 0, sizeof(long long) * 5 * (size_t)atom_numbers);
    if (cudaGetLastError() != cudaSuccess) {
        sb_set_error("sb_nb14_create: device copy failed");
        sb_nb14_destroy(m);
        return SB_ERR_CUDA;
    }
    *out = m;
    return SB_OK;
}

extern "C" int sb_nb14_destroy(sb_nb14* m) {
    if (!m) return SB_OK;
    void* ps[] = {m->d_a, m->d_b, m->d_A, m->d_B, m->d_cf, m->d_pair_e, m->d_red, m->d_fix};
    for (void* p : ps) sb_free(p);
    delete m;
    return SB_OK;
}

extern "C" int sb_nb14_force(sb_nb14* m, const uint32_t* d_uint_crd, const float* d_charge,
                             const float scaler[3], float* d_frc, float* d_atom_energy,
                             float* d_atom_virial, void* stream) {
    if (!m || !d_uint_crd || !d_charge || !scaler || !d_frc) {
        sb_set_error("sb_nb14_force: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    if (m->n14 > 0) {
        const int tb = 128, blocks = (m->n14 + tb - 1) / tb;
        const bool ev = d_atom_energy || d_atom_virial;
        if (ev)
            k_nb14_force<true><<<blocks, tb, 0, s>>>(m->n14, m->n, d_uint_crd, d_charge,
                                                      scaler[0], scaler[1], scaler[2], m->d_a,
                                                      m->d_b, m->d_A, m->d_B, m->d_cf, m->d_fix);
        else
            k_nb14_force<false><<<blocks, tb, 0, s>>>(m->n14, m->n, d_uint_crd, d_charge,
                                                       scaler[0], scaler[1], scaler[2], m->d_a,
                                                       m->d_b, m->d_A, m->d_B, m->d_cf,
                                                       m->d_fix);
        SB_CHECK_LAUNCH();
    }
    k_nb14_finalize<<<(m->n + 255) / 256, 256, 0, s>>>(m->n, m->d_fix, d_frc, d_atom_energy,
                                                       d_atom_virial);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

extern "C" int sb_nb14_energy(sb_nb14* m, const uint32_t* d_uint_crd, const float* d_charge,
                              const float scaler[3], double* h_lj, double* h_cf, void* stream) {
    if (!m || !d_uint_crd || !scaler || (h_cf && !d_charge)) {
        sb_set_error("sb_nb14_energy: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    double out[2] = {0.0, 0.0};
    for (int c = 0; c < 2; c++) {
        double* h = c ? h_cf : h_lj;
        if (!h) continue;
        if (m->n14 > 0) {
            k_nb14_energy<<<(m->n14 + 127) / 128, 128, 0, s>>>(
                m->n14, d_uint_crd, d_charge, scaler[0], scaler[1], scaler[2], m->d_a, m->d_b,
                m->d_A, m->d_B, m->d_cf, c, m->d_pair_e);
            SB_CHECK_LAUNCH();
            SB_TRY(sb_reduce_sum_f32(m->d_pair_e, m->n14, m->d_red + c, s));
            SB_CHECK_CUDA(cudaMemcpyAsync(&out[c], m->d_red + c, sizeof(double),
                                          cudaMemcpyDeviceToHost, s));
        }
    }
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    if (h_lj) *h_lj = out[0];
    if (h_cf) *h_cf = out[1];
    return SB_OK;
}

// ---------------------------------------------------------------------------------------------
// virtual atoms
// ---------------------------------------------------------------------------------------------
// record per virtual atom (types of virtual_atoms.cuh:8-85): v = the virtual atom, f[0..2] its
// parents, p0/p1 = the type's parameters (type 0: 2h; 1: a; 2: a, b; 3: d, k)
struct SbVsiteRec {
    int type, v, f0, f1, f2;
    float p0, p1;
};

struct sb_vsite {
    int n = 0, nv = 0, nlevels = 0;
    SbVsiteRec* d_rec = nullptr;       // records grouped by level (level 1 first)
    std::vector<int> lvl_beg;          // [nlevels+1] record ranges per level
    // per level: parent atoms and, per parent, its (record, role) shares in a fixed order
    int* d_par = nullptr;              // parent atom of each gather slot
    int* d_par_beg = nullptr;          // [slots+1] share range of each parent
    int* d_share = nullptr;            // record index * 4 + role (role 0..2)
    std::vector<int> par_lvl_beg;      // [nlevels+1] parent-slot ranges per level
};

__device__ __forceinline__ float3 vs_disp(const uint32_t* uc, int from, int to, float sx, float sy,
                                          float sz) {
    // Get_Periodic_Displacement(uint_crd[to], uint_crd[from], scaler)
    return make_float3((float)(int)(uc[3 * to] - uc[3 * from]) * sx,
                       (float)(int)(uc[3 * to + 1] - uc[3 * from + 1]) * sy,
                       (float)(int)(uc[3 * to + 2] - uc[3 * from + 2]) * sz);
}

// v*_Coordinate_Refresh (virtual_atoms.cu:2-73)
__global__ void k_vs_refresh(int nrec, const SbVsiteRec* __restrict__ rec,
                             const uint32_t* __restrict__ uc, float sx, float sy, float sz,
                             float* __restrict__ crd) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    const SbVsiteRec R = rec[r];
    float x = crd[3 * R.f0], y = crd[3 * R.f0 + 1], z = crd[3 * R.f0 + 2];
    if (R.type == 0) {
        z = R.p0 - z;
    } else if (R.type == 1) {
        const float3 d = vs_disp(uc, R.f0, R.f1, sx, sy, sz);
        x += R.p0 * d.x;
        y += R.p0 * d.y;
        z += R.p0 * d.z;
    } else if (R.type == 2) {
        const float3 d1 = vs_disp(uc, R.f0, R.f1, sx, sy, sz);
        const float3 d2 = vs_disp(uc, R.f0, R.f2, sx, sy, sz);
        x += R.p0 * d1.x + R.p1 * d2.x;
        y += R.p0 * d1.y + R.p1 * d2.y;
        z += R.p0 * d1.z + R.p1 * d2.z;
    } else {
        const float3 r21 = vs_disp(uc, R.f0, R.f1, sx, sy, sz);
        const float3 r32 = vs_disp(uc, R.f1, R.f2, sx, sy, sz);
        const float tx = r21.x + R.p1 * r32.x, ty = r21.y + R.p1 * r32.y,
                    tz = r21.z + R.p1 * r32.z;
        const float f = R.p0 * rnorm3df(tx, ty, tz);
        x += f * tx;
        y += f * ty;
        z += f * tz;
    }
    crd[3 * R.v] = x;
    crd[3 * R.v + 1] = y;
    crd[3 * R.v + 2] = z;
}

// share of parent role `role` in the force fv of virtual atom R (v*_Force_Redistribute,
// virtual_atoms.cu:75-180)
__device__ __forceinline__ float3 vs_share(const SbVsiteRec& R, int role, float3 fv,
                                           const uint32_t* uc, float sx, float sy, float sz) {
    if (R.type == 0) return make_float3(fv.x, fv.y, -fv.z);
    if (R.type == 1) {
        const float w = role == 0 ? R.p0 : 1.0f - R.p0;
        return make_float3(w * fv.x, w * fv.y, w * fv.z);
    }
    if (R.type == 2) {
        const float w = role == 0 ? 1.0f - R.p0 - R.p1 : role == 1 ? R.p0 : R.p1;
        return make_float3(w * fv.x, w * fv.y, w * fv.z);
    }
    const float3 r21 = vs_disp(uc, R.f0, R.f1, sx, sy, sz);
    const float3 r32 = vs_disp(uc, R.f1, R.f2, sx, sy, sz);
    const float3 rv1 = vs_disp(uc, R.f0, R.v, sx, sy, sz);
    const float tx = r21.x + R.p1 * r32.x, ty = r21.y + R.p1 * r32.y, tz = r21.z + R.p1 * r32.z;
    const float factor = R.p0 * rnorm3df(tx, ty, tz);
    const float proj = (rv1.x * fv.x + rv1.y * fv.y + rv1.z * fv.z) /
                       (rv1.x * rv1.x + rv1.y * rv1.y + rv1.z * rv1.z);
    const float3 t = make_float3(factor * (fv.x - proj * rv1.x), factor * (fv.y - proj * rv1.y),
                                 factor * (fv.z - proj * rv1.z));
    if (role == 0) return make_float3(fv.x - t.x, fv.y - t.y, fv.z - t.z);
    const float w = role == 1 ? 1.0f - R.p1 : R.p1;
    return make_float3(w * t.x, w * t.y, w * t.z);
}

__global__ void k_vs_gather(int slot0, int nslots, const int* __restrict__ par,
                            const int* __restrict__ par_beg, const int* __restrict__ share,
                            const SbVsiteRec* __restrict__ rec, const uint32_t* __restrict__ uc,
                            float sx, float sy, float sz, float* __restrict__ frc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslots) return;
    const int sl = slot0 + t;
    const int p = par[sl];
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int k = par_beg[sl]; k < par_beg[sl + 1]; k++) {
        const int code = share[k];
        const SbVsiteRec R = rec[code >> 2];
        const float3 fv = make_float3(frc[3 * R.v], frc[3 * R.v + 1], frc[3 * R.v + 2]);
        const float3 s = vs_share(R, code & 3, fv, uc, sx, sy, sz);
        ax += s.x;
        ay += s.y;
        az += s.z;
    }
    frc[3 * p] += ax;
    frc[3 * p + 1] += ay;
    frc[3 * p + 2] += az;
}

__global__ void k_vs_zero(int r0, int nrec, const SbVsiteRec* __restrict__ rec,
                          float* __restrict__ frc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrec) return;
    const int v = rec[r0 + t].v;
    frc[3 * v] = 0.f;
    frc[3 * v + 1] = 0.f;
    frc[3 * v + 2] = 0.f;
}

extern "C" int sb_vsite_create(int atom_numbers, int virtual_numbers, const int* h_type,
                               const int* h_atoms, const float* h_param, sb_vsite** out) {
    if (!out || atom_numbers <= 0 || virtual_numbers < 0 ||
        (virtual_numbers > 0 && (!h_type || !h_atoms || !h_param))) {
        sb_set_error("sb_vsite_create: invalid arguments");
        return SB_ERR_ARG;
    }
    const int nparents[4] = {1, 2, 3, 3};
    std::vector<int> level(atom_numbers, 0);
    // levels as the reference's first pass computes them (virtual_atoms.cu:246-290): a virtual
    // atom is one level above its highest parent; records may come in any order, so iterate
    // until stable (at most virtual_numbers passes; a cycle is an error)
    for (int it = 0;; it++) {
        bool changed = false;
        for (int r = 0; r < virtual_numbers; r++) {
            const int t = h_type[r];
            if (t < 0 || t > 3) {
                sb_set_error("sb_vsite_create: record %d has type %d (0..3)", r, t);
                return SB_ERR_ARG;
            }
            const int* a = h_atoms + 4 * r;
            for (int k = 0; k <= nparents[t]; k++)
                if (a[k] < 0 || a[k] >= atom_numbers) {
                    sb_set_error("sb_vsite_create: record %d references atom %d", r, a[k]);
                    return SB_ERR_ARG;
                }
            int lv = 0;
            for (int k = 1; k <= nparents[t]; k++) lv = std::max(lv, level[a[k]]);
            if (level[a[0]] != lv + 1) {
                level[a[0]] = lv + 1;
                changed = true;
            }
        }
        if (!changed) break;
        if (it > virtual_numbers) {
            sb_set_error("sb_vsite_create: virtual atoms depend on one another in a cycle");
            return SB_ERR_ARG;
        }
    }
    sb_vsite* m = new sb_vsite();
    m->n = atom_numbers;
    m->nv = virtual_numbers;
    int nl = 0;
    for (int r = 0; r < virtual_numbers; r++) nl = std::max(nl, level[h_atoms[4 * r]]);
    m->nlevels = nl;
    // records grouped by level, in input order inside a level
    std::vector<SbVsiteRec> rec;
    m->lvl_beg.assign(nl + 1, 0);
    for (int L = 1; L <= nl; L++) {
        m->lvl_beg[L - 1] = (int)rec.size();
        for (int r = 0; r < virtual_numbers; r++) {
            const int* a = h_atoms + 4 * r;
            if (level[a[0]] != L) continue;
            const int t = h_type[r];
            SbVsiteRec R;
            R.type = t;
            R.v = a[0];
            R.f0 = a[1];
            R.f1 = t >= 1 ? a[2] : a[1];
            R.f2 = t >= 2 ? a[3] : a[1];
            // type 0 stores 2h (virtual_atoms.cu:403)
            R.p0 = t == 0 ? 2.0f * h_param[2 * r] : h_param[2 * r];
            R.p1 = h_param[2 * r + 1];
            rec.push_back(R);
        }
    }
    m->lvl_beg[nl] = (int)rec.size();
    // per level: parents and their shares in record order
    std::vector<int> par, par_beg, share;
    m->par_lvl_beg.assign(nl + 1, 0);
    for (int L = 1; L <= nl; L++) {
        m->par_lvl_beg[L - 1] = (int)par.size();
        std::vector<std::vector<int>> by_parent(atom_numbers);
        std::vector<int> order;
        for (int r = m->lvl_beg[L - 1]; r < m->lvl_beg[L]; r++) {
            const SbVsiteRec& R = rec[r];
            const int np = nparents[R.type];
            const int f[3] = {R.f0, R.f1, R.f2};
            for (int k = 0; k < np; k++) {
                if (by_parent[f[k]].empty()) order.push_back(f[k]);
                by_parent[f[k]].push_back(r * 4 + k);
            }
        }
        for (int p : order) {
            par.push_back(p);
            par_beg.push_back((int)share.size());
            for (int c : by_parent[p]) share.push_back(c);
        }
    }
    m->par_lvl_beg[nl] = (int)par.size();
    par_beg.push_back((int)share.size());
    int st = SB_OK;
    if ((st = sb_malloc((void**)&m->d_rec, sizeof(SbVsiteRec) * std::max<size_t>(1, rec.size()),
                        "virtual atoms")) ||
        (st = sb_malloc((void**)&m->d_par, sizeof(int) * std::max<size_t>(1, par.size()),
                        "virtual parents")) ||
        (st = sb_malloc((void**)&m->d_par_beg, sizeof(int) * par_beg.size(), "parent ranges")) ||
        (st = sb_malloc((void**)&m->d_share, sizeof(int) * std::max<size_t>(1, share.size()),
                        "parent shares"))) {
        sb_vsite_destroy(m);
        return st;
    }
    if (!rec.empty())
        cudaMemcpy(m->d_rec, rec.data(), sizeof(SbVsiteRec) * rec.size(), cudaMemcpyHostToDevice);
    if (!par.empty()) cudaMemcpy(m->d_par, par.data(), sizeof(int) * par.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(m->d_par_beg, par_beg.data(), sizeof(int) * par_beg.size(), cudaMemcpyHostToDevice);
    if (!share.empty())
        cudaMemcpy(m->d_share, share.data(), sizeof(int) * share.size(), cudaMemcpyHostToDevice);
    if (cudaGetLastError() != cudaSuccess) {
        sb_set_error("sb_vsite_create: device copy failed");
        sb_vsite_destroy(m);
        return SB_ERR_CUDA;
    }
    *out = m;
    return SB_OK;
}

extern "C" int sb_vsite_destroy(sb_vsite* m) {
    if (!m) return SB_OK;
    void* ps[] = {m->d_rec, m->d_par, m->d_par_beg, m->d_share};
    for (void* p : ps) sb_free(p);
    delete m;
    return SB_OK;
}

extern "C" int sb_vsite_coordinate_refresh(sb_vsite* m, const uint32_t* d_uint_crd,
                                           const float scaler[3], float* d_crd, void* stream) {
    if (!m || !d_uint_crd || !scaler || !d_crd) {
        sb_set_error("sb_vsite_coordinate_refresh: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    for (int L = 0; L < m->nlevels; L++) {  // lowest level first (virtual_atoms.cu:498-509)
        const int r0 = m->lvl_beg[L], nr = m->lvl_beg[L + 1] - r0;
        if (nr <= 0) continue;
        k_vs_refresh<<<(nr + 127) / 128, 128, 0, s>>>(nr, m->d_rec + r0, d_uint_crd, scaler[0],
                                                      scaler[1], scaler[2], d_crd);
        SB_CHECK_LAUNCH();
    }
    return SB_OK;
}

extern "C" int sb_vsite_force_redistribute(sb_vsite* m, const uint32_t* d_uint_crd,
                                           const float scaler[3], float* d_frc, void* stream) {
    if (!m || !d_uint_crd || !scaler || !d_frc) {
        sb_set_error("sb_vsite_force_redistribute: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    for (int L = m->nlevels - 1; L >= 0; L--) {  // highest level first (virtual_atoms.cu:513-530)
        const int s0 = m->par_lvl_beg[L], ns = m->par_lvl_beg[L + 1] - s0;
        const int r0 = m->lvl_beg[L], nr = m->lvl_beg[L + 1] - r0;
        if (ns > 0) {
            k_vs_gather<<<(ns + 127) / 128, 128, 0, s>>>(s0, ns, m->d_par, m->d_par_beg,
                                                         m->d_share, m->d_rec, d_uint_crd,
                                                         scaler[0], scaler[1], scaler[2], d_frc);
            SB_CHECK_LAUNCH();
        }
        if (nr > 0) {
            k_vs_zero<<<(nr + 127) / 128, 128, 0, s>>>(r0, nr, m->d_rec, d_frc);
            SB_CHECK_LAUNCH();
        }
    }
    return SB_OK;
}
