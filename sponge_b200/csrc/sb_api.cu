// C ABI glue: error reporting, allocation, FP64 reductions and the whole-step entry point.

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "sb_internal.cuh"

static thread_local char g_err[1024] = "";

void sb_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char* sb_last_error(void) { return g_err; }

extern "C" int sb_version(void) { return 100; }

int sb_malloc(void** p, size_t bytes, const char* what) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        sb_set_error("cudaMalloc of %zu bytes for %s failed: %s", bytes, what,
                     cudaGetErrorString(e));
        return SB_ERR_ALLOC;
    }
    return SB_OK;
}

void sb_free(void* p) {
    if (p) cudaFree(p);
}

__global__ void __launch_bounds__(1024) k_reduce_f32(const float* __restrict__ x, int n,
                                                     double* __restrict__ out) {
    __shared__ double red[1024];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += (double)x[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

int sb_reduce_sum_f32(const float* d_x, int n, double* d_out, cudaStream_t s) {
    k_reduce_f32<<<1, 1024, 0, s>>>(d_x, n, d_out);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

// force part of one step (the list is used as it stands)
static int nonbonded_force(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                           const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                           const int* el, const int* en, float* d_frc, int need_energy,
                           int need_virial, float* d_atom_energy, float* d_atom_virial,
                           float* d_virial, float* d_potential, void* stream) {
    float* d_direct = nullptr;
    float* d_corr = nullptr;
    SB_TRY(sb_pme_atom_energy_arrays(pme, &d_direct, &d_corr));
    if (lj->form == SB_FORM_FIXED && pme->form == SB_FORM_FIXED && nl->form == SB_FORM_FIXED &&
        lj->n == nl->n && pme->n == nl->n) {
        // fused fixed form: pair and exclusion forces meet in the list's slot-order fixed-point
        // buffer; the reciprocal gather finalises it into d_frc
        SB_TRY(sb_nl_ensure_built(nl));
        cudaStream_t s = sb_stream(stream);
        const int ev = need_energy > 0 || need_virial > 0;
        // the reciprocal grid chain (with the exclusion correction in its gather) reads the
        // atom-order coordinates and charges, so it needs no packing: with overlap on it runs on
        // the module's side stream from the start while the packing and the pair kernel run
        // here (the force buffer takes integer adds, so the order cannot change a bit)
        const bool fork = pme->overlap && pme->side;
        cudaStream_t g = fork ? pme->side : s;
        if (fork) {
            SB_CHECK_CUDA(cudaEventRecord(pme->ev_fork, s));
            SB_CHECK_CUDA(cudaStreamWaitEvent(g, pme->ev_fork, 0));
        }
        // the exclusion correction runs inside the reciprocal gather; the per-atom correction
        // energy is only read on energy/virial steps
        int st = sb_pme_zero_atom_energy(pme, ev ? d_corr : nullptr, g);
        if (!st)
            st = sb_pme_fused_grid_atoms(pme, nl, ev, g, d_uint_crd, d_charge, es, el, en,
                                         ev ? d_corr : nullptr);
        if (fork) {
            // join even after a failed launch so that a capture in progress stays well formed
            SB_CHECK_CUDA(cudaEventRecord(pme->ev_join, g));
        }
        // the pair kernel's packed slots (issued after the fork, so the side chain starts first)
        int st2 = sb_nl_pack(nl, d_uint_crd, d_charge, lj->d_type, s);
        if (!st2)
            st2 = sb_lj_fused_pair(lj, nl, pme->beta, need_energy, d_atom_energy, need_virial,
                                   d_atom_virial, d_direct, s);
        if (!st2)
            st2 = sb_lj_long_range_correction(lj, need_virial, d_virial, need_energy,
                                              d_potential, stream);
        if (fork) SB_CHECK_CUDA(cudaStreamWaitEvent(s, pme->ev_join, 0));
        if (st) return st;
        if (st2) return st2;
        return sb_pme_fused_finish(pme, nl, d_frc, d_charge, need_virial, need_energy, d_virial,
                                   d_potential, s);
    }
    SB_TRY(sb_lj_pme_direct_force(lj, nl, lj->n, d_uint_crd, d_charge, d_frc, pme->beta,
                                  need_energy, d_atom_energy, need_virial, d_atom_virial,
                                  d_direct, stream));
    SB_TRY(sb_lj_long_range_correction(lj, need_virial, d_virial, need_energy, d_potential,
                                       stream));
    const float sc[3] = {(1.0f / 4294967296.0f) * pme->box[0],
                         (1.0f / 4294967296.0f) * pme->box[1],
                         (1.0f / 4294967296.0f) * pme->box[2]};
    SB_TRY(sb_pme_excluded_force(pme, d_uint_crd, sc, d_charge, es, el, en, d_frc, d_corr,
                                 stream));
    SB_TRY(sb_pme_reciprocal_force(pme, d_uint_crd, d_charge, d_frc, need_virial, need_energy,
                                   d_virial, d_potential, stream));
    return SB_OK;
}

extern "C" int sb_nonbonded_step(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                                 float* d_crd, const uint32_t* d_uint_crd, const float* d_charge,
                                 const int* es, const int* el, const int* en, float* d_frc,
                                 int need_energy, int need_virial, float* d_atom_energy,
                                 float* d_atom_virial, float* d_virial, float* d_potential,
                                 void* stream) {
    if (!nl || !lj || !pme || !d_crd || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_nonbonded_step: null argument");
        return SB_ERR_ARG;
    }
    // Main_Iteration's list update follows the previous step's integration; the list built
    // here is used for this step's forces (the order a driver calling update then force sees)
    SB_TRY(sb_nl_update(nl, d_crd, es, el, en, 0, 0, stream));
    return nonbonded_force(nl, lj, pme, d_uint_crd, d_charge, es, el, en, d_frc, need_energy,
                           need_virial, d_atom_energy, d_atom_virial, d_virial, d_potential,
                           stream);
}

extern "C" int sb_nonbonded_set_overlap(sb_pme* pme, int on) {
    if (!pme) {
        sb_set_error("sb_nonbonded_set_overlap: null handle");
        return SB_ERR_ARG;
    }
    pme->overlap = on ? 1 : 0;
    return SB_OK;
}

extern "C" int sb_nonbonded_force(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                                  const uint32_t* d_uint_crd, const float* d_charge,
                                  const int* es, const int* el, const int* en, float* d_frc,
                                  int need_energy, int need_virial, float* d_atom_energy,
                                  float* d_atom_virial, float* d_virial, float* d_potential,
                                  void* stream) {
    if (!nl || !lj || !pme || !d_uint_crd || !d_charge || !d_frc) {
        sb_set_error("sb_nonbonded_force: null argument");
        return SB_ERR_ARG;
    }
    return nonbonded_force(nl, lj, pme, d_uint_crd, d_charge, es, el, en, d_frc, need_energy,
                           need_virial, d_atom_energy, d_atom_virial, d_virial, d_potential,
                           stream);
}
