// Internal definitions shared by the sponge_b200 CUDA sources (sm_100a).
//
// Data layout in HBM (chosen form):
//   * original atom order (caller-owned): uint_crd[3N] u32, charge[N] f32, frc[3N] f32
//   * cell-sorted "slots": atoms are bucketed into xy columns (~ (8/rho)^(1/3) wide), sorted
//     by (z, atom id) inside each column, and every column is padded to a multiple of 8 slots.
//     Slot s holds atom slot_atom[s] (-1 for padding). 8 consecutive slots form a cluster.
//   * per-call packed SoA in slot order: xq[s] = {ux, uy, uz, float_bits(q)} (uint4, one
//     128-bit load) and stype[s] (int)
//   * cluster pair list: for cluster c, cl_count[c] entries at cl_ent[c*ent_cap ...]; entry =
//     (slot j) | (mask << 24), mask bit k set iff pair (slot 8c+k, j) is in the half list
//     (slot j > slot 8c+k, not excluded, FP32 distance^2 < (rc+skin)^2)
//   * fixed-point accumulators: int64 fx/fy/fz per slot, 2^-32 kcal/mol/A per unit
//   * PME: int64 charge grid [K0][K1][K2] (2^-40 e*18.2223 per unit), complex half spectrum
//     [K0][K1][K2/2+1] float2, real potential grid [K0][K1][K2] float
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sponge_b200.h"

#define SB_FORCE_SCALE 4294967296.0f          // 2^32 units per kcal/mol/A
#define SB_FORCE_UNSCALE (1.0 / 4294967296.0)  // double
#define SB_GRID_SCALE 1099511627776.0f        // 2^40 units per charge unit on the PME grid
#define SB_GRID_UNSCALE (1.0f / 1099511627776.0f)

#define SB_CLUSTER 8
#define SB_CL_EXACT (1 << 30)        // cluster flag: pair kernel must use exact minimum image
#define SB_CL_COUNT_MASK 0xffffff
#define SB_MAX_SLOTS (1 << 24)  // slot index must fit 24 bits of a list entry
#define SB_COLUMN_SORT_CAP 4096 // max atoms per sort column (bitonic sort in shared memory)
#define SB_ZBIN_SHIFT 25        // z bins per column: the top 7 bits of the fixed-point z
#define SB_ZBINS (1 << (32 - SB_ZBIN_SHIFT))
#define SB_MAX_RADIX 8
#define SB_FFT_MAX_STAGES 12

// ---------------------------------------------------------------------------------------------
// error handling
// ---------------------------------------------------------------------------------------------
void sb_set_error(const char* fmt, ...);

#define SB_CHECK_CUDA(call)                                                              \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess) {                                                         \
            sb_set_error("%s failed at %s:%d: %s", #call, __FILE__, __LINE__,            \
                         cudaGetErrorString(_e));                                        \
            return SB_ERR_CUDA;                                                          \
        }                                                                                \
    } while (0)

#define SB_CHECK_LAUNCH()                                                                \
    do {                                                                                 \
        cudaError_t _e = cudaGetLastError();                                             \
        if (_e != cudaSuccess) {                                                         \
            sb_set_error("kernel launch failed at %s:%d: %s", __FILE__, __LINE__,        \
                         cudaGetErrorString(_e));                                        \
            return SB_ERR_CUDA;                                                          \
        }                                                                                \
    } while (0)

#define SB_TRY(expr)                  \
    do {                              \
        int _s = (expr);              \
        if (_s != SB_OK) return _s;   \
    } while (0)

int sb_malloc(void** p, size_t bytes, const char* what);
void sb_free(void* p);

// ---------------------------------------------------------------------------------------------
// FFT plan (hand-written mixed-radix shared-memory FFT)
// ---------------------------------------------------------------------------------------------
struct SbFftAxis {
    int n = 0;
    int nrad = 0;
    int rad[SB_FFT_MAX_STAGES] = {0};
    int* d_perm = nullptr;     // DIT input position p holds element perm[p]; DIF output likewise
    int* d_iperm = nullptr;    // inverse: element e sits at position iperm[e]
    float2* d_tw = nullptr;    // e^{-2 pi i t / n}, t < n (FP64-computed)
};

// per-grid pointers of a batched FFT launch: grids of one size transformed by one launch, grid
// blockIdx.y of the launch taking entry blockIdx.y (the twiddles are shared by the size)
struct SbFftBatchIo {
    long long* qfix;
    float2* spec;
    float* real;
    const float* bc;
    double* epart;
};

struct SbFftPlan {
    int K[3] = {0, 0, 0};
    int H = 0;                 // K2/2 + 1
    SbFftAxis z;               // complex length K2/2 (real transform along z via the half trick)
    SbFftAxis y;               // length K1
    SbFftAxis x;               // length K0
    float2* d_post = nullptr;  // e^{-2 pi i k / K2}, k < K2/2 (real-transform twiddles)
    size_t plane_smem = 0;     // bytes of the plane kernels' dynamic shared memory
    // kernel shape of each pass: 0 = register line transform (sizes that have one, unless the
    // generic family is requested), else the stage kernels with 8 or 16 lines per block (picked
    // by timing; both give the same bits) or 32 rows (z)
    int yt = 16;
    int xt = 16;
    int zt = 32;
    int variant = 0;           // SB_FFT_AUTO / SB_FFT_GENERIC / SB_FFT_LINES
    int fused = 0;             // 1: y and x passes fused per kz plane (k_plane4), spectrum
                               // stored plane by plane [kz][x][y]
};

// sets the kernel shape of every pass for the plan's variant, timing the stage kernels' line
// tiles where they run; d_spec is overwritten
int sb_fft_plan_tune(SbFftPlan* p, float2* d_spec, const float* d_bc, cudaStream_t s);

int sb_fft_plan_create(SbFftPlan* p, const int K[3]);
void sb_fft_plan_destroy(SbFftPlan* p);

// forward plane pass: int64 charge grid -> half spectrum (z R2C + y forward); clears the grid
int sb_fft_plane_forward(const SbFftPlan* p, long long* d_qfix, float2* d_spec, cudaStream_t s);
// the same three stages for `nb` grids of this plan's shape in one launch each (io: a device
// table of nb entries); SB_ERR_ARG for a plan with a stage-kernel axis (no batched form)
int sb_fft_batch_forward(const SbFftPlan* p, const SbFftBatchIo* d_io, int nb, cudaStream_t s);
int sb_fft_batch_convolve(const SbFftPlan* p, const SbFftBatchIo* d_io, int nb, int want_energy,
                          cudaStream_t s);
int sb_fft_batch_inverse(const SbFftPlan* p, const SbFftBatchIo* d_io, int nb, cudaStream_t s);
bool sb_fft_batchable(const SbFftPlan* p);
// x pass: forward x, multiply by the Green's function table, energy partials, inverse x
int sb_fft_x_convolve(const SbFftPlan* p, float2* d_spec, const float* d_bc, double* d_epart,
                      int want_energy, cudaStream_t s, int* nparts_out);
// inverse plane pass: half spectrum -> real grid (y inverse + z C2R)
int sb_fft_plane_inverse(const SbFftPlan* p, const float2* d_spec, float* d_real,
                         cudaStream_t s);
int sb_fft_xconv_parts(const SbFftPlan* p);

// ---------------------------------------------------------------------------------------------
// module structs
// ---------------------------------------------------------------------------------------------
struct sb_neighbor_list {
    int n = 0;
    float box[3];
    float cutoff = 10.f, skin = 2.f, cs = 12.f, cs2 = 144.f;
    int refresh_interval = 0, refresh_count = 0;
    float skin_permit = 1.f;        // internal value (2x the mdin value, neighbor_list.cu:718)
    float half_skin_square = 1.f;
    int form = SB_FORM_FIXED;
    int max_neighbor_numbers = 800;
    // column grid
    int ncx = 1, ncy = 1, ncol = 1;
    int nxr = 1, nyr = 1;
    int slot_cap = 0;               // n + 8*ncol
    int clu_cap = 0;                // slot_cap / 8
    int ent_cap = 0;                // entries per cluster
    // device buffers
    float* old_crd = nullptr;       // VECTOR[N]
    uint32_t* ucrd = nullptr;       // UNSIGNED_INT_VECTOR[N] of the last rebuild
    int* col_of = nullptr;          // [N]
    int* col_rank = nullptr;        // [N]
    int* col_count = nullptr;       // [ncol] real atoms
    int* col_start = nullptr;       // [ncol+1] padded slot starts
    unsigned long long* sort_tmp = nullptr;  // [slot_cap] (z << 32 | atom) scatter buffer
    int* slot_atom = nullptr;       // [slot_cap]
    int* atom_slot = nullptr;       // [N]
    uint32_t* slot_u = nullptr;     // [3*slot_cap] fixed-point coordinates at build, slot order
    int* excl_lo = nullptr;         // [N] min / max exclusion partner (INT_MAX / -1 if none)
    int* excl_hi = nullptr;
    int* zbin = nullptr;            // [ncol][SB_ZBINS+1] first slot of each z bin of a column
    int* cl_count = nullptr;        // [clu_cap]
    uint32_t* cl_ent = nullptr;     // [clu_cap * ent_cap]
    int* meta = nullptr;            // [0] clusters, [1] status flags, [2] refresh flag,
                                    // [3] padded slots, [4..5] pair count (int64),
                                    // [6] prune request, [7] pruned by the last pair launch
    // per force call packed data
    uint4* xq = nullptr;            // [slot_cap]
    int* stype = nullptr;           // [slot_cap]
    long long* fix = nullptr;       // [3*slot_cap] x,y,z planes
    // pruned list (sb_nl_set_prune): the entries of cl_ent with an active slot within
    // cutoff + prune_buffer at the last prune, written by the packed pair kernel when meta[6] is
    // set (by a rebuild, by k_pack when an atom has moved more than prune_buffer / 2 since the
    // last prune, or every prune_interval updates) and read by it in the other steps. Its masks
    // keep only the slots within that radius, and each cluster's entries are sorted by which
    // slot pairs they use (the packed kernel skips a slot pair that no entry of a batch uses).
    float prune_buffer = 0.f;
    int prune_interval = 0, prune_count = 0;
    int* cl_count_in = nullptr;     // [clu_cap]
    uint32_t* cl_ent_in = nullptr;  // [clu_cap * ent_cap]
    uint32_t* cl_ent_tmp = nullptr; // [clu_cap * ent_cap] a prune's entries before the sort
    uint4* xq_prune = nullptr;      // [slot_cap] packed coordinates at the last prune
    // ATOM_GROUP compatibility export
    void* ag = nullptr;             // ATOM_GROUP[N]
    int* ag_serial = nullptr;       // [N * max_neighbor_numbers]
    int ag_valid = 0;
    int built = 0;
    int needs_rebuild = 0;
    unsigned long long build_id = 0;
};

struct sb_lennard_jones {
    int n = 0;
    int ntypes = 0;
    int form = SB_FORM_FIXED;
    float cutoff = 10.f;
    float box[3];
    float volume = 1.f;
    double long_range_factor = 0;
    float* d_A = nullptr;           // lower-triangular x12
    float* d_B = nullptr;           // lower-triangular x6
    float2* d_AB = nullptr;         // full square [ntypes*ntypes] {A12, B6}
    int* d_type = nullptr;          // [N]
    double* d_red = nullptr;        // FP64 reduction scratch
    float* d_energy_atom = nullptr; // [N] scratch for Get_Energy
    int ipl = 2;                    // pair kernel shape: 8 or 4 i atoms per lane, 2 = packed
                                    // FP32x2 slot pairs, 1 = compacted in-cutoff pairs
};

struct sb_pme {
    int n = 0;
    int form = SB_FORM_FIXED;
    float box[3];
    float cutoff = 10.f, tolerance = 1e-5f;
    float beta = 0.f;
    int K[3];
    size_t G = 0;                   // K0*K1*K2
    size_t Gh = 0;                  // K0*K1*(K2/2+1)
    double neutralizing_factor = 0; // -pi/(2 beta^2 V)
    SbFftPlan plan;
    long long* d_qfix = nullptr;    // int64 charge grid (chosen form), kept zero between calls
    float* d_qf = nullptr;          // float charge grid (plain form)
    float2* d_spec = nullptr;       // half spectrum
    float* d_theta = nullptr;       // real convolved grid
    float* d_bc = nullptr;          // [K0][K1][H] Green's function x B-spline moduli (FP64-built)
    double* d_epart = nullptr;      // per-block reciprocal energy partials
    int nparts = 0;
    double* d_ered = nullptr;       // [8] FP64 energy slots: rec, self, direct, corr
    float* d_direct_atom_energy = nullptr;
    float* d_correction_atom_energy = nullptr;
    long long* d_fix = nullptr;     // [3N] exclusion-correction accumulator (original order)
    float* energy_scratch = nullptr; // [3N] discarded forces of energy queries (first query)
    void* cufft_r2c = nullptr;      // plain form: cuFFT handles (stored as int)
    void* cufft_c2r = nullptr;
    int cufft_ok = 0;
    // fused step: the reciprocal grid chain runs on `side` (highest priority, non-blocking)
    // between a fork and a join event, concurrently with the pair kernel on the caller's stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int overlap = 1;
    int num_sms = 148;             // SMs of the device (grids of the side-stream kernels)
    int rec_nparts = 0;             // energy partials written by the last grid chain
};

// kernels/launchers shared across files
int sb_nl_ensure_built(sb_neighbor_list* nl);
int sb_nl_pack(sb_neighbor_list* nl, const uint32_t* d_uint_crd, const float* d_charge,
               const int* d_type, cudaStream_t s);
int sb_nl_finalize_forces(sb_neighbor_list* nl, float* d_frc, cudaStream_t s);
int sb_nl_retire_prune(sb_neighbor_list* nl, cudaStream_t s);
int sb_nl_build_atom_group(sb_neighbor_list* nl, cudaStream_t s);

// fused fixed-form step pieces: the pair kernel and the exclusion correction accumulate into the
// list's slot-order fixed-point buffer; the reciprocal spread reads the list's packed slot data
// and its gather finalises the buffer into d_frc
int sb_lj_fused_direct(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                       const float* d_charge, float pme_beta, int need_atom_energy,
                       float* d_atom_energy, int need_virial, float* d_atom_lj_virial,
                       float* d_atom_direct_pme_energy, cudaStream_t s);
// the pair kernel alone, on coordinates already packed by sb_nl_pack
int sb_lj_fused_pair(sb_lennard_jones* lj, sb_neighbor_list* nl, float pme_beta,
                     int need_atom_energy, float* d_atom_energy, int need_virial,
                     float* d_atom_lj_virial, float* d_atom_direct_pme_energy, cudaStream_t s);
// reciprocal part in two pieces: the grid chain (spread from the atom-order fixed-point
// coordinates and charges, FFT, convolution, inverse FFT into d_theta, gather of the forces into
// the list's slot-order fixed-point buffer, with the exclusion correction when the CSR is given;
// d_excl_energy: per-atom correction energy, zeroed first by sb_pme_zero_atom_energy, or null)
// and the finish (finalisation of that buffer into d_frc, energy and virial sums), which must
// follow the pair kernel
int sb_pme_fused_grid_atoms(sb_pme* pme, sb_neighbor_list* nl, int want_energy, cudaStream_t s,
                            const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                            const int* el, const int* en, float* d_excl_energy);
int sb_pme_zero_atom_energy(sb_pme* pme, float* d_atom_energy, cudaStream_t s);
int sb_pme_fused_finish(sb_pme* pme, sb_neighbor_list* nl, float* d_frc, const float* d_charge,
                        int need_virial, int need_energy, float* d_virial, float* d_potential,
                        cudaStream_t s);
// grid chain and finish in one call (the exclusion correction included when the CSR is given)
int sb_pme_fused_reciprocal(sb_pme* pme, sb_neighbor_list* nl, float* d_frc,
                            const uint32_t* d_uint_crd, const float* d_charge, const int* es,
                            const int* el, const int* en, int need_virial, int need_energy,
                            float* d_virial, float* d_potential, cudaStream_t s);

// FEP step: PME cross terms of dU/dlambda after sb_pme_fused_reciprocal (acc[0] reciprocal,
// acc[1] exclusion correction, 2^32 fixed point)
int sb_pme_ti_terms_slot(sb_pme* p, sb_neighbor_list* nl, const float* slot_dq,
                         const uint32_t* uc, const float* q, const float* dq, const int* es,
                         const int* el, const int* en, long long* acc, cudaStream_t s);

// 64-bit integer add to global memory with no value returned (PTX red): the fixed-point grid and
// force sums, where a returned value would only make the thread wait for the atomic's round trip
__device__ __forceinline__ void sb_red_add(long long* p, long long v) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)),
                 "l"(v));
}

// slot s of a packed list (k_pack): coordinates, charge bits and type in slot order (zeros in an
// empty slot); with a pruned list (pruned), an atom that moved more than sqrt(move2) since the
// last prune (its packed coordinates then: o) sets the prune request. The slot's atom a and o
// are loaded by the caller, beside the slot count (the packing kernels run a thread per slot of
// the allocation, so these loads need not wait for the count).
__device__ __forceinline__ void sb_pack_slot(int s, int a, uint4 o,
                                             const uint32_t* __restrict__ uc,
                                             const float* __restrict__ q,
                                             const int* __restrict__ type,
                                             uint4* __restrict__ xq, int* __restrict__ stype,
                                             bool pruned, float sx, float sy, float sz,
                                             float move2, int* __restrict__ prune_req) {
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    int t = 0;
    if (a >= 0) {
        v.x = uc[3 * a];
        v.y = uc[3 * a + 1];
        v.z = uc[3 * a + 2];
        v.w = q ? __float_as_uint(q[a]) : 0u;
        t = type ? type[a] : 0;
        if (pruned) {
            const float dx = __int2float_rn((int)(v.x - o.x)) * sx;
            const float dy = __int2float_rn((int)(v.y - o.y)) * sy;
            const float dz = __int2float_rn((int)(v.z - o.z)) * sz;
            if (dx * dx + dy * dy + dz * dz > move2) prune_req[0] = 1;
        }
    }
    xq[s] = v;
    stype[s] = t;
}

// slot s of the fixed-point force planes (k_finalize) added to the atom's float force, the
// accumulator cleared for the next step; the slot's atom a and its sums fx, fy, fz are loaded by
// the caller, beside the slot count
__device__ __forceinline__ void sb_finalize_slot(int s, int a, long long fx, long long fy,
                                                 long long fz, long long* __restrict__ fix,
                                                 int slot_cap, float* __restrict__ frc) {
    if (fx | fy | fz) {
        fix[s] = 0;
        fix[slot_cap + s] = 0;
        fix[2 * slot_cap + s] = 0;
    }
    if (a >= 0) {
        frc[3 * a] += (float)((double)fx * SB_FORCE_UNSCALE);
        frc[3 * a + 1] += (float)((double)fy * SB_FORCE_UNSCALE);
        frc[3 * a + 2] += (float)((double)fz * SB_FORCE_UNSCALE);
    }
}

// a prune request served by the pair launch before (meta[7] set) is retired
__device__ __forceinline__ void sb_retire_prune(int* __restrict__ meta) {
    if (meta[7]) {
        meta[6] = 0;
        meta[7] = 0;
    }
}

// Ewald exclusion correction of one atom inside a reciprocal gather (k_gather_atom): the
// arithmetic of k_excluded<true>, its int64 terms added to the atoms' slot accumulators
struct SbExclPass {
    const int* slot_atom;
    const int* atom_slot;
    const int* es;
    const int* el;
    const int* en;
    float sx, sy, sz, beta, beta2, beta3;
    float* ene;  // per-atom correction energy (energy steps) or null
};

// One FEP box of a batched step (sb_fep_batch_*): the device pointers and constants that the
// batched kernels of every stage read, gathered from the box's list, soft-core and PME modules
// and from the caller's buffers bound to the batch.
#define SB_FEP_BATCH_THREADS 256  // threads per block of the batched per-atom and per-slot kernels
struct SbFepBox {
    // neighbor list
    int* meta;
    const int* cl_count;
    const uint32_t* cl_ent;
    uint4* xq;
    int* stype;
    const int* slot_atom;
    long long* fix;
    const uint4* xq_prune;  // null without a pruned list
    float move2;            // squared displacement that requests a prune
    float usx, usy, usz;    // length of one fixed-point coordinate unit in the list's box
    int slot_cap;
    // soft core
    const int* typeA;
    const int* typeB;
    const int* mask;
    const float* dq;
    int* slot_ext;
    float* slot_dq;
    const float2* ABa;
    const float2* ABb;
    long long* hfix;  // [4] dH/dlambda parts: LJ, direct, reciprocal, correction
    double* sums;     // [3] FP64 sums of q dq, q, dq (self term)
    // split form (sb_softcore split != 0): the A-state square table with a zero ghost type
    // (ntA) for the packed kernel, each atom's A type or the ghost type, the perturbed atoms
    int split;
    int ghost;
    const int* tu;
    const float2* ABu;
    const int* pert;
    int npert;
    int2* ppairs;  // pairs with a perturbed atom found this step: {perturbed index, slot}
    int* pcount;
    int pcap;
    // reciprocal space
    long long* qfix;
    const float* theta;
    int K0, K1, K2;
    float ix, iy, iz;
    SbExclPass X;
    // the caller's buffers and the finishing constants
    const uint32_t* uc;
    const float* q;
    float* frc;
    double* dudl;
    int n;
    double self_coef, neutral2, lrc;
};

// FEP split form: the packed pair kernel over the unperturbed pairs of a box packed by the FEP
// step (sb_pair.cu); the batched form over several boxes' clusters, grouped by common parameters
bool sb_pair_fep_packed(const sb_neighbor_list* nl, float cutoff, float beta);
int sb_pair_fep(sb_neighbor_list* nl, const float2* d_AB, int ntypes, float cutoff, float beta,
                cudaStream_t s);
struct SbX2Batch;
int sb_pair_batch_create(int nb, const int* box_ids, sb_neighbor_list* const* nls,
                         const float2* const* tables, const int* ntypes, const float* cutoffs,
                         const float* betas, SbX2Batch** out);
int sb_pair_batch_launch(const SbX2Batch* x, cudaStream_t s);
int sb_pair_batch_launches(const SbX2Batch* x);
void sb_pair_batch_destroy(SbX2Batch* x);

// batched stages over all boxes; tab[b] = {box, block of that box} for every launched block
int sb_pme_batch_spread(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, cudaStream_t s);
int sb_pme_batch_gather(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, int dh,
                        cudaStream_t s);
int sb_pme_batch_slots(const SbFepBox* d_boxes, const int2* d_tab, int nblocks, int dh,
                       cudaStream_t s);

// FP64 reduction helpers (deterministic: fixed block/thread order)
int sb_reduce_sum_f32(const float* d_x, int n, double* d_out, cudaStream_t s);

static inline cudaStream_t sb_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
