/*
 * sponge_b200 — C ABI of a B200 (sm_100a) implementation of SPONGE's nonbonded hot path:
 * the cell-grid neighbor-list rebuild, the Lennard-Jones + PME direct-space pair
 * force/energy/virial, and PME reciprocal space.
 *
 * The three handle types mirror SPONGE's three module structs; every entry point names the
 * reference method it replaces (paths relative to the SPONGE project root, SPONGE/...).
 * Plain pointers and sizes only: device pointers are prefixed d_, host pointers h_. Streams are
 * passed as void* holding a cudaStream_t (NULL = legacy default stream, as the reference uses).
 *
 * Units and layouts follow the reference: lengths in Angstrom, energies in kcal/mol, charges
 * pre-multiplied by 18.2223, coordinates as unsigned-int fixed point (3 x uint32 per atom,
 * UNSIGNED_INT_VECTOR), forces as float VECTOR (3 x float per atom) accumulated with +=,
 * per-atom energies/virials as float[N] accumulated with +=, d_virial / d_potential as single
 * device floats accumulated with +=.
 *
 * Every function returns SB_OK (0) or an SB_ERR_* code; sb_last_error() gives the message.
 */
#ifndef SPONGE_B200_H
#define SPONGE_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define SB_API __attribute__((visibility("default")))
#else
#define SB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SB_OK 0
#define SB_ERR_ARG 1      /* invalid argument (null handle, bad size, mismatched atom count) */
#define SB_ERR_CUDA 2     /* a CUDA runtime call or kernel launch failed */
#define SB_ERR_ALLOC 3    /* device or host allocation failed */
#define SB_ERR_OVERFLOW 4 /* a fixed-capacity buffer overflowed (see sb_nl_status) */
#define SB_ERR_STATE 5    /* call order violated (e.g. force before the first list build) */

/* Accumulation forms (the `form` argument of the create functions). */
#define SB_FORM_FIXED 0 /* FP32 pair math, 64-bit fixed-point accumulation: bit-identical runs */
#define SB_FORM_PLAIN 1 /* FP32 pair math, float atomics, per-atom lists, library FFT */

/* Status flags reported by sb_nl_status (OR-ed). */
#define SB_STATUS_LIST_OVERFLOW 1    /* a cluster's pair-entry capacity was exceeded */
#define SB_STATUS_COLUMN_OVERFLOW 2  /* a sort column held more atoms than the sort capacity */
#define SB_STATUS_ATOMGROUP_OVERFLOW 4 /* an atom exceeded max_neighbor_numbers in the export */

/* Particle_Mesh_Ewald::PME_ENERGY_PART (SPONGE/PME_force/PME_force.cuh:86-93) */
#define SB_PME_TOTAL 0
#define SB_PME_DIRECT 1
#define SB_PME_RECIPROCAL 2
#define SB_PME_CORRECTION 3
#define SB_PME_SELF 4

typedef struct sb_neighbor_list sb_neighbor_list;
typedef struct sb_lennard_jones sb_lennard_jones;
typedef struct sb_pme sb_pme;
typedef struct sb_adjoint sb_adjoint;
typedef struct sb_softcore sb_softcore;

/* Library version (integer) and the message of the last failed call on this host thread. */
SB_API int sb_version(void);
SB_API const char* sb_last_error(void);

/* ------------------------------------------------------------------------------------------
 * Neighbor list — replaces NEIGHBOR_LIST (SPONGE/neighbor_list/neighbor_list.cuh:44-106)
 * ---------------------------------------------------------------------------------------- */

/* NEIGHBOR_LIST::Initial (SPONGE/neighbor_list/neighbor_list.cu:688-750). skin_permit is the
 * mdin value (the reference doubles it internally, :718); pass 0.5 for the reference default.
 * max_neighbor_numbers sizes the ATOM_GROUP compatibility export (reference default 800). */
SB_API int sb_nl_create(int atom_numbers, const float box_length[3], float cutoff, float skin,
                 int refresh_interval, float skin_permit, int max_neighbor_numbers, int form,
                 sb_neighbor_list** out);

/* NEIGHBOR_LIST::Clear (neighbor_list.cu:767-819) */
SB_API int sb_nl_destroy(sb_neighbor_list* nl);

/* NEIGHBOR_LIST::Neighbor_List_Update (neighbor_list.cu:618-664). d_crd is VECTOR[N] and is
 * wrapped into the box in place on every rebuild, as the reference does. The exclusion CSR is
 * SPONGE's (MD_core/MD_core.cu:308-351): for atom i, d_excluded_list[start[i] .. start[i] +
 * numbers[i]) lists the excluded partners j > i. Policy: forced_update rebuilds; else with
 * refresh_interval > 0 and !forced_check every refresh_interval-th call rebuilds; else the
 * rebuild happens when an atom moved more than skin_permit*skin/2 since the last rebuild. */
SB_API int sb_nl_update(sb_neighbor_list* nl, float* d_crd, const int* d_excluded_list_start,
                 const int* d_excluded_list, const int* d_excluded_numbers, int forced_update,
                 int forced_check, void* stream);

/* NEIGHBOR_LIST::Update_Volume (neighbor_list.cu:753-764): box change without re-gridding.
 * The next update call rebuilds. */
SB_API int sb_nl_update_volume(sb_neighbor_list* nl, const float box_length[3]);

/* Materialises the reference's public member `ATOM_GROUP* d_nl` (neighbor_list.cuh:75): an
 * ATOM_GROUP[N] device array ({int atom_numbers; int* atom_serial}) whose per-atom lists hold
 * the same half pair set (j > i, exclusions removed, within cutoff+skin). The array and its
 * serial storage are owned by the handle; *d_atom_group receives its device address. Consumers
 * that read d_nl directly (Get_Energy, FEP_CORE, TI_CORE) use this. */
SB_API int sb_nl_atom_group(sb_neighbor_list* nl, void** d_atom_group, void* stream);

/* Number of half pairs currently in the list (synchronises the stream). */
SB_API int sb_nl_pair_count(sb_neighbor_list* nl, int64_t* h_count, void* stream);

/* Copies the half pair set as sorted keys i*N + j (i < j, original atom ids) into h_keys
 * (capacity cap). *h_count receives the count; fails with SB_ERR_OVERFLOW if cap is short. */
SB_API int sb_nl_export_pairs(sb_neighbor_list* nl, int64_t* h_keys, int64_t cap, int64_t* h_count,
                       void* stream);

/* Pruned pair list (no reference counterpart; off by default). With prune_buffer > 0 the packed
 * pair kernel (shape 2) walks a list holding only the entries with a pair within
 * cutoff + prune_buffer at the last prune, instead of the full cutoff + skin list. A prune runs
 * inside the pair launch after every rebuild, when an atom has moved more than prune_buffer / 2
 * since the last prune (tested while packing coordinates), and every prune_interval list updates
 * (0: never on a count, which the displacement test makes safe; a count only adds prunes). A
 * prune keeps in each entry only the slots within that radius and sorts each cluster's entries
 * by the slot pairs they use, so that the walk can skip slot pairs a whole batch does not use.
 * Every pair within the cut-off stays in the walked list, so the pair set evaluated is
 * unchanged; the i-atom sums run over other entries in another order, so forces may differ from
 * the unpruned walk in FP32 rounding, and do not depend on whether a launch pruned. With the
 * displacement-check policy (refresh_interval 0) the skin left for motion before a rebuild
 * becomes skin - prune_buffer. Requires 0 <= prune_buffer <= skin; 0 turns pruning off. */
SB_API int sb_nl_set_prune(sb_neighbor_list* nl, float prune_buffer, int prune_interval);

/* OR of SB_STATUS_* flags raised since the last call (synchronises the stream, clears them). */
SB_API int sb_nl_status(sb_neighbor_list* nl, int* h_flags, void* stream);

/* The list's own fixed-point coordinates (UNSIGNED_INT_VECTOR[N], NEIGHBOR_LIST::uint_crd). */
SB_API int sb_nl_uint_crd(sb_neighbor_list* nl, const uint32_t** d_uint_crd);

/* ------------------------------------------------------------------------------------------
 * Lennard-Jones + PME direct space — replaces LENNARD_JONES_INFORMATION
 * (SPONGE/Lennard_Jones_force/Lennard_Jones_force.cuh:41-149)
 * ---------------------------------------------------------------------------------------- */

/* LENNARD_JONES_INFORMATION::Initial (Lennard_Jones_force.cu:1067-1139). h_LJ_A / h_LJ_B are
 * the lower-triangular tables as the module stores them (already x12 and x6, pair index
 * max*(max+1)/2 + min), h_atom_LJ_type the per-atom type. The long-range correction factor is
 * computed in FP64 from type counts. */
SB_API int sb_lj_create(int atom_numbers, int atom_type_numbers, const float* h_LJ_A,
                 const float* h_LJ_B, const int* h_atom_LJ_type, float cutoff,
                 const float box_length[3], int form, sb_lennard_jones** out);

/* LENNARD_JONES_INFORMATION::Clear (Lennard_Jones_force.cu:1141-1176) */
SB_API int sb_lj_destroy(sb_lennard_jones* lj);

/* LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (Lennard_Jones_force.cu:1318-1352): LJ + Ewald direct force over the list of `nl`, added to
 * d_frc. need_atom_energy adds LJ + direct Coulomb energy per atom into d_atom_energy;
 * need_virial adds the LJ virial per atom into d_atom_lj_virial and overwrites
 * d_atom_direct_pme_energy with the direct Coulomb energy per atom. */
SB_API int sb_lj_pme_direct_force(sb_lennard_jones* lj, sb_neighbor_list* nl, int atom_numbers,
                           const uint32_t* d_uint_crd, const float* d_charge, float* d_frc,
                           float pme_beta, int need_atom_energy, float* d_atom_energy,
                           int need_virial, float* d_atom_lj_virial,
                           float* d_atom_direct_pme_energy, void* stream);

/* LENNARD_JONES_INFORMATION::Long_Range_Correction (Lennard_Jones_force.cu:1178-1191) */
SB_API int sb_lj_long_range_correction(sb_lennard_jones* lj, int need_pressure, float* d_virial,
                                int need_potential, float* d_potential, void* stream);

/* LENNARD_JONES_INFORMATION::Get_Energy (Lennard_Jones_force.cu:1407-1433): LJ energy within
 * the cutoff over the list plus the long-range correction, reduced in FP64. */
SB_API int sb_lj_get_energy(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                     float* h_energy, void* stream);

/* LENNARD_JONES_INFORMATION::Update_Volume */
SB_API int sb_lj_update_volume(sb_lennard_jones* lj, const float box_length[3]);

/* Pair-kernel shape of the fixed-point form (no reference counterpart; a tuning knob):
 * i atoms held per lane, 8 (one lane per list entry) or 4 (two lanes per entry, fewer registers,
 * more resident warps); 2: the eight-atom layout evaluated two (i, j) slots at a time on the
 * packed FP32x2 instructions (the default); or 1: the compacted kernel, which first filters each
 * batch of entries to the pairs inside the cutoff and then evaluates one such pair per lane.
 * Results are identical to FP32 rounding whichever shape runs. */
SB_API int sb_lj_set_kernel_variant(sb_lennard_jones* lj, int atoms_per_lane);

/* Autotuner: times each pair-kernel shape on the current list and keeps the fastest; writes the
 * choice to *h_chosen. Synchronises the stream; leaves d_frc untouched. The shapes sum in
 * different orders, so a process that needs the same bits as another sets the shape explicitly
 * (sb_lj_set_kernel_variant) rather than tuning (the default shape is 2). */
SB_API int sb_lj_tune(sb_lennard_jones* lj, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                      const float* d_charge, float pme_beta, int* h_chosen, void* stream);

/* Public members read by other modules: long_range_factor (FP64-computed, returned as float). */
SB_API int sb_lj_long_range_factor(sb_lennard_jones* lj, float* h_factor);

/* ------------------------------------------------------------------------------------------
 * PME — replaces Particle_Mesh_Ewald (SPONGE/PME_force/PME_force.cuh:25-123)
 * ---------------------------------------------------------------------------------------- */

/* Particle_Mesh_Ewald::Initial (PME_force.cu:108-306). fft* <= 0 picks the size as the
 * reference's Get_Fft_Patameter does; tolerance is PME_Direct_Tolerance (default 1e-5). The
 * B-spline moduli and the Green's-function table are computed in FP64. */
SB_API int sb_pme_create(int atom_numbers, const float box_length[3], float cutoff, float tolerance,
                  int fftx, int ffty, int fftz, int form, sb_pme** out);

/* Particle_Mesh_Ewald::Clear */
SB_API int sb_pme_destroy(sb_pme* pme);

/* Public members beta, fftx/ffty/fftz, and the device arrays d_direct_atom_energy (filled by
 * sb_lj_pme_direct_force with need_virial) and d_correction_atom_energy (filled by
 * sb_pme_excluded_force), which the reference reads in its energy and virial sums. */
SB_API int sb_pme_info(sb_pme* pme, float* h_beta, int* h_fft3);
SB_API int sb_pme_atom_energy_arrays(sb_pme* pme, float** d_direct_atom_energy,
                              float** d_correction_atom_energy);

/* FFT kernel family of the fixed-point form (no reference counterpart; a tuning knob):
 * SB_FFT_AUTO (the default) runs the register line transforms on every axis whose size has one
 * (N = N1 * N2 with small 2/3/5-smooth factors) and the generic mixed-radix stage kernels on the
 * others, and, for square x-y planes (30, 32, 36, 40, 48, 50, 54, 60, 64, 80, 96, 128) with
 * register transforms on every axis, fuses the y and x passes of each kz plane into one block
 * (same transforms, same bits as SB_FFT_LINES); SB_FFT_LINES runs the register line transforms pass by pass; SB_FFT_GENERIC runs
 * only the stage kernels. The choice is a fixed rule, not a timing, so the same grid gives the
 * same bits in every process. Synchronises the device and clears the spectrum buffer; call it
 * outside stream capture. The register and generic families agree to FP32 rounding. */
#define SB_FFT_AUTO 0
#define SB_FFT_GENERIC 1
#define SB_FFT_LINES 2
SB_API int sb_pme_set_fft_variant(sb_pme* pme, int variant);

/* Particle_Mesh_Ewald::PME_Excluded_Force_With_Atom_Energy (PME_force.cu:697-708): Ewald
 * correction for every exclusion CSR entry, force added to d_frc, per-atom correction energy
 * written (reset then +=) to d_atom_energy (the reference passes d_correction_atom_energy). */
SB_API int sb_pme_excluded_force(sb_pme* pme, const uint32_t* d_uint_crd, const float scaler[3],
                          const float* d_charge, const int* d_excluded_list_start,
                          const int* d_excluded_list, const int* d_excluded_numbers,
                          float* d_frc, float* d_atom_energy, void* stream);

/* Particle_Mesh_Ewald::PME_Reciprocal_Force_With_Energy_And_Virial (PME_force.cu:722-773):
 * B-spline spread, 3D real FFT, Green's-function convolution, inverse FFT, force gather (added
 * to d_frc). need_energy adds correction + self + reciprocal energy to *d_potential;
 * need_virial adds direct + correction + self + reciprocal energy to *d_virial. */
SB_API int sb_pme_reciprocal_force(sb_pme* pme, const uint32_t* d_uint_crd, const float* d_charge,
                            float* d_frc, int need_virial, int need_energy, float* d_virial,
                            float* d_potential, void* stream);

/* Particle_Mesh_Ewald::Get_Energy (PME_force.cu:892-994). which_part is SB_PME_*. The DIRECT
 * part is evaluated over the list of `nl` (may be NULL for other parts; it must hold as many
 * atoms as `pme`). h_parts (optional, 5 doubles) receives total, direct, reciprocal, correction,
 * self as computed (FP64). The forces that the reciprocal and exclusion passes produce on the
 * way are discarded into a 3N-float array of the module, allocated on the first call and kept
 * until sb_pme_destroy. */
SB_API int sb_pme_get_energy(sb_pme* pme, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                      const float* d_charge, const float scaler[3],
                      const int* d_excluded_list_start, const int* d_excluded_list,
                      const int* d_excluded_numbers, int which_part, float* h_energy,
                      double* h_parts, void* stream);

/* Allocation-free variant of sb_pme_get_energy (no counterpart in the reference). Same
 * arguments and results. sb_pme_get_energy allocates and frees a 3N-float array on every call
 * for the forces its reciprocal and exclusion passes produce and then discard; this variant uses
 * a fixed 1.5 MiB device block of the library instead, for callers that cannot allocate:
 * programs whose device memory is all handed to their own pool allocator, and loops that must
 * not pay for cudaFree, which waits for the whole device. The block exists on a device once the
 * library's device code is loaded there, which happens at the latest in sb_pme_create.
 *   - at most 131072 atoms (larger modules are rejected with SB_ERR_ARG); `nl` must hold as many
 *     atoms as `pme` when the DIRECT part (or TOTAL) is asked for (else SB_ERR_ARG);
 *   - the first call on each device looks up the block's device address (with that device
 *     current) and keeps it for the life of the process; make that first call before beginning
 *     any stream capture. The kept address does not survive cudaDeviceReset or anything else
 *     that destroys the device's primary context: do not call this entry point after that;
 *   - the DIRECT part (and TOTAL) reads the list's ATOM_GROUP export, which allocates on first
 *     use: call sb_nl_atom_group once beforehand, or the call fails with SB_ERR_STATE;
 *   - every call on a device shares the one block: calls whose GPU work overlaps (other streams,
 *     other host threads) race on it. Each call clears the part it uses before use. */
SB_API int sb_pme_get_energy_noalloc(sb_pme* pme, sb_neighbor_list* nl,
                      const uint32_t* d_uint_crd, const float* d_charge, const float scaler[3],
                      const int* d_excluded_list_start, const int* d_excluded_list,
                      const int* d_excluded_numbers, int which_part, float* h_energy,
                      double* h_parts, void* stream);

/* The member PME_BC of Particle_Mesh_Ewald (PME_force.cu:253-286), which TI_CORE reads: the
 * device address of the module's Green's-function table (B-spline moduli included, built in
 * FP64), float [fftx][ffty][fftz/2+1] in the layout of a real-to-complex transform's half
 * spectrum, element [0] = 0. Owned by the module; sb_pme_update_box rewrites it in place. */
SB_API int sb_pme_bc_table(sb_pme* pme, const float** d_bc);

/* Particle_Mesh_Ewald::Update_Box_Length / Update_Volume (PME_force.cu:996-1042) */
SB_API int sb_pme_update_box(sb_pme* pme, const float box_length[3]);

/* ------------------------------------------------------------------------------------------
 * Whole nonbonded force evaluation of one MD step, as Main_Calculate_Force + Main_Iteration
 * call the three modules (SPONGE/main.cu:180-193 and :376): list update by its policy, LJ +
 * direct, long-range correction, exclusion correction, reciprocal space. Forces are added to
 * d_frc. The flags and outputs have the meanings of the module calls above.
 * ---------------------------------------------------------------------------------------- */
SB_API int sb_nonbonded_step(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme, float* d_crd,
                      const uint32_t* d_uint_crd, const float* d_charge,
                      const int* d_excluded_list_start, const int* d_excluded_list,
                      const int* d_excluded_numbers, float* d_frc, int need_energy,
                      int need_virial, float* d_atom_energy, float* d_atom_virial,
                      float* d_virial, float* d_potential, void* stream);

/* The force part of sb_nonbonded_step with the list as it stands (no update): a fixed sequence
 * of kernel launches with no host synchronisation, so a driver may capture it in a CUDA graph
 * and replay it between list updates. */
SB_API int sb_nonbonded_force(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                       const uint32_t* d_uint_crd, const float* d_charge,
                       const int* d_excluded_list_start, const int* d_excluded_list,
                       const int* d_excluded_numbers, float* d_frc, int need_energy,
                       int need_virial, float* d_atom_energy, float* d_atom_virial,
                       float* d_virial, float* d_potential, void* stream);

/* Overlap switch of the fixed-form force part (no reference counterpart; a scheduling knob, on
 * by default): the exclusion correction and the reciprocal grid chain (spread, FFT, convolution,
 * inverse FFT) run on a high-priority stream owned by the PME module, forked from and joined back
 * to the caller's stream, concurrently with the pair kernel. Forces are bit-identical either way
 * (integer accumulation); a graph captured from the caller's stream holds both branches. */
SB_API int sb_nonbonded_set_overlap(sb_pme* pme, int on);

/* ------------------------------------------------------------------------------------------
 * NON_BOND_14 (SPONGE/nb14/nb14.cuh:41-86): scaled 1-4 LJ and Coulomb pairs
 * ---------------------------------------------------------------------------------------- */
typedef struct sb_nb14 sb_nb14;

/* NON_BOND_14::Initial (nb14.cu:172-246) from arrays: pair atoms a, b; per-pair A (x12) and B
 * (x6), i.e. lj_scale * LJ_A[type pair] as Initial computes them from the LJ tables, and the
 * Coulomb scale factor. */
SB_API int sb_nb14_create(int atom_numbers, int nb14_numbers, const int* h_atom_a,
                          const int* h_atom_b, const float* h_A, const float* h_B,
                          const float* h_cf_scale, sb_nb14** out);
SB_API int sb_nb14_destroy(sb_nb14* nb14);
/* Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial (nb14.cu:467-480): frc += on both atoms,
 * atom_energy / atom_virial += on the first atom of each pair (either may be NULL). */
SB_API int sb_nb14_force(sb_nb14* nb14, const uint32_t* d_uint_crd, const float* d_charge,
                         const float scaler[3], float* d_frc, float* d_atom_energy,
                         float* d_atom_virial, void* stream);
/* Get_14_LJ_Energy / Get_14_CF_Energy (nb14.cu:482-520), summed in FP64; either output may be
 * NULL. Synchronises the stream. */
SB_API int sb_nb14_energy(sb_nb14* nb14, const uint32_t* d_uint_crd, const float* d_charge,
                          const float scaler[3], double* h_lj_energy, double* h_cf_energy,
                          void* stream);

/* ------------------------------------------------------------------------------------------
 * VIRTUAL_INFORMATION (SPONGE/virtual_atoms/virtual_atoms.cuh:86-142): virtual atoms of types
 * 0 (mirror of atom 1 in z = h), 1 (r_1 + a r_21), 2 (r_1 + a r_21 + b r_31) and 3
 * (r_1 + d (r_21 + k r_32)/|r_21 + k r_32|)
 * ---------------------------------------------------------------------------------------- */
typedef struct sb_vsite sb_vsite;

/* VIRTUAL_INFORMATION::Initial (virtual_atoms.cu:181-490) from arrays: per record its type,
 * atoms[4] = {virtual atom, from_1, from_2, from_3} (unused parents ignored) and param[2] = the
 * type's numbers as the virtual_atom_in_file line gives them (type 0: h; 1: a; 2: a, b; 3: d,
 * k). Levels (a virtual atom built from virtual atoms sits one level above them) are computed
 * here. */
SB_API int sb_vsite_create(int atom_numbers, int virtual_numbers, const int* h_type,
                           const int* h_atoms, const float* h_param, sb_vsite** out);
SB_API int sb_vsite_destroy(sb_vsite* vsite);
/* Coordinate_Refresh: crd of every virtual atom from its parents, lowest level first. */
SB_API int sb_vsite_coordinate_refresh(sb_vsite* vsite, const uint32_t* d_uint_crd,
                                       const float scaler[3], float* d_crd, void* stream);
/* Force_Redistribute: the force on each virtual atom moves to its parents and the virtual
 * atom's force is zeroed, highest level first. */
SB_API int sb_vsite_force_redistribute(sb_vsite* vsite, const uint32_t* d_uint_crd,
                                       const float scaler[3], float* d_frc, void* stream);

/* ------------------------------------------------------------------------------------------
 * Integration with rigid-water constraints: the NVE leap-frog of MD_INFORMATION
 * (SPONGE/MD_core/MD_core.cu:13-32) and SETTLE (SPONGE/constrain/SETTLE.cuh:33-64), in
 * Main_Iteration's order (SPONGE/main.cu:283-325). dt is the integrator's internal time step
 * (MD_INFORMATION::dt: the mdin dt in ps times SPONGE's time unit conversion).
 * ---------------------------------------------------------------------------------------- */
typedef struct sb_settle sb_settle;

/* SETTLE::Initial (SETTLE.cu:183-354) from CONSTRAIN's pair list (atom i, atom j, length r, in
 * CONSTRAIN's order; CONSTRAIN::Add_HBond_To_Constrain_Pair puts there every bond with an atom
 * lighter than 3.3): closed triangles of constrained pairs become rigid triangles, isolated
 * pairs rigid pairs, the rest is left to another constraint scheme (counted by sb_settle_info).
 * exp_gamma is the thermostat's velocity factor (1 for NVE), as CONSTRAIN::Initial_Constrain
 * takes it. */
SB_API int sb_settle_create(int atom_numbers, int constrain_pair_numbers, const int* h_pair_i,
                            const int* h_pair_j, const float* h_pair_r, const float* h_mass,
                            float dt, float exp_gamma, sb_settle** out);
SB_API int sb_settle_destroy(sb_settle* settle);
SB_API int sb_settle_info(sb_settle* settle, int* h_triangles, int* h_pairs, int* h_remaining);
/* SETTLE::Remember_Last_Coordinates: edge vectors of the step start (fixed point). */
SB_API int sb_settle_remember(sb_settle* settle, const uint32_t* d_uint_crd,
                              const float scaler[3], void* stream);
/* SETTLE::Do_SETTLE: constrain crd and vel after the integrator; with need_pressure the
 * constraint virial / (3V) is added to *d_pressure. */
SB_API int sb_settle_apply(sb_settle* settle, const float* d_mass, float* d_crd,
                           const float box[3], float* d_vel, int need_pressure,
                           float* d_pressure, void* stream);
/* MD_INFORMATION::NVE_iteration::Leap_Frog (MD_core.cu:1535-1547): acc = F/m, vel += dt acc,
 * crd += dt vel (d_acc may be NULL). */
SB_API int sb_md_leap_frog(int atom_numbers, const float* d_inverse_mass, const float* d_frc,
                           float* d_vel, float* d_crd, float* d_acc, float dt, void* stream);
/* Remember + leap-frog + SETTLE in one launch (no reference counterpart as one call; the
 * same bits as the three calls in sequence). Refuses a system whose constraints are not all
 * rigid triangles or pairs. */
SB_API int sb_md_nve_settle_step(sb_settle* settle, const uint32_t* d_uint_crd,
                                 const float scaler[3], const float* d_inverse_mass,
                                 const float* d_mass, const float* d_frc, float* d_vel,
                                 float* d_crd, float* d_acc, const float box[3],
                                 int need_pressure, float* d_pressure, void* stream);

/* Crd_To_Uint_Crd (SPONGE/common.cu:264-287) with the quarter coefficient 0.25*2^32/L, as
 * MD_INFORMATION::MD_Information_Crd_To_Uint_Crd produces md_info.uint_crd. */
SB_API int sb_crd_to_uint_crd(int atom_numbers, const float box_length[3], const float* d_crd,
                       uint32_t* d_uint_crd, void* stream);

/* ------------------------------------------------------------------------------------------
 * Soft-core LJ for FEP/TI — replaces LJ_SOFT_CORE (SPONGE/Lennard_Jones_force/LJ_soft_core.cuh:
 * 42-159) and the PME cross terms of TI_CORE (SPONGE/TI_core/TI_core.cu:670-730)
 * ---------------------------------------------------------------------------------------- */

/* LJ_SOFT_CORE::Initial (LJ_soft_core.cu:1420-1610). Two end states A and B with their own type
 * sets: h_LJ_AA / h_LJ_AB the lower-triangular A-state tables (x12, x6 as the LJ module stores
 * them) over atom_type_numbers_A types, h_LJ_BA / h_LJ_BB the B-state tables; per atom the A and B
 * types, the perturbation mask (pairs whose masks differ are soft-cored) and the charge change
 * h_charge_B_A = q_B - q_A. Soft core: r_A^6 = r^6 + alpha lambda^p sigma_A^6 and
 * r_B^6 = r^6 + alpha (1 - lambda)^p sigma_B^6 with sigma^6 = max(A/(2B), sigma_min^6) of the
 * pair (sigma^6 when either coefficient is zero). lambda is lambda_lj. */
SB_API int sb_sc_create(int atom_numbers, int atom_type_numbers_A, const float* h_LJ_AA,
                        const float* h_LJ_AB, int atom_type_numbers_B, const float* h_LJ_BA,
                        const float* h_LJ_BB, const int* h_atom_LJ_type_A,
                        const int* h_atom_LJ_type_B, const int* h_mask,
                        const float* h_charge_B_A, float cutoff, const float box_length[3],
                        float lambda, float alpha, float p, float sigma, float sigma_min, int form,
                        sb_softcore** out);
SB_API int sb_sc_destroy(sb_softcore* sc);

/* Moves the module to another coupling parameter (one lambda window); recomputes the
 * lambda-mixed long-range correction factor. */
SB_API int sb_sc_set_lambda(sb_softcore* sc, float lambda);

/* The split form of sb_fep_step / sb_fep_batch_step (no reference counterpart): the perturbed
 * atoms are those with a mask or a charge change, or whose (A, B) type pair makes the B-state
 * table differ from the A-state table against the other atoms. With at most 512 of them and at
 * most one atom in eight, the pairs of two unperturbed atoms (whose soft-core energy is their
 * A-state energy, with no dH/dlambda) run through the packed LJ + Ewald kernel and the pairs with
 * a perturbed atom through a soft-core pass over the perturbed atoms. *h_split = 1 when the
 * module uses it, *h_n_perturbed = the perturbed atom count. */
SB_API int sb_sc_split_form(const sb_softcore* sc, int* h_split, int* h_n_perturbed);

/* LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial: soft-core LJ + Ewald
 * direct force over the list of `nl` added to d_frc (d_charge holds the charges at lambda), with
 * the per-atom energy / LJ virial / direct energy outputs of sb_lj_pme_direct_force. */
SB_API int sb_sc_pme_direct_force(sb_softcore* sc, sb_neighbor_list* nl, int atom_numbers,
                                  const uint32_t* d_uint_crd, const float* d_charge, float* d_frc,
                                  float pme_beta, int need_atom_energy, float* d_atom_energy,
                                  int need_virial, float* d_atom_lj_virial,
                                  float* d_atom_direct_pme_energy, void* stream);

/* LJ_SOFT_CORE::Long_Range_Correction with the lambda-mixed dispersion factor. */
SB_API int sb_sc_long_range_correction(sb_softcore* sc, int need_pressure, float* d_virial,
                                       int need_potential, float* d_potential, void* stream);

/* LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct (LJ_soft_core.cu:1137-1283) and
 * Partial_H_Partial_Lambda_Long_Range_Correction (:1939-1953): h_dhdl[0] = LJ, h_dhdl[1] = direct
 * Coulomb (including the charge change at fixed geometry), h_dhdl[2] = long-range correction.
 * Exact derivatives of the soft-core energy (FP64 sums). Synchronises the stream. */
SB_API int sb_sc_dh_dlambda(sb_softcore* sc, sb_neighbor_list* nl, const uint32_t* d_uint_crd,
                            const float* d_charge, float pme_beta, double* h_dhdl, void* stream);

/* TI_CORE::Get_Cross_PME_Partial_H_Partial_Lambda: for charges d_charge changing by
 * d_charge_B_A per unit lambda, h_parts[0] = reciprocal sum_i dq_i phi_i (phi the SPME potential),
 * h_parts[1] = self + neutralising derivative, h_parts[2] = exclusion-correction derivative.
 * Synchronises the stream. */
SB_API int sb_pme_ti_cross(sb_pme* pme, const uint32_t* d_uint_crd, const float* d_charge,
                           const float* d_charge_B_A, const int* d_excluded_list_start,
                           const int* d_excluded_list, const int* d_excluded_numbers,
                           double* h_parts, void* stream);

/* One FEP force evaluation at the module's lambda with dU/dlambda, fixed-point form, no host
 * synchronisation: soft-core LJ + direct, long-range correction, exclusion correction and
 * reciprocal space (charges d_charge at lambda) added to d_frc; *d_dudl (one device double)
 * receives dU/dlambda = soft-core LJ + direct + PME cross terms + long-range correction. The list
 * of `nl` must be current (sb_nl_update is not called). */
SB_API int sb_fep_step(sb_neighbor_list* nl, sb_softcore* sc, sb_pme* pme,
                       const uint32_t* d_uint_crd, const float* d_charge,
                       const int* d_excluded_list_start, const int* d_excluded_list,
                       const int* d_excluded_numbers, float* d_frc, double* d_dudl, void* stream);

/* Many FEP windows stepped together (the loop over lambda windows of a SPONGE_FEP / SPONGE_TI
 * campaign, main_fep.cu:56-132, one process per window there): sb_fep_step of every box, one
 * launch per stage over all boxes (pack, soft-core pair, spread, gather, finalize, dU/dlambda
 * finish) plus one launch per FFT stage per group of equal grid sizes. Box k reads
 * d_uint_crd[k], d_charge[k] and its exclusion lists, adds its forces into d_frc[k] and writes
 * its dU/dlambda to the device double d_dudl[k] (d_dudl: n_boxes pointers, or NULL for forces
 * only). Each box gets the same bits as its own sb_fep_step. The pair stage, the soft-core
 * passes and the reciprocal chain run on library-owned streams forked from and joined back
 * into `stream` (capturable in a CUDA graph).
 * The batch records the modules' buffers, capacities, boxes and lambdas at creation: after a
 * box or lambda change (sb_*_update_volume, sb_sc_set_lambda) or sb_nl_set_prune, create it
 * again (sb_fep_batch_step refuses with SB_ERR_STATE). Every list must be built before
 * sb_fep_batch_create; later list updates (same capacities) need nothing. The caller's arrays
 * (d_uint_crd, d_charge, ...) are read through device pointers stored at creation, so a captured
 * CUDA graph of sb_fep_batch_step stays valid as long as those buffers do. */
typedef struct sb_fep_batch sb_fep_batch;
SB_API int sb_fep_batch_create(int n_boxes, sb_neighbor_list* const* nls,
                               sb_softcore* const* scs, sb_pme* const* pmes,
                               const uint32_t* const* d_uint_crd, const float* const* d_charge,
                               const int* const* d_excluded_list_start,
                               const int* const* d_excluded_list,
                               const int* const* d_excluded_numbers, float* const* d_frc,
                               double* const* d_dudl, sb_fep_batch** out);
SB_API int sb_fep_batch_step(sb_fep_batch* batch, void* stream);
/* kernel launches of one sb_fep_batch_step */
SB_API int sb_fep_batch_launches(const sb_fep_batch* batch);
SB_API int sb_fep_batch_destroy(sb_fep_batch* batch);

/* ------------------------------------------------------------------------------------------
 * Differentiation for force-field fitting (no reference counterpart: SPONGE has no gradients
 * with respect to parameters). Fixed-point form of all three modules only.
 * ---------------------------------------------------------------------------------------- */

/* Parameter update for fitting: replaces the LJ pair tables (same layout and scaling as
 * sb_lj_create: lower-triangular, already x12 and x6) and recomputes the long-range correction
 * factor. The atom types are unchanged. Copies from the host (synchronous). */
SB_API int sb_lj_set_tables(sb_lennard_jones* lj, const float* h_LJ_A, const float* h_LJ_B);

/* Adjoint context for one set of modules (scratch sized from them; re-create it after any of
 * the modules is re-created). */
SB_API int sb_adjoint_create(sb_neighbor_list* nl, sb_lennard_jones* lj, sb_pme* pme,
                             sb_adjoint** out);
SB_API int sb_adjoint_destroy(sb_adjoint* adj);

/* Jacobian-vector product of the nonbonded energy E and forces F (the sum of what the LJ,
 * long-range-correction, exclusion and reciprocal calls produce) at d_uint_crd with the current
 * list of nl: for L with dL/dE = grad_energy and dL/dF = d_grad_frc [3N] float, writes
 *   d_grad_crd    [3N] double  dL/dx in (unit of L)/A
 *   d_grad_charge [N]  double  dL/dq per atom (charges in the module's scaled units)
 *   d_grad_lj     [2 * ntypes^2] double  dL/dA12 then dL/dB6, square [type_i][type_j] tables
 *                 of the scaled values A*12, B*6; an entry (a, b) collects the half-list pairs
 *                 whose first atom has type a, so a symmetric table's gradient is g[a][b] +
 *                 g[b][a] (a != b)
 * Outputs are overwritten. The list must be current for d_uint_crd (as for the force calls). */
SB_API int sb_adjoint_backward(sb_adjoint* adj, sb_neighbor_list* nl, sb_lennard_jones* lj,
                               sb_pme* pme, const uint32_t* d_uint_crd, const float* d_charge,
                               const int* d_excluded_list_start, const int* d_excluded_list,
                               const int* d_excluded_numbers, double grad_energy,
                               const float* d_grad_frc, double* d_grad_crd,
                               double* d_grad_charge, double* d_grad_lj, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPONGE_B200_H */
