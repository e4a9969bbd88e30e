// Reference harness (test infrastructure): drives the reference's own, unchanged
// NEIGHBOR_LIST, LENNARD_JONES_INFORMATION and Particle_Mesh_Ewald modules (compiled from the
// reference tree by oracle/ref_harness/Makefile) on a system written by run.py, the way
// Main_Calculate_Force and Main_Iteration call them (SPONGE/main.cu:162-210, :376), and dumps
// their outputs. It is the source of the golden vectors and of the reference timing on the GPU.
//
// usage: harness <in.bin> <outdir> [timing_steps]
// in.bin: int32 N, ntypes, nexcl, fftx, ffty, fftz, refresh_interval, max_neighbor_numbers,
//         max_atom_in_grid_numbers; float box[3], cutoff, skin, tolerance;
//         float crd[3N], charge[N]; int32 type[N]; float A[T(T+1)/2], B[...] (unscaled);
//         int32 excl_start[N], excl_numbers[N], excl_list[nexcl]
//         optional, after that: int32 n14, a[n14], b[n14], float lj_scale[n14], cf[n14];
//         int32 nv, type[nv], atoms[4 nv], float param[2 nv] (the 1-4 pairs and virtual atoms,
//         run through NON_BOND_14 and VIRTUAL_INFORMATION when present); int32 nbond,
//         a[nbond], b[nbond], float r0[nbond], mass[N], vel[3N], dt (internal unit), with
//         which CONSTRAIN (bonds to atoms lighter than 3.3) and SETTLE run one NVE step on the
//         nonbonded forces (after the virtual-atom redistribution when there are virtual atoms)
// outputs (outdir): frc.f32 [3N] force of one evaluation with energy and virial requested,
//         frc_plain.f32 [3N] force-only evaluation, pairs.i64 (sorted keys i*N+j),
//         summary.txt (key value lines); with 1-4 pairs: nb14_frc.f32 [3N], nb14_ae.f32 [N],
//         nb14_av.f32 [N] (Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial from zero);
//         with virtual atoms: vs_frc.f32 [3N] (frc.f32 after Force_Redistribute),
//         vs_crd.f32 [3N] (the wrapped coordinates after Coordinate_Refresh); with bonds:
//         settle_crd.f32 / settle_vel.f32 [3N] after Remember_Last_Coordinates, the leap-frog
//         of MD_core.cu:13-32 and Do_SETTLE, and settle_pressure in summary.txt

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "control.cuh"
#include "Lennard_Jones_force/Lennard_Jones_force.cuh"
#include "constrain/SETTLE.cuh"
#include "constrain/constrain.cuh"
#include "PME_force/PME_force.cuh"
#include "nb14/nb14.cuh"
#include "neighbor_list/neighbor_list.cuh"
#include "virtual_atoms/virtual_atoms.cuh"

#define CK(x)                                                                      \
    do {                                                                           \
        cudaError_t e = (x);                                                       \
        if (e != cudaSuccess) {                                                    \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e),     \
                    __FILE__, __LINE__);                                           \
            exit(3);                                                               \
        }                                                                          \
    } while (0)

template <class T>
static void rd(FILE* f, T* p, size_t n) {
    if (n && fread(p, sizeof(T), n, f) != n) {
        fprintf(stderr, "short input\n");
        exit(2);
    }
}

template <class T>
static T* dev_copy(const std::vector<T>& h) {
    T* d = nullptr;
    CK(cudaMalloc((void**)&d, sizeof(T) * std::max<size_t>(1, h.size())));
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return d;
}

static void wr(const char* dir, const char* name, const void* p, size_t bytes) {
    char path[1024];
    snprintf(path, sizeof(path), "%s/%s", dir, name);
    FILE* f = fopen(path, "wb");
    if (!f) {
        fprintf(stderr, "cannot write %s\n", path);
        exit(2);
    }
    fwrite(p, 1, bytes, f);
    fclose(f);
}

// MD_Iteration_Leap_Frog (SPONGE/MD_core/MD_core.cu:13-32) is file-static in the reference, so
// the harness states it again, operation for operation
__global__ void harness_leap_frog(const int atom_numbers, VECTOR* vel, VECTOR* crd, VECTOR* frc,
                                  VECTOR* acc, const float* inverse_mass, const float dt) {
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers) {
        acc[i].x = inverse_mass[i] * frc[i].x;
        acc[i].y = inverse_mass[i] * frc[i].y;
        acc[i].z = inverse_mass[i] * frc[i].z;
        vel[i].x = vel[i].x + dt * acc[i].x;
        vel[i].y = vel[i].y + dt * acc[i].y;
        vel[i].z = vel[i].z + dt * acc[i].z;
        crd[i].x = crd[i].x + dt * vel[i].x;
        crd[i].y = crd[i].y + dt * vel[i].y;
        crd[i].z = crd[i].z + dt * vel[i].z;
    }
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: harness in.bin outdir [timing_steps]\n");
        return 1;
    }
    const int timing_steps = argc > 3 ? atoi(argv[3]) : 0;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[9];
    float fh[6];
    rd(f, hdr, 9);
    rd(f, fh, 6);
    const int N = hdr[0], T = hdr[1], NE = hdr[2];
    const int np = T * (T + 1) / 2;
    std::vector<float> crd(3 * (size_t)N), q(N), A(np), B(np);
    std::vector<int> type(N), es(N), en(N), el(std::max(NE, 1));
    rd(f, crd.data(), crd.size());
    rd(f, q.data(), q.size());
    rd(f, type.data(), type.size());
    rd(f, A.data(), A.size());
    rd(f, B.data(), B.size());
    rd(f, es.data(), es.size());
    rd(f, en.data(), en.size());
    rd(f, el.data(), NE);
    // optional 1-4 pairs and virtual atoms
    int n14 = 0, nv = 0;
    std::vector<int> a14, b14, vtype, vatoms;
    std::vector<float> ljs14, cf14, vparam;
    if (fread(&n14, sizeof(int), 1, f) == 1 && n14 > 0) {
        a14.resize(n14);
        b14.resize(n14);
        ljs14.resize(n14);
        cf14.resize(n14);
        rd(f, a14.data(), n14);
        rd(f, b14.data(), n14);
        rd(f, ljs14.data(), n14);
        rd(f, cf14.data(), n14);
    }
    if (fread(&nv, sizeof(int), 1, f) == 1 && nv > 0) {
        vtype.resize(nv);
        vatoms.resize(4 * (size_t)nv);
        vparam.resize(2 * (size_t)nv);
        rd(f, vtype.data(), nv);
        rd(f, vatoms.data(), vatoms.size());
        rd(f, vparam.data(), vparam.size());
    }
    int nbond = 0;
    std::vector<int> bond_a, bond_b;
    std::vector<float> bond_r, mass, vel;
    float md_dt = 0.f;
    if (fread(&nbond, sizeof(int), 1, f) == 1 && nbond > 0) {
        bond_a.resize(nbond);
        bond_b.resize(nbond);
        bond_r.resize(nbond);
        mass.resize(N);
        vel.resize(3 * (size_t)N);
        rd(f, bond_a.data(), nbond);
        rd(f, bond_b.data(), nbond);
        rd(f, bond_r.data(), nbond);
        rd(f, mass.data(), N);
        rd(f, vel.data(), vel.size());
        rd(f, &md_dt, 1);
    }
    fclose(f);
    el.resize(NE);

    // LJ_in_file in the reference's text format (Lennard_Jones_force.cu:1082-1105)
    char ljpath[1024];
    snprintf(ljpath, sizeof(ljpath), "%s/lj_in.txt", argv[2]);
    FILE* lf = fopen(ljpath, "w");
    fprintf(lf, "%d %d\n", N, T);
    for (int i = 0; i < np; i++) fprintf(lf, "%.9e\n", A[i]);
    for (int i = 0; i < np; i++) fprintf(lf, "%.9e\n", B[i]);
    for (int i = 0; i < N; i++) fprintf(lf, "%d\n", type[i]);
    fclose(lf);

    CONTROLLER controller;
    char buf[64];
    controller.Set_Command("LJ_in_file", ljpath);
    snprintf(buf, sizeof(buf), "%d", hdr[3]);
    controller.Set_Command("PME_fftx", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[4]);
    controller.Set_Command("PME_ffty", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[5]);
    controller.Set_Command("PME_fftz", buf);
    snprintf(buf, sizeof(buf), "%g", fh[5]);
    controller.Set_Command("PME_Direct_Tolerance", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[6]);
    controller.Set_Command("neighbor_list_refresh_interval", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[7]);
    controller.Set_Command("neighbor_list_max_neighbor_numbers", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[8]);
    controller.Set_Command("neighbor_list_max_atom_in_grid_numbers", buf);
    // nb14_in_file (nb14.cu:179-187, :203-206) and virtual_atom_in_file (virtual_atoms.cu:
    // 192-200) in the reference's text formats
    char nb14path[1024], vspath[1024];
    if (n14 > 0) {
        snprintf(nb14path, sizeof(nb14path), "%s/nb14_in.txt", argv[2]);
        FILE* nf = fopen(nb14path, "w");
        fprintf(nf, "%d\n", n14);
        for (int i = 0; i < n14; i++)
            fprintf(nf, "%d %d %.9g %.9g\n", a14[i], b14[i], ljs14[i], cf14[i]);
        fclose(nf);
        controller.Set_Command("nb14_in_file", nb14path);
    }
    if (nv > 0) {
        snprintf(vspath, sizeof(vspath), "%s/vatom_in.txt", argv[2]);
        FILE* vf = fopen(vspath, "w");
        const int npar[4] = {1, 2, 3, 3};
        for (int i = 0; i < nv; i++) {
            fprintf(vf, "%d", vtype[i]);
            for (int k = 0; k <= npar[vtype[i]]; k++) fprintf(vf, " %d", vatoms[4 * i + k]);
            fprintf(vf, " %.9g", vparam[2 * i]);
            if (vtype[i] >= 2) fprintf(vf, " %.9g", vparam[2 * i + 1]);
            fprintf(vf, "\n");
        }
        fclose(vf);
        controller.Set_Command("virtual_atom_in_file", vspath);
    }

    VECTOR box = {fh[0], fh[1], fh[2]};
    const float cutoff = fh[3], skin = fh[4];

    VECTOR* d_crd = (VECTOR*)dev_copy(crd);
    float* d_q = dev_copy(q);
    int* d_es = dev_copy(es);
    int* d_en = dev_copy(en);
    int* d_el = dev_copy(el);
    UNSIGNED_INT_VECTOR* d_uc = nullptr;
    float *d_frc, *d_ae, *d_av, *d_vir, *d_pot;
    CK(cudaMalloc((void**)&d_uc, sizeof(UNSIGNED_INT_VECTOR) * N));
    CK(cudaMalloc((void**)&d_frc, sizeof(VECTOR) * N));
    CK(cudaMalloc((void**)&d_ae, sizeof(float) * N));
    CK(cudaMalloc((void**)&d_av, sizeof(float) * N));
    CK(cudaMalloc((void**)&d_vir, sizeof(float)));
    CK(cudaMalloc((void**)&d_pot, sizeof(float)));

    NEIGHBOR_LIST nl;
    nl.Initial(&controller, N, box, cutoff, skin);
    nl.Neighbor_List_Update((VECTOR*)d_crd, d_es, d_el, d_en, NEIGHBOR_LIST::FORCED_UPDATE);
    LENNARD_JONES_INFORMATION lj;
    lj.Initial(&controller, cutoff, box);
    Particle_Mesh_Ewald pme;
    pme.Initial(&controller, N, box, cutoff);
    CK(cudaDeviceSynchronize());

    // MD_INFORMATION's fixed point (MD_core.cu:485-490, :1528-1531) and displacement scaler
    VECTOR cof = CONSTANT_UINT_MAX_FLOAT / box;
    VECTOR quarter = 0.25f * cof;
    VECTOR scaler = 1.0f / cof;
    Crd_To_Uint_Crd<<<(N + 127) / 128, 128>>>(N, quarter, d_crd, d_uc);

    auto evaluate = [&](int need_energy, int need_virial) {
        cudaMemset(d_frc, 0, sizeof(VECTOR) * N);
        cudaMemset(d_ae, 0, sizeof(float) * N);
        cudaMemset(d_av, 0, sizeof(float) * N);
        cudaMemset(d_vir, 0, sizeof(float));
        cudaMemset(d_pot, 0, sizeof(float));
        lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(N, d_uc, d_q, (VECTOR*)d_frc, nl.d_nl,
                                                           pme.beta, need_energy, d_ae,
                                                           need_virial, d_av,
                                                           pme.d_direct_atom_energy);
        lj.Long_Range_Correction(need_virial, d_vir, need_energy, d_pot);
        pme.PME_Excluded_Force_With_Atom_Energy(d_uc, scaler, d_q, d_es, d_el, d_en,
                                                (VECTOR*)d_frc, pme.d_correction_atom_energy);
        pme.PME_Reciprocal_Force_With_Energy_And_Virial(d_uc, d_q, (VECTOR*)d_frc, need_virial,
                                                        need_energy, d_vir, d_pot);
    };

    std::vector<float> h(3 * (size_t)N), hae(N), hav(N);
    float vir = 0, pot = 0;
    evaluate(0, 0);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(h.data(), d_frc, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
    wr(argv[2], "frc_plain.f32", h.data(), sizeof(float) * h.size());
    evaluate(1, 1);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(h.data(), d_frc, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hae.data(), d_ae, sizeof(float) * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hav.data(), d_av, sizeof(float) * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&vir, d_vir, sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&pot, d_pot, sizeof(float), cudaMemcpyDeviceToHost));
    wr(argv[2], "frc.f32", h.data(), sizeof(float) * h.size());
    double sae = 0, sav = 0;
    for (int i = 0; i < N; i++) {
        sae += hae[i];
        sav += hav[i];
    }
    // energies by part through the modules' own Get_Energy
    float e_rec = pme.Get_Energy(d_uc, d_q, nl.d_nl, scaler, d_es, d_el, d_en,
                                 Particle_Mesh_Ewald::RECIPROCAL);
    float e_self = pme.Get_Energy(d_uc, d_q, nl.d_nl, scaler, d_es, d_el, d_en,
                                  Particle_Mesh_Ewald::SELF);
    float e_dir = pme.Get_Energy(d_uc, d_q, nl.d_nl, scaler, d_es, d_el, d_en,
                                 Particle_Mesh_Ewald::DIRECT);
    float e_corr = pme.Get_Energy(d_uc, d_q, nl.d_nl, scaler, d_es, d_el, d_en,
                                  Particle_Mesh_Ewald::CORRECTION);
    float e_lj = lj.Get_Energy(d_uc, nl.d_nl);

    // the pair list (ATOM_GROUP d_nl, neighbor_list.cuh:75)
    std::vector<ATOM_GROUP> g(N);
    CK(cudaMemcpy(g.data(), nl.d_nl, sizeof(ATOM_GROUP) * N, cudaMemcpyDeviceToHost));
    std::vector<long long> keys;
    std::vector<int> tmp;
    long long overflow = 0;
    for (int i = 0; i < N; i++) {
        int c = g[i].atom_numbers;
        if (c > nl.max_neighbor_numbers) {
            overflow++;
            c = nl.max_neighbor_numbers;
        }
        tmp.resize(std::max(c, 1));
        if (c) CK(cudaMemcpy(tmp.data(), g[i].atom_serial, sizeof(int) * c, cudaMemcpyDeviceToHost));
        for (int k = 0; k < c; k++) keys.push_back((long long)i * N + tmp[k]);
    }
    std::sort(keys.begin(), keys.end());
    wr(argv[2], "pairs.i64", keys.data(), sizeof(long long) * keys.size());

    // 1-4 pairs and virtual atoms (SPONGE/main.cu:81, :127, :195, :207, :375)
    float e14_lj = 0.f, e14_cf = 0.f;
    if (n14 > 0) {
        NON_BOND_14 nb14;
        nb14.Initial(&controller, lj.h_LJ_A, lj.h_LJ_B, lj.h_atom_LJ_type);
        cudaMemset(d_frc, 0, sizeof(VECTOR) * N);
        cudaMemset(d_ae, 0, sizeof(float) * N);
        cudaMemset(d_av, 0, sizeof(float) * N);
        nb14.Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial(d_uc, d_q, scaler, (VECTOR*)d_frc,
                                                                 d_ae, d_av);
        CK(cudaDeviceSynchronize());
        std::vector<float> f14(3 * (size_t)N), e14(N), v14(N);
        CK(cudaMemcpy(f14.data(), d_frc, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(e14.data(), d_ae, sizeof(float) * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(v14.data(), d_av, sizeof(float) * N, cudaMemcpyDeviceToHost));
        wr(argv[2], "nb14_frc.f32", f14.data(), sizeof(float) * f14.size());
        wr(argv[2], "nb14_ae.f32", e14.data(), sizeof(float) * e14.size());
        wr(argv[2], "nb14_av.f32", v14.data(), sizeof(float) * v14.size());
        e14_lj = nb14.Get_14_LJ_Energy(d_uc, scaler);
        e14_cf = nb14.Get_14_CF_Energy(d_uc, d_q, scaler);
    }
    if (nv > 0) {
        VIRTUAL_INFORMATION vatom;
        int freedom = 3 * N;
        vatom.Initial(&controller, N, &freedom);
        // the LJ + PME forces of the energy/virial evaluation, redistributed
        CK(cudaMemcpy(d_frc, h.data(), sizeof(float) * 3 * N, cudaMemcpyHostToDevice));
        vatom.Force_Redistribute(d_uc, scaler, (VECTOR*)d_frc);
        CK(cudaDeviceSynchronize());
        std::vector<float> fv(3 * (size_t)N), cv(3 * (size_t)N);
        CK(cudaMemcpy(fv.data(), d_frc, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
        wr(argv[2], "vs_frc.f32", fv.data(), sizeof(float) * fv.size());
        vatom.Coordinate_Refresh(d_uc, scaler, (VECTOR*)d_crd);
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(cv.data(), d_crd, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
        wr(argv[2], "vs_crd.f32", cv.data(), sizeof(float) * cv.size());
        h = fv;  // the integrator below takes the redistributed forces
    }
    float settle_pressure = 0.f;
    if (nbond > 0) {
        // CONSTRAIN + SETTLE as main.cu:92-103 set them up for an NVE run (exp_gamma 1)
        CONSTRAIN constrain;
        constrain.Add_HBond_To_Constrain_Pair(&controller, nbond, bond_a.data(), bond_b.data(),
                                              bond_r.data(), mass.data());
        // no angle constraints: main.cu:95 adds them only under the constrain_angle command
        int freedom = 3 * N;
        constrain.Initial_Constrain(&controller, N, md_dt, box, 1.0f, 0, mass.data(), &freedom);
        SETTLE settle;
        settle.Initial(&controller, &constrain, mass.data());
        // the coordinates of this evaluation (wrapped), their fixed point, the forces h
        CK(cudaMemcpy(d_crd, crd.data(), sizeof(float) * 3 * N, cudaMemcpyHostToDevice));
        Crd_Periodic_Map<<<(N + 127) / 128, 128>>>(N, d_crd, box);
        Crd_To_Uint_Crd<<<(N + 127) / 128, 128>>>(N, quarter, d_crd, d_uc);
        std::vector<float> inv(N);
        for (int i = 0; i < N; i++) inv[i] = mass[i] == 0 ? 0.0f : (float)(1.0 / mass[i]);  // MD_core.cu:952-955
        float* d_mass = dev_copy(mass);
        float* d_inv = dev_copy(inv);
        float* d_vel = dev_copy(vel);
        float* d_f = dev_copy(h);
        float* d_acc = nullptr;
        CK(cudaMalloc((void**)&d_acc, sizeof(float) * 3 * N));
        cudaMemset(d_pot, 0, sizeof(float));
        settle.Remember_Last_Coordinates(d_uc, scaler);
        harness_leap_frog<<<(N + 127) / 128, 128>>>(N, (VECTOR*)d_vel, (VECTOR*)d_crd,
                                                     (VECTOR*)d_f, (VECTOR*)d_acc, d_inv, md_dt);
        settle.Do_SETTLE(d_mass, (VECTOR*)d_crd, box, (VECTOR*)d_vel, 1, d_pot);
        CK(cudaDeviceSynchronize());
        std::vector<float> sc(3 * (size_t)N), sv(3 * (size_t)N);
        CK(cudaMemcpy(sc.data(), d_crd, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(sv.data(), d_vel, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&settle_pressure, d_pot, sizeof(float), cudaMemcpyDeviceToHost));
        wr(argv[2], "settle_crd.f32", sc.data(), sizeof(float) * sc.size());
        wr(argv[2], "settle_vel.f32", sv.data(), sizeof(float) * sv.size());
        printf("settle: %d triangles, %d pairs\n", settle.triangle_numbers, settle.pair_numbers);
    }

    double ms_step = -1, ms_force = -1;
    if (timing_steps > 0) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        for (int k = 0; k < 5; k++) evaluate(0, 0);
        // force-only evaluation
        cudaEventRecord(a);
        for (int k = 0; k < timing_steps; k++) evaluate(0, 0);
        cudaEventRecord(b);
        CK(cudaEventSynchronize(b));
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        ms_force = ms / timing_steps;
        // a step: list update by its policy (every refresh_interval) + forces
        cudaEventRecord(a);
        for (int k = 0; k < timing_steps; k++) {
            nl.Neighbor_List_Update((VECTOR*)d_crd, d_es, d_el, d_en);
            evaluate(0, 0);
        }
        cudaEventRecord(b);
        CK(cudaEventSynchronize(b));
        cudaEventElapsedTime(&ms, a, b);
        ms_step = ms / timing_steps;
    }
    CK(cudaDeviceSynchronize());

    char path[1024];
    snprintf(path, sizeof(path), "%s/summary.txt", argv[2]);
    FILE* s = fopen(path, "w");
    fprintf(s, "atoms %d\nbeta %.9g\nfftx %d\nffty %d\nfftz %d\n", N, pme.beta, pme.fftx, pme.ffty,
            pme.fftz);
    fprintf(s, "atom_energy_sum %.9g\natom_virial_sum %.9g\nd_virial %.9g\nd_potential %.9g\n",
            sae, sav, vir, pot);
    fprintf(s, "e_rec %.9g\ne_self %.9g\ne_direct %.9g\ne_corr %.9g\ne_lj_with_lrc %.9g\n", e_rec,
            e_self, e_dir, e_corr, e_lj);
    fprintf(s, "long_range_factor %.9g\npairs %zu\nnl_overflow_atoms %lld\n",
            lj.long_range_factor, keys.size(), overflow);
    fprintf(s, "ms_force_only %.6f\nms_step %.6f\ntiming_steps %d\n", ms_force, ms_step,
            timing_steps);
    fprintf(s, "nb14_pairs %d\nnb14_lj %.9g\nnb14_cf %.9g\nvirtual_atoms %d\n", n14, e14_lj,
            e14_cf, nv);
    fprintf(s, "bonds %d\nsettle_pressure %.9g\n", nbond, settle_pressure);
    fclose(s);
    printf("harness done: %d atoms, %zu pairs\n", N, keys.size());
    return 0;
}
