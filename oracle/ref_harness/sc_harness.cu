// Soft-core reference harness (test infrastructure): drives the reference's own, unchanged
// LJ_SOFT_CORE (SPONGE/Lennard_Jones_force/LJ_soft_core.cu) over the reference's NEIGHBOR_LIST,
// and the PME cross terms of TI_CORE (SPONGE/TI_core/TI_core.cu:670-730) over the reference's
// Particle_Mesh_Ewald, on one FEP box written by run.py, and dumps their outputs. Compiled from
// the reference tree by oracle/ref_harness/Makefile into oracle/_ref/; the golden fixtures of the
// soft-core path come from it.
//
// usage: sc_harness <in.bin> <outdir>
// in.bin: int32 N, TA, TB, nexcl, fftx, ffty, fftz, max_neighbor_numbers,
//         max_atom_in_grid_numbers; float box[3], cutoff, skin, tolerance, lambda, alpha, p,
//         sigma, sigma_min; float crd[3N], charge[N] (at lambda), charge_B_A[N];
//         int32 typeA[N], typeB[N], subsys[N]; float AA[TA(TA+1)/2], AB[...] (state A, unscaled
//         A and B), BA[TB(TB+1)/2], BB[...] (state B); int32 excl_start[N], excl_numbers[N],
//         excl_list[nexcl]
// outputs (outdir): sc_frc.f32 [3N] LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial
//         from zero with energy and virial requested; sc_ae.f32, sc_av.f32, sc_adir.f32 [N] its
//         atom energy, LJ virial and direct Coulomb energy; pairs.i64 (the list's sorted keys);
//         summary.txt: the dH/dlambda parts (Get_Partial_H_Partial_Lambda_With_Columb_Direct,
//         Partial_H_Partial_Lambda_Long_Range_Correction), the long-range correction, the
//         energies of Get_Energy_With_Coulomb_Direct, and TI_CORE's PME cross terms.
//
// TI_CORE::Initial reads a whole TI run's files; the harness instead sets the members that
// Get_Cross_PME_Partial_H_Partial_Lambda reads. Its cross_pme.charge_sum_B_A is allocated by
// cross_pme.Initial and read at TI_core.cu:704 but written nowhere in the reference; the
// harness clears it after the allocation, which is what freshly allocated device memory reads
// as, so the neutralising cross term the reference adds is f * sum(q) * 0.

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "control.cuh"
#include "Lennard_Jones_force/LJ_soft_core.cuh"
#include "PME_force/PME_force.cuh"
#include "TI_core/TI_core.cuh"
#include "neighbor_list/neighbor_list.cuh"

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

template <class T>
static std::vector<T> dev_get(const T* d, size_t n) {
    std::vector<T> h(n);
    CK(cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
    return h;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: sc_harness in.bin outdir\n");
        return 1;
    }
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[9];
    float fh[11];
    rd(f, hdr, 9);
    rd(f, fh, 11);
    const int N = hdr[0], TA = hdr[1], TB = hdr[2], NE = hdr[3];
    const int npa = TA * (TA + 1) / 2, npb = TB * (TB + 1) / 2;
    std::vector<float> crd(3 * (size_t)N), q(N), dq(N), AA(npa), AB(npa), BA(npb), BB(npb);
    std::vector<int> ta(N), tb(N), sub(N), es(N), en(N), el(std::max(NE, 1));
    rd(f, crd.data(), crd.size());
    rd(f, q.data(), N);
    rd(f, dq.data(), N);
    rd(f, ta.data(), N);
    rd(f, tb.data(), N);
    rd(f, sub.data(), N);
    rd(f, AA.data(), npa);
    rd(f, AB.data(), npa);
    rd(f, BA.data(), npb);
    rd(f, BB.data(), npb);
    rd(f, es.data(), N);
    rd(f, en.data(), N);
    rd(f, el.data(), NE);
    fclose(f);
    el.resize(NE);

    // LJ_soft_core_in_file and subsys_division_in_file in the reference's text formats
    // (LJ_soft_core.cu:1491-1547)
    char scpath[1024], subpath[1024];
    snprintf(scpath, sizeof(scpath), "%s/lj_soft_core_in.txt", argv[2]);
    FILE* sf = fopen(scpath, "w");
    fprintf(sf, "%d %d %d\n", N, TA, TB);
    for (int i = 0; i < npa; i++) fprintf(sf, "%.9e\n", AA[i]);
    for (int i = 0; i < npa; i++) fprintf(sf, "%.9e\n", AB[i]);
    for (int i = 0; i < npb; i++) fprintf(sf, "%.9e\n", BA[i]);
    for (int i = 0; i < npb; i++) fprintf(sf, "%.9e\n", BB[i]);
    for (int i = 0; i < N; i++) fprintf(sf, "%d %d\n", ta[i], tb[i]);
    fclose(sf);
    snprintf(subpath, sizeof(subpath), "%s/subsys_in.txt", argv[2]);
    sf = fopen(subpath, "w");
    fprintf(sf, "%d\n", N);
    for (int i = 0; i < N; i++) fprintf(sf, "%d\n", sub[i]);
    fclose(sf);

    CONTROLLER controller;
    char buf[64];
    controller.Set_Command("LJ_soft_core_in_file", scpath);
    controller.Set_Command("subsys_division_in_file", subpath);
    snprintf(buf, sizeof(buf), "%.9g", fh[6]);
    controller.Set_Command("lambda_lj", buf);
    snprintf(buf, sizeof(buf), "%.9g", fh[7]);
    controller.Set_Command("soft_core_alpha", buf);
    snprintf(buf, sizeof(buf), "%.9g", fh[8]);
    controller.Set_Command("soft_core_powfer", buf);
    snprintf(buf, sizeof(buf), "%.9g", fh[9]);
    controller.Set_Command("soft_core_sigma", buf);
    snprintf(buf, sizeof(buf), "%.9g", fh[10]);
    controller.Set_Command("soft_core_sigma_min", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[4]);
    controller.Set_Command("PME_fftx", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[5]);
    controller.Set_Command("PME_ffty", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[6]);
    controller.Set_Command("PME_fftz", buf);
    snprintf(buf, sizeof(buf), "%g", fh[5]);
    controller.Set_Command("PME_Direct_Tolerance", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[7]);
    controller.Set_Command("neighbor_list_max_neighbor_numbers", buf);
    snprintf(buf, sizeof(buf), "%d", hdr[8]);
    controller.Set_Command("neighbor_list_max_atom_in_grid_numbers", buf);

    VECTOR box = {fh[0], fh[1], fh[2]};
    const float cutoff = fh[3], skin = fh[4];
    VECTOR* d_crd = (VECTOR*)dev_copy(crd);
    float* d_q = dev_copy(q);
    float* d_dq = dev_copy(dq);
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
    nl.Neighbor_List_Update(d_crd, d_es, d_el, d_en, NEIGHBOR_LIST::FORCED_UPDATE);
    LJ_SOFT_CORE sc;
    sc.Initial(&controller, cutoff, box);
    Particle_Mesh_Ewald pme;
    pme.Initial(&controller, N, box, cutoff);
    CK(cudaDeviceSynchronize());
    if (!sc.is_initialized) {
        fprintf(stderr, "LJ_SOFT_CORE not initialised\n");
        return 4;
    }

    // MD_INFORMATION's fixed point (MD_core.cu:485-490, :1528-1531)
    VECTOR cof = CONSTANT_UINT_MAX_FLOAT / box;
    VECTOR quarter = 0.25f * cof;
    VECTOR scaler = 1.0f / cof;
    Crd_To_Uint_Crd<<<(N + 127) / 128, 128>>>(N, quarter, d_crd, d_uc);

    // the force step of the soft-core module (main_ti/main_fep drive energies; MD drives this)
    cudaMemset(d_frc, 0, sizeof(VECTOR) * N);
    cudaMemset(d_ae, 0, sizeof(float) * N);
    cudaMemset(d_av, 0, sizeof(float) * N);
    cudaMemset(pme.d_direct_atom_energy, 0, sizeof(float) * N);
    sc.LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
        N, d_uc, d_q, (VECTOR*)d_frc, nl.d_nl, pme.beta, 1, d_ae, 1, d_av,
        pme.d_direct_atom_energy);
    cudaMemset(d_vir, 0, sizeof(float));
    cudaMemset(d_pot, 0, sizeof(float));
    sc.Long_Range_Correction(1, d_vir, 1, d_pot);
    CK(cudaDeviceSynchronize());
    wr(argv[2], "sc_frc.f32", dev_get((float*)d_frc, 3 * (size_t)N).data(), sizeof(float) * 3 * N);
    wr(argv[2], "sc_ae.f32", dev_get(d_ae, N).data(), sizeof(float) * N);
    wr(argv[2], "sc_av.f32", dev_get(d_av, N).data(), sizeof(float) * N);
    wr(argv[2], "sc_adir.f32", dev_get(pme.d_direct_atom_energy, N).data(), sizeof(float) * N);
    const float lrc_pot = dev_get(d_pot, 1)[0], lrc_vir = dev_get(d_vir, 1)[0];

    // energies and dH/dlambda as main_fep.cu:97-104 and main_ti.cu:129-133 ask for them
    const float e_sc = sc.Get_Energy_With_Coulomb_Direct(d_uc, nl.d_nl, d_q);
    const float e_lrc = sc.Long_Range_Correction();
    const float dhdl_lj = sc.Get_Partial_H_Partial_Lambda_With_Columb_Direct(d_uc, d_q, nl.d_nl,
                                                                             d_dq, 1);
    const float dhdl_direct = *sc.h_sigma_of_dH_dlambda_direct;
    const float dhdl_lrc = sc.Partial_H_Partial_Lambda_Long_Range_Correction();

    // TI_CORE's PME cross terms (TI_core.cu:670-730) with lj_pertubated 0, so that the direct
    // cross term is evaluated as well
    TI_CORE ti;
    ti.atom_numbers = N;
    ti.box_length = box;
    ti.uint_crd = d_uc;
    ti.d_charge = d_q;
    ti.d_charge_B_A = d_dq;
    ti.charge_pertubated = 1;
    ti.pbc.uint_dr_to_dr_cof = scaler;
    ti.nb.cutoff = cutoff;
    ti.nb.skin = skin;
    ti.nb.d_excluded_list_start = d_es;
    ti.nb.d_excluded_list = d_el;
    ti.nb.d_excluded_numbers = d_en;
    ti.cross_pme.Initial(N, pme.PME_Nall);
    CK(cudaMemset(ti.cross_pme.charge_sum_B_A, 0, sizeof(float)));
    const float pme_cross = ti.Get_Cross_PME_Partial_H_Partial_Lambda(&pme, nl.d_nl, 0, 1);
    CK(cudaDeviceSynchronize());

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

    char path[1024];
    snprintf(path, sizeof(path), "%s/summary.txt", argv[2]);
    FILE* s = fopen(path, "w");
    fprintf(s, "atoms %d\nbeta %.9g\nsc_beta %.9g\nlambda %.9g\n", N, pme.beta, sc.pme_beta,
            sc.lambda);
    fprintf(s, "e_with_coulomb_direct %.9g\ne_lj %.9g\ne_lj_intersys %.9g\ne_lj_intrasys %.9g\n",
            e_sc, sc.h_LJ_energy_sum, sc.h_LJ_energy_sum_intersys, sc.h_LJ_energy_sum_intrasys);
    fprintf(s, "e_direct %.9g\ne_direct_intersys %.9g\ne_direct_intrasys %.9g\n",
            sc.h_direct_ene_sum, sc.h_direct_ene_sum_intersys, sc.h_direct_ene_sum_intrasys);
    fprintf(s, "lrc_energy %.9g\nlrc_potential %.9g\nlrc_virial %.9g\n", e_lrc, lrc_pot, lrc_vir);
    fprintf(s, "long_range_factor %.9g\nlong_range_factor_ti %.9g\n", sc.long_range_factor,
            sc.long_range_factor_TI);
    fprintf(s, "dhdl_lj %.9g\ndhdl_direct %.9g\ndhdl_lrc %.9g\n", dhdl_lj, dhdl_direct, dhdl_lrc);
    fprintf(s, "pme_cross %.9g\ncross_rec %.9g\ncross_self %.9g\ncross_corr %.9g\n"
               "cross_direct %.9g\n",
            pme_cross, ti.cross_pme.cross_reciprocal_ene, ti.cross_pme.cross_self_ene,
            ti.cross_pme.cross_correction_ene, ti.cross_pme.cross_direct_ene);
    fprintf(s, "pairs %zu\nnl_overflow_atoms %lld\n", keys.size(), overflow);
    fclose(s);
    printf("sc harness done: %d atoms, %zu pairs\n", N, keys.size());
    return 0;
}
