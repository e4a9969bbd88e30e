// Drop-in replacement for SPONGE's Particle_Mesh_Ewald (SPONGE/PME_force/PME_force.cuh:25-123):
// same struct, the public members the MD driver reads (beta, fft sizes, d_direct_atom_energy,
// d_correction_atom_energy, energy parts) and method signatures; spread, FFT, convolution and
// gather are libsponge_b200's, reached through the C ABI.
//
// TI_CORE::Get_Cross_PME_Partial_H_Partial_Lambda (TI_core.cu:670-730) works on the reference's
// own PME internals: it launches PME_Atom_Near, PME_Q_Spread, PME_BCFQ and PME_Energy_Product on
// the members PME_atom_near, PME_kxyz, PME_uxyz, PME_frxyz, PME_Q, PME_FQ, PME_FBCFQ, PME_BC and
// the cuFFT plans. The same members and kernels are declared here (with the reference header's
// names and signatures, which TI_core.cu compiles against); Initial allocates them only for runs
// whose mdin perturbs charges (charge_pertubated), PME_BC is the library's FP64-built Green's
// function table, and the kernels are this drop-in's own (PME_force.cu).
#ifndef PME_FORCE_CUH
#define PME_FORCE_CUH
#include <cufft.h>

#include "../common.cuh"
#include "../control.cuh"

struct sb_pme;

struct Particle_Mesh_Ewald
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int is_controller_printf_initialized = 0;
    int last_modify_date = 20261203;

    int fftx = -1;
    int ffty = -1;
    int fftz = -1;
    int PME_Nall = 0;
    int PME_Nin = 0;
    int PME_Nfft = 0;

    int atom_numbers = 0;
    VECTOR boxlength;
    VECTOR PME_inverse_box_vector;

    float beta;
    float cutoff = 10.0;
    float tolerance = 0.00001f;
    float neutralizing_factor = 0;

    float *d_direct_atom_energy = NULL;      // owned by the library
    float *d_correction_atom_energy = NULL;  // owned by the library
    // device copies of the energy parts of the last Get_Energy (single floats, as the reference)
    float *d_reciprocal_ene = NULL;
    float *d_self_ene = NULL;
    float *d_direct_ene = NULL;
    float *d_correction_ene = NULL;
    float *d_ee_ene = NULL;
    float reciprocal_ene = 0;
    float self_ene = 0;
    float direct_ene = 0;
    float correction_ene = 0;
    float ee_ene;

    sb_pme *handle = NULL;

    // the internals TI_CORE reads (allocated by Initial when the mdin perturbs charges)
    dim3 thread_PME = {8, 8};
    cufftHandle PME_plan_r2c = 0;
    cufftHandle PME_plan_c2r = 0;
    int ti_internals = 0;
    float *PME_BC = NULL;  // the library's table, [fftx][ffty][fftz/2+1]
    UNSIGNED_INT_VECTOR *PME_kxyz = NULL;
    UNSIGNED_INT_VECTOR *PME_uxyz = NULL;
    VECTOR *PME_frxyz = NULL;
    float *PME_Q = NULL;
    float *PME_FBCFQ = NULL;
    cufftComplex *PME_FQ = NULL;
    int **PME_atom_near = NULL;
    int *PME_atom_near_block = NULL;
    float *charge_sum = NULL;

    enum PME_ENERGY_PART
    {
        TOTAL = 0,
        DIRECT = 1,
        RECIPROCAL = 2,
        CORRECTION = 3,
        SELF = 4,
    };

    void Initial(CONTROLLER *controller, int atom_numbers, VECTOR boxlength, float cutoff, const char *module_name = NULL);
    void Clear();
    void PME_Excluded_Force_With_Atom_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const VECTOR sacler, const float *charge,
        const int *excluded_list_start, const int *excluded_list, const int *excluded_atom_numbers,
        VECTOR *frc, float *atom_energy);
    void PME_Reciprocal_Force_With_Energy_And_Virial(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge,
        VECTOR *force, int need_virial, int need_energy, float *d_virial, float *d_potential);
    float Get_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge,
        const ATOM_GROUP *nl, const VECTOR scaler,
        const int *excluded_list_start, const int *excluded_list, const int *excluded_atom_numbers, int which_part = 0, int is_download = 1);
    void Update_Volume(VECTOR boxlength);
    void Update_Box_Length(VECTOR boxlength);
    void Initial_TI_Internals();
    void Clear_TI_Internals();
};

// kernels of the reference header that TI_CORE launches on the members above
__global__ void PME_Atom_Near(const UNSIGNED_INT_VECTOR *uint_crd, int **PME_atom_near, const int PME_Nin,
    const float periodic_factor_inverse_x, const float periodic_factor_inverse_y, const float periodic_factor_inverse_z,
    const int atom_numbers, const int fftx, const int ffty, const int fftz,
    const UNSIGNED_INT_VECTOR *PME_kxyz, UNSIGNED_INT_VECTOR *PME_uxyz, VECTOR *PME_frxyz);
__global__ void PME_Q_Spread(int **PME_atom_near, const float *charge, const VECTOR *PME_frxyz,
    float *PME_Q, const UNSIGNED_INT_VECTOR *PME_kxyz, const int atom_numbers);
__global__ void PME_Energy_Product(const int element_number, const float *list1, const float *list2, float *sum);
__global__ void PME_BCFQ(cufftComplex *PME_FQ, float *PME_BC, int PME_Nfft);

#endif
