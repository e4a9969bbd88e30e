// Drop-in replacement for SPONGE's Particle_Mesh_Ewald (SPONGE/PME_force/PME_force.cuh:25-123):
// same struct, the public members the MD driver reads (beta, fft sizes, d_direct_atom_energy,
// d_correction_atom_energy, energy parts) and method signatures; spread, FFT, convolution and
// gather are libsponge_b200's, reached through the C ABI. The cuFFT plans and per-atom stencil
// arrays of the reference are internal to the library and not exposed; the TI cross terms
// that TI_CORE derives from them are computed by sb_pme_ti_cross.
#ifndef PME_FORCE_CUH
#define PME_FORCE_CUH
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
};

#endif
