// Drop-in replacement for SPONGE's LENNARD_JONES_INFORMATION
// (SPONGE/Lennard_Jones_force/Lennard_Jones_force.cuh:41-149): same struct, public members
// (h_LJ_A / h_LJ_B x12/x6, h_atom_LJ_type read by nb14) and method signatures; the pair work is
// libsponge_b200's fixed-point cluster kernel, reached through the C ABI.
#ifndef LENNARD_JONES_FORCE_CUH
#define LENNARD_JONES_FORCE_CUH
#include "../common.cuh"
#include "../control.cuh"

#ifndef UINT_VECTOR_LJ_TYPE_DEFINE
#define UINT_VECTOR_LJ_TYPE_DEFINE
struct UINT_VECTOR_LJ_TYPE
{
    unsigned int uint_x;
    unsigned int uint_y;
    unsigned int uint_z;
    int LJ_type;
    float charge;
};
__device__ __host__ VECTOR Get_Periodic_Displacement(const UINT_VECTOR_LJ_TYPE uvec_a, const UINT_VECTOR_LJ_TYPE uvec_b, const VECTOR scaler);
__global__ void Copy_LJ_Type_To_New_Crd(const int atom_numbers, UINT_VECTOR_LJ_TYPE *new_crd, const int *LJ_type);
__global__ void Copy_Crd_And_Charge_To_New_Crd(const int atom_numbers, const UNSIGNED_INT_VECTOR *crd, UINT_VECTOR_LJ_TYPE *new_crd, const float *charge);
__global__ void Copy_Crd_To_New_Crd(const int atom_numbers, const UNSIGNED_INT_VECTOR *crd, UINT_VECTOR_LJ_TYPE *new_crd);
#endif

struct sb_lennard_jones;

struct LENNARD_JONES_INFORMATION
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int is_controller_printf_initialized = 0;
    int last_modify_date = 20261203;

    int atom_numbers = 0;
    int atom_type_numbers = 0;
    int pair_type_numbers = 0;

    int *h_atom_LJ_type = NULL;
    int *d_atom_LJ_type = NULL;
    float *h_LJ_A = NULL;   // lower-triangular, x12
    float *h_LJ_B = NULL;   // lower-triangular, x6
    float *d_LJ_A = NULL;
    float *d_LJ_B = NULL;

    float *h_LJ_energy_atom = NULL;
    float h_LJ_energy_sum = 0;
    float *d_LJ_energy_atom = NULL;
    float *d_LJ_energy_sum = NULL;

    dim3 thread_LJ = {32, 32};

    float cutoff = 10.0;
    VECTOR uint_dr_to_dr_cof;
    float volume = 0;
    UINT_VECTOR_LJ_TYPE *uint_crd_with_LJ = NULL;
    float long_range_factor = 0;

    sb_lennard_jones *handle = NULL;

    void Initial(CONTROLLER *controller, float cutoff, VECTOR box_length, const char *module_name = NULL);
    void Initial_From_AMBER_Parm(const char *file_name, CONTROLLER controller);
    void Clear();
    void LJ_Malloc();
    void Parameter_Host_To_Device();

    void LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(const int atom_numbers, const UNSIGNED_INT_VECTOR *uint_crd, const float *charge, VECTOR *frc,
        const ATOM_GROUP *nl, const float pme_beta, const int need_atom_energy, float *atom_energy,
        const int need_virial, float *atom_lj_virial, float *atom_direct_pme_energy);
    void Long_Range_Correction(int need_pressure, float *d_virial, int need_potential, float *d_potential);
    float Get_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const ATOM_GROUP *nl, int is_download = 1);
    void Update_Volume(VECTOR box_length);
    void LJ_Force_With_PME_Direct_Force(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge, VECTOR *frc, const ATOM_GROUP *nl, const float pme_beta);
    void LJ_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const ATOM_GROUP *nl);
    void Long_Range_Correction(float volume);
    void Energy_Device_To_Host();
};
#endif //LENNARD_JONES_FORCE_CUH
