// Drop-in LENNARD_JONES_INFORMATION forwarding to libsponge_b200 (see Lennard_Jones_force.cuh).
#include "Lennard_Jones_force.cuh"

#include "../neighbor_list/neighbor_list.cuh"
#include "sponge_b200.h"

#include <vector>

// helpers other modules link against (nb14 declares them too)
__device__ __host__ VECTOR Get_Periodic_Displacement(const UINT_VECTOR_LJ_TYPE uvec_a, const UINT_VECTOR_LJ_TYPE uvec_b, const VECTOR scaler)
{
    VECTOR dr;
    dr.x = ((int)(uvec_a.uint_x - uvec_b.uint_x)) * scaler.x;
    dr.y = ((int)(uvec_a.uint_y - uvec_b.uint_y)) * scaler.y;
    dr.z = ((int)(uvec_a.uint_z - uvec_b.uint_z)) * scaler.z;
    return dr;
}

__global__ void Copy_LJ_Type_To_New_Crd(const int atom_numbers, UINT_VECTOR_LJ_TYPE *new_crd, const int *LJ_type)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
        new_crd[i].LJ_type = LJ_type[i];
}

__global__ void Copy_Crd_And_Charge_To_New_Crd(const int atom_numbers, const UNSIGNED_INT_VECTOR *crd, UINT_VECTOR_LJ_TYPE *new_crd, const float *charge)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].uint_x = crd[i].uint_x;
        new_crd[i].uint_y = crd[i].uint_y;
        new_crd[i].uint_z = crd[i].uint_z;
        new_crd[i].charge = charge[i];
    }
}

__global__ void Copy_Crd_To_New_Crd(const int atom_numbers, const UNSIGNED_INT_VECTOR *crd, UINT_VECTOR_LJ_TYPE *new_crd)
{
    int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < atom_numbers)
    {
        new_crd[i].uint_x = crd[i].uint_x;
        new_crd[i].uint_y = crd[i].uint_y;
        new_crd[i].uint_z = crd[i].uint_z;
    }
}

void LENNARD_JONES_INFORMATION::LJ_Malloc()
{
    Malloc_Safely((void **)&h_LJ_energy_atom, sizeof(float) * atom_numbers);
    Malloc_Safely((void **)&h_atom_LJ_type, sizeof(int) * atom_numbers);
    Malloc_Safely((void **)&h_LJ_A, sizeof(float) * pair_type_numbers);
    Malloc_Safely((void **)&h_LJ_B, sizeof(float) * pair_type_numbers);
    Cuda_Malloc_Safely((void **)&d_LJ_energy_sum, sizeof(float));
    Cuda_Malloc_Safely((void **)&d_LJ_energy_atom, sizeof(float) * atom_numbers);
    Cuda_Malloc_Safely((void **)&d_atom_LJ_type, sizeof(int) * atom_numbers);
    Cuda_Malloc_Safely((void **)&d_LJ_A, sizeof(float) * pair_type_numbers);
    Cuda_Malloc_Safely((void **)&d_LJ_B, sizeof(float) * pair_type_numbers);
}

void LENNARD_JONES_INFORMATION::Parameter_Host_To_Device()
{
    cudaMemcpy(d_LJ_A, h_LJ_A, sizeof(float) * pair_type_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(d_LJ_B, h_LJ_B, sizeof(float) * pair_type_numbers, cudaMemcpyHostToDevice);
    cudaMemcpy(d_atom_LJ_type, h_atom_LJ_type, sizeof(int) * atom_numbers, cudaMemcpyHostToDevice);
}

void LENNARD_JONES_INFORMATION::Initial(CONTROLLER *controller, float cutoff, VECTOR box_length, const char *module_name)
{
    if (module_name == NULL)
        strcpy(this->module_name, "LJ");
    else
        strcpy(this->module_name, module_name);
    controller[0].printf("START INITIALIZING LENNARD JONES INFORMATION (sponge_b200):\n");
    if (controller[0].Command_Exist(this->module_name, "in_file"))
    {
        FILE *fp = NULL;
        Open_File_Safely(&fp, controller[0].Command(this->module_name, "in_file"), "r");
        if (fscanf(fp, "%d %d", &atom_numbers, &atom_type_numbers) != 2)
        {
            fprintf(stderr, "sponge_b200: malformed LJ_in_file header\n");
            exit(1);
        }
        pair_type_numbers = atom_type_numbers * (atom_type_numbers + 1) / 2;
        LJ_Malloc();
        int ok = 1;
        for (int i = 0; i < pair_type_numbers; i++)
        {
            ok &= fscanf(fp, "%f", h_LJ_A + i) == 1;
            h_LJ_A[i] *= 12.0f;
        }
        for (int i = 0; i < pair_type_numbers; i++)
        {
            ok &= fscanf(fp, "%f", h_LJ_B + i) == 1;
            h_LJ_B[i] *= 6.0f;
        }
        for (int i = 0; i < atom_numbers; i++)
            ok &= fscanf(fp, "%d", h_atom_LJ_type + i) == 1;
        fclose(fp);
        if (!ok)
        {
            fprintf(stderr, "sponge_b200: truncated LJ_in_file\n");
            exit(1);
        }
        controller[0].printf("    atom_numbers is %d\n    atom_LJ_type_number is %d\n", atom_numbers, atom_type_numbers);
        Parameter_Host_To_Device();
        is_initialized = 1;
    }
    else if (controller[0].Command_Exist("amber_parm7"))
    {
        Initial_From_AMBER_Parm(controller[0].Command("amber_parm7"), controller[0]);
    }
    if (is_initialized)
    {
        this->cutoff = cutoff;
        this->uint_dr_to_dr_cof = 1.0f / CONSTANT_UINT_MAX_FLOAT * box_length;
        this->volume = box_length.x * box_length.y * box_length.z;
        float box[3] = {box_length.x, box_length.y, box_length.z};
        Sponge_B200_Check(sb_lj_create(atom_numbers, atom_type_numbers, h_LJ_A, h_LJ_B, h_atom_LJ_type,
                                       cutoff, box, SB_FORM_FIXED, &handle),
                          "LENNARD_JONES_INFORMATION::Initial");
        sb_lj_long_range_factor(handle, &long_range_factor);
        controller[0].printf("    long range correction factor is: %e\n", long_range_factor);
        if (!is_controller_printf_initialized)
        {
            controller[0].Step_Print_Initial(this->module_name, "%.2f");
            is_controller_printf_initialized = 1;
            controller[0].printf("    structure last modify date is %d\n", last_modify_date);
        }
    }
    controller[0].printf("END INITIALIZING LENNARD JONES INFORMATION\n\n");
}

// AMBER parm7 sections are "%FLAG NAME", one "%FORMAT(...)" line, then the values as
// whitespace-separated fields. Reads `count` values of the current section into `out`; returns
// the number read.
static int parm7_read_doubles(FILE *fp, double *out, int count)
{
    int got = 0;
    while (got < count && fscanf(fp, "%lf", out + got) == 1)
        got++;
    return got;
}

// LENNARD_JONES_INFORMATION::Initial_From_AMBER_Parm (Lennard_Jones_force.cu:1201-1276): the
// atom count and type count from POINTERS (its first two values), the per-atom type index
// (ATOM_TYPE_INDEX, 1-based in the file) and the pair tables LENNARD_JONES_ACOEF / _BCOEF, read
// in file order as the lower-triangular type-pair tables and scaled by 12 and 6 in double
// before rounding to float, as the reference reads them.
void LENNARD_JONES_INFORMATION::Initial_From_AMBER_Parm(const char *file_name, CONTROLLER controller)
{
    FILE *fp = NULL;
    Open_File_Safely(&fp, file_name, "r");
    controller.printf("    Start reading LJ information from AMBER file:\n");
    char line[CHAR_LENGTH_MAX];
    int have_pointers = 0, have_types = 0, have_a = 0, have_b = 0;
    std::vector<double> vals;
    while (fgets(line, CHAR_LENGTH_MAX, fp))
    {
        char flag[CHAR_LENGTH_MAX], name[CHAR_LENGTH_MAX];
        if (sscanf(line, "%s %s", flag, name) != 2 || strcmp(flag, "%FLAG") != 0)
            continue;
        const int pointers = strcmp(name, "POINTERS") == 0;
        const int types = strcmp(name, "ATOM_TYPE_INDEX") == 0;
        const int acoef = strcmp(name, "LENNARD_JONES_ACOEF") == 0;
        const int bcoef = strcmp(name, "LENNARD_JONES_BCOEF") == 0;
        if (!(pointers || types || acoef || bcoef))
            continue;
        if (!fgets(line, CHAR_LENGTH_MAX, fp))  // the %FORMAT line
            break;
        if (pointers)
        {
            vals.resize(2);
            if (parm7_read_doubles(fp, vals.data(), 2) != 2)
                break;
            atom_numbers = (int)vals[0];
            atom_type_numbers = (int)vals[1];
            pair_type_numbers = atom_type_numbers * (atom_type_numbers + 1) / 2;
            controller.printf("        atom_numbers is %d\n        atom_LJ_type_number is %d\n",
                              atom_numbers, atom_type_numbers);
            LJ_Malloc();
            have_pointers = 1;
        }
        else if (!have_pointers)
        {
            break;  // the tables are sized by POINTERS, which comes first in a parm7 file
        }
        else if (types)
        {
            vals.resize(atom_numbers);
            have_types = parm7_read_doubles(fp, vals.data(), atom_numbers) == atom_numbers;
            for (int i = 0; i < atom_numbers && have_types; i++)
                h_atom_LJ_type[i] = (int)vals[i] - 1;
        }
        else
        {
            vals.resize(pair_type_numbers);
            const int ok = parm7_read_doubles(fp, vals.data(), pair_type_numbers) == pair_type_numbers;
            float *dst = acoef ? h_LJ_A : h_LJ_B;
            const double scale = acoef ? 12.0 : 6.0;
            for (int i = 0; i < pair_type_numbers && ok; i++)
                dst[i] = (float)(scale * vals[i]);
            (acoef ? have_a : have_b) = ok;
        }
    }
    fclose(fp);
    if (!(have_pointers && have_types && have_a && have_b))
    {
        fprintf(stderr, "sponge_b200: %s lacks POINTERS, ATOM_TYPE_INDEX or the LJ A/B tables, "
                        "or one of them is truncated\n", file_name);
        exit(1);
    }
    for (int i = 0; i < atom_numbers; i++)
    {
        if (h_atom_LJ_type[i] < 0 || h_atom_LJ_type[i] >= atom_type_numbers)
        {
            fprintf(stderr, "sponge_b200: %s: atom %d has LJ type %d of %d\n", file_name, i,
                    h_atom_LJ_type[i] + 1, atom_type_numbers);
            exit(1);
        }
    }
    controller.printf("    End reading LJ information from AMBER file\n");
    Parameter_Host_To_Device();
    is_initialized = 1;
}

void LENNARD_JONES_INFORMATION::Clear()
{
    if (is_initialized)
    {
        is_initialized = 0;
        sb_lj_destroy(handle);
        handle = NULL;
        free(h_atom_LJ_type);
        free(h_LJ_A);
        free(h_LJ_B);
        free(h_LJ_energy_atom);
        cudaFree(d_atom_LJ_type);
        cudaFree(d_LJ_A);
        cudaFree(d_LJ_B);
        cudaFree(d_LJ_energy_atom);
        cudaFree(d_LJ_energy_sum);
        h_atom_LJ_type = NULL;
        h_LJ_A = NULL;
        h_LJ_B = NULL;
        h_LJ_energy_atom = NULL;
        d_atom_LJ_type = NULL;
        d_LJ_A = NULL;
        d_LJ_B = NULL;
        d_LJ_energy_atom = NULL;
        d_LJ_energy_sum = NULL;
    }
}

void LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(const int atom_numbers, const UNSIGNED_INT_VECTOR *uint_crd, const float *charge, VECTOR *frc,
    const ATOM_GROUP *nl, const float pme_beta, const int need_atom_energy, float *atom_energy,
    const int need_virial, float *atom_lj_virial, float *atom_direct_pme_energy)
{
    if (!is_initialized)
        return;
    Sponge_B200_Check(sb_lj_pme_direct_force(handle, Sponge_B200_Neighbor_List_Of(nl), atom_numbers,
                                             (const uint32_t *)uint_crd, charge, (float *)frc, pme_beta,
                                             need_atom_energy, atom_energy, need_virial, atom_lj_virial,
                                             atom_direct_pme_energy, NULL),
                      "LJ_PME_Direct_Force_With_Atom_Energy_And_Virial");
}

void LENNARD_JONES_INFORMATION::LJ_Force_With_PME_Direct_Force(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge, VECTOR *frc, const ATOM_GROUP *nl, const float pme_beta)
{
    LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(atom_numbers, uint_crd, charge, frc, nl, pme_beta, 0, NULL, 0, NULL, NULL);
}

void LENNARD_JONES_INFORMATION::Long_Range_Correction(int need_pressure, float *d_virial, int need_potential, float *d_potential)
{
    if (is_initialized)
        Sponge_B200_Check(sb_lj_long_range_correction(handle, need_pressure, d_virial, need_potential, d_potential, NULL),
                          "LENNARD_JONES_INFORMATION::Long_Range_Correction");
}

void LENNARD_JONES_INFORMATION::Long_Range_Correction(float volume)
{
    if (is_initialized)
    {
        float e = 0;
        cudaMemcpy(&e, d_LJ_energy_sum, sizeof(float), cudaMemcpyDeviceToHost);
        e += long_range_factor / volume;
        cudaMemcpy(d_LJ_energy_sum, &e, sizeof(float), cudaMemcpyHostToDevice);
    }
}

float LENNARD_JONES_INFORMATION::Get_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const ATOM_GROUP *nl, int is_download)
{
    if (!is_initialized)
        return NAN;
    float e = 0;
    Sponge_B200_Check(sb_lj_get_energy(handle, Sponge_B200_Neighbor_List_Of(nl), (const uint32_t *)uint_crd, &e, NULL),
                      "LENNARD_JONES_INFORMATION::Get_Energy");
    h_LJ_energy_sum = e;
    cudaMemcpy(d_LJ_energy_sum, &e, sizeof(float), cudaMemcpyHostToDevice);
    return is_download ? e : 0;
}

void LENNARD_JONES_INFORMATION::LJ_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const ATOM_GROUP *nl)
{
    Get_Energy(uint_crd, nl, 0);
}

void LENNARD_JONES_INFORMATION::Energy_Device_To_Host()
{
    cudaMemcpy(&h_LJ_energy_sum, d_LJ_energy_sum, sizeof(float), cudaMemcpyDeviceToHost);
}

void LENNARD_JONES_INFORMATION::Update_Volume(VECTOR box_length)
{
    if (!is_initialized)
        return;
    this->uint_dr_to_dr_cof = 1.0f / CONSTANT_UINT_MAX_FLOAT * box_length;
    this->volume = box_length.x * box_length.y * box_length.z;
    float box[3] = {box_length.x, box_length.y, box_length.z};
    Sponge_B200_Check(sb_lj_update_volume(handle, box), "LENNARD_JONES_INFORMATION::Update_Volume");
}
