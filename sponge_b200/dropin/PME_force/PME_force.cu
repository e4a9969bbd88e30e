// Drop-in Particle_Mesh_Ewald forwarding to libsponge_b200 (see PME_force.cuh).
#include "PME_force.cuh"

#include "../neighbor_list/neighbor_list.cuh"
#include "sponge_b200.h"

void Particle_Mesh_Ewald::Initial(CONTROLLER *controller, int atom_numbers, VECTOR boxlength, float cutoff, const char *module_name)
{
    if (module_name == NULL)
        strcpy(this->module_name, "PME");
    else
        strcpy(this->module_name, module_name);
    controller[0].printf("START INITIALIZING PME (sponge_b200):\n");
    this->cutoff = cutoff;
    tolerance = 0.00001f;
    if (controller[0].Command_Exist(this->module_name, "Direct_Tolerance"))
        tolerance = atof(controller[0].Command(this->module_name, "Direct_Tolerance"));
    fftx = ffty = fftz = -1;
    if (controller[0].Command_Exist(this->module_name, "fftx"))
        fftx = atoi(controller[0].Command(this->module_name, "fftx"));
    if (controller[0].Command_Exist(this->module_name, "ffty"))
        ffty = atoi(controller[0].Command(this->module_name, "ffty"));
    if (controller[0].Command_Exist(this->module_name, "fftz"))
        fftz = atoi(controller[0].Command(this->module_name, "fftz"));
    this->atom_numbers = atom_numbers;
    this->boxlength = boxlength;
    float box[3] = {boxlength.x, boxlength.y, boxlength.z};
    Sponge_B200_Check(sb_pme_create(atom_numbers, box, cutoff, tolerance, fftx, ffty, fftz, SB_FORM_FIXED, &handle),
                      "Particle_Mesh_Ewald::Initial");
    int k[3];
    sb_pme_info(handle, &beta, k);
    fftx = k[0];
    ffty = k[1];
    fftz = k[2];
    PME_Nall = fftx * ffty * fftz;
    PME_Nin = ffty * fftz;
    PME_Nfft = fftx * ffty * (fftz / 2 + 1);
    PME_inverse_box_vector.x = (float)fftx / boxlength.x;
    PME_inverse_box_vector.y = (float)ffty / boxlength.y;
    PME_inverse_box_vector.z = (float)fftz / boxlength.z;
    float volume = boxlength.x * boxlength.y * boxlength.z;
    neutralizing_factor = -0.5 * CONSTANT_Pi / (beta * beta * volume);
    sb_pme_atom_energy_arrays(handle, &d_direct_atom_energy, &d_correction_atom_energy);
    Cuda_Malloc_Safely((void **)&d_reciprocal_ene, sizeof(float));
    Cuda_Malloc_Safely((void **)&d_self_ene, sizeof(float));
    Cuda_Malloc_Safely((void **)&d_direct_ene, sizeof(float));
    Cuda_Malloc_Safely((void **)&d_correction_ene, sizeof(float));
    Cuda_Malloc_Safely((void **)&d_ee_ene, sizeof(float));
    cudaMemset(d_direct_ene, 0, sizeof(float));
    controller[0].printf("    fftx: %d\n    ffty: %d\n    fftz: %d\n    beta: %f\n", fftx, ffty, fftz, beta);
    is_initialized = 1;
    if (!is_controller_printf_initialized)
    {
        controller[0].Step_Print_Initial(this->module_name, "%.2f");
        is_controller_printf_initialized = 1;
        controller[0].printf("    structure last modify date is %d\n", last_modify_date);
    }
    controller[0].printf("END INITIALIZING PME\n\n");
}

void Particle_Mesh_Ewald::Clear()
{
    if (is_initialized)
    {
        is_initialized = 0;
        sb_pme_destroy(handle);
        handle = NULL;
        d_direct_atom_energy = NULL;
        d_correction_atom_energy = NULL;
        cudaFree(d_reciprocal_ene);
        cudaFree(d_self_ene);
        cudaFree(d_direct_ene);
        cudaFree(d_correction_ene);
        cudaFree(d_ee_ene);
        d_reciprocal_ene = d_self_ene = d_direct_ene = d_correction_ene = d_ee_ene = NULL;
    }
}

void Particle_Mesh_Ewald::PME_Excluded_Force_With_Atom_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const VECTOR sacler, const float *charge,
    const int *excluded_list_start, const int *excluded_list, const int *excluded_atom_numbers,
    VECTOR *frc, float *atom_energy)
{
    if (!is_initialized)
        return;
    float sc[3] = {sacler.x, sacler.y, sacler.z};
    Sponge_B200_Check(sb_pme_excluded_force(handle, (const uint32_t *)uint_crd, sc, charge, excluded_list_start,
                                            excluded_list, excluded_atom_numbers, (float *)frc, atom_energy, NULL),
                      "PME_Excluded_Force_With_Atom_Energy");
}

void Particle_Mesh_Ewald::PME_Reciprocal_Force_With_Energy_And_Virial(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge,
    VECTOR *force, int need_virial, int need_energy, float *d_virial, float *d_potential)
{
    if (!is_initialized)
        return;
    Sponge_B200_Check(sb_pme_reciprocal_force(handle, (const uint32_t *)uint_crd, charge, (float *)force, need_virial,
                                              need_energy, d_virial, d_potential, NULL),
                      "PME_Reciprocal_Force_With_Energy_And_Virial");
}

float Particle_Mesh_Ewald::Get_Energy(const UNSIGNED_INT_VECTOR *uint_crd, const float *charge,
    const ATOM_GROUP *nl, const VECTOR scaler,
    const int *excluded_list_start, const int *excluded_list, const int *excluded_atom_numbers, int which_part, int is_download)
{
    if (!is_initialized)
        return NAN;
    float sc[3] = {scaler.x, scaler.y, scaler.z};
    float e = 0;
    double parts[5];
    sb_neighbor_list *h = NULL;
    if (which_part == TOTAL || which_part == DIRECT)
        h = Sponge_B200_Neighbor_List_Of(nl);
    Sponge_B200_Check(sb_pme_get_energy(handle, h, (const uint32_t *)uint_crd, charge, sc, excluded_list_start,
                                        excluded_list, excluded_atom_numbers, which_part, &e, parts, NULL),
                      "Particle_Mesh_Ewald::Get_Energy");
    if (which_part == TOTAL || which_part == DIRECT)
        direct_ene = (float)parts[1];
    if (which_part == TOTAL || which_part == RECIPROCAL)
        reciprocal_ene = (float)parts[2];
    if (which_part == TOTAL || which_part == CORRECTION)
        correction_ene = (float)parts[3];
    if (which_part == TOTAL || which_part == SELF)
        self_ene = (float)parts[4];
    if (which_part == TOTAL)
        ee_ene = e;
    cudaMemcpy(d_direct_ene, &direct_ene, sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_reciprocal_ene, &reciprocal_ene, sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_correction_ene, &correction_ene, sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_self_ene, &self_ene, sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_ee_ene, &ee_ene, sizeof(float), cudaMemcpyHostToDevice);
    return is_download ? e : 0;
}

void Particle_Mesh_Ewald::Update_Volume(VECTOR box_length)
{
    // the reference passes its own member box here (PME_force.cu:996-999); the new box is used
    Update_Box_Length(box_length);
}

void Particle_Mesh_Ewald::Update_Box_Length(VECTOR boxlength)
{
    if (!is_initialized)
        return;
    this->boxlength = boxlength;
    PME_inverse_box_vector.x = (float)fftx / boxlength.x;
    PME_inverse_box_vector.y = (float)ffty / boxlength.y;
    PME_inverse_box_vector.z = (float)fftz / boxlength.z;
    float volume = boxlength.x * boxlength.y * boxlength.z;
    neutralizing_factor = -0.5 * CONSTANT_Pi / (beta * beta * volume);
    float box[3] = {boxlength.x, boxlength.y, boxlength.z};
    Sponge_B200_Check(sb_pme_update_box(handle, box), "Particle_Mesh_Ewald::Update_Box_Length");
}
