// Drop-in Particle_Mesh_Ewald forwarding to libsponge_b200 (see PME_force.cuh).
#include "PME_force.cuh"

#include "../neighbor_list/neighbor_list.cuh"
#include "sponge_b200.h"

// ---------------------------------------------------------------------------------------------
// The reference-layout PME internals for TI_CORE (see PME_force.cuh). The kernels keep the
// reference header's contracts: a grid coordinate u = uint * K / 2^32 in FP32, base = (int)u,
// fraction u - base; the 64 stencil points (base - k) mod K of the 4th-order B-spline; charge
// spread with float atomics; the half spectrum times the Green's function table; a dot product
// summed by one block.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float ti_bspline4(int k, float f)
{
    // weight of stencil offset k (0..3) at fraction f: the cardinal cubic B-spline pieces
    const float f2 = f * f, f3 = f2 * f;
    switch (k)
    {
    case 0: return f3 * (1.0f / 6.0f);
    case 1: return -0.5f * f3 + 0.5f * f2 + 0.5f * f + (1.0f / 6.0f);
    case 2: return 0.5f * f3 - f2 + (2.0f / 3.0f);
    default: return -f3 * (1.0f / 6.0f) + 0.5f * f2 - 0.5f * f + (1.0f / 6.0f);
    }
}

__global__ void PME_Atom_Near(const UNSIGNED_INT_VECTOR *uint_crd, int **PME_atom_near, const int PME_Nin,
    const float periodic_factor_inverse_x, const float periodic_factor_inverse_y, const float periodic_factor_inverse_z,
    const int atom_numbers, const int fftx, const int ffty, const int fftz,
    const UNSIGNED_INT_VECTOR *PME_kxyz, UNSIGNED_INT_VECTOR *PME_uxyz, VECTOR *PME_frxyz)
{
    const int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i >= atom_numbers)
        return;
    const float ux = (float)uint_crd[i].uint_x * periodic_factor_inverse_x;
    const float uy = (float)uint_crd[i].uint_y * periodic_factor_inverse_y;
    const float uz = (float)uint_crd[i].uint_z * periodic_factor_inverse_z;
    const int bx = (int)ux, by = (int)uy, bz = (int)uz;
    PME_frxyz[i].x = ux - bx;
    PME_frxyz[i].y = uy - by;
    PME_frxyz[i].z = uz - bz;
    UNSIGNED_INT_VECTOR last = PME_uxyz[i];
    if ((int)last.uint_x == bx && (int)last.uint_y == by && (int)last.uint_z == bz)
        return;  // same base cell as the last call: the stencil indices stand
    PME_uxyz[i].uint_x = bx;
    PME_uxyz[i].uint_y = by;
    PME_uxyz[i].uint_z = bz;
    int *near = PME_atom_near[i];
    for (int k = 0; k < 64; k++)
    {
        const UNSIGNED_INT_VECTOR o = PME_kxyz[k];
        int gx = bx - (int)o.uint_x, gy = by - (int)o.uint_y, gz = bz - (int)o.uint_z;
        gx += gx < 0 ? fftx : (gx >= fftx ? -fftx : 0);
        gy += gy < 0 ? ffty : (gy >= ffty ? -ffty : 0);
        gz += gz < 0 ? fftz : (gz >= fftz ? -fftz : 0);
        near[k] = gx * PME_Nin + gy * fftz + gz;
    }
}

__global__ void PME_Q_Spread(int **PME_atom_near, const float *charge, const VECTOR *PME_frxyz,
    float *PME_Q, const UNSIGNED_INT_VECTOR *PME_kxyz, const int atom_numbers)
{
    const int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i >= atom_numbers)
        return;
    const int *near = PME_atom_near[i];
    const VECTOR f = PME_frxyz[i];
    const float q = charge[i];
    for (int k = threadIdx.y; k < 64; k += blockDim.y)
    {
        const UNSIGNED_INT_VECTOR o = PME_kxyz[k];
        const float w = q * ti_bspline4(o.uint_x, f.x) * ti_bspline4(o.uint_y, f.y) *
                        ti_bspline4(o.uint_z, f.z);
        atomicAdd(&PME_Q[near[k]], w);
    }
}

__global__ void PME_BCFQ(cufftComplex *PME_FQ, float *PME_BC, int PME_Nfft)
{
    const int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < PME_Nfft)
    {
        const float b = PME_BC[i];
        PME_FQ[i].x *= b;
        PME_FQ[i].y *= b;
    }
}

__global__ void PME_Energy_Product(const int element_number, const float *list1, const float *list2, float *sum)
{
    // one block: a strided partial per thread, a warp-shuffle and shared-memory tree, one store
    __shared__ float part[32];
    float v = 0.f;
    for (int i = threadIdx.x; i < element_number; i += blockDim.x)
        v += list1[i] * list2[i];
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        v = threadIdx.x < (blockDim.x + 31) / 32 ? part[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0)
            sum[0] = v;
    }
}

__global__ static void ti_fill_kxyz(UNSIGNED_INT_VECTOR *kxyz, UNSIGNED_INT_VECTOR *uxyz, int n,
                                    int **near, int *block)
{
    const int i = blockDim.x * blockIdx.x + threadIdx.x;
    if (i < 64)
    {
        kxyz[i].uint_x = i >> 4;
        kxyz[i].uint_y = (i >> 2) & 3;
        kxyz[i].uint_z = i & 3;
    }
    if (i < n)
    {
        // no base cell yet: the first PME_Atom_Near computes every stencil
        uxyz[i].uint_x = uxyz[i].uint_y = uxyz[i].uint_z = 1u << 30;
        near[i] = block + 64 * (size_t)i;
    }
}

void Particle_Mesh_Ewald::Initial_TI_Internals()
{
    if (ti_internals)
        return;
    Cuda_Malloc_Safely((void **)&PME_kxyz, sizeof(UNSIGNED_INT_VECTOR) * 64);
    Cuda_Malloc_Safely((void **)&PME_uxyz, sizeof(UNSIGNED_INT_VECTOR) * atom_numbers);
    Cuda_Malloc_Safely((void **)&PME_frxyz, sizeof(VECTOR) * atom_numbers);
    Cuda_Malloc_Safely((void **)&PME_Q, sizeof(float) * PME_Nall);
    Cuda_Malloc_Safely((void **)&PME_FBCFQ, sizeof(float) * PME_Nall);
    Cuda_Malloc_Safely((void **)&PME_FQ, sizeof(cufftComplex) * PME_Nfft);
    Cuda_Malloc_Safely((void **)&PME_atom_near, sizeof(int *) * atom_numbers);
    Cuda_Malloc_Safely((void **)&PME_atom_near_block, sizeof(int) * 64 * (size_t)atom_numbers);
    Cuda_Malloc_Safely((void **)&charge_sum, sizeof(float));
    const int n = atom_numbers > 64 ? atom_numbers : 64;
    ti_fill_kxyz<<<(n + 255) / 256, 256>>>(PME_kxyz, PME_uxyz, atom_numbers, PME_atom_near,
                                           PME_atom_near_block);
    if (cufftPlan3d(&PME_plan_r2c, fftx, ffty, fftz, CUFFT_R2C) != CUFFT_SUCCESS ||
        cufftPlan3d(&PME_plan_c2r, fftx, ffty, fftz, CUFFT_C2R) != CUFFT_SUCCESS)
    {
        fprintf(stderr, "sponge_b200: cuFFT plans of the TI internals could not be created\n");
        exit(1);
    }
    const float *bc = NULL;
    Sponge_B200_Check(sb_pme_bc_table(handle, &bc), "Particle_Mesh_Ewald::Initial_TI_Internals");
    PME_BC = (float *)bc;
    ti_internals = 1;
}

void Particle_Mesh_Ewald::Clear_TI_Internals()
{
    if (!ti_internals)
        return;
    cufftDestroy(PME_plan_r2c);
    cufftDestroy(PME_plan_c2r);
    void *ps[] = {PME_kxyz, PME_uxyz, PME_frxyz, PME_Q, PME_FBCFQ, PME_FQ, PME_atom_near,
                  PME_atom_near_block, charge_sum};
    for (void *q : ps)
        cudaFree(q);
    PME_kxyz = PME_uxyz = NULL;
    PME_frxyz = NULL;
    PME_Q = PME_FBCFQ = charge_sum = NULL;
    PME_FQ = NULL;
    PME_atom_near = NULL;
    PME_atom_near_block = NULL;
    PME_BC = NULL;
    ti_internals = 0;
}

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
    if (controller[0].Command_Exist("charge_pertubated") && atoi(controller[0].Command("charge_pertubated")) != 0)
        Initial_TI_Internals();
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
        Clear_TI_Internals();
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
