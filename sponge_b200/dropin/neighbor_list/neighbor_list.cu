// Drop-in NEIGHBOR_LIST forwarding to libsponge_b200 (see neighbor_list.cuh).
#include "neighbor_list.cuh"

#include <map>

#include "sponge_b200.h"

static std::map<const void *, sb_neighbor_list *> &registry()
{
    static std::map<const void *, sb_neighbor_list *> r;
    return r;
}

sb_neighbor_list *Sponge_B200_Neighbor_List_Of(const ATOM_GROUP *d_nl)
{
    std::map<const void *, sb_neighbor_list *>::iterator it = registry().find((const void *)d_nl);
    if (it == registry().end())
    {
        fprintf(stderr, "sponge_b200: the ATOM_GROUP list passed is not owned by a NEIGHBOR_LIST\n");
        exit(1);
    }
    return it->second;
}

void Sponge_B200_Check(int status, const char *what)
{
    if (status != SB_OK)
    {
        fprintf(stderr, "sponge_b200: %s failed (%d): %s\n", what, status, sb_last_error());
        exit(1);
    }
}

void NEIGHBOR_LIST::Initial(CONTROLLER *controller, int md_atom_numbers, VECTOR box_length, float cut, float skin, const char *module_name)
{
    if (module_name == NULL)
        strcpy(this->module_name, "neighbor_list");
    else
        strcpy(this->module_name, module_name);
    controller[0].printf("START INITIALIZING NEIGHBOR LIST (sponge_b200):\n");
    atom_numbers = md_atom_numbers;
    float permit = 0.5f;
    if (controller[0].Command_Exist(this->module_name, "refresh_interval"))
        refresh_interval = atoi(controller[0].Command(this->module_name, "refresh_interval"));
    if (controller[0].Command_Exist(this->module_name, "max_atom_in_grid_numbers"))
        max_atom_in_grid_numbers = atoi(controller[0].Command(this->module_name, "max_atom_in_grid_numbers"));
    if (controller[0].Command_Exist(this->module_name, "max_neighbor_numbers"))
        max_neighbor_numbers = atoi(controller[0].Command(this->module_name, "max_neighbor_numbers"));
    if (controller[0].Command_Exist(this->module_name, "skin_permit"))
        permit = atof(controller[0].Command(this->module_name, "skin_permit"));
    if (controller[0].Command_Exist(this->module_name, "atom_group_export"))
        atom_group_export = atoi(controller[0].Command(this->module_name, "atom_group_export"));
    skin_permit = 2.f * permit;
    this->skin = skin;
    this->cutoff = cut;
    cutoff_square = cutoff * cutoff;
    cutoff_with_skin = cutoff + skin;
    half_cutoff_with_skin = 0.5 * cutoff_with_skin;
    cutoff_with_skin_square = cutoff_with_skin * cutoff_with_skin;
    half_skin_square = 0.25 * skin * skin;
    this->box_length = box_length;
    this->quarter_crd_to_uint_crd_cof = 0.25f * CONSTANT_UINT_MAX_FLOAT / box_length;
    this->uint_dr_to_dr_cof = 1.0f / CONSTANT_UINT_MAX_FLOAT * box_length;
    float box[3] = {box_length.x, box_length.y, box_length.z};
    Sponge_B200_Check(sb_nl_create(atom_numbers, box, cutoff, skin, refresh_interval, permit,
                                   max_neighbor_numbers, SB_FORM_FIXED, &handle),
                      "NEIGHBOR_LIST::Initial");
    // pruned pair list (sb_nl_set_prune; off unless neighbor_list_prune_buffer is given)
    float prune_buffer = 0.f;
    int prune_interval = 0;
    if (controller[0].Command_Exist(this->module_name, "prune_buffer"))
        prune_buffer = atof(controller[0].Command(this->module_name, "prune_buffer"));
    if (controller[0].Command_Exist(this->module_name, "prune_interval"))
        prune_interval = atoi(controller[0].Command(this->module_name, "prune_interval"));
    if (prune_buffer > 0.f)
    {
        Sponge_B200_Check(sb_nl_set_prune(handle, prune_buffer, prune_interval),
                          "NEIGHBOR_LIST::Initial (prune)");
        controller[0].printf("    pruned pair list: cutoff + %.2f, renewed every %d updates and on moves of %.2f\n",
                             prune_buffer, prune_interval, 0.5f * prune_buffer);
    }
    const uint32_t *uc = NULL;
    sb_nl_uint_crd(handle, &uc);
    uint_crd = (UNSIGNED_INT_VECTOR *)uc;
    is_initialized = 1;
    controller[0].printf("    refresh interval %d, cutoff %.2f, skin %.2f\n", refresh_interval, cutoff, skin);
    if (!is_controller_printf_initialized)
    {
        is_controller_printf_initialized = 1;
        controller[0].printf("    structure last modify date is %d\n", last_modify_date);
    }
    controller[0].printf("END INITIALIZING NEIGHBOR LIST\n\n");
}

void NEIGHBOR_LIST::Initial_Malloc()
{
}

void NEIGHBOR_LIST::Neighbor_List_Update(VECTOR *crd, int *d_excluded_list_start, int *d_excluded_list, int *d_excluded_numbers,
    int forced_update, int forced_check)
{
    if (!is_initialized)
        return;
    Sponge_B200_Check(sb_nl_update(handle, (float *)crd, d_excluded_list_start, d_excluded_list,
                                   d_excluded_numbers, forced_update, forced_check, NULL),
                      "NEIGHBOR_LIST::Neighbor_List_Update");
    if (d_nl == NULL || atom_group_export)
    {
        void *p = NULL;
        Sponge_B200_Check(sb_nl_atom_group(handle, &p, NULL), "NEIGHBOR_LIST atom group export");
        if (d_nl == NULL)
        {
            d_nl = (ATOM_GROUP *)p;
            registry()[(const void *)d_nl] = handle;
        }
    }
}

void NEIGHBOR_LIST::Update_Volume(VECTOR box_length)
{
    this->box_length = box_length;
    this->quarter_crd_to_uint_crd_cof = 0.25f * CONSTANT_UINT_MAX_FLOAT / box_length;
    this->uint_dr_to_dr_cof = 1.0f / CONSTANT_UINT_MAX_FLOAT * box_length;
    float box[3] = {box_length.x, box_length.y, box_length.z};
    if (is_initialized)
        Sponge_B200_Check(sb_nl_update_volume(handle, box), "NEIGHBOR_LIST::Update_Volume");
}

void NEIGHBOR_LIST::Clear()
{
    if (is_initialized)
    {
        is_initialized = 0;
        if (d_nl)
            registry().erase((const void *)d_nl);
        sb_nl_destroy(handle);
        handle = NULL;
        d_nl = NULL;
        uint_crd = NULL;
    }
}
