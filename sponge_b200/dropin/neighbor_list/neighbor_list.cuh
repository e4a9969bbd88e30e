// Drop-in replacement for SPONGE's NEIGHBOR_LIST (SPONGE/neighbor_list/neighbor_list.cuh:44-106).
// Same struct name, public members read by other modules and method signatures; the work is done
// by libsponge_b200 through its C ABI (include/sponge_b200.h). Place this directory over
// SPONGE/neighbor_list and link libsponge_b200.so.
#ifndef NEIGHBOR_LIST_CUH
#define NEIGHBOR_LIST_CUH
#include "../common.cuh"
#include "../control.cuh"

struct sb_neighbor_list;

struct NEIGHBOR_LIST
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int is_controller_printf_initialized = 0;
    int last_modify_date = 20261203;

    int atom_numbers = 0;
    int refresh_interval = 0;
    int refresh_count = 0;

    float skin = 2.0;
    float cutoff = 10.0;
    float cutoff_square;
    float cutoff_with_skin;
    float half_cutoff_with_skin;
    float cutoff_with_skin_square;
    float half_skin_square;
    float skin_permit = 1.;
    VECTOR box_length;
    VECTOR quarter_crd_to_uint_crd_cof;
    VECTOR uint_dr_to_dr_cof;

    int refresh_flag;
    UNSIGNED_INT_VECTOR *uint_crd = NULL;  // the list's own fixed-point coordinates (device)
    ATOM_GROUP *d_nl = NULL;               // per-atom half list j > i (device), kept current when
                                           // atom_group_export = 1 (mdin neighbor_list_atom_group_export)
    int max_neighbor_numbers = 800;
    int max_atom_in_grid_numbers = 64;     // accepted for compatibility; the column sort has no cap
    int atom_group_export = 1;

    sb_neighbor_list *handle = NULL;

    void Initial(CONTROLLER *controller, int md_atom_numbers, VECTOR box_length, float cut, float skin, const char *module_name = NULL);
    void Initial_Malloc();
    void Clear();
    void Neighbor_List_Update(VECTOR *crd, int *d_excluded_list_start, int *d_excluded_list, int *d_excluded_numbers,
        int forced_update = 0, int forced_check = 0);
    void Update_Volume(VECTOR box_length);

    enum NEIGHBOR_LIST_UPDATE_PARAMETER
    {
        CONDITIONAL_UPDATE = 0,
        FORCED_UPDATE = 1
    };
    enum NEIGHBOR_LIST_CHECK_PARAMETER
    {
        CONDITIONAL_CHECK = 0,
        FORCED_CHECK = 1
    };
};

// The LJ and PME drop-ins receive `const ATOM_GROUP *nl` (= NEIGHBOR_LIST::d_nl) and find the
// list handle behind it here.
sb_neighbor_list *Sponge_B200_Neighbor_List_Of(const ATOM_GROUP *d_nl);
// Prints the library's last error and exits, as the reference's fatal paths do.
void Sponge_B200_Check(int status, const char *what);

#endif //NEIGHBOR_LIST_CUH
