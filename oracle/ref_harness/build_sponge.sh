#!/bin/bash
# Builds the unchanged SPONGE drivers (SPONGE/main.cu, main_fep.cu and main_ti.cu with every
# module they link, per the reference's Makefile object lists) twice, into oracle/_ref/
# (git-ignored, travels to the GPU box):
#   sponge_stock, sponge_fep_stock, sponge_ti_stock   the reference exactly as shipped (target
#                  sm_100a, -include cfloat)
#   sponge_b200, sponge_fep_b200, sponge_ti_b200      the same drivers with neighbor_list/,
#                  Lennard_Jones_force.cu/.cuh and PME_force/ replaced by sponge_b200/dropin and
#                  linked to libsponge_b200.so
# Sources are compiled where they lie through a shadow tree of symlinks; nothing is copied.
# usage: oracle/ref_harness/build_sponge.sh [stock|b200|both]   (needs the reference tree)
set -e
REF=${REF:-/root/reference/SPONGE}
HERE=$(cd "$(dirname "$0")" && pwd)
REPO=$(cd "$HERE/../.." && pwd)
OUT=$REPO/oracle/_ref
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
JOBS=${JOBS:-8}
FLAGS="-arch=sm_100a -rdc=true --use_fast_math -O3 -std=c++14 -include cfloat -w"
OBJS="main common control MD_core/MD_core bond/bond bond/bond_soft angle/angle angle/Urey_Bradley_force
dihedral/dihedral dihedral/improper_dihedral cmap/cmap nb14/nb14 neighbor_list/neighbor_list
Lennard_Jones_force/Lennard_Jones_force Lennard_Jones_force/LJ_soft_core PME_force/PME_force
thermostats/Langevin_MD thermostats/Middle_Langevin_MD thermostats/Andersen_thermostat
thermostats/Berendsen_thermostat thermostats/nose_hoover_chain barostats/MC_barostat
barostats/Berendsen_barostat barostats/andersen_barostat restrain/restrain constrain/constrain
constrain/simple_constrain constrain/SETTLE constrain/SHAKE virtual_atoms/virtual_atoms
crd_molecular_map/crd_molecular_map"
FEP_OBJS="main_fep common control FEP_core/FEP_core bond/bond bond/bond_soft angle/angle
dihedral/dihedral nb14/nb14 neighbor_list/neighbor_list Lennard_Jones_force/LJ_soft_core
PME_force/PME_force"
TI_OBJS="main_ti common control TI_core/TI_core bond/bond bond/bond_soft angle/angle
dihedral/dihedral nb14/nb14 neighbor_list/neighbor_list Lennard_Jones_force/LJ_soft_core
PME_force/PME_force"

shadow() {  # $1 = variant dir
    local S=$1
    rm -rf "$S"
    mkdir -p "$S"
    (cd "$REF" && find . -type d) | while read -r d; do mkdir -p "$S/$d"; done
    (cd "$REF" && find . -type f \( -name '*.cu' -o -name '*.cuh' \)) | while read -r f; do
        ln -s "$REF/$f" "$S/$f"
    done
}

build_variant() {  # $1 = stock|b200
    local V=$1
    local S=$OUT/src_$V
    shadow "$S"
    local LINK=""
    if [ "$V" = "b200" ]; then
        for f in neighbor_list/neighbor_list.cu neighbor_list/neighbor_list.cuh \
                 Lennard_Jones_force/Lennard_Jones_force.cu Lennard_Jones_force/Lennard_Jones_force.cuh \
                 PME_force/PME_force.cu PME_force/PME_force.cuh; do
            rm -f "$S/$f"
            ln -s "$REPO/sponge_b200/dropin/$f" "$S/$f"
        done
        LINK="-L$REPO/sponge_b200 -lsponge_b200 -Xlinker -rpath=$REPO/sponge_b200 -Xlinker -rpath=\$ORIGIN/../../sponge_b200"
    fi
    mkdir -p "$S/obj"
    echo $OBJS $FEP_OBJS $TI_OBJS | tr ' ' '\n' | sort -u | xargs -P "$JOBS" -I{} sh -c \
        "mkdir -p \$(dirname '$S/obj/{}.o') && $NVCC $FLAGS -I$REPO/include -c '$S/{}.cu' -o '$S/obj/{}.o'"
    local OL=""
    for o in $OBJS; do OL="$OL $S/obj/$o.o"; done
    $NVCC -arch=sm_100a -rdc=true -o "$OUT/sponge_$V" $OL -lcufft -lcudadevrt $LINK
    echo "built $OUT/sponge_$V"
    OL=""
    for o in $FEP_OBJS; do OL="$OL $S/obj/$o.o"; done
    $NVCC -arch=sm_100a -rdc=true -o "$OUT/sponge_fep_$V" $OL -lcufft -lcudadevrt $LINK
    echo "built $OUT/sponge_fep_$V"
    OL=""
    for o in $TI_OBJS; do OL="$OL $S/obj/$o.o"; done
    $NVCC -arch=sm_100a -rdc=true -o "$OUT/sponge_ti_$V" $OL -lcufft -lcudadevrt $LINK
    echo "built $OUT/sponge_ti_$V"
}

mkdir -p "$OUT"
case "${1:-both}" in
    stock) build_variant stock ;;
    b200) build_variant b200 ;;
    both) build_variant stock; build_variant b200 ;;
esac
