"""Real-system fixture from the reference's own input files (SPONGE/covid-tip4p/) and the
reference's forces on it (test infrastructure).

SPONGE ships one real system, a 98,282-atom protein in TIP4P water (virtual M sites included as
charged particles), with no expected outputs. Two steps make it a parity case for the nonbonded
path and for the two modules beside it, the 1-4 pairs and the virtual atoms:

    python tests/golden/make_covid.py inputs      # here: reads the reference tree, writes
                                                  #   covid_tip4p_inputs.npz (coordinates,
                                                  #   charges, LJ tables and types, exclusions)
    python tests/golden/make_covid.py reference [out.npz]
                                                  # on a GPU machine with oracle/_ref built:
                                                  #   runs the reference's unchanged modules,
                                                  #   writes reference_covid_tip4p.npz

The inputs follow the reference's file formats (SPONGE/MD_core/MD_core.cu:1213-1257 coordinates
with the box on the line after them, :1051-1080 charges, :308-351 exclusions as per-atom
"count j1 j2 ..." lists of later atoms; SPONGE/Lennard_Jones_force/Lennard_Jones_force.cu
:1082-1105 "N T", then A and B over the T(T+1)/2 type pairs, then the N types). The cut-off
(10 A), skin (2 A) and Ewald tolerance (1e-5) are SPONGE's defaults; the PME grid is the one
Get_Fft_Patameter picks for the box. The 1-4 pairs (covid-tip4p_nb14.txt: "count", then
"a b lj_scale cf_scale") and virtual atoms (covid-tip4p_vatom.txt: one "type v from... params" line
each) come from the same directory. For one NVE step with SETTLE the bonds (covid-tip4p_bond.txt:
"count", then "a b k r0"; only the pairs CONSTRAIN keeps are used), the masses
(covid-tip4p_mass.txt) and the equilibrated velocities (npt_velocity.txt) are added, with a
2 fs step; the bonded forces are not part of the comparison.
"""

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
INPUTS = os.path.join(HERE, "covid_tip4p_inputs.npz")
REFERENCE = os.path.join(HERE, "reference_covid_tip4p.npz")
# the reference tree is read where the harness scripts read it (REF, as in
# oracle/ref_harness/build_all.sh)
SOURCE = os.path.join(os.environ.get("REF", "/root/reference/SPONGE"), "covid-tip4p")
# Get_Fft_Patameter's grid for the fixture's box (108.43 x 91.25 x 84.41 A)
FFT = (112, 96, 96)
# the MD step: 2 fs in SPONGE's internal time unit (MD_core.cu reads dt in ps and multiplies by
# CONSTANT_TIME_CONVERTION = 20.455 in FP32)
MD_DT = np.float32(np.float32(0.002) * np.float32(20.455))
# atoms whose SETTLE outputs are stored (a seeded sample, so the file stays small)
SETTLE_SAMPLE = 8192


def read_reference_files(src=SOURCE, prefix="covid-tip4p", coordinates="npt_coordinate.txt"):
    """The LJ + PME inputs of the reference's covid-tip4p system, as arrays, read with
    sponge_b200.sponge_io. The coordinates are the equilibrated ones the reference ships beside
    the topology (npt_coordinate.txt): the starting structure (covid-tip4p_coordinate.txt) still
    has clashes of 0.34 A between non-excluded atoms, whose 1e12 kcal/mol/A forces would swamp any
    comparison."""
    sys.path.insert(0, ROOT)
    from sponge_b200 import sponge_io
    p = lambda name: os.path.join(src, "%s_%s.txt" % (prefix, name))  # noqa: E731
    crd, box = sponge_io.read_coordinate(os.path.join(src, coordinates))
    charge = sponge_io.read_values(p("charge"))
    A, B, lj_type, t = sponge_io.read_lj(p("lj"))
    _, numbers, excl_list = sponge_io.read_exclude(p("exclude"))
    a14, b14, ljs14, cf14 = sponge_io.read_nb14(p("nb14"))
    vt, va, vp = sponge_io.read_vatom(p("vatom"))
    ba, bb, _, br = sponge_io.read_bond(p("bond"))
    mass = sponge_io.read_values(p("mass"))
    vel = sponge_io.read_velocity(os.path.join(src, "npt_velocity.txt"))
    return dict(crd=crd, box=box, charge=charge, lj_A=A, lj_B=B, lj_type=lj_type,
                n_types=np.int32(t), excl_numbers=numbers, excl_list=excl_list, nb14_a=a14,
                nb14_b=b14, nb14_lj_scale=ljs14, nb14_cf=cf14, vs_type=vt, vs_atoms=va,
                vs_param=vp, bond_a=ba, bond_b=bb, bond_r=br, mass=mass, vel=vel)


def load_system(path=INPUTS):
    """The fixture as a system dict of the form sponge_b200.systems builds."""
    z = np.load(path)
    n = z["charge"].size
    numbers = z["excl_numbers"].astype(np.int32)
    start = np.zeros(n, np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    box = z["box"].astype(np.float32)
    crd = np.mod(z["crd"].astype(np.float64), box.astype(np.float64)).astype(np.float32)
    crd = np.where(crd >= box, np.float32(0.0), crd).astype(np.float32)
    return dict(
        name="covid_tip4p", crd=crd, charge=z["charge"].astype(np.float32),
        lj_type=z["lj_type"].astype(np.int32), n_types=int(z["n_types"]),
        lj_A=z["lj_A"].astype(np.float32), lj_B=z["lj_B"].astype(np.float32),
        excl_start=start, excl_numbers=numbers, excl_list=z["excl_list"].astype(np.int32),
        box=box, cutoff=10.0, skin=2.0, fft=FFT, tolerance=1e-5,
        nb14_a=z["nb14_a"].astype(np.int32), nb14_b=z["nb14_b"].astype(np.int32),
        nb14_lj_scale=z["nb14_lj_scale"].astype(np.float32),
        nb14_cf=z["nb14_cf"].astype(np.float32), vs_type=z["vs_type"].astype(np.int32),
        vs_atoms=z["vs_atoms"].astype(np.int32), vs_param=z["vs_param"].astype(np.float32),
        bond_a=z["bond_a"].astype(np.int32), bond_b=z["bond_b"].astype(np.int32),
        bond_r=z["bond_r"].astype(np.float32), mass=z["mass"].astype(np.float32),
        vel=z["vel"].astype(np.float32), md_dt=MD_DT)


def settle_sample(n):
    """The atoms whose SETTLE step outputs the reference file keeps."""
    return np.sort(np.random.default_rng(2024).choice(n, SETTLE_SAMPLE, replace=False))


def write_inputs():
    r = read_reference_files()
    np.savez_compressed(INPUTS, crd=r["crd"], box=r["box"], charge=r["charge"],
                        lj_A=r["lj_A"], lj_B=r["lj_B"], lj_type=r["lj_type"].astype(np.int8),
                        n_types=r["n_types"], excl_numbers=r["excl_numbers"].astype(np.int16),
                        excl_list=r["excl_list"].astype(np.int32), nb14_a=r["nb14_a"],
                        nb14_b=r["nb14_b"], nb14_lj_scale=r["nb14_lj_scale"],
                        nb14_cf=r["nb14_cf"], vs_type=r["vs_type"].astype(np.int8),
                        vs_atoms=r["vs_atoms"], vs_param=r["vs_param"], bond_a=r["bond_a"],
                        bond_b=r["bond_b"], bond_r=r["bond_r"], mass=r["mass"], vel=r["vel"])
    print(INPUTS, os.path.getsize(INPUTS))


def compact_modules(r, s):
    """The 1-4 and virtual-atom outputs stored compactly: the 1-4 arrays only on the atoms of
    1-4 pairs (nb14_atoms), the refreshed coordinates only of the virtual atoms; the
    redistributed forces in full."""
    out = {}
    if "nb14_frc" in r:
        atoms = np.unique(np.concatenate([s["nb14_a"], s["nb14_b"]])).astype(np.int32)
        out["nb14_atoms"] = atoms
        for k in ("nb14_frc", "nb14_ae", "nb14_av"):
            out[k] = np.asarray(r[k], np.float32)[atoms]
    if "vs_frc" in r:
        out["vs_frc"] = np.asarray(r["vs_frc"], np.float32)
        out["vs_crd"] = np.asarray(r["vs_crd"], np.float32)[s["vs_atoms"][:, 0]]
    if "settle_crd" in r:
        atoms = settle_sample(len(s["charge"]))
        out["settle_atoms"] = atoms.astype(np.int32)
        out["settle_crd"] = np.asarray(r["settle_crd"], np.float32)[atoms]
        out["settle_vel"] = np.asarray(r["settle_vel"], np.float32)[atoms]
    return out


def write_reference(path=REFERENCE):
    sys.path.insert(0, ROOT)
    import oracle  # noqa: E402
    from oracle.ref_harness import run as refrun  # noqa: E402
    s = load_system()
    uc = oracle.crd_to_uint(oracle.periodic_map(s["crd"], s["box"]), s["box"])
    keys = oracle.pairs(uc, s, "cells")
    r = refrun.run(s, uc, keys)
    ref_pairs = r["pairs"]
    out = dict(
        frc=r["frc"],
        n_pairs=np.int64(ref_pairs.size),
        pairs_sha256=hashlib.sha256(np.sort(ref_pairs).tobytes()).hexdigest(),
        pairs_only_ref=np.setdiff1d(ref_pairs, keys),
        pairs_only_oracle=np.setdiff1d(keys, ref_pairs),
        capacities=np.array(r["capacities"], np.int64),
    )
    out.update(compact_modules(r, s))
    for k, v in r["summary"].items():
        out["summary_" + k] = np.float64(v)
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "pairs", ref_pairs.size)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "inputs"
    if what == "inputs":
        write_inputs()
    elif what == "reference":
        write_reference(sys.argv[2] if len(sys.argv) > 2 else REFERENCE)
    else:
        raise SystemExit("usage: make_covid.py inputs|reference")


def compact_file(src, dst=REFERENCE):
    """Rewrites a reference file whose 1-4 and virtual-atom arrays are stored in full."""
    z = dict(np.load(src))
    z.pop("frc_plain", None)  # within FP32 rounding of frc; not kept for this system
    s = load_system()
    r = {k: z.pop(k) for k in ("nb14_frc", "nb14_ae", "nb14_av", "vs_frc", "vs_crd") if k in z}
    z.update(compact_modules(r, s))
    np.savez_compressed(dst, **z)
