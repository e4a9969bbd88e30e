"""Writers for SPONGE's text input formats, so that a generated system can be run by an unchanged
SPONGE driver (with the stock modules or with the sponge_b200 drop-ins).

Formats (SPONGE/MD_core/MD_core.cu:1213-1257 coordinates, :1051-1080 charge, :308-351 exclude;
SPONGE/Lennard_Jones_force/Lennard_Jones_force.cu:1082-1105 LJ; bond and residue files as in
SPONGE/covid-tip4p/):
    coordinate  "N\\n" + N lines "x y z" + "Lx Ly Lz 90 90 90"
    mass/charge "N\\n" + N values (charges already x18.2223)
    LJ          "N T\\n" + A[T(T+1)/2] + B[...] + type[N]
    exclude     "N total\\n" + per atom "count j1 j2 ..."
    bond        "nbonds\\n" + "i j k r0"
    residue     "N nres\\n" + residue sizes
Rigid water is constrained by SETTLE, which finds the O-H-H triangles from the three bonds of
each water (O-H1, O-H2, H1-H2).
"""

import os

import numpy as np

MASS_O = 15.9994
MASS_H = 1.008
MASS_SOLUTE = 12.011
R_HH = 2 * 0.9572 * np.sin(np.deg2rad(104.52) / 2)


def _waters(system):
    """Index of the first water atom and the number of waters (waters are stored O,H,H last)."""
    t = np.asarray(system["lj_type"])
    n = len(t)
    # solute atoms have types >= 2 and come first
    first = int(np.argmax((t == 0) | (t == 1))) if np.any(t < 2) else n
    return first, (n - first) // 3


def write_inputs(system, outdir, prefix="sys"):
    os.makedirs(outdir, exist_ok=True)
    n = len(system["charge"])
    box = np.asarray(system["box"], np.float64)
    p = lambda name: os.path.join(outdir, "%s_%s.txt" % (prefix, name))  # noqa: E731
    crd = np.asarray(system["crd"], np.float64)
    with open(p("coordinate"), "w") as f:
        f.write("%d 0.0\n" % n)
        np.savetxt(f, crd, fmt="%.7f")
        f.write("%.7f %.7f %.7f 90.0 90.0 90.0\n" % tuple(box))
    first, nw = _waters(system)
    mass = np.full(n, MASS_SOLUTE)
    for w in range(nw):
        o = first + 3 * w
        mass[o], mass[o + 1], mass[o + 2] = MASS_O, MASS_H, MASS_H
    with open(p("mass"), "w") as f:
        f.write("%d\n" % n)
        np.savetxt(f, mass, fmt="%.6f")
    with open(p("charge"), "w") as f:
        f.write("%d\n" % n)
        np.savetxt(f, np.asarray(system["charge"], np.float64), fmt="%.7f")
    T = int(system["n_types"])
    with open(p("LJ"), "w") as f:
        f.write("%d %d\n" % (n, T))
        np.savetxt(f, np.asarray(system["lj_A"], np.float64), fmt="%.9e")
        np.savetxt(f, np.asarray(system["lj_B"], np.float64), fmt="%.9e")
        np.savetxt(f, np.asarray(system["lj_type"]), fmt="%d")
    es, en, el = system["excl_start"], system["excl_numbers"], system["excl_list"]
    with open(p("exclude"), "w") as f:
        f.write("%d %d\n" % (n, len(el)))
        for i in range(n):
            f.write(" ".join([str(en[i])] + [str(x) for x in el[es[i]:es[i] + en[i]]]) + "\n")
    with open(p("bond"), "w") as f:
        f.write("%d\n" % (3 * nw))
        for w in range(nw):
            o = first + 3 * w
            f.write("%d %d 553.0 0.9572\n%d %d 553.0 0.9572\n%d %d 553.0 %.6f\n"
                    % (o, o + 1, o, o + 2, o + 1, o + 2, R_HH))
    with open(p("residue"), "w") as f:
        f.write("%d %d\n" % (n, first + nw))
        f.write("1\n" * first)
        f.write("3\n" * nw)
    return {k: p(k) for k in ("coordinate", "mass", "charge", "LJ", "exclude", "bond", "residue")}


def write_mdin(path, files, system, steps=10000, dt=0.002, refresh_interval=20,
               max_neighbor_numbers=1200, max_atom_in_grid_numbers=128, extra=None):
    fft = system.get("fft")
    lines = [
        "%s nonbonded benchmark" % system.get("name", "system"),
        "mode = NVT",
        "dt = %g" % dt,
        "step_limit = %d" % steps,
        "write_information_interval = 1000",
        "write_restart_file_interval = %d" % (steps * 10),
        "cutoff = %g" % system["cutoff"],
        "skin = %g" % system["skin"],
        "neighbor_list_refresh_interval = %d" % refresh_interval,
        "neighbor_list_max_neighbor_numbers = %d" % max_neighbor_numbers,
        "neighbor_list_max_atom_in_grid_numbers = %d" % max_atom_in_grid_numbers,
        "thermostat = middle_langevin",
        "middle_langevin_gamma = 1",
        "middle_langevin_seed = 1",
        "target_temperature = 300.0",
        "constrain_mode = SETTLE",
        "dont_check_input = 1",
        "end_pause = 0",
    ]
    if fft:
        lines += ["PME_fftx = %d" % fft[0], "PME_ffty = %d" % fft[1], "PME_fftz = %d" % fft[2]]
    for k, key in (("coordinate", "coordinate_in_file"), ("mass", "mass_in_file"),
                   ("charge", "charge_in_file"), ("LJ", "LJ_in_file"),
                   ("exclude", "exclude_in_file"), ("bond", "bond_in_file"),
                   ("residue", "residue_in_file")):
        lines.append("%s = %s" % (key, files[k]))
    for k, v in (extra or {}).items():
        lines.append("%s = %s" % (k, v))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
