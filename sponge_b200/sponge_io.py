"""Readers and writers for SPONGE's text input formats: a generated system can be run by an
unchanged SPONGE driver (with the stock modules or with the sponge_b200 drop-ins), and a SPONGE
system (such as the reference's covid-tip4p) can be read into the system dict the engine takes.

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


def bonds_and_masses(system):
    """The rigid-water bonds (O-H1, O-H2, H1-H2 per water, as the bond file lists them) and the
    per-atom masses of a generated system. Returns (bond_a, bond_b, bond_r0, mass)."""
    n = len(system["charge"])
    first, nw = _waters(system)
    mass = np.full(n, MASS_SOLUTE, np.float32)
    o = first + 3 * np.arange(nw, dtype=np.int32)
    mass[o], mass[o + 1], mass[o + 2] = MASS_O, MASS_H, MASS_H
    a = np.stack([o, o, o + 1], 1).reshape(-1).astype(np.int32)
    b = np.stack([o + 1, o + 2, o + 2], 1).reshape(-1).astype(np.int32)
    r = np.tile(np.array([0.9572, 0.9572, R_HH], np.float32), nw)
    return a, b, r, mass


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


# ---------------------------------------------------------------------------------------------
# readers
# ---------------------------------------------------------------------------------------------
def _parm7_section(f, name, fmt, values, per_line, width, conv):
    f.write("%%FLAG %s\n%%FORMAT(%s)\n" % (name, fmt))
    values = list(values)
    for k in range(0, len(values), per_line):
        f.write("".join(conv(v).rjust(width) for v in values[k:k + per_line]) + "\n")
    if not values:
        f.write("\n")


def write_amber_parm7(path, system):
    """The LJ part of an AMBER parm7 topology for ``system``: POINTERS (NATOM, NTYPES, the other
    counts 0), ATOM_TYPE_INDEX (1-based), NONBONDED_PARM_INDEX and LENNARD_JONES_ACOEF / _BCOEF
    (unscaled A = 4 eps sigma^12, B = 4 eps sigma^6, lower-triangular type-pair order). SPONGE's
    LJ module reads exactly these when an mdin names ``amber_parm7`` and no ``LJ_in_file``
    (Lennard_Jones_force.cu:1201-1276); the other modules read their own ``*_in_file`` first, and
    with the counts 0 the angle, dihedral, 1-4 and CMAP readers initialise nothing."""
    n = len(system["charge"])
    T = int(system["n_types"])
    A = np.asarray(system["lj_A"], np.float32)
    B = np.asarray(system["lj_B"], np.float32)
    ico = np.zeros(T * T, np.int64)
    for i in range(T):
        for j in range(T):
            hi, lo = max(i, j), min(i, j)
            ico[i * T + j] = hi * (hi + 1) // 2 + lo + 1
    pointers = [n, T] + [0] * 29
    e16 = lambda v: "%.8E" % float(v)  # noqa: E731  (9 significant digits: exact for float32)
    with open(path, "w") as f:
        f.write("%VERSION  VERSION_STAMP = V0001.000\n")
        _parm7_section(f, "TITLE", "20a4", [], 20, 4, str)
        _parm7_section(f, "POINTERS", "10I8", pointers, 10, 8, str)
        _parm7_section(f, "ATOM_TYPE_INDEX", "10I8",
                       (np.asarray(system["lj_type"], np.int64) + 1).tolist(), 10, 8, str)
        _parm7_section(f, "NONBONDED_PARM_INDEX", "10I8", ico.tolist(), 10, 8, str)
        _parm7_section(f, "LENNARD_JONES_ACOEF", "5E16.8", A.tolist(), 5, 16, e16)
        _parm7_section(f, "LENNARD_JONES_BCOEF", "5E16.8", B.tolist(), 5, 16, e16)
    return path


def read_coordinate(path):
    """Coordinate or restart file (MD_core.cu:1213-1257): first line "N" or "N time", N lines of
    "x y z", then "Lx Ly Lz alpha beta gamma". Returns (crd [N,3] float32, box [3] float32)."""
    with open(path) as f:
        lines = f.read().split("\n")
    n = int(lines[0].split()[0])
    crd = np.array(" ".join(lines[1:1 + n]).split(), np.float64).reshape(n, 3)
    box = np.array(lines[1 + n].split()[:3], np.float64)
    return crd.astype(np.float32), box.astype(np.float32)


def read_velocity(path):
    """Velocity restart file: "N [time]", then N lines of "vx vy vz" (A per internal time
    unit). Returns vel [N,3] float32."""
    with open(path) as f:
        lines = f.read().split("\n")
    n = int(lines[0].split()[0])
    return np.array(" ".join(lines[1:1 + n]).split(), np.float32).reshape(n, 3)


def write_velocity(path, vel):
    """Velocity file as velocity_in_file reads it (MD_core.cu:867-892): "N", then N lines
    "vx vy vz" in A per internal time unit."""
    vel = np.asarray(vel, np.float64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("%d\n" % vel.shape[0])
        np.savetxt(f, vel, fmt="%.7f")
    return path


def maxwell_boltzmann(mass, temperature, seed):
    """Velocities (A per internal time unit) drawn at ``temperature`` K for ``mass`` (amu),
    centre-of-mass momentum removed: sqrt(kB T / m) per component, kB in kcal/mol/K."""
    m = np.asarray(mass, np.float64)
    inv = np.divide(1.0, m, out=np.zeros_like(m), where=m != 0)
    rng = np.random.default_rng(seed)
    vel = rng.normal(size=(m.size, 3)) * np.sqrt(0.0019872041 * temperature * inv)[:, None]
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    return vel


def append_crd_traj(path, crd):
    """One frame of the binary coordinate trajectory (`crd`, mdcrd.dat), as
    Append_Crd_Traj_File writes it (MD_core.cu:1347-1357): N x 3 float32, no header, frames
    appended one after another. Also the layout of the velocity and force trajectories."""
    with open(path, "ab") as f:
        np.ascontiguousarray(crd, np.float32).reshape(-1, 3).tofile(f)


def read_crd_traj(path, atom_numbers):
    """All frames of a binary coordinate (or velocity, force) trajectory: [F, N, 3] float32."""
    a = np.fromfile(path, np.float32)
    per = 3 * int(atom_numbers)
    if a.size % per:
        raise ValueError("%s: %d floats is not a whole number of %d-atom frames"
                         % (path, a.size, atom_numbers))
    return a.reshape(-1, int(atom_numbers), 3)


def append_box_traj(path, box):
    """One line of the box trajectory (`box`, mdbox.txt) as Append_Box_Traj_File writes it
    (MD_core.cu:1398-1408): "Lx Ly Lz 90 90 90" with %f lengths."""
    b = np.asarray(box, np.float32).reshape(3)
    with open(path, "a") as f:
        f.write("%f %f %f %.0f %.0f %.0f\n" % (b[0], b[1], b[2], 90.0, 90.0, 90.0))


def read_box_traj(path):
    """The box lengths of every frame of a box trajectory: [F, 3] float32."""
    rows = [l.split() for l in open(path) if l.strip()]
    return np.array([[float(x) for x in r[:3]] for r in rows], np.float32).reshape(-1, 3)


def write_restart(prefix, crd, vel, box, time_ps=0.0):
    """SPONGE's own restart pair as Export_Restart_File writes it without an AMBER restart
    (MD_core.cu:1466-1486): "<prefix>_coordinate.txt" ("N time", N lines "%12.7f %12.7f
    %12.7f", the box line) and "<prefix>_velocity.txt" ("N time", N velocity lines)."""
    crd = np.asarray(crd, np.float32).reshape(-1, 3)
    vel = np.asarray(vel, np.float32).reshape(-1, 3)
    b = np.asarray(box, np.float32).reshape(3)
    n = crd.shape[0]
    with open(prefix + "_coordinate.txt", "w") as f:
        f.write("%d %.3f\n" % (n, time_ps))
        for x in crd:
            f.write("%12.7f %12.7f %12.7f\n" % tuple(x))
        f.write("%12.7f %12.7f %12.7f %12.7f %12.7f %12.7f" % (b[0], b[1], b[2], 90.0, 90.0, 90.0))
    with open(prefix + "_velocity.txt", "w") as f:
        f.write("%d %.3f\n" % (n, time_ps))
        for v in vel:
            f.write("%12.7f %12.7f %12.7f\n" % tuple(v))
    return prefix + "_coordinate.txt", prefix + "_velocity.txt"


def read_restart(prefix):
    """The restart pair of `write_restart` (or of a SPONGE run with `rst = <prefix>`):
    (crd [N,3], vel [N,3], box [3], time in ps)."""
    crd, box = read_coordinate(prefix + "_coordinate.txt")
    vel = read_velocity(prefix + "_velocity.txt")
    with open(prefix + "_coordinate.txt") as f:
        head = f.readline().split()
    return crd, vel, box, float(head[1]) if len(head) > 1 else 0.0


def write_fep_inputs(system, outdir, frames, prefix="fep"):
    """Inputs of SPONGE's FEP and TI drivers (main_fep.cu, main_ti.cu) for an FEP box of
    ``sponge_b200.systems.fep_box`` and a list of coordinate frames (same box each):

    * charge_in_file (the charges at the box's lambda), chargeA_in_file, chargeB_in_file
      (TI_core.cu:421-470), subsys_division_in_file (the perturbed-atom mask,
      LJ_soft_core.cu:1549-1575), exclude_in_file;
    * LJ_soft_core_in_file: "N TA TB", the A state's A and B tables, the B state's, then
      "typeA typeB" per atom (LJ_soft_core.cu:1491-1547), unscaled;
    * the binary coordinate trajectory and the box trajectory that the drivers read frame by
      frame (``crd`` and ``box``).
    Returns a dict of paths."""
    os.makedirs(outdir, exist_ok=True)
    n = len(system["charge"])
    p = lambda name: os.path.join(outdir, "%s_%s" % (prefix, name))  # noqa: E731

    def values(path, v, fmt):
        with open(path, "w") as f:
            f.write("%d\n" % n)
            np.savetxt(f, np.asarray(v).reshape(-1), fmt=fmt)
        return path

    out = {
        "charge": values(p("charge.txt"), np.asarray(system["charge"], np.float64), "%.9g"),
        "chargeA": values(p("chargeA.txt"), np.asarray(system["charge_A"], np.float64), "%.9g"),
        "chargeB": values(p("chargeB.txt"), np.asarray(system["charge_B"], np.float64), "%.9g"),
        "subsys": values(p("subsys.txt"), np.asarray(system["mask"], np.int64), "%d"),
    }
    es, en, el = system["excl_start"], system["excl_numbers"], system["excl_list"]
    out["exclude"] = p("exclude.txt")
    with open(out["exclude"], "w") as f:
        f.write("%d %d\n" % (n, len(el)))
        for i in range(n):
            f.write(" ".join([str(en[i])] + [str(x) for x in el[es[i]:es[i] + en[i]]]) + "\n")
    out["lj_soft"] = p("LJ_soft_core.txt")
    with open(out["lj_soft"], "w") as f:
        f.write("%d %d %d\n" % (n, int(system["n_types"]), int(system["n_types_B"])))
        for key in ("lj_A", "lj_B", "lj_A_B", "lj_B_B"):
            np.savetxt(f, np.asarray(system[key], np.float64), fmt="%.9e")
        np.savetxt(f, np.stack([system["lj_type"], system["lj_type_B"]], 1), fmt="%d")
    out["crd"], out["box"] = p("crd.dat"), p("box.txt")
    for path in (out["crd"], out["box"]):
        if os.path.exists(path):
            os.remove(path)
    for fr in frames:
        append_crd_traj(out["crd"], fr)
        append_box_traj(out["box"], system["box"])
    return out


def read_bond(path):
    """Bond file: "count", then "a b k r0" per bond. Returns (a, b, k, r0)."""
    tok = open(path).read().split()
    n = int(tok[0])
    rows = np.array(tok[1:1 + 4 * n], np.float64).reshape(n, 4)
    return (rows[:, 0].astype(np.int32), rows[:, 1].astype(np.int32),
            rows[:, 2].astype(np.float32), rows[:, 3].astype(np.float32))


def read_values(path):
    """Per-atom value file (mass, charge; MD_core.cu:1051-1080): "N", then N numbers."""
    tok = open(path).read().split()
    n = int(tok[0])
    return np.array(tok[1:1 + n], np.float32)


def read_lj(path):
    """LJ file (Lennard_Jones_force.cu:1082-1105): "N T", A and B over the T(T+1)/2 type pairs,
    then the N types. Returns (A, B, types, T)."""
    tok = open(path).read().split()
    n, t = int(tok[0]), int(tok[1])
    npair = t * (t + 1) // 2
    A = np.array(tok[2:2 + npair], np.float32)
    B = np.array(tok[2 + npair:2 + 2 * npair], np.float32)
    types = np.array(tok[2 + 2 * npair:2 + 2 * npair + n], np.int32)
    return A, B, types, t


def read_exclude(path):
    """Exclusion file (MD_core.cu:308-351): "N total", then per atom "count j1 j2 ...".
    Returns the CSR (start, numbers, list)."""
    tok = open(path).read().split()
    n, total = int(tok[0]), int(tok[1])
    numbers = np.zeros(n, np.int32)
    lists = []
    p = 2
    for i in range(n):
        c = int(tok[p])
        numbers[i] = c
        lists.append(np.array(tok[p + 1:p + 1 + c], np.int32))
        p += 1 + c
    lst = np.concatenate(lists) if lists else np.zeros(0, np.int32)
    if lst.size != total:
        raise ValueError("%s: %d exclusions listed, header says %d" % (path, lst.size, total))
    start = np.zeros(n, np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    return start, numbers, lst.astype(np.int32)


def read_nb14(path):
    """1-4 file (nb14.cu:179-206): "count", then "a b lj_scale cf_scale" per pair.
    Returns (a, b, lj_scale, cf_scale)."""
    tok = open(path).read().split()
    n = int(tok[0])
    rows = np.array(tok[1:1 + 4 * n], np.float64).reshape(n, 4)
    return (rows[:, 0].astype(np.int32), rows[:, 1].astype(np.int32),
            rows[:, 2].astype(np.float32), rows[:, 3].astype(np.float32))


def read_vatom(path):
    """Virtual-atom file (virtual_atoms.cu:246-290): one "type v from_1 [from_2 from_3] params"
    line per virtual atom. Returns (types [V], atoms [V,4], params [V,2]) as
    sponge_b200.VirtualAtoms takes them (unused parents repeat from_1, unused params are 0)."""
    npar = {0: 1, 1: 2, 2: 3, 3: 3}
    nparam = {0: 1, 1: 1, 2: 2, 3: 2}
    types, atoms, params = [], [], []
    with open(path) as f:
        for line in f:
            w = line.split()
            if len(w) < 2:
                continue
            t = int(w[0])
            k = npar[t]
            idx = [int(x) for x in w[1:2 + k]]
            par = [float(x) for x in w[2 + k:2 + k + nparam[t]]]
            types.append(t)
            atoms.append(idx + [idx[1]] * (4 - len(idx)))
            params.append(par + [0.0] * (2 - len(par)))
    return (np.array(types, np.int32), np.array(atoms, np.int32).reshape(-1, 4),
            np.array(params, np.float32).reshape(-1, 2))


def write_nb14(path, a, b, lj_scale, cf_scale):
    with open(path, "w") as f:
        f.write("%d\n" % len(a))
        for row in zip(a, b, lj_scale, cf_scale):
            f.write("%d %d %.9g %.9g\n" % row)


def write_vatom(path, types, atoms, params):
    npar = {0: 1, 1: 2, 2: 3, 3: 3}
    nparam = {0: 1, 1: 1, 2: 2, 3: 2}
    with open(path, "w") as f:
        for t, a, p in zip(types, np.asarray(atoms).reshape(-1, 4), np.asarray(params).reshape(-1, 2)):
            t = int(t)
            f.write(" ".join([str(t)] + [str(int(x)) for x in a[:1 + npar[t]]] +
                             ["%.9g" % x for x in p[:nparam[t]]]) + "\n")


def read_system(directory, prefix, coordinate=None, cutoff=10.0, skin=2.0, tolerance=1e-5,
                fft=None):
    """A SPONGE input set (prefix_coordinate/charge/LJ/exclude[/nb14/vatom].txt) as the system
    dict sponge_b200.systems builds; ``coordinate`` overrides the coordinate file (a restart).
    Files that are absent are left out (no 1-4 pairs or virtual atoms)."""
    p = lambda name: os.path.join(directory, "%s_%s.txt" % (prefix, name))  # noqa: E731
    crd, box = read_coordinate(coordinate or p("coordinate"))
    charge = read_values(p("charge"))
    lj = p("LJ") if os.path.exists(p("LJ")) else p("lj")
    A, B, types, t = read_lj(lj)
    start, numbers, lst = read_exclude(p("exclude"))
    box64 = box.astype(np.float64)
    crd = np.mod(crd.astype(np.float64), box64)
    crd = np.where(crd >= box64, 0.0, crd).astype(np.float32)
    s = dict(name=prefix, crd=crd, charge=charge, lj_type=types, n_types=t, lj_A=A, lj_B=B,
             excl_start=start, excl_numbers=numbers, excl_list=lst, box=box,
             cutoff=float(cutoff), skin=float(skin), fft=fft, tolerance=float(tolerance))
    if os.path.exists(p("nb14")):
        s["nb14_a"], s["nb14_b"], s["nb14_lj_scale"], s["nb14_cf"] = read_nb14(p("nb14"))
    if os.path.exists(p("vatom")):
        s["vs_type"], s["vs_atoms"], s["vs_param"] = read_vatom(p("vatom"))
    return s
