"""Runs the reference harness (oracle/_ref/ref_harness) on a generated system (test infrastructure).

The reference kernels have no bounds checks on their fixed-capacity buffers (per-atom lists of
max_neighbor_numbers, cell buckets of max_atom_in_grid_numbers: neighbor_list.cu:297-329,
:378-386), so the capacities passed here are computed from the system first (largest half list
and fullest cell, with margin): the harness never runs with a capacity the system can overflow.
The list is refreshed on a fixed interval so the device-side launch path is not exercised.
"""

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "_ref", "ref_harness")


def available():
    return os.path.exists(BIN)


def safe_capacities(system, uc, pair_keys):
    n = uc.shape[0]
    per_atom = np.bincount((pair_keys // n).astype(np.int64), minlength=n)
    max_nb = int(per_atom.max()) if per_atom.size else 0
    cs = np.float32(system["cutoff"]) + np.float32(system["skin"])
    box = np.asarray(system["box"], np.float64)
    N = np.maximum(1, np.floor(box / (0.5 * float(cs))).astype(np.int64))
    cell = [((uc[:, d].astype(np.uint64) * np.uint64(N[d])) >> np.uint64(32)).astype(np.int64)
            for d in range(3)]
    key = (cell[2] * N[1] + cell[1]) * N[0] + cell[0]
    max_cell = int(np.bincount(key).max())
    return int(max_nb * 1.25) + 64, int(max_cell * 1.5) + 16


def write_input(path, system, max_nb, max_grid, refresh_interval=20):
    n = len(system["charge"])
    T = int(system["n_types"])
    fft = system.get("fft") or (-1, -1, -1)
    el = np.asarray(system["excl_list"], np.int32)
    with open(path, "wb") as f:
        np.array([n, T, el.size, fft[0], fft[1], fft[2], refresh_interval, max_nb, max_grid],
                 np.int32).tofile(f)
        np.array([*system["box"], system["cutoff"], system["skin"], system["tolerance"]],
                 np.float32).tofile(f)
        np.asarray(system["crd"], np.float32).tofile(f)
        np.asarray(system["charge"], np.float32).tofile(f)
        np.asarray(system["lj_type"], np.int32).tofile(f)
        np.asarray(system["lj_A"], np.float32).tofile(f)
        np.asarray(system["lj_B"], np.float32).tofile(f)
        np.asarray(system["excl_start"], np.int32).tofile(f)
        np.asarray(system["excl_numbers"], np.int32).tofile(f)
        el.tofile(f)
        # optional 1-4 pairs and virtual atoms
        a14 = np.asarray(system.get("nb14_a", np.zeros(0)), np.int32)
        np.array([a14.size], np.int32).tofile(f)
        if a14.size:
            a14.tofile(f)
            np.asarray(system["nb14_b"], np.int32).tofile(f)
            np.asarray(system["nb14_lj_scale"], np.float32).tofile(f)
            np.asarray(system["nb14_cf"], np.float32).tofile(f)
        vt = np.asarray(system.get("vs_type", np.zeros(0)), np.int32)
        np.array([vt.size], np.int32).tofile(f)
        if vt.size:
            vt.tofile(f)
            np.asarray(system["vs_atoms"], np.int32).reshape(-1).tofile(f)
            np.asarray(system["vs_param"], np.float32).reshape(-1).tofile(f)
        # optional bonds, masses, velocities and time step for one CONSTRAIN + SETTLE step
        ba = np.asarray(system.get("bond_a", np.zeros(0)), np.int32)
        np.array([ba.size], np.int32).tofile(f)
        if ba.size:
            ba.tofile(f)
            np.asarray(system["bond_b"], np.int32).tofile(f)
            np.asarray(system["bond_r"], np.float32).tofile(f)
            np.asarray(system["mass"], np.float32).tofile(f)
            np.asarray(system["vel"], np.float32).reshape(-1).tofile(f)
            np.array([system["md_dt"]], np.float32).tofile(f)


def run(system, uc, pair_keys, timing_steps=0, outdir=None, timeout=900):
    """Runs the harness; returns dict(frc, frc_plain, pairs, summary)."""
    max_nb, max_grid = safe_capacities(system, uc, pair_keys)
    outdir = outdir or tempfile.mkdtemp(prefix="refh_")
    os.makedirs(outdir, exist_ok=True)
    inp = os.path.join(outdir, "in.bin")
    write_input(inp, system, max_nb, max_grid)
    r = subprocess.run([BIN, inp, outdir, str(int(timing_steps))], stdin=subprocess.DEVNULL,
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference harness failed (%d): %s" % (r.returncode, r.stderr[-2000:]))
    n = len(system["charge"])
    summ = {}
    for line in open(os.path.join(outdir, "summary.txt")):
        k, v = line.split()
        summ[k] = float(v)
    out = dict(
        frc=np.fromfile(os.path.join(outdir, "frc.f32"), np.float32).reshape(n, 3),
        frc_plain=np.fromfile(os.path.join(outdir, "frc_plain.f32"), np.float32).reshape(n, 3),
        pairs=np.fromfile(os.path.join(outdir, "pairs.i64"), np.int64),
        summary=summ, capacities=(max_nb, max_grid), outdir=outdir)
    for name, shape in (("nb14_frc", (n, 3)), ("nb14_ae", (n,)), ("nb14_av", (n,)),
                        ("vs_frc", (n, 3)), ("vs_crd", (n, 3)), ("settle_crd", (n, 3)),
                        ("settle_vel", (n, 3))):
        path = os.path.join(outdir, name + ".f32")
        if os.path.exists(path):
            out[name] = np.fromfile(path, np.float32).reshape(shape)
    return out


SC_BIN = os.path.join(os.path.dirname(HERE), "_ref", "sc_harness")


def sc_available():
    return os.path.exists(SC_BIN)


def write_sc_input(path, system, max_nb, max_grid):
    """Input of sc_harness for an FEP box of sponge_b200.systems.fep_box (charges at lambda)."""
    n = len(system["charge"])
    TA, TB = int(system["n_types"]), int(system["n_types_B"])
    fft = system["fft"]
    el = np.asarray(system["excl_list"], np.int32)
    with open(path, "wb") as f:
        np.array([n, TA, TB, el.size, fft[0], fft[1], fft[2], max_nb, max_grid],
                 np.int32).tofile(f)
        np.array([*system["box"], system["cutoff"], system["skin"], system["tolerance"],
                  system["lam"], system["sc_alpha"], system["sc_p"], system["sc_sigma"],
                  system["sc_sigma_min"]], np.float32).tofile(f)
        np.asarray(system["crd"], np.float32).tofile(f)
        np.asarray(system["charge"], np.float32).tofile(f)
        np.asarray(system["dq"], np.float32).tofile(f)
        np.asarray(system["lj_type"], np.int32).tofile(f)
        np.asarray(system["lj_type_B"], np.int32).tofile(f)
        np.asarray(system["mask"], np.int32).tofile(f)
        np.asarray(system["lj_A"], np.float32).tofile(f)
        np.asarray(system["lj_B"], np.float32).tofile(f)
        np.asarray(system["lj_A_B"], np.float32).tofile(f)
        np.asarray(system["lj_B_B"], np.float32).tofile(f)
        np.asarray(system["excl_start"], np.int32).tofile(f)
        np.asarray(system["excl_numbers"], np.int32).tofile(f)
        el.tofile(f)


def run_softcore(system, uc, pair_keys, outdir=None, timeout=600):
    """Runs sc_harness on an FEP box; returns dict(frc, ae, av, adir, pairs, summary). The list
    capacities are computed from the system as in run()."""
    max_nb, max_grid = safe_capacities(system, uc, pair_keys)
    outdir = outdir or tempfile.mkdtemp(prefix="refsc_")
    os.makedirs(outdir, exist_ok=True)
    inp = os.path.join(outdir, "in.bin")
    write_sc_input(inp, system, max_nb, max_grid)
    r = subprocess.run([SC_BIN, inp, outdir], stdin=subprocess.DEVNULL, capture_output=True,
                       text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("soft-core harness failed (%d): %s" % (r.returncode, r.stderr[-2000:]))
    n = len(system["charge"])
    summ = {}
    for line in open(os.path.join(outdir, "summary.txt")):
        k, v = line.split()
        summ[k] = float(v)
    rdf = lambda name, shape: np.fromfile(os.path.join(outdir, name), np.float32).reshape(shape)  # noqa: E731
    return dict(frc=rdf("sc_frc.f32", (n, 3)), ae=rdf("sc_ae.f32", (n,)),
                av=rdf("sc_av.f32", (n,)), adir=rdf("sc_adir.f32", (n,)),
                pairs=np.fromfile(os.path.join(outdir, "pairs.i64"), np.int64), summary=summ,
                capacities=(max_nb, max_grid))
