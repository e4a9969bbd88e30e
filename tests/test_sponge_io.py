"""SPONGE's text input formats: what sponge_b200.sponge_io writes, it reads back (CPU test).

Covers the coordinate/restart file (with and without the time on the first line), mass and charge
files, the LJ file, the exclusion CSR, the 1-4 file and the virtual-atom file (every type), and
read_system assembling them into the engine's system dict.
"""

import os

import numpy as np

from sponge_b200 import sponge_io, systems


def test_round_trip_system(tmp_path):
    s = systems.small_water()
    files = sponge_io.write_inputs(s, str(tmp_path), prefix="w")
    r = sponge_io.read_system(str(tmp_path), "w", cutoff=s["cutoff"], skin=s["skin"],
                              fft=s["fft"])
    assert np.allclose(r["crd"], s["crd"], atol=1e-6)
    assert np.array_equal(r["box"], np.asarray(s["box"], np.float32))
    assert np.allclose(r["charge"], s["charge"], atol=1e-6)
    assert np.allclose(r["lj_A"], s["lj_A"], rtol=1e-8)
    assert np.allclose(r["lj_B"], s["lj_B"], rtol=1e-8)
    assert np.array_equal(r["lj_type"], s["lj_type"])
    assert r["n_types"] == s["n_types"]
    for k in ("excl_start", "excl_numbers", "excl_list"):
        assert np.array_equal(r[k], s[k]), k
    m = sponge_io.read_values(files["mass"])
    assert m.size == len(s["charge"]) and np.all(m > 0)
    assert "nb14_a" not in r and "vs_type" not in r


def test_restart_coordinates(tmp_path):
    path = os.path.join(str(tmp_path), "rst.txt")
    crd = np.array([[1.5, 2.25, 3.0], [4.0, 5.5, 6.125]], np.float32)
    with open(path, "w") as f:
        f.write("2 25.505\n")
        np.savetxt(f, crd, fmt="%.7f")
        f.write("10.0 20.0 30.0 90.0 90.0 90.0\n")
    c, b = sponge_io.read_coordinate(path)
    assert np.array_equal(c, crd) and np.array_equal(b, np.array([10, 20, 30], np.float32))


def test_round_trip_nb14_and_virtual_atoms(tmp_path):
    a = np.array([0, 3, 7], np.int32)
    b = np.array([5, 9, 11], np.int32)
    ljs = np.array([0.5, 0.5, 1.0], np.float32)
    cf = np.array([0.833333, 0.833333, 1.0], np.float32)
    p14 = os.path.join(str(tmp_path), "x_nb14.txt")
    sponge_io.write_nb14(p14, a, b, ljs, cf)
    ra, rb, rl, rc = sponge_io.read_nb14(p14)
    assert np.array_equal(ra, a) and np.array_equal(rb, b)
    assert np.array_equal(rl, ljs) and np.array_equal(rc, cf)
    types = np.array([0, 1, 2, 3], np.int32)
    atoms = np.array([[20, 1, 1, 1], [21, 2, 3, 2], [22, 4, 5, 6], [23, 7, 8, 9]], np.int32)
    params = np.array([[1.5, 0], [0.25, 0], [0.1066, 0.1066], [0.6, 0.4]], np.float32)
    pv = os.path.join(str(tmp_path), "x_vatom.txt")
    sponge_io.write_vatom(pv, types, atoms, params)
    rt, ratoms, rp = sponge_io.read_vatom(pv)
    assert np.array_equal(rt, types) and np.array_equal(ratoms, atoms)
    assert np.allclose(rp, params)


def test_trajectory_and_restart_round_trip(tmp_path):
    """The binary coordinate trajectory (float32 frames appended, MD_core.cu:1347-1357), the box
    trajectory (one "Lx Ly Lz 90 90 90" line per frame, :1398-1408) and SPONGE's own restart
    pair (:1466-1486): written frames read back, restart values to the 1e-7 of %12.7f."""
    rng = np.random.default_rng(3)
    n = 17
    frames = rng.uniform(0, 30, (3, n, 3)).astype(np.float32)
    boxes = np.array([[30.0, 30.5, 31.0], [30.1, 30.6, 31.1], [29.9, 30.4, 30.9]], np.float32)
    traj = os.path.join(str(tmp_path), "mdcrd.dat")
    boxf = os.path.join(str(tmp_path), "mdbox.txt")
    for f, b in zip(frames, boxes):
        sponge_io.append_crd_traj(traj, f)
        sponge_io.append_box_traj(boxf, b)
    assert os.path.getsize(traj) == frames.nbytes
    assert np.array_equal(sponge_io.read_crd_traj(traj, n), frames)
    assert np.allclose(sponge_io.read_box_traj(boxf), boxes, atol=1e-6)
    vel = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    prefix = os.path.join(str(tmp_path), "restart")
    sponge_io.write_restart(prefix, frames[2], vel, boxes[2], time_ps=12.5)
    c, v, b, t = sponge_io.read_restart(prefix)
    assert np.allclose(c, frames[2], atol=6e-8 * 30) and np.allclose(v, vel, atol=1e-7)
    assert np.allclose(b, boxes[2], atol=1e-6) and t == 12.5
