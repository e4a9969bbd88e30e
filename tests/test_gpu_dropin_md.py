"""The drop-in modules inside the reference's own MD driver.

oracle/ref_harness/build_sponge.sh builds SPONGE's unchanged main.cu and modules twice into
oracle/_ref/: `sponge_stock` (the reference as shipped) and `sponge_b200` (NEIGHBOR_LIST,
LENNARD_JONES_INFORMATION and Particle_Mesh_Ewald replaced by sponge_b200/dropin, linked to
libsponge_b200.so). Both run the same generated water box (3,000 atoms, rc 8 A, PME 32^3, harmonic
bonds, NVE, 1 fs) from the same input files for 40 steps, and the energies they print every
10 steps (potential, LJ, PME, bond, temperature) agree within 2e-4 of their size: the printed PME
energy of the stock build sits about 1.5e-4 from the FP64 value (its B-spline moduli and energy
sums are FP32; the reference's own energies meet the FP64 oracle only to 1e-4 in
tests/test_golden.py), while the drop-in's match FP64 to 1e-5. The drop-in with the pruned pair
list (neighbor_list_prune_buffer 0.5, prune_interval 5) prints the same energies as without it,
and so do both builds with the LJ parameters read from an AMBER parm7 topology (amber_parm7)
instead of LJ_in_file.
Skipped where the two binaries have not been built.
"""

import os
import subprocess

import numpy as np
import pytest

from sponge_b200 import sponge_io, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STOCK = os.path.join(ROOT, "oracle", "_ref", "sponge_stock")
B200 = os.path.join(ROOT, "oracle", "_ref", "sponge_b200")


def _mdin(paths, outdir, extra=""):
    text = """water box, drop-in parity run
mode = NVE
dt = 1e-3
step_limit = 40
write_information_interval = 10
cutoff = 8.0
skin = 2.0
neighbor_list_refresh_interval = 10
neighbor_list_max_neighbor_numbers = 1200
PME_fftx = 32
PME_ffty = 32
PME_fftz = 32
coordinate_in_file = {coordinate}
mass_in_file = {mass}
charge_in_file = {charge}
LJ_in_file = {LJ}
exclude_in_file = {exclude}
bond_in_file = {bond}
residue_in_file = {residue}
mdout = {out}/mdout.txt
mdinfo = {out}/mdinfo.txt
box = {out}/mdbox.txt
crd = {out}/mdcrd.dat
rst = {out}/restart
end_pause = 0
dont_check_input = 1
device = 0
{extra}
""".format(out=outdir, extra=extra, **paths)
    if paths.get("LJ") is None:  # LJ from amber_parm7 (in `extra`) instead of LJ_in_file
        text = "\n".join(l for l in text.split("\n") if not l.startswith("LJ_in_file"))
    if "mode =" in extra:  # another mode replaces the NVE default
        text = "\n".join(l for l in text.split("\n") if l != "mode = NVE")
    if "step_limit =" in extra:
        text = "\n".join(l for l in text.split("\n") if l != "step_limit = 40")
    return text


# NPT with the Berendsen barostat every 2 steps (deterministic, so the two builds see the same
# box moves up to the rounding of their pressures): every move calls Main_Volume_Change
# (main.cu:438-448), that is NEIGHBOR_LIST::Update_Volume, LENNARD_JONES_INFORMATION::Update_Volume
# and Particle_Mesh_Ewald::Update_Volume on the drop-ins, and the pressure reads their virial.
NPT = """mode = NPT
thermostat = berendsen_thermostat
berendsen_thermostat_tau = 0.1
target_temperature = 300
barostat = berendsen_barostat
target_pressure = 1.0
berendsen_barostat_tau = 1.0
berendsen_barostat_compressibility = 4.5e-5
berendsen_barostat_update_interval = 2"""


def _run(binary, paths, outdir, extra=""):
    os.makedirs(outdir, exist_ok=True)
    mdin = os.path.join(outdir, "mdin.txt")
    with open(mdin, "w") as f:
        f.write(_mdin(paths, outdir, extra))
    r = subprocess.run([binary, "-mdin", mdin], cwd=outdir, stdin=subprocess.DEVNULL,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = [l.split() for l in open(os.path.join(outdir, "mdout.txt")) if l.strip()]
    head = lines[0]
    rows = np.array([[float(x) for x in l] for l in lines[1:]], np.float64)
    return {k: rows[:, i] for i, k in enumerate(head)}


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    if not (os.path.exists(STOCK) and os.path.exists(B200)):
        pytest.skip("oracle/_ref/sponge_stock and sponge_b200 not built "
                    "(oracle/ref_harness/build_sponge.sh both)")
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    base = tmp_path_factory.mktemp("dropin_md")
    paths = sponge_io.write_inputs(systems.config0(), str(base / "inputs"), prefix="water")
    parm7 = sponge_io.write_amber_parm7(str(base / "inputs" / "water.parm7"), systems.config0())
    # the thermostat of the NPT run needs a temperature: velocities at 300 K (seeded)
    mass = sponge_io.bonds_and_masses(systems.config0())[3]
    vel = sponge_io.write_velocity(str(base / "inputs" / "water_velocity.txt"),
                                   sponge_io.maxwell_boltzmann(mass, 300.0, 2024))
    npt = NPT + "\nvelocity_in_file = " + vel
    no_lj = dict(paths, LJ=None)
    out = {
        "stock": _run(STOCK, paths, str(base / "stock")),
        "b200": _run(B200, paths, str(base / "b200")),
        "b200_pruned": _run(B200, paths, str(base / "b200_pruned"),
                            "neighbor_list_prune_buffer = 0.5\nneighbor_list_prune_interval = 5"),
        "stock_parm7": _run(STOCK, no_lj, str(base / "stock_parm7"), "amber_parm7 = " + parm7),
        "b200_parm7": _run(B200, no_lj, str(base / "b200_parm7"), "amber_parm7 = " + parm7),
        "stock_npt": _run(STOCK, paths, str(base / "stock_npt"), npt),
        "b200_npt": _run(B200, paths, str(base / "b200_npt"), npt),
    }
    # restart: 20 steps, then 20 more from the restart files the first run wrote
    _run(B200, paths, str(base / "b200_first20"), "step_limit = 20")
    rst = str(base / "b200_first20" / "restart")
    again = dict(paths, coordinate=rst + "_coordinate.txt")
    out["b200_restarted"] = _run(B200, again, str(base / "b200_restarted"),
                                 "step_limit = 20\nvelocity_in_file = %s_velocity.txt" % rst)
    out["dirs"] = {k: str(base / k) for k in ("stock", "b200", "b200_first20",
                                               "b200_restarted")}
    return out


def test_drop_in_matches_stock_driver(runs):
    a, b = runs["stock"], runs["b200"]
    assert len(a["step"]) >= 4 and list(a["step"]) == list(b["step"])
    for key in ("potential", "LJ", "PME", "bond"):
        scale = np.abs(a[key]).max()
        err = np.abs(a[key] - b[key]).max()
        print("%-10s stock %s b200 %s" % (key, a[key], b[key]))
        assert err <= 2e-4 * scale + 0.05, key
    assert np.allclose(a["temperature"], b["temperature"], rtol=1e-3, atol=0.05)


def test_pruned_list_in_driver(runs):
    b, p = runs["b200"], runs["b200_pruned"]
    for key in ("potential", "LJ", "PME", "bond", "temperature"):
        assert np.allclose(b[key], p[key], rtol=1e-5, atol=0.02), key


def test_lj_from_amber_parm7(runs):
    """LENNARD_JONES_INFORMATION::Initial_From_AMBER_Parm: with the LJ tables and types read from
    an AMBER parm7 topology instead of LJ_in_file, the drop-in prints the energies of its
    LJ_in_file run, and the stock build does the same with its own reader."""
    for a, b in ((runs["b200"], runs["b200_parm7"]), (runs["stock"], runs["stock_parm7"])):
        assert list(a["step"]) == list(b["step"])
        for key in ("potential", "LJ", "PME", "bond", "temperature"):
            assert np.allclose(a[key], b[key], rtol=1e-5, atol=0.02), key
    a, b = runs["stock_parm7"], runs["b200_parm7"]
    for key in ("potential", "LJ", "PME", "bond"):
        scale = np.abs(a[key]).max()
        assert np.abs(a[key] - b[key]).max() <= 2e-4 * scale + 0.05, key


def test_npt_box_moves_in_driver(runs):
    """Berendsen NPT: the box changes every 2 steps through Main_Volume_Change and the modules'
    Update_Volume; the drop-in prints the stock build's density, pressure, LJ and bond energies.
    The stock PME keeps the box it was initialised with (Particle_Mesh_Ewald::Update_Volume
    passes its own member box on, PME_force.cu:996-999), while the drop-in takes the new one, so
    the printed PME energy (and the potential) differ by the change of the reciprocal energy
    with the box: the box moves by about 0.3 % here, which moves the reciprocal energy by about
    2 kcal/mol; 1e-3 of the potential bounds it."""
    a, b = runs["stock_npt"], runs["b200_npt"]
    assert list(a["step"]) == list(b["step"])
    assert "density" in a and "pressure" in a
    assert np.ptp(a["density"]) > 0  # the box did move
    # density is printed with 4 decimals: one unit of the last digit apart at most
    assert np.allclose(a["density"], b["density"], rtol=0, atol=1.5e-4)
    assert np.allclose(a["pressure"], b["pressure"], rtol=1e-3, atol=10.0)
    for key in ("LJ", "bond"):
        scale = np.abs(a[key]).max()
        assert np.abs(a[key] - b[key]).max() <= 2e-4 * scale + 0.05, key
    for key in ("potential", "PME"):
        scale = np.abs(a["potential"]).max()
        assert np.abs(a[key] - b[key]).max() <= 1e-3 * scale, key
    assert np.allclose(a["temperature"], b["temperature"], rtol=1e-3, atol=0.05)


def test_trajectory_and_restart_files(runs):
    """The output files of the driver on the drop-ins, read back by sponge_b200.sponge_io: the
    binary coordinate trajectory and box file have one frame per printed step; the last frame
    is the state of the restart pair written at the same step; the stock and drop-in
    trajectories agree; and a run continued from the restart files of its first 20 steps follows
    the uninterrupted 40-step run (the restart stores %12.7f text, so the two drift apart from
    1e-7 A; within 1e-3 A after 20 steps of 1 fs)."""
    n = 3000
    d = runs["dirs"]
    ta = sponge_io.read_crd_traj(os.path.join(d["b200"], "mdcrd.dat"), n)
    tb = sponge_io.read_box_traj(os.path.join(d["b200"], "mdbox.txt"))
    assert ta.shape == (4, n, 3) and tb.shape == (4, 3)
    assert np.allclose(tb, np.asarray(systems.config0()["box"], np.float32), atol=1e-4)
    c, v, b, t = sponge_io.read_restart(os.path.join(d["b200"], "restart"))
    assert np.abs(c - ta[-1]).max() < 1e-5
    assert t == pytest.approx(0.04, abs=1e-9)
    ts = sponge_io.read_crd_traj(os.path.join(d["stock"], "mdcrd.dat"), n)
    L = np.asarray(systems.config0()["box"], np.float64)
    dd = ts.astype(np.float64) - ta
    dd -= L * np.round(dd / L)
    assert np.abs(dd).max() < 1e-3
    tr = sponge_io.read_crd_traj(os.path.join(d["b200_restarted"], "mdcrd.dat"), n)
    assert tr.shape == (2, n, 3)
    dd = tr.astype(np.float64) - ta[2:]
    dd -= L * np.round(dd / L)
    assert np.abs(dd).max() < 1e-3
