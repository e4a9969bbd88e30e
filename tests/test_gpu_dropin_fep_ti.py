"""SPONGE's FEP and TI drivers on the drop-ins.

oracle/ref_harness/build_sponge.sh builds the reference's unchanged main_fep.cu and main_ti.cu
with their modules twice (sponge_fep_stock / sponge_ti_stock as shipped; sponge_fep_b200 /
sponge_ti_b200 with NEIGHBOR_LIST and Particle_Mesh_Ewald replaced by the drop-ins). Both read the
same FEP box (600 waters + a 20-atom solute vanishing in lambda, lambda 0.4, soft core alpha 0.5,
p 1, sigma 3 A) and a 3-frame coordinate trajectory written by sponge_b200.sponge_io.

* FEP (main_fep.cu:56-132): per frame the soft-core LJ energy of the reference's LJ_SOFT_CORE over
  the drop-in's ATOM_GROUP list, the direct Coulomb energy, and the PME energy parts that the
  drop-in's Get_Energy(which_part) returns (main_fep.cu:114-121). Within 2e-4 of each column's
  scale (the stock PME energies are FP32 sums); the totals, small differences of the self and
  correction energies, within 1e-5 of those.
* TI (main_ti.cu:129-150): dH/dlambda per frame, with TI_CORE::Get_Cross_PME_Partial_H_Partial_Lambda
  (TI_core.cu:670-730) running unchanged on the drop-in's copies of the PME internals it reads
  (PME_force.cuh); within 1e-4 of each column's scale. The drop-in's parts are also checked
  against the FP64 oracle at frame 1 (the reference's self cross term is the oracle's without the
  neutralising term, as tests/test_golden_fep.py measures).
Skipped where the binaries have not been built.
"""

import os
import subprocess

import numpy as np
import pytest

from sponge_b200 import sponge_io, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = {k: os.path.join(ROOT, "oracle", "_ref", "sponge_%s" % k)
       for k in ("fep_stock", "fep_b200", "ti_stock", "ti_b200")}
LAMBDA = 0.4


def _system():
    return systems.fep_box(600, LAMBDA, 1004077)


def _frames(s):
    rng = np.random.default_rng(31)
    box = np.asarray(s["box"], np.float64)
    out = [np.asarray(s["crd"], np.float32)]
    for _ in range(2):
        c = np.mod(s["crd"].astype(np.float64) + rng.normal(0, 0.03, s["crd"].shape), box)
        out.append(np.where(c >= box, 0.0, c).astype(np.float32))
    return out


def _mdin(s, files, outdir, capacities):
    fft = s["fft"]
    return "\n".join([
        "FEP/TI drop-in parity run",
        "atom_numbers = %d" % len(s["charge"]),
        "frame_numbers = 3",
        "crd = %s" % files["crd"],
        "box = %s" % files["box"],
        "charge_pertubated = 1",
        "charge_in_file = %s" % files["charge"],
        "chargeA_in_file = %s" % files["chargeA"],
        "chargeB_in_file = %s" % files["chargeB"],
        "subsys_division_in_file = %s" % files["subsys"],
        "exclude_in_file = %s" % files["exclude"],
        "LJ_soft_core_in_file = %s" % files["lj_soft"],
        "lambda_lj = %g" % LAMBDA,
        "target_temperature = 300",
        "target_pressure = 1",
        "soft_core_alpha = %g" % s["sc_alpha"],
        "soft_core_powfer = %g" % s["sc_p"],
        "soft_core_sigma = %g" % s["sc_sigma"],
        "cutoff = %g" % s["cutoff"],
        "skin = %g" % s["skin"],
        "PME_fftx = %d" % fft[0], "PME_ffty = %d" % fft[1], "PME_fftz = %d" % fft[2],
        "neighbor_list_max_neighbor_numbers = %d" % capacities[0],
        "neighbor_list_max_atom_in_grid_numbers = %d" % capacities[1],
        "mdout = %s/mdout.txt" % outdir,
        "mdinfo = %s/mdinfo.txt" % outdir,
        "TI = %s/ti_result.txt" % outdir,
        "FEP = %s/fep_result.txt" % outdir,
        "end_pause = 0",
        "dont_check_input = 1",
        "device = 0",
        ""])


def _run(binary, s, files, outdir, capacities):
    os.makedirs(outdir, exist_ok=True)
    mdin = os.path.join(outdir, "mdin.txt")
    with open(mdin, "w") as f:
        f.write(_mdin(s, files, outdir, capacities))
    r = subprocess.run([binary, "-mdin", mdin], cwd=outdir, stdin=subprocess.DEVNULL,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    lines = [l.split() for l in open(os.path.join(outdir, "mdout.txt")) if l.strip()]
    head = lines[0]
    # a value too wide for its print format comes out as stars; no compared column has one
    rows = np.array([[float(x) if "*" not in x else np.nan for x in l] for l in lines[1:]],
                    np.float64)
    print(binary, "\n", open(os.path.join(outdir, "mdout.txt")).read())
    return {k: rows[:, i] for i, k in enumerate(head)}


@pytest.fixture(scope="module")
def runs(tmp_path_factory, oracle_lib):
    if not all(os.path.exists(b) for b in BIN.values()):
        pytest.skip("the FEP/TI driver builds are missing (oracle/ref_harness/build_sponge.sh)")
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle.ref_harness import run as refrun
    s = _system()
    frames = _frames(s)
    base = tmp_path_factory.mktemp("fep_ti")
    files = sponge_io.write_fep_inputs(s, str(base / "inputs"), frames)
    # the reference's list has no capacity checks: capacities from the frames, with margin
    caps = [0, 0]
    for fr in frames:
        uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(fr, s["box"]), s["box"])
        c = refrun.safe_capacities(s, uc, oracle_lib.pairs(uc, s, "cells"))
        caps = [max(caps[0], c[0]), max(caps[1], c[1])]
    out = {k: _run(b, s, files, str(base / k), caps) for k, b in BIN.items()}
    out["system"], out["frames"] = s, frames
    return out


def _close(a, b, cols, rel, absol=0.02):
    for key in cols:
        scale = max(np.abs(a[key]).max(), np.abs(b[key]).max())
        err = np.abs(a[key] - b[key]).max()
        print("%-14s stock %s b200 %s" % (key, a[key], b[key]))
        assert err <= rel * scale + absol, (key, err, scale)


def test_fep_driver_on_drop_ins(runs):
    a, b = runs["fep_stock"], runs["fep_b200"]
    assert list(a["frame"]) == [1, 2, 3] and list(b["frame"]) == [1, 2, 3]
    _close(a, b, ("LJ(sc.)", "Coul(direct.)", "LR_corr(sc.)", "PME(reci.)", "PME(self.)",
                  "PME(corr.)"), 2e-4)
    # the total and the Coulomb sum are small differences of the self and correction energies
    # (about 3.6e4 kcal/mol each, of opposite sign), whose FP32 rounding in the stock build
    # (a few 1e-6 of them) carries over: bounded by 1e-5 of |self| + |corr|
    big = np.abs(a["PME(self.)"]).max() + np.abs(a["PME(corr.)"]).max()
    for key in ("ene", "Coul(all.)"):
        assert np.abs(a[key] - b[key]).max() <= 1e-5 * big + 0.02, key


def test_ti_driver_on_drop_ins(runs):
    a, b = runs["ti_stock"], runs["ti_b200"]
    assert list(a["frame"]) == [1, 2, 3] and list(b["frame"]) == [1, 2, 3]
    _close(a, b, ("dH_dlambda", "LJ(sc.)", "Coul(direct.)", "LR_corr(sc.)", "PME(reci.)",
                  "PME(self.)", "PME(corr.)"), 1e-4)


def test_ti_driver_against_fp64_oracle(runs, oracle_lib):
    """Frame 1 of the drop-in TI run against the FP64 oracle of the same box at lambda 0.4."""
    b = runs["ti_b200"]
    s = runs["system"]
    ref = oracle_lib.fep_reference(s, lam=LAMBDA)
    q = np.asarray(ref["charge"], np.float64)
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    neutral = 2.0 * (-np.pi / (2.0 * float(ref["beta"]) ** 2 * V)) * q.sum() * \
        np.asarray(s["dq"], np.float64).sum()
    pairs = (("LJ(sc.)", ref["dhdl_lj"]), ("Coul(direct.)", ref["dhdl_direct"]),
             ("LR_corr(sc.)", ref["dhdl_lrc"]), ("PME(reci.)", ref["cross_rec"]),
             ("PME(self.)", ref["cross_self"] - neutral), ("PME(corr.)", ref["cross_corr"]))
    for key, want in pairs:
        assert b[key][0] == pytest.approx(want, rel=1e-4, abs=2e-2), key
