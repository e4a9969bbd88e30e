"""The FP64 SETTLE step of the oracle (oracle.nve_settle) checked on its own and against the
reference's CONSTRAIN + SETTLE modules on the covid-tip4p system (no GPU needed).

SETTLE (SPONGE/constrain/SETTLE.cu) restores each rigid water's three distances and each isolated
rigid pair's distance after the unconstrained leap-frog, moving only within the molecule: the
molecule's centre of mass is that of the unconstrained step. The reference outputs
(tests/golden/reference_covid_tip4p.npz: settle_crd / settle_vel on a seeded sample of atoms,
settle_pressure) come from the reference's own modules run by oracle/ref_harness on the same
forces (the nonbonded forces after the virtual-atom redistribution, vs_frc).
"""

import importlib.util
import os

import numpy as np
import pytest

from sponge_b200 import constrain_pairs_from_bonds, sponge_io, systems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KB = 0.0019872041  # kcal/mol/K
DT = float(np.float32(np.float32(0.002) * np.float32(20.455)))


def water_case(oracle, seed=11):
    s = systems.config0()
    a, b, r, mass = sponge_io.bonds_and_masses(s)
    pi, pj, pr = constrain_pairs_from_bonds(a, b, r, mass)
    n = len(s["charge"])
    rng = np.random.default_rng(seed)
    vel = (rng.normal(size=(n, 3)) * np.sqrt(KB * 300.0 / mass)[:, None]).astype(np.float32)
    crd = oracle.periodic_map(s["crd"], s["box"])
    uc = oracle.crd_to_uint(crd, s["box"])
    frc = oracle.reference_energies(s, uc=uc)["f_total"].astype(np.float32)
    return s, (pi, pj, pr), mass, vel, crd.astype(np.float32), uc, frc


def distances(crd, box, i, j):
    d = crd[j] - crd[i]
    L = np.asarray(box, np.float64)
    d -= L * np.round(d / L)
    return np.sqrt((d ** 2).sum(1))


def test_constrain_pairs_from_bonds():
    s = systems.config0()
    a, b, r, mass = sponge_io.bonds_and_masses(s)
    pi, pj, pr = constrain_pairs_from_bonds(a, b, r, mass)
    assert pi.size == a.size  # every water bond has a hydrogen
    heavy = mass.copy()
    heavy[:] = 16.0
    assert constrain_pairs_from_bonds(a, b, r, heavy)[0].size == 0
    heavy[b[0]] = 0.0  # massless atoms are not hydrogens (constrain.cu:99)
    assert constrain_pairs_from_bonds(a, b, r, heavy)[0].size == 0


def test_water_settle_restores_geometry(oracle_lib):
    s, (pi, pj, pr), mass, vel, crd, uc, frc = water_case(oracle_lib)
    n = len(mass)
    c, v, acc, vir, nt, npair = oracle_lib.nve_settle(uc, s["box"], pi, pj, pr, mass, DT, frc,
                                                      crd, vel)
    assert (nt, npair) == (n // 3, 0)
    d = distances(c, s["box"], pi, pj)
    assert np.abs(d - pr).max() < 1e-6
    # unconstrained leap-frog for comparison: SETTLE keeps each water's centre of mass
    inv = np.where(mass == 0, 0.0, 1.0 / mass.astype(np.float64))
    v0 = vel + DT * inv[:, None] * frc
    c0 = crd + DT * v0
    o = np.arange(0, n, 3)
    m = mass.astype(np.float64)
    com = lambda x: (m[o, None] * x[o] + m[o + 1, None] * x[o + 1] + m[o + 2, None] * x[o + 2])  # noqa: E731
    assert np.abs(com(c) - com(c0)).max() < 1e-9 * np.abs(com(c0)).max()
    assert np.abs(com(v) - com(v0)).max() < 1e-9 * np.abs(com(v0)).max()
    # the velocity update is the position correction over dt (SETTLE.cu:432-466)
    assert np.allclose(v - v0, (c - c0) / DT, atol=1e-9)
    assert np.isfinite(vir) and vir != 0.0


def _covid():
    spec = importlib.util.spec_from_file_location("make_covid", os.path.join(HERE, "make_covid.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system()


def test_covid_settle_matches_reference(oracle_lib):
    golden = np.load(os.path.join(HERE, "reference_covid_tip4p.npz"))
    if "settle_crd" not in golden.files:
        pytest.skip("reference outputs without the SETTLE step")
    s = _covid()
    pi, pj, pr = constrain_pairs_from_bonds(s["bond_a"], s["bond_b"], s["bond_r"], s["mass"])
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s["crd"], s["box"]), s["box"])
    frc = golden["vs_frc"].astype(np.float64)
    c, v, acc, vir, nt, npair = oracle_lib.nve_settle(uc, s["box"], pi, pj, pr, s["mass"],
                                                      float(s["md_dt"]), frc, s["crd"], s["vel"])
    assert (nt, npair) == (21389, 2408)
    atoms = golden["settle_atoms"]
    L = np.asarray(s["box"], np.float64)
    dc = c[atoms] - golden["settle_crd"]
    dc -= L * np.round(dc / L)
    # FP32 reference against FP64: coordinates to 1.3e-5 A, velocities to 7.9e-5 relative RMS
    # (the velocity correction is a coordinate difference over dt)
    assert np.abs(dc).max() < 5e-5
    dv = v[atoms] - golden["settle_vel"]
    assert np.sqrt((dv ** 2).mean()) < 1e-4 * np.sqrt((v[atoms] ** 2).mean())
    V = float(np.prod(L))
    p = vir * float(np.float32(0.33333)) / V
    assert p == pytest.approx(float(golden["summary_settle_pressure"]), rel=1e-5)
