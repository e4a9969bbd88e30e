"""The oracle pinned against the REFERENCE's own outputs (CPU test).

tests/golden/reference_*.npz were produced by running SPONGE's unchanged NEIGHBOR_LIST,
LENNARD_JONES_INFORMATION and Particle_Mesh_Ewald modules on a B200 (tests/golden/make_golden.py
through oracle/ref_harness). The systems are regenerated here from their seeds.

Tolerances: the reference computes in FP32 with float atomics, so its forces are compared at
relative RMS 1e-5 against the FP64 oracle; its FP32 energy reductions at relative 1e-4; its
long-range LJ factor (an FP32 atomic sum over all N^2 atom pairs) at 1e-3 (1e-2 for the 98,282-atom
real system, tests/golden/make_covid.py). Its pair list may
differ from the pinned criterion only in pairs within FP32 rounding of the threshold.
"""

import os

import numpy as np
import pytest

from sponge_b200 import systems

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def covid_tip4p():
    """The reference's own real system (tests/golden/make_covid.py), 98,282 atoms."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_covid", os.path.join(HERE, "make_covid.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system()


CASES = {
    "small": lambda: systems.small_water(),
    "config0": systems.config0,
    "config1": systems.config1,
    "config3": systems.config3,
    "covid_tip4p": covid_tip4p,
}
# the reference's long-range LJ factor is an FP32 atomic sum over all N^2 atom pairs: its
# rounding grows with N (9.7e9 pairs for the 98,282-atom system)
LRC_TOL = {"covid_tip4p": 1e-2}


def fixture(name):
    path = os.path.join(HERE, "reference_%s.npz" % name)
    if not os.path.exists(path):
        pytest.fail("missing golden fixture %s (run tests/golden/make_golden.py on a GPU)" % path)
    return np.load(path)


@pytest.fixture(scope="module", params=list(CASES))
def case(request, oracle_lib):
    s = CASES[request.param]()
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s["crd"], s["box"]), s["box"])
    ref = oracle_lib.reference_energies(s, uc=uc)
    return request.param, s, uc, ref, fixture(request.param)


def boundary_r2(uc, keys, s):
    """FP32 r^2 of pairs (pinned expression) and the list threshold."""
    n = uc.shape[0]
    i, j = keys // n, keys % n
    sc = (np.float32(1.0) / np.float32(4294967296.0)) * np.asarray(s["box"], np.float32)
    with np.errstate(over="ignore"):
        d = [(uc[j, k].astype(np.int64) - uc[i, k].astype(np.int64)).astype(np.int32)
             .astype(np.float32) * sc[k] for k in range(3)]
    r2 = (d[0] * d[0] + d[1] * d[1]).astype(np.float32) + (d[2] * d[2]).astype(np.float32)
    cs = np.float32(s["cutoff"]) + np.float32(s["skin"])
    return r2.astype(np.float32), np.float32(cs * cs)


def test_pair_list_matches_reference(case):
    name, s, uc, ref, g = case
    if "pairs" in g.files:
        rp = g["pairs"]
        only_ref = np.setdiff1d(rp, ref["pairs"])
        only_orc = np.setdiff1d(ref["pairs"], rp)
    else:
        only_ref, only_orc = g["pairs_only_ref"], g["pairs_only_oracle"]
        assert int(g["n_pairs"]) == ref["pairs"].size + only_ref.size - only_orc.size
    # every disagreement is a pair within FP32 rounding of (rc+skin)^2
    for keys in (only_ref, only_orc):
        if keys.size:
            r2, thr = boundary_r2(uc, keys, s)
            assert np.all(np.abs(r2 - thr) <= 4 * np.spacing(thr))
    assert only_ref.size + only_orc.size <= max(2, ref["pairs"].size // 100000)


def test_reference_forces_match_oracle(case):
    name, s, uc, ref, g = case
    for key in ("frc", "frc_plain"):
        if key not in g.files:  # the real system keeps only the energy/virial evaluation
            continue
        f = g[key].astype(np.float64)
        err = np.sqrt(((f - ref["f_total"]) ** 2).sum() / (ref["f_total"] ** 2).sum())
        assert err < 1e-5, (key, err)


def test_reference_energies_match_oracle(case):
    name, s, uc, ref, g = case
    get = lambda k: float(g["summary_" + k])  # noqa: E731
    assert get("beta") == pytest.approx(ref["beta"], rel=1e-7)
    assert get("e_rec") == pytest.approx(ref["e_rec"], rel=1e-4)
    assert get("e_self") == pytest.approx(ref["e_self"], rel=1e-4)
    assert get("e_direct") == pytest.approx(ref["e_direct"], rel=1e-4, abs=1e-2)
    assert get("e_corr") == pytest.approx(ref["e_corr"], rel=1e-4)
    assert get("long_range_factor") == pytest.approx(ref["lrc_factor"], rel=LRC_TOL.get(name, 1e-3))
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    lrc_ref = get("long_range_factor") / V
    assert get("e_lj_with_lrc") - lrc_ref == pytest.approx(ref["e_lj"], rel=1e-4, abs=1e-2)
    assert get("atom_virial_sum") == pytest.approx(ref["virial_lj"], rel=1e-4, abs=1e-2)
    # d_potential = LRC + correction + self + reciprocal; d_virial = 6 LRC + direct + those
    pot = lrc_ref + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    vir = 6 * lrc_ref + ref["e_direct"] + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    scale = abs(ref["e_self"]) + abs(ref["e_corr"])
    assert abs(get("d_potential") - pot) < 1e-5 * scale + 1e-4 * abs(pot)
    assert abs(get("d_virial") - vir) < 1e-5 * scale + 1e-4 * abs(vir)
    # per-atom energy sum = LJ + direct Coulomb
    assert get("atom_energy_sum") == pytest.approx(ref["e_lj"] + ref["e_direct"], rel=1e-4,
                                                    abs=1e-2)


def test_reference_nb14_and_virtual_atoms_match_oracle(oracle_lib):
    """The reference's NON_BOND_14 and VIRTUAL_INFORMATION on the real system against the FP64
    oracle (tests/golden/make_covid.py): 1-4 forces, per-atom energies and virials, the 1-4
    energy sums, the redistributed nonbonded forces and the refreshed virtual-atom positions."""
    from sponge_b200 import nb14_pair_tables
    s = covid_tip4p()
    g = fixture("covid_tip4p")
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s["crd"], s["box"]), s["box"])
    A, B = nb14_pair_tables(s["nb14_a"], s["nb14_b"], s["nb14_lj_scale"],
                            np.float32(12.0) * s["lj_A"], np.float32(6.0) * s["lj_B"],
                            s["lj_type"])
    f, ae, av, elj, ecf = oracle_lib.nb14(uc, s["box"], s["charge"], s["nb14_a"], s["nb14_b"],
                                          A, B, s["nb14_cf"])
    at = g["nb14_atoms"]
    rel = lambda a, b: float(np.sqrt(((np.asarray(a, np.float64) - b) ** 2).sum()  # noqa: E731
                                     / (np.asarray(b, np.float64) ** 2).sum()))
    assert rel(g["nb14_frc"], f[at]) < 1e-5
    assert rel(g["nb14_ae"], ae[at]) < 1e-5
    assert rel(g["nb14_av"], av[at]) < 1e-5
    assert float(g["summary_nb14_lj"]) == pytest.approx(elj, rel=1e-5)
    assert float(g["summary_nb14_cf"]) == pytest.approx(ecf, rel=1e-5)
    fv = oracle_lib.vsite(uc, s["box"], s["vs_type"], s["vs_atoms"], s["vs_param"],
                          frc=g["frc"].astype(np.float64))
    assert rel(g["vs_frc"], fv) < 1e-6
    crd = oracle_lib.periodic_map(s["crd"], s["box"]).astype(np.float64)
    cv = oracle_lib.vsite(uc, s["box"], s["vs_type"], s["vs_atoms"], s["vs_param"], crd=crd)
    L = np.asarray(s["box"], np.float64)
    d = g["vs_crd"].astype(np.float64) - cv[s["vs_atoms"][:, 0]]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4
