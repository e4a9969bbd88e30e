"""The FP64 FEP/TI oracle (soft-core LJ + direct Coulomb, PME cross terms) checked on CPU.

* dU/dlambda (soft-core LJ and direct Coulomb, PME reciprocal/self/exclusion cross terms,
  long-range correction) against central finite differences of U(lambda);
* forces against finite differences of U in positions;
* end states: at lambda = 0 the soft-core sum is the plain LJ + direct sum of state A, at
  lambda = 1 that of state B (the softening vanishes at the state it belongs to);
* with nothing perturbed the soft-core sum equals the plain sum and dH/dlambda is zero.
"""

import numpy as np
import pytest

from sponge_b200 import systems


@pytest.fixture(scope="module")
def box():
    return systems.fep_box(600, 0.4, 77)


@pytest.mark.parametrize("lam", [0.25, 0.8])
def test_dU_dlambda_matches_finite_differences(box, oracle_lib, lam):
    r = oracle_lib.fep_reference(box, lam=lam)
    # LJ terms do not depend on the (float32) charges: a small step is exact to FP64 rounding
    h = 1e-5
    a = oracle_lib.fep_reference(box, uc=r["uc"], lam=lam + h)
    b = oracle_lib.fep_reference(box, uc=r["uc"], lam=lam - h)
    assert (a["e_lj"] - b["e_lj"]) / (2 * h) == pytest.approx(r["dhdl_lj"], rel=1e-6)
    assert (a["e_lrc"] - b["e_lrc"]) / (2 * h) == pytest.approx(r["dhdl_lrc"], rel=1e-8)
    # charge-dependent terms: a larger step keeps the float32 rounding of q(lambda) small
    h = 1e-3
    a = oracle_lib.fep_reference(box, uc=r["uc"], lam=lam + h)
    b = oracle_lib.fep_reference(box, uc=r["uc"], lam=lam - h)
    scale = sum(abs(r[k]) for k in ("dhdl_lj", "dhdl_direct", "cross_rec", "cross_self",
                                     "cross_corr", "dhdl_lrc"))
    for e, d in (("e_direct", "dhdl_direct"), ("e_rec", "cross_rec"), ("e_self", "cross_self"),
                 ("e_corr", "cross_corr")):
        fd = (a[e] - b[e]) / (2 * h)
        assert abs(fd - r[d]) <= 1e-4 * max(abs(r[d]), 1e-3 * scale), (e, fd, r[d])
    fd = (a["U"] - b["U"]) / (2 * h)
    assert abs(fd - r["dU"]) <= 1e-4 * scale


def test_forces_match_position_finite_differences(box, oracle_lib):
    r = oracle_lib.fep_reference(box)
    uc = r["uc"]
    L = np.asarray(box["box"], np.float64)
    rng = np.random.default_rng(5)
    # a solute atom (soft-core pairs) and a water atom
    for atom in (3, 20 + int(rng.integers(0, 1700))):
        for d in range(3):
            step = 1024  # fixed-point units: 1024 L / 2^32 A
            h = step * L[d] / 4294967296.0
            up = uc.copy()
            dn = uc.copy()
            up[atom, d] = np.uint32(int(up[atom, d]) + step)
            dn[atom, d] = np.uint32(int(dn[atom, d]) - step)
            Ua = oracle_lib.fep_reference(box, uc=up)["U"]
            Ub = oracle_lib.fep_reference(box, uc=dn)["U"]
            fd = -(Ua - Ub) / (2 * h)
            f = r["f_total"][atom, d]
            assert abs(fd - f) <= 1e-4 * max(abs(f), 1.0), (atom, d, fd, f)


def test_end_states_are_plain_sums(box, oracle_lib):
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(box["crd"], box["box"]), box["box"])
    beta = oracle_lib.get_beta(box["cutoff"], box["tolerance"])
    pk = oracle_lib.pairs(uc, box)
    for lam, qkey, akey, bkey, tkey in ((0.0, "charge_A", "lj_A", "lj_B", "lj_type"),
                                       (1.0, "charge_B", "lj_A_B", "lj_B_B", "lj_type_B")):
        f_sc, p = oracle_lib.softcore(uc, box, pk, beta, lam=lam, charge=box[qkey])
        plain = dict(box, charge=box[qkey], lj_A=box[akey], lj_B=box[bkey], lj_type=box[tkey],
                     n_types=box["n_types"] if lam == 0.0 else box["n_types_B"])
        f_d, _, d = oracle_lib.direct(uc, plain, pk, beta)
        assert p["e_lj"] == pytest.approx(d["e_lj"], rel=1e-12, abs=1e-9)
        assert p["e_direct"] == pytest.approx(d["e_direct"], rel=1e-12, abs=1e-9)
        assert np.allclose(f_sc, f_d, rtol=1e-10, atol=1e-9)


def test_unperturbed_is_plain(oracle_lib):
    w = systems.config0()
    n = len(w["charge"])
    fake = dict(w, lj_type_B=w["lj_type"], lj_A_B=w["lj_A"], lj_B_B=w["lj_B"],
                mask=np.zeros(n, np.int32), dq=np.zeros(n, np.float32), lam=0.37,
                sc_alpha=0.5, sc_p=1.0, sc_sigma=3.0, sc_sigma_min=0.0)
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(w["crd"], w["box"]), w["box"])
    beta = oracle_lib.get_beta(w["cutoff"], w["tolerance"])
    pk = oracle_lib.pairs(uc, w)
    f_sc, p = oracle_lib.softcore(uc, fake, pk, beta)
    f_d, _, d = oracle_lib.direct(uc, w, pk, beta)
    assert np.allclose(f_sc, f_d, rtol=1e-12, atol=1e-10)
    assert p["e_lj"] == pytest.approx(d["e_lj"], rel=1e-12)
    assert p["dhdl_lj"] == 0.0 and p["dhdl_direct"] == 0.0
