"""CPU tests of the FP64 oracle against known answers (runs without a GPU).

The reference ships no tests or golden outputs; its known answers for this path are the values
its own initialisation code produces (Get_Beta, Get_Fft_Patameter), the B-spline identities,
and the physics the path implements (converged Ewald sums). The oracle is also checked against
numpy (FFT) and against pure-Python restatements on tiny cases.
"""

import numpy as np
import pytest

from sponge_b200 import systems


def test_get_beta_known_values(oracle_lib):
    # Get_Beta (SPONGE/PME_force/PME_force.cu:71-100) at tolerance 1e-5 for rc = 8, 10, 9
    assert oracle_lib.get_beta(8.0) == pytest.approx(0.34864, abs=2e-5)
    assert oracle_lib.get_beta(10.0) == pytest.approx(0.27511, abs=2e-5)
    assert oracle_lib.get_beta(9.0) == pytest.approx(0.30768, abs=2e-5)
    # defining property: erfc(beta rc)/rc == tol
    from scipy.special import erfc
    for rc in (8.0, 9.0, 10.0, 12.0):
        b = oracle_lib.get_beta(rc, 1e-5)
        assert erfc(b * rc) / rc == pytest.approx(1e-5, rel=1e-3)


def test_fft_size_known_values(oracle_lib):
    # Get_Fft_Patameter (SPONGE/common.cu:513-534)
    assert oracle_lib.fft_size(31.04) == 32
    assert oracle_lib.fft_size(98.6) == 100
    assert oracle_lib.fft_size(215.3) == 216
    assert oracle_lib.fft_size(60.0) == 64
    for L in np.linspace(10, 300, 97):
        k = oracle_lib.fft_size(float(L))
        m = k
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        # the power-of-two snap (60..68 -> 64, ...) can land slightly below L
        assert m == 1 and k % 4 == 0 and k >= 0.9 * L


def test_bspline_identities():
    # the weights of PME_force.cu:8-14 sum to 1, their derivatives to 0
    for fr in np.linspace(0, 1, 11):
        f2, f3 = fr * fr, fr ** 3
        w = [f3 / 6, -f3 / 2 + f2 / 2 + fr / 2 + 1 / 6, f3 / 2 - f2 + 2 / 3, -f3 / 6 + f2 / 2 - fr / 2 + 1 / 6]
        dw = [f2 / 2, -1.5 * f2 + fr + 0.5, 1.5 * f2 - 2 * fr, -0.5 * f2 + fr - 0.5]
        assert sum(w) == pytest.approx(1.0, abs=1e-14)
        assert sum(dw) == pytest.approx(0.0, abs=1e-14)


def test_bspline_moduli_closed_form(oracle_lib):
    for K in (16, 32, 96, 100):
        b = oracle_lib.bspline_moduli(K)
        k = np.arange(K)
        # |1/6 + 2/3 e^{i t} + 1/6 e^{2 i t}| = |2/3 + 1/3 cos t|
        expect = 1.0 / (2.0 / 3.0 + np.cos(2 * np.pi * k / K) / 3.0) ** 2
        assert np.allclose(b, expect, rtol=1e-12)


def test_fft_matches_numpy(oracle_lib):
    rng = np.random.default_rng(0)
    for shape in [(8, 6, 10), (12, 15, 14), (16, 16, 16)]:
        g = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        assert np.allclose(oracle_lib.fft3(g, -1), np.fft.fftn(g), atol=1e-10)
        assert np.allclose(oracle_lib.fft3(g, +1), np.fft.ifftn(g) * g.size, atol=1e-10)


def test_fixed_point_and_wrap(oracle_lib):
    box = np.array([31.04, 31.04, 31.04], np.float32)
    crd = np.array([[0.0, 15.0, 31.039], [-0.5, 31.5, 10.0]], np.float32)
    w = oracle_lib.periodic_map(crd, box)
    assert np.all(w >= 0) and np.all(w < box)
    uc = oracle_lib.crd_to_uint(w, box)
    # Crd_To_Uint_Crd: (int)(x * 0.25*2^32/L) << 2 in float
    cof = np.float32(0.25 * 4294967296.0) / box
    expect = ((w * cof).astype(np.float32).astype(np.int64).astype(np.uint32) << np.uint32(2))
    assert np.array_equal(uc, expect.astype(np.uint32))
    assert np.all(uc % 4 == 0)


def _tiny_pairs_python(uc, sys):
    """Pure-Python restatement of the half pair set (FP32 criterion, exclusion rule)."""
    n = uc.shape[0]
    s = (np.float32(1.0) / np.float32(4294967296.0)) * np.asarray(sys["box"], np.float32)
    cs = np.float32(sys["cutoff"]) + np.float32(sys["skin"])
    thr = np.float32(cs * cs)
    out = []
    for i in range(n):
        ex = set(sys["excl_list"][sys["excl_start"][i]:sys["excl_start"][i] + sys["excl_numbers"][i]].tolist())
        for j in range(i + 1, n):
            d = [np.float32(np.int32(np.uint32(uc[j, k]) - np.uint32(uc[i, k])).astype(np.float32)) * s[k]
                 for k in range(3)]
            r2 = np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1]))
            r2 = np.float32(r2 + np.float32(d[2] * d[2]))
            if r2 < thr and j not in ex:
                out.append(i * n + j)
    return np.array(out, np.int64)


def test_pair_sets_agree(oracle_lib):
    sys_ = systems.small_water(n_side=3, fft=(12, 12, 12))
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(sys_["crd"], sys_["box"]), sys_["box"])
    pb = oracle_lib.pairs(uc, sys_, "brute")
    pc = oracle_lib.pairs(uc, sys_, "cells")
    with np.errstate(over="ignore"):
        pp = _tiny_pairs_python(uc, sys_)
    assert np.array_equal(pb, pc)
    assert np.array_equal(pb, pp)
    # exclusions removed: no intramolecular pair in the list
    n = uc.shape[0]
    i, j = pb // n, pb % n
    assert not np.any((i // 3 == j // 3))


def test_pair_sets_agree_config0(oracle_lib):
    s0 = systems.config0()
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s0["crd"], s0["box"]), s0["box"])
    pb = oracle_lib.pairs(uc, s0, "brute")
    pc = oracle_lib.pairs(uc, s0, "cells")
    assert np.array_equal(pb, pc)
    assert 190 < len(pb) / 3000 < 230  # ~210 half-list entries per atom at rc+skin = 10 A


def test_direct_force_matches_finite_difference(oracle_lib):
    """Forces are minus the gradient of the energies the oracle reports."""
    s = systems.small_water(n_side=3, fft=(12, 12, 12), cutoff=4.5, skin=0.5)
    crd = oracle_lib.periodic_map(s["crd"], s["box"]).astype(np.float64)
    beta = oracle_lib.get_beta(s["cutoff"])
    L = np.asarray(s["box"], np.float64)

    def to_uint(c):  # FP64 fixed point (resolution L/2^30) so that the step h is resolved
        return ((np.floor(np.mod(c, L) / L * 2.0 ** 30).astype(np.uint64) << np.uint64(2))
                .astype(np.uint32))

    uc0 = to_uint(crd)
    keys = oracle_lib.pairs(uc0, s)

    def energy(c):
        _, _, d = oracle_lib.direct(to_uint(c), s, keys, beta)
        return d["e_lj"] + d["e_direct"]

    f, _, _ = oracle_lib.direct(uc0, s, keys, beta)
    h = 1e-4
    rng = np.random.default_rng(3)
    for a in rng.choice(len(crd), 4, replace=False):
        for k in range(3):
            cp, cm = crd.copy(), crd.copy()
            cp[a, k] += h
            cm[a, k] -= h
            fd = -(energy(cp) - energy(cm)) / (2 * h)
            assert fd == pytest.approx(f[a, k], rel=2e-3, abs=2e-3)


def test_spme_converges_to_ewald(oracle_lib):
    """SPME reciprocal force approaches the exact Ewald reciprocal sum (method error)."""
    s = systems.config0()
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s["crd"], s["box"]), s["box"])
    beta = oracle_lib.get_beta(s["cutoff"])
    fe, ee = oracle_lib.ewald_recip(uc, s, beta, 12)
    errs = []
    for K in (32, 48, 64):
        fr, er = oracle_lib.pme(uc, s, beta, fft=(K, K, K))
        errs.append(np.sqrt(((fr - fe) ** 2).sum() / (fe ** 2).sum()))
        assert er == pytest.approx(ee, rel=5e-3)
    assert errs[0] < 5e-3 and errs[1] < errs[0] and errs[2] < errs[1]


def test_total_potential_parts(oracle_lib):
    s = systems.config0()
    r = oracle_lib.reference_energies(s)
    # the exclusion and self terms nearly cancel for neutral rigid waters
    assert r["e_corr"] > 0 and r["e_self"] < 0
    assert abs(r["e_corr"] + r["e_self"]) < 0.05 * abs(r["e_self"])
    assert r["e_lrc"] < 0
    assert r["n_in_cutoff"] < len(r["pairs"])
