"""GPU parity tests: the CUDA path through the C ABI against the FP64 oracle.

Tolerances (stated per the accuracy bar of the hot path): relative RMS force error <= 1e-5
against FP64 evaluation of the same discretised method (same list, cutoff, beta, grid, order);
energies and virial parts within 1e-5 relative; pair sets bit-exact; forces of the fixed-point
form bit-identical run to run and under atom relabelling.
"""

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sponge_b200
    sponge_b200.lib()  # fails loudly if the library is missing
    return torch


SYSTEMS = {
    "small": lambda: systems.small_water(),
    "config0": systems.config0,
    "config3": systems.config3,
}


@pytest.fixture(scope="module", params=list(SYSTEMS))
def case(request, torch_cuda, oracle_lib):
    from sponge_b200 import NonbondedEngine
    s = SYSTEMS[request.param]()
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    torch_cuda.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.reference_energies(s, uc=uc)
    return request.param, s, eng, ref


def test_wrap_and_fixed_point_match_reference(case, oracle_lib):
    name, s, eng, ref = case
    wrapped = oracle_lib.periodic_map(s["crd"], s["box"])
    assert np.array_equal(eng.crd.cpu().numpy(), wrapped)
    uc_expected = oracle_lib.crd_to_uint(wrapped, s["box"])
    assert np.array_equal(eng.uint_crd.cpu().numpy().view(np.uint32), uc_expected)
    assert np.array_equal(eng.nl.uint_crd().cpu().numpy().view(np.uint32), uc_expected)


def test_pair_set_bit_exact_vs_bruteforce(case, oracle_lib):
    name, s, eng, ref = case
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    brute = oracle_lib.pairs(uc, s, "brute")
    got = eng.nl.export_pairs()
    assert eng.nl.status() == 0
    assert got.shape == brute.shape
    assert np.array_equal(got, brute)


def test_atom_group_export_matches_pair_set(case, torch_cuda):
    name, s, eng, ref = case
    from sponge_b200 import DeviceArray
    torch = torch_cuda
    n = eng.n
    addr = eng.nl.d_nl
    ag = torch.as_tensor(DeviceArray(addr, (n, 2), "<i8"), device="cuda").cpu().numpy()
    counts = (ag[:, 0] & 0xffffffff).astype(np.int64)
    base = int(ag[0, 1])
    maxnb = eng.nl.max_neighbor_numbers
    serial = torch.as_tensor(DeviceArray(base, (n, maxnb), "<i4"), device="cuda").cpu().numpy()
    keys = []
    for i in range(n):
        js = serial[i, :counts[i]]
        assert np.all(js > i)
        keys.append(i * n + js.astype(np.int64))
    keys = np.sort(np.concatenate(keys))
    assert np.array_equal(keys, np.sort(ref["pairs"]))


def _forces(eng, parts, need_energy=0, need_virial=0):
    eng.reset()
    eng.forces(need_energy=need_energy, need_virial=need_virial, parts=parts)
    return eng.frc.cpu().numpy().astype(np.float64)


def test_direct_force(case):
    name, s, eng, ref = case
    out = {}
    # every pair-kernel shape (1 = compacted pairs, 2 = packed FP32x2 slot pairs)
    for ipl in (8, 4, 2, 1):
        eng.lj.set_kernel_variant(ipl)
        out[ipl] = _forces(eng, ("direct",))
        assert rel_rms(out[ipl], ref["f_direct"]) < FORCE_TOL
        assert np.array_equal(_forces(eng, ("direct",)), out[ipl])  # bit-identical repeat
    assert rel_rms(out[4], out[8]) < 1e-6
    assert rel_rms(out[2], out[8]) < 1e-6
    assert rel_rms(out[1], out[8]) < 1e-6
    chosen = eng.lj.tune(eng.nl, eng.uint_crd, eng.charge, eng.pme.beta)
    assert chosen in (1, 2, 4, 8)
    # tuning leaves no residue in the accumulators
    assert np.array_equal(_forces(eng, ("direct",)), out[chosen])


def test_excluded_force(case):
    name, s, eng, ref = case
    f = _forces(eng, ("excluded",))
    assert rel_rms(f, ref["f_excl"]) < FORCE_TOL


def test_reciprocal_force(case):
    name, s, eng, ref = case
    import sponge_b200
    out = {}
    # every FFT kernel family (register line transforms exist for every grid here; the grids
    # are square, so the default fuses the y and x passes per plane); the default stays in place
    # for the other tests
    energies = {}
    for v in (sponge_b200.FFT_GENERIC, sponge_b200.FFT_LINES, sponge_b200.FFT_AUTO):
        eng.pme.set_fft_variant(v)
        out[v] = _forces(eng, ("reciprocal",))
        assert rel_rms(out[v], ref["f_rec"]) < FORCE_TOL
        assert np.array_equal(_forces(eng, ("reciprocal",)), out[v])  # bit-identical repeat
        e, parts = eng.pme.Get_Energy(eng.uint_crd, eng.charge, eng.nl, eng.scaler, *eng.excl,
                                      which_part=sponge_b200.PME_TOTAL, parts=True)
        assert parts["reciprocal"] == pytest.approx(ref["e_rec"], rel=1e-5)
        energies[v] = parts["reciprocal"]
    assert rel_rms(out[sponge_b200.FFT_AUTO], out[sponge_b200.FFT_GENERIC]) < 1e-6
    # the fused plane kernel runs the same line transforms as the pass-by-pass kernels
    assert np.array_equal(out[sponge_b200.FFT_AUTO], out[sponge_b200.FFT_LINES])
    assert energies[sponge_b200.FFT_AUTO] == pytest.approx(energies[sponge_b200.FFT_LINES],
                                                           rel=1e-12)


def test_total_force(case):
    name, s, eng, ref = case
    f = _forces(eng, ("direct", "lrc", "excluded", "reciprocal"))
    err = rel_rms(f, ref["f_total"])
    print("%s total force rel RMS vs FP64: %.3e" % (name, err))
    assert err < FORCE_TOL


@pytest.mark.parametrize("ipl", [1, 2, 4, 8])
def test_energies_and_virial(case, ipl):
    name, s, eng, ref = case
    torch = eng.torch
    eng.lj.set_kernel_variant(ipl)
    eng.reset()
    eng.forces(need_energy=1, need_virial=1)
    torch.cuda.synchronize()
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    # per-part checks (FP64 reductions of FP32 per-atom terms)
    direct = float(eng.pme.d_direct_atom_energy.double().sum())
    corr = float(eng.pme.d_correction_atom_energy.double().sum())
    lj_plus_direct = float(eng.atom_energy.double().sum())
    assert direct == pytest.approx(ref["e_direct"], rel=1e-5, abs=1e-3)
    assert corr == pytest.approx(ref["e_corr"], rel=1e-5)
    assert lj_plus_direct - direct == pytest.approx(ref["e_lj"], rel=1e-5, abs=1e-3)
    lj_virial = float(eng.atom_virial.double().sum())
    assert lj_virial == pytest.approx(ref["virial_lj"], rel=1e-5, abs=1e-3)
    pot = ref["e_lj"] + ref["e_direct"] + ref["e_lrc"] + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    vir = ref["virial_lj"] + ref["virial_lrc"] + ref["e_direct"] + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    scale = abs(ref["e_self"]) + abs(ref["e_corr"])
    assert abs(eng.potential() - pot) < 2e-6 * scale + 1e-5 * abs(pot)
    assert abs(eng.virial() - vir) < 2e-6 * scale + 1e-5 * abs(vir)


def test_get_energy_parts(case):
    name, s, eng, ref = case
    import sponge_b200
    e, parts = eng.pme.Get_Energy(eng.uint_crd, eng.charge, eng.nl, eng.scaler, *eng.excl,
                                  which_part=sponge_b200.PME_TOTAL, parts=True)
    assert parts["reciprocal"] == pytest.approx(ref["e_rec"], rel=1e-5)
    assert parts["self"] == pytest.approx(ref["e_self"], rel=1e-6)
    assert parts["correction"] == pytest.approx(ref["e_corr"], rel=1e-5)
    assert parts["direct"] == pytest.approx(ref["e_direct"], rel=1e-5, abs=1e-3)
    elj = eng.lj.Get_Energy(eng.uint_crd, eng.nl)
    assert elj == pytest.approx(ref["e_lj"] + ref["e_lrc"], rel=1e-5, abs=1e-3)
    assert eng.lj.long_range_factor == pytest.approx(ref["lrc_factor"], rel=1e-6)


def test_fixed_point_forces_bit_identical(case):
    name, s, eng, ref = case
    allp = ("direct", "lrc", "excluded", "reciprocal")
    a = _forces(eng, allp, 1, 1)
    b = _forces(eng, allp, 1, 1)
    c = _forces(eng, allp, 0, 0)
    eng.update_list(forced=1)
    d = _forces(eng, allp, 0, 0)
    assert np.array_equal(a, b)
    assert np.array_equal(c, d)
    # energy/virial steps run another instantiation of the pair kernel: same forces to FP32
    # rounding, not necessarily the same bits
    assert rel_rms(a, c) < 1e-6


def test_relabelled_atoms_give_identical_forces(torch_cuda, oracle_lib):
    from sponge_b200 import NonbondedEngine
    s = systems.config0()
    n = len(s["charge"])
    rng = np.random.default_rng(11)
    perm = rng.permutation(n)  # new atom k is old atom perm[k]
    inv = np.argsort(perm)
    t = dict(s)
    t["crd"] = s["crd"][perm]
    t["charge"] = s["charge"][perm]
    t["lj_type"] = s["lj_type"][perm]
    # exclusions relabelled; each pair stored under its lower new id
    lists = [[] for _ in range(n)]
    for i in range(n):
        for j in s["excl_list"][s["excl_start"][i]:s["excl_start"][i] + s["excl_numbers"][i]]:
            a, b = inv[i], inv[j]
            lists[min(a, b)].append(max(a, b))
    t["excl_numbers"] = np.array([len(l) for l in lists], np.int32)
    t["excl_start"] = np.concatenate([[0], np.cumsum(t["excl_numbers"])[:-1]]).astype(np.int32)
    t["excl_list"] = np.array([x for l in lists for x in sorted(l)], np.int32)
    out = []
    for sysd in (s, t):
        eng = NonbondedEngine(sysd)
        eng.update_list(forced=1)
        eng.to_uint()
        out.append(_forces(eng, ("direct", "lrc", "excluded", "reciprocal")))
    assert np.array_equal(out[0][perm], out[1])


@pytest.mark.parametrize("name", ["config0", "config3"])
def test_plain_form_matches_oracle(name, torch_cuda, oracle_lib):
    from sponge_b200 import FORM_PLAIN, NonbondedEngine
    s = SYSTEMS[name]()
    eng = NonbondedEngine(s, form=FORM_PLAIN)
    eng.update_list(forced=1)
    eng.to_uint()
    torch_cuda.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.reference_energies(s, uc=uc)
    f = _forces(eng, ("direct", "lrc", "excluded", "reciprocal"), 1, 1)
    err = rel_rms(f, ref["f_total"])
    print("%s plain form total force rel RMS vs FP64: %.3e" % (name, err))
    assert err < FORCE_TOL
    assert float(eng.atom_virial.double().sum()) == pytest.approx(ref["virial_lj"], rel=1e-5)


@pytest.mark.parametrize("name", ["small", "config0", "config3"])
def test_fused_step_matches_module_sequence(name, torch_cuda, oracle_lib):
    """The fused fixed-form step (pair and exclusion forces summed in one fixed-point buffer,
    finalised by the reciprocal gather) agrees with the module-by-module sequence to float
    rounding of the final conversion, is bit-identical run to run, and meets the FP64 bar."""
    from sponge_b200 import NonbondedEngine
    s = SYSTEMS[name]()
    eng = NonbondedEngine(s, refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    a = _forces(eng, ("direct", "lrc", "excluded", "reciprocal"), 1, 1)
    pa, va = eng.potential(), eng.virial()
    runs = []
    for _ in range(2):
        eng.reset()
        eng.step(need_energy=1, need_virial=1)
        runs.append(eng.frc.cpu().numpy().astype(np.float64))
    assert np.array_equal(runs[0], runs[1])
    assert rel_rms(runs[0], a) < 1e-6
    p0, v0 = eng.potential(), eng.virial()
    assert p0 == pytest.approx(pa, rel=1e-6)
    assert v0 == pytest.approx(va, rel=1e-6)
    # the serial schedule (no side stream) gives the same bits as the overlapped default
    eng.pme.set_overlap(False)
    eng.reset()
    eng.step(need_energy=1, need_virial=1)
    assert np.array_equal(eng.frc.cpu().numpy().astype(np.float64), runs[0])
    assert eng.potential() == p0 and eng.virial() == v0
    eng.pme.set_overlap(True)
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.reference_energies(s, uc=uc)
    assert rel_rms(runs[0], ref["f_total"]) < FORCE_TOL
    # force-only steps give the same forces as energy/virial steps to float rounding
    eng.reset()
    eng.step()
    assert rel_rms(eng.frc.cpu().numpy(), runs[0]) < 1e-6


@pytest.mark.parametrize("form", ["fixed", "fixed-serial", "plain"])
def test_force_graph_replay_matches_eager_step(form, torch_cuda):
    """The force part captured once as a CUDA graph and replayed after each list update gives
    the eager step's forces (bit-identical in the fixed form, whose captured graph holds the
    side-stream branch unless the serial schedule is chosen)."""
    from sponge_b200 import FORM_FIXED, FORM_PLAIN, NonbondedEngine
    s = systems.config0()
    eng = NonbondedEngine(s, form=FORM_PLAIN if form == "plain" else FORM_FIXED,
                          refresh_interval=3)
    if form == "fixed-serial":
        eng.pme.set_overlap(False)
    eng.update_list(forced=1)
    eng.to_uint()
    eng.capture_force_graph()
    for k in range(5):  # crosses a list rebuild (every 3rd update)
        eng.crd[:30] += 0.05
        eng.to_uint()
        eng.step_graph()
        g = eng.frc.cpu().numpy().copy()
        eng.frc.zero_()
        eng.force()
        e = eng.frc.cpu().numpy()
        if form != "plain":
            assert np.array_equal(g, e), k
        else:
            assert rel_rms(g, e) < 1e-6, k


def test_refresh_policy(torch_cuda, oracle_lib):
    """refresh_interval > 0 rebuilds on calls 0, k, 2k ...; interval 0 rebuilds only when an
    atom moved more than skin/2 (neighbor_list.cu:618-664)."""
    from sponge_b200 import NonbondedEngine
    s = systems.config0()
    eng = NonbondedEngine(s, refresh_interval=3)
    eng.update_list(forced=0)  # first call always builds
    p0 = eng.nl.pair_count()
    eng.crd[:3] += 1.5  # move one water
    eng.update_list()  # call 1: no rebuild
    eng.update_list()  # call 2: no rebuild
    assert eng.nl.pair_count() == p0
    eng.update_list()  # call 3: rebuild
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(eng.crd.cpu().numpy(), s["box"]), s["box"])
    assert np.array_equal(eng.nl.export_pairs(), oracle_lib.pairs(uc, s))
    eng2 = NonbondedEngine(s, refresh_interval=0)
    eng2.update_list(forced=1)
    q0 = eng2.nl.export_pairs()
    eng2.crd[0] += 0.2  # below skin/2 = 1.0: no rebuild
    eng2.update_list()
    assert np.array_equal(eng2.nl.export_pairs(), q0)
    eng2.crd[0] += 1.2  # beyond skin/2: rebuild
    eng2.update_list()
    uc2 = oracle_lib.crd_to_uint(oracle_lib.periodic_map(eng2.crd.cpu().numpy(), s["box"]), s["box"])
    assert np.array_equal(eng2.nl.export_pairs(), oracle_lib.pairs(uc2, s))


@pytest.mark.slow
def test_config1_full_size(torch_cuda, oracle_lib):
    from sponge_b200 import NonbondedEngine
    s = systems.config1()
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    torch_cuda.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    assert eng.nl.status() == 0
    keys = eng.nl.export_pairs()
    assert np.array_equal(keys, oracle_lib.pairs(uc, s, "cells"))
    f = _forces(eng, ("direct", "lrc", "excluded", "reciprocal"))
    fr, en, _ = oracle_lib.nonbonded(uc, s, oracle_lib.get_beta(s["cutoff"]))
    err = rel_rms(f, fr)
    print("config1 total force rel RMS vs FP64: %.3e" % err)
    assert err < FORCE_TOL


@pytest.mark.parametrize("K", [30, 36, 40, 48, 50, 54, 60, 64, 80, 96, 128])
def test_plane_fft_sizes(K, torch_cuda, oracle_lib):
    """Every square plane size the fused y-x kernel serves besides 32 (config0's own grid):
    the same bits as the pass-by-pass register transforms, and the FP64 reciprocal force."""
    import sponge_b200
    from sponge_b200 import NonbondedEngine
    s = dict(systems.config0(), fft=(K, K, K))
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    out = {}
    for v in (sponge_b200.FFT_LINES, sponge_b200.FFT_AUTO):
        eng.pme.set_fft_variant(v)
        out[v] = _forces(eng, ("reciprocal",))
    assert np.array_equal(out[sponge_b200.FFT_AUTO], out[sponge_b200.FFT_LINES])
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    beta = oracle_lib.get_beta(s["cutoff"], s["tolerance"])
    f_rec = oracle_lib.pme(uc, s, beta, fft=(K, K, K))[0]
    assert rel_rms(out[sponge_b200.FFT_AUTO], f_rec) < FORCE_TOL
