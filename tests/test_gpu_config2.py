"""The large throughput case on the GPU: 1,000,512 atoms (333,504 waters) in a 215.3 A cube,
rc 10 A, skin 2 A, PME 216^3, in both forms (fixed-point accumulation and plain float atomics).

Checked against the FP64 oracle on the same fixed-point coordinates:
* the pair set bit-exact against the oracle's cell-list enumeration (itself equal to the
  brute-force O(N^2) one on every smaller system), with no capacity flag raised;
* total forces (LJ + Ewald direct, long-range correction, exclusion correction, SPME 216^3)
  within 1e-5 relative RMS for both forms, and the energy parts within 1e-5 relative;
* the ATOM_GROUP export (SPONGE's per-atom half list, max_neighbor_numbers per atom) holding the
  same pair set at this size;
* the reciprocal force of every FFT kernel family on grids of 100-216 points per axis.
The reference has no capacity check at max_neighbor_numbers (neighbor_list.cu:276-277) and plans
cuFFT at any size (PME_force.cu:194-195); here the list capacities raise status flags instead.
"""

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

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
    sponge_b200.lib()
    return torch


@pytest.fixture(scope="module")
def big(torch_cuda, oracle_lib):
    from sponge_b200 import NonbondedEngine
    s = systems.config2()
    assert len(s["charge"]) == 1000512
    eng = NonbondedEngine(s, refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    torch_cuda.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    beta = oracle_lib.get_beta(s["cutoff"], s["tolerance"])
    f_ref, e_ref, _ = oracle_lib.nonbonded(uc, s, beta)
    return s, eng, uc, beta, f_ref, e_ref


def test_config2_pair_set_and_capacity(big, oracle_lib):
    s, eng, uc, beta, f_ref, e_ref = big
    assert eng.nl.status() == 0
    keys = eng.nl.export_pairs()
    ref = oracle_lib.pairs(uc, s, "cells")
    assert keys.shape == ref.shape
    assert np.array_equal(keys, ref)


def test_config2_fixed_form_forces_and_energies(big):
    s, eng, uc, beta, f_ref, e_ref = big
    torch = eng.torch
    eng.reset()
    eng.forces(need_energy=1, need_virial=1)
    torch.cuda.synchronize()
    f = eng.frc.cpu().numpy()
    err = rel_rms(f, f_ref)
    print("config2 fixed form: total force rel RMS vs FP64 %.3e" % err)
    assert err < FORCE_TOL
    direct = float(eng.pme.d_direct_atom_energy.double().sum())
    corr = float(eng.pme.d_correction_atom_energy.double().sum())
    lj = float(eng.atom_energy.double().sum()) - direct
    assert direct == pytest.approx(e_ref["e_direct"], rel=1e-5)
    assert corr == pytest.approx(e_ref["e_corr"], rel=1e-5)
    assert lj == pytest.approx(e_ref["e_lj"], rel=1e-5)
    assert float(eng.atom_virial.double().sum()) == pytest.approx(e_ref["virial_lj"], rel=1e-5)
    # the fused step (overlapped reciprocal chain, pruned pair list) and its repeat
    runs = []
    for _ in range(2):
        eng.reset()
        eng.step()
        runs.append(eng.frc.cpu().numpy())
    assert np.array_equal(runs[0], runs[1])
    assert rel_rms(runs[0], f_ref) < FORCE_TOL


def test_config2_atom_group_export(big, torch_cuda):
    """SPONGE's ATOM_GROUP half list at 1 M atoms: counts and serials against the pair set."""
    s, eng, uc, beta, f_ref, e_ref = big
    from sponge_b200 import DeviceArray
    torch = torch_cuda
    n = eng.n
    addr = eng.nl.d_nl
    assert eng.nl.status() == 0
    ag = torch.as_tensor(DeviceArray(addr, (n, 2), "<i8"), device="cuda")
    counts = (ag[:, 0] & 0xffffffff).to(torch.int64)
    base = int(ag[0, 1].item())
    maxnb = eng.nl.max_neighbor_numbers
    assert int(counts.max()) <= maxnb
    serial = torch.as_tensor(DeviceArray(base, (n, maxnb), "<i4"), device="cuda")
    col = torch.arange(maxnb, device="cuda")[None, :]
    valid = col < counts[:, None]
    i = torch.arange(n, device="cuda", dtype=torch.int64)[:, None].expand(n, maxnb)
    j = serial.to(torch.int64)
    assert bool((j[valid] > i[valid]).all())
    keys = (i[valid] * n + j[valid]).sort().values.cpu().numpy()
    assert np.array_equal(keys, eng.nl.export_pairs())


def test_config2_plain_form(big, oracle_lib, torch_cuda):
    s, eng, uc, beta, f_ref, e_ref = big
    from sponge_b200 import FORM_PLAIN, NonbondedEngine
    pe = NonbondedEngine(s, form=FORM_PLAIN, refresh_interval=20)
    pe.update_list(forced=1)
    pe.to_uint()
    assert np.array_equal(pe.uint_crd.cpu().numpy().view(np.uint32), uc)
    assert pe.nl.status() == 0
    pe.reset()
    pe.forces(need_energy=0, need_virial=1)
    torch_cuda.cuda.synchronize()
    err = rel_rms(pe.frc.cpu().numpy(), f_ref)
    print("config2 plain form: total force rel RMS vs FP64 %.3e" % err)
    assert err < FORCE_TOL
    assert float(pe.atom_virial.double().sum()) == pytest.approx(e_ref["virial_lj"], rel=1e-5)
    del pe


@pytest.mark.parametrize("K", [100, 120, 144, 160, 180, 216])
def test_large_grid_reciprocal(K, torch_cuda, oracle_lib):
    """The reciprocal force on grids of 100-216 points per axis (the config-2 grid and the sizes
    Get_Fft_Patameter gives for 95-215 A boxes), every FFT kernel family, on the 3,000-atom box."""
    import sponge_b200
    from sponge_b200 import NonbondedEngine
    s = dict(systems.config0(), fft=(K, K, K))
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    beta = oracle_lib.get_beta(s["cutoff"], s["tolerance"])
    f_rec, e_rec = oracle_lib.pme(uc, s, beta, fft=(K, K, K))[:2]
    out = {}
    for v in (sponge_b200.FFT_GENERIC, sponge_b200.FFT_LINES, sponge_b200.FFT_AUTO):
        eng.pme.set_fft_variant(v)
        eng.reset()
        eng.forces(parts=("reciprocal",))
        out[v] = eng.frc.cpu().numpy().astype(np.float64)
        assert rel_rms(out[v], f_rec) < FORCE_TOL, v
        _, parts = eng.pme.Get_Energy(eng.uint_crd, eng.charge, eng.nl, eng.scaler, *eng.excl,
                                      which_part=sponge_b200.PME_TOTAL, parts=True)
        assert parts["reciprocal"] == pytest.approx(e_rec, rel=1e-5)
    assert np.array_equal(out[sponge_b200.FFT_AUTO], out[sponge_b200.FFT_LINES])
