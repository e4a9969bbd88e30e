"""GPU parity on the reference's own real system: SPONGE's covid-tip4p protein in TIP4P water
(98,282 atoms, 19 LJ types, 196,818 exclusions, 108.4 x 91.2 x 84.4 A box, rc 10 A, skin 2 A,
PME 112 x 96 x 96; tests/golden/make_covid.py).

Checked: the pair set bit-exact against the oracle; LJ + PME forces of the fused step and of the
module calls against the FP64 oracle (relative RMS <= 1e-5) and against the forces the
reference's own CUDA modules produced on this input (tests/golden/reference_covid_tip4p.npz,
<= 2e-5: both sides are FP32 within 1e-5 of FP64); energies and virial; bit-identical repeats;
the 1-4 pairs and virtual atoms against the oracle and the reference's modules.
The grid's x size (112 = 2^4 7) has no register transform, so the generic FFT kernels run on
that axis.
"""

import importlib.util
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def _load():
    spec = importlib.util.spec_from_file_location("make_covid", os.path.join(HERE, "make_covid.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system()


@pytest.fixture(scope="module")
def covid(oracle_lib):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sponge_b200 import NonbondedEngine
    s = _load()
    eng = NonbondedEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    torch.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.reference_energies(s, uc=uc)
    golden = np.load(os.path.join(HERE, "reference_covid_tip4p.npz"))
    return s, eng, ref, golden, torch


def _forces(eng, parts, need_energy=0, need_virial=0):
    eng.reset()
    eng.forces(need_energy=need_energy, need_virial=need_virial, parts=parts)
    return eng.frc.cpu().numpy().astype(np.float64)


def test_grid_and_pairs(covid, oracle_lib):
    s, eng, ref, golden, torch = covid
    assert (eng.pme.fftx, eng.pme.ffty, eng.pme.fftz) == (112, 96, 96)
    assert eng.nl.status() == 0
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    assert np.array_equal(eng.nl.export_pairs(), oracle_lib.pairs(uc, s, "cells"))


def test_fused_step_forces(covid):
    s, eng, ref, golden, torch = covid
    runs = []
    for _ in range(2):
        eng.reset()
        eng.step(need_energy=1, need_virial=1)
        runs.append(eng.frc.cpu().numpy().astype(np.float64))
    assert np.array_equal(runs[0], runs[1])
    err = rel_rms(runs[0], ref["f_total"])
    print("covid-tip4p fused step force rel RMS vs FP64: %.3e" % err)
    assert err < 1e-5
    assert rel_rms(runs[0], golden["frc"]) < 2e-5
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    pot = ref["e_lj"] + ref["e_direct"] + ref["e_lrc"] + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    vir = ref["virial_lj"] + ref["virial_lrc"] + ref["e_direct"] + ref["e_corr"] + ref["e_self"] + ref["e_rec"]
    scale = abs(ref["e_self"]) + abs(ref["e_corr"])
    assert abs(eng.potential() - pot) < 2e-6 * scale + 1e-5 * abs(pot)
    assert abs(eng.virial() - vir) < 2e-6 * scale + 1e-5 * abs(vir)
    assert V > 0


@pytest.mark.parametrize("ipl", [2, 8])
def test_module_forces(covid, ipl):
    s, eng, ref, golden, torch = covid
    import sponge_b200
    eng.lj.set_kernel_variant(ipl)
    assert rel_rms(_forces(eng, ("direct",)), ref["f_direct"]) < 1e-5
    assert rel_rms(_forces(eng, ("excluded",)), ref["f_excl"]) < 1e-5
    for v in (sponge_b200.FFT_GENERIC, sponge_b200.FFT_AUTO):
        eng.pme.set_fft_variant(v)
        assert rel_rms(_forces(eng, ("reciprocal",)), ref["f_rec"]) < 1e-5
    f = _forces(eng, ("direct", "lrc", "excluded", "reciprocal"))
    assert rel_rms(f, ref["f_total"]) < 1e-5
    assert rel_rms(f, golden["frc"]) < 2e-5
    eng.lj.set_kernel_variant(2)


def test_plain_form(covid, oracle_lib):
    s, eng, ref, golden, torch = covid
    from sponge_b200 import FORM_PLAIN, NonbondedEngine
    pe = NonbondedEngine(s, form=FORM_PLAIN)
    pe.update_list(forced=1)
    pe.to_uint()
    f = _forces(pe, ("direct", "lrc", "excluded", "reciprocal"))
    assert rel_rms(f, ref["f_total"]) < 1e-5
    assert rel_rms(f, golden["frc"]) < 2e-5


# --- the modules beside the nonbonded path: 1-4 pairs and virtual atoms (SPONGE/main.cu:195,
# :207, :375) ----------------------------------------------------------------------------------

def _nb14_tables(s):
    from sponge_b200 import nb14_pair_tables
    return nb14_pair_tables(s["nb14_a"], s["nb14_b"], s["nb14_lj_scale"],
                            np.float32(12.0) * s["lj_A"], np.float32(6.0) * s["lj_B"],
                            s["lj_type"])


def test_nb14(covid, oracle_lib):
    s, eng, ref, golden, torch = covid
    from sponge_b200 import NonBond14
    A, B = _nb14_tables(s)
    m = NonBond14(len(s["charge"]), s["nb14_a"], s["nb14_b"], A, B, s["nb14_cf"])
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    f0, ae0, av0, elj, ecf = oracle_lib.nb14(uc, s["box"], s["charge"], s["nb14_a"],
                                             s["nb14_b"], A, B, s["nb14_cf"])
    n = len(s["charge"])
    runs = []
    for _ in range(2):
        frc = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        ae = torch.zeros(n, dtype=torch.float32, device="cuda")
        av = torch.zeros(n, dtype=torch.float32, device="cuda")
        m.Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial(eng.uint_crd, eng.charge,
                                                               eng.scaler, frc, ae, av)
        runs.append((frc.cpu().numpy().astype(np.float64), ae.cpu().numpy().astype(np.float64),
                     av.cpu().numpy().astype(np.float64)))
    assert all(np.array_equal(x, y) for x, y in zip(runs[0], runs[1]))
    f, ae, av = runs[0]
    assert rel_rms(f, f0) < 1e-6
    assert rel_rms(ae, ae0) < 1e-6
    assert rel_rms(av, av0) < 1e-6
    assert rel_rms(f[golden["nb14_atoms"]], golden["nb14_frc"]) < 1e-5
    assert m.Get_14_LJ_Energy(eng.uint_crd, eng.scaler) == pytest.approx(elj, rel=1e-6)
    assert m.Get_14_CF_Energy(eng.uint_crd, eng.charge, eng.scaler) == pytest.approx(ecf,
                                                                                      rel=1e-6)


def test_virtual_atoms(covid, oracle_lib):
    s, eng, ref, golden, torch = covid
    from sponge_b200 import VirtualAtoms
    n = len(s["charge"])
    vs = VirtualAtoms(n, s["vs_type"], s["vs_atoms"], s["vs_param"])
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    # forces: the nonbonded forces with the virtual atoms' shares moved to their parents
    frc = torch.tensor(ref["f_total"].astype(np.float32), device="cuda")
    vs.Force_Redistribute(eng.uint_crd, eng.scaler, frc)
    f = frc.cpu().numpy().astype(np.float64)
    f0 = oracle_lib.vsite(uc, s["box"], s["vs_type"], s["vs_atoms"], s["vs_param"],
                          frc=ref["f_total"].astype(np.float32).astype(np.float64))
    assert rel_rms(f, f0) < 1e-6
    assert np.all(f[s["vs_atoms"][:, 0]] == 0.0)
    fg = oracle_lib.vsite(uc, s["box"], s["vs_type"], s["vs_atoms"], s["vs_param"],
                          frc=golden["frc"].astype(np.float64))
    assert rel_rms(golden["vs_frc"], fg) < 1e-6
    # coordinates (compared modulo the box: a virtual atom sits beside its parent's image)
    crd = eng.crd.clone()
    vs.Coordinate_Refresh(eng.uint_crd, eng.scaler, crd)
    c = crd.cpu().numpy().astype(np.float64)
    c0 = oracle_lib.vsite(uc, s["box"], s["vs_type"], s["vs_atoms"], s["vs_param"],
                          crd=eng.crd.cpu().numpy().astype(np.float64))
    L = np.asarray(s["box"], np.float64)
    d = c - c0
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4
    dg = golden["vs_crd"].astype(np.float64) - c0[s["vs_atoms"][:, 0]]
    dg -= L * np.round(dg / L)
    assert np.abs(dg).max() < 1e-4
