"""Box changes: the barostat path of SPONGE's MD driver on the GPU modules.

Main_Volume_Change / Main_Box_Length_Change (SPONGE/main.cu:438-460) scale the coordinates, then
call NEIGHBOR_LIST::Update_Volume (neighbor_list.cu:645-656) and Neighbor_List_Update,
LENNARD_JONES_INFORMATION::Update_Volume (Lennard_Jones_force.cu:1450) and
Particle_Mesh_Ewald::Update_Volume / Update_Box_Length (PME_force.cu:996-1042);
Main_Volume_Change_Largely (main.cu:462-471) clears the list and PME modules and initialises them
again. After each, the forces, energies and virial are checked against the FP64 oracle evaluated
from scratch at the new box (relative RMS force error <= 1e-5, energy parts <= 1e-5 relative),
and the pair set bit-exact against the brute-force enumeration at the new box.
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
    sponge_b200.lib()
    return torch


def _scaled(s, factor):
    """The system after a barostat move: coordinates and box scaled by ``factor`` (per axis)."""
    f = np.asarray(factor, np.float32).reshape(1, 3)
    t = dict(s)
    t["box"] = (np.asarray(s["box"], np.float32) * f[0]).astype(np.float32)
    t["crd"] = (np.asarray(s["crd"], np.float32) * f).astype(np.float32)
    return t


def _check_against_oracle(eng, t, oracle_lib, parts_checked=True):
    torch = eng.torch
    eng.update_list()
    eng.to_uint()
    eng.reset()
    eng.forces(need_energy=1, need_virial=1)
    torch.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    assert eng.nl.status() == 0
    assert np.array_equal(eng.nl.export_pairs(), oracle_lib.pairs(uc, t, "brute"))
    ref = oracle_lib.reference_energies(t, uc=uc)
    f = eng.frc.cpu().numpy()
    err = rel_rms(f, ref["f_total"])
    assert err < FORCE_TOL, err
    pot = (ref["e_lj"] + ref["e_direct"] + ref["e_lrc"] + ref["e_corr"] + ref["e_self"] +
           ref["e_rec"])
    vir = (ref["virial_lj"] + ref["virial_lrc"] + ref["e_direct"] + ref["e_corr"] +
           ref["e_self"] + ref["e_rec"])
    scale = abs(ref["e_self"]) + abs(ref["e_corr"])
    assert abs(eng.potential() - pot) < 2e-6 * scale + 1e-5 * abs(pot)
    assert abs(eng.virial() - vir) < 2e-6 * scale + 1e-5 * abs(vir)
    if parts_checked:
        import sponge_b200
        _, parts = eng.pme.Get_Energy(eng.uint_crd, eng.charge, eng.nl, eng.scaler, *eng.excl,
                                      which_part=sponge_b200.PME_TOTAL, parts=True)
        assert parts["reciprocal"] == pytest.approx(ref["e_rec"], rel=1e-5)
        assert parts["self"] == pytest.approx(ref["e_self"], rel=1e-6)
        assert eng.lj.Get_Energy(eng.uint_crd, eng.nl) == pytest.approx(
            ref["e_lj"] + ref["e_lrc"], rel=1e-5, abs=1e-3)
    return f, err


@pytest.mark.parametrize("factor", [1.02, 0.98, (1.03, 0.99, 1.01)])
@pytest.mark.parametrize("form", ["fixed", "plain"])
def test_box_change_matches_oracle_at_new_box(factor, form, torch_cuda, oracle_lib):
    from sponge_b200 import FORM_FIXED, FORM_PLAIN, NonbondedEngine
    s = systems.config0()
    eng = NonbondedEngine(s, form=FORM_FIXED if form == "fixed" else FORM_PLAIN,
                          refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    eng.forces()
    t = _scaled(s, np.broadcast_to(np.asarray(factor, np.float32), (3,)))
    # the caller scales its coordinates (Scale_List / Scale_Coordinate_Atomically), then the
    # modules take the new box
    eng.crd.copy_(torch_cuda.tensor(t["crd"], device="cuda"))
    eng.update_box(t["box"])
    _check_against_oracle(eng, t, oracle_lib)


def test_box_change_in_fused_step_and_graph(torch_cuda, oracle_lib):
    """The fused step (sb_nonbonded_step) and a captured force graph after a box change: the
    graph captured at the old box is captured again, and gives the eager step's bits."""
    from sponge_b200 import NonbondedEngine
    s = systems.config0()
    eng = NonbondedEngine(s, refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    eng.capture_force_graph()
    eng.step_graph()
    t = _scaled(s, np.full(3, 0.985, np.float32))
    eng.crd.copy_(torch_cuda.tensor(t["crd"], device="cuda"))
    eng.update_box(t["box"])
    eng.to_uint()
    eng.step_graph()  # rebuilds the list (box changed) and captures the graph again
    g = eng.frc.cpu().numpy().copy()
    eng.reset()
    eng.step()
    e = eng.frc.cpu().numpy()
    assert np.array_equal(g, e)
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.reference_energies(t, uc=uc)
    assert rel_rms(e, ref["f_total"]) < FORCE_TOL


def test_repeated_box_moves_and_back(torch_cuda, oracle_lib):
    """A Monte Carlo barostat's rejected move scales by f and then by 1/f (main.cu:240-275):
    after the pair of moves the modules give the original forces to float rounding."""
    from sponge_b200 import NonbondedEngine
    s = systems.config0()
    eng = NonbondedEngine(s, refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    eng.reset()
    eng.forces()
    f0 = eng.frc.cpu().numpy().copy()
    crd0 = eng.crd.clone()
    box0 = np.asarray(s["box"], np.float32)
    for f in (1.015, 0.99, 1.005):
        t = _scaled(s, np.full(3, f, np.float32))
        eng.crd.copy_(torch_cuda.tensor(t["crd"], device="cuda"))
        eng.update_box(t["box"])
        _check_against_oracle(eng, t, oracle_lib, parts_checked=False)
    eng.crd.copy_(crd0)
    eng.update_box(box0)
    eng.update_list()
    eng.to_uint()
    eng.reset()
    eng.forces()
    assert np.array_equal(eng.frc.cpu().numpy(), f0)


def test_clear_and_initial_again(torch_cuda, oracle_lib):
    """Main_Volume_Change_Largely: the list and PME modules are cleared and initialised again at
    the new box; the LJ module only takes the new volume."""
    from sponge_b200 import NeighborList, NonbondedEngine, ParticleMeshEwald
    s = systems.config0()
    eng = NonbondedEngine(s, refresh_interval=20)
    eng.update_list(forced=1)
    eng.to_uint()
    eng.forces()
    t = _scaled(s, np.full(3, 1.12, np.float32))
    eng.crd.copy_(torch_cuda.tensor(t["crd"], device="cuda"))
    eng.update_box(t["box"])
    eng.nl.Clear()
    eng.pme.Clear()
    eng.nl = NeighborList(eng.n, t["box"], t["cutoff"], t["skin"], 20, max_neighbor_numbers=1200)
    eng.nl.set_prune(0.5, 5)
    eng.pme = ParticleMeshEwald(eng.n, t["box"], t["cutoff"], t["tolerance"], t["fft"])
    eng.update_list(forced=1)
    _check_against_oracle(eng, t, oracle_lib)
