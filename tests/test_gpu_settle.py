"""GPU parity of the NVE leap-frog + SETTLE step (sb_md_leap_frog, sb_settle_*, the fused
sb_md_nve_settle_step) against the FP64 oracle and the reference's modules.

Water box (3,000 atoms, rigid TIP3P-like waters, forces of the LJ + PME evaluation, 300 K
velocities): the fused step equals the three module calls bit for bit; coordinates, velocities
and the constraint pressure follow the oracle; every constrained distance is restored.
covid-tip4p (98,282 atoms): 21,389 waters, 2,408 isolated rigid pairs and 3,698 constraint pairs
SETTLE leaves to another scheme; the module calls follow the oracle and the reference's own
CONSTRAIN + SETTLE outputs on the same forces; the fused step refuses the system (it would skip
the remaining pairs).
"""

import importlib.util
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _helpers():
    spec = importlib.util.spec_from_file_location("tso", os.path.join(HERE,
                                                                      "test_settle_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


H = _helpers()


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def _scaler(box):
    # MD_INFORMATION's uint_dr_to_dr_cof as the reference computes it: 1 / (2^32 / box)
    box = np.asarray(box, np.float32)
    return np.float32(1.0) / (np.float32(4294967296.0) / box)


class Case:
    def __init__(self, torch, box, pairs, mass, vel, crd, uc, frc, dt):
        self.t = torch
        self.box = np.asarray(box, np.float32)
        self.pairs = pairs
        self.mass = np.asarray(mass, np.float32)
        self.n = self.mass.size
        self.dt = dt
        m64 = self.mass.astype(np.float64)
        inv = np.divide(1.0, m64, out=np.zeros_like(m64), where=m64 != 0).astype(np.float32)
        dev = lambda x: torch.tensor(np.ascontiguousarray(x), device="cuda")  # noqa: E731
        self.vel0, self.crd0 = dev(np.asarray(vel, np.float32)), dev(np.asarray(crd, np.float32))
        self.uc = dev(np.ascontiguousarray(uc, np.uint32).view(np.int32))
        self.frc = dev(np.asarray(frc, np.float32))
        self.inv, self.mass_t = dev(inv), dev(self.mass)

    def module_calls(self, settle):
        from sponge_b200 import md_leap_frog
        t = self.t
        vel, crd = self.vel0.clone(), self.crd0.clone()
        acc = t.zeros_like(vel)
        p = t.zeros(1, dtype=t.float32, device="cuda")
        settle.Remember_Last_Coordinates(self.uc, _scaler(self.box))
        md_leap_frog(self.n, self.inv, self.frc, vel, crd, self.dt, acc=acc)
        settle.Do_SETTLE(self.mass_t, crd, self.box, vel, 1, p)
        t.cuda.synchronize()
        return [x.cpu().numpy() for x in (crd, vel, acc, p)]

    def fused(self, settle):
        t = self.t
        vel, crd = self.vel0.clone(), self.crd0.clone()
        acc = t.zeros_like(vel)
        p = t.zeros(1, dtype=t.float32, device="cuda")
        settle.nve_step(self.uc, _scaler(self.box), self.inv, self.mass_t, self.frc, vel, crd,
                        self.box, acc=acc, need_pressure=1, pressure=p)
        t.cuda.synchronize()
        return [x.cpu().numpy() for x in (crd, vel, acc, p)]


def _wrapped_err(a, b, box):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    L = np.asarray(box, np.float64)
    d -= L * np.round(d / L)
    return np.abs(d).max()


def _rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.fixture(scope="module")
def water(torch, oracle_lib):
    s, pairs, mass, vel, crd, uc, frc = H.water_case(oracle_lib)
    return s, Case(torch, s["box"], pairs, mass, vel, crd, uc, frc, H.DT), (vel, crd, uc, frc)


def test_water_fused_equals_module_calls(water):
    from sponge_b200 import Settle
    s, case, _ = water
    pi, pj, pr = case.pairs
    st = Settle(case.n, pi, pj, pr, case.mass, case.dt)
    assert (st.triangle_numbers, st.pair_numbers, st.remaining_pairs) == (case.n // 3, 0, 0)
    a = case.module_calls(st)
    b = case.fused(st)
    c = case.module_calls(st)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, z)
        assert np.array_equal(x, y)


def test_water_matches_oracle(water, oracle_lib):
    from sponge_b200 import Settle
    s, case, (vel, crd, uc, frc) = water
    pi, pj, pr = case.pairs
    st = Settle(case.n, pi, pj, pr, case.mass, case.dt)
    c, v, acc, p = case.module_calls(st)
    c0, v0, a0, vir, nt, npair = oracle_lib.nve_settle(uc, s["box"], pi, pj, pr, case.mass,
                                                       case.dt, frc, crd, vel)
    ec, ev = _wrapped_err(c, c0, s["box"]), _rel_rms(v, v0)
    print("water SETTLE: crd max err %.3e A, vel rel RMS %.3e" % (ec, ev))
    # FP32 SETTLE: the velocity correction is a coordinate difference over dt, so its error is
    # the coordinates' FP32 rounding over dt (the reference's own, on covid-tip4p: 7.9e-5)
    assert ec < 5e-5
    assert ev < 1e-4
    assert _rel_rms(acc, a0) < 1e-6
    d = H.distances(c.astype(np.float64), s["box"], pi, pj)
    assert np.abs(d - pr).max() < 5e-5
    # the pressure is a sum of per-constraint virials that largely cancel: FP32 terms give a
    # few 1e-5 relative on the sum
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    assert float(p[0]) == pytest.approx(vir * float(np.float32(0.33333)) / V, rel=1e-4)


@pytest.fixture(scope="module")
def covid(torch, oracle_lib):
    s = H._covid()
    from sponge_b200 import constrain_pairs_from_bonds
    pairs = constrain_pairs_from_bonds(s["bond_a"], s["bond_b"], s["bond_r"], s["mass"])
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(s["crd"], s["box"]), s["box"])
    golden = np.load(os.path.join(HERE, "golden", "reference_covid_tip4p.npz"))
    frc = golden["vs_frc"]
    case = Case(torch, s["box"], pairs, s["mass"], s["vel"], s["crd"], uc, frc,
                float(s["md_dt"]))
    return s, case, golden, uc


def test_covid_module_calls(covid, oracle_lib):
    from sponge_b200 import Settle, SpongeError
    s, case, golden, uc = covid
    pi, pj, pr = case.pairs
    st = Settle(case.n, pi, pj, pr, case.mass, case.dt)
    assert (st.triangle_numbers, st.pair_numbers, st.remaining_pairs) == (21389, 2408, 3698)
    c, v, acc, p = case.module_calls(st)
    assert all(np.array_equal(x, y) for x, y in zip((c, v, acc, p), case.module_calls(st)))
    c0, v0, a0, vir, nt, npair = oracle_lib.nve_settle(uc, s["box"], pi, pj, pr, case.mass,
                                                       case.dt, golden["vs_frc"], s["crd"],
                                                       s["vel"])
    ec, ev = _wrapped_err(c, c0, s["box"]), _rel_rms(v, v0)
    print("covid SETTLE: crd max err %.3e A, vel rel RMS %.3e" % (ec, ev))
    assert ec < 5e-5
    assert ev < 1e-4
    V = float(np.prod(np.asarray(s["box"], np.float64)))
    assert float(p[0]) == pytest.approx(vir * float(np.float32(0.33333)) / V, rel=1e-4)
    if "settle_crd" in golden.files:
        atoms = golden["settle_atoms"]
        eg = _wrapped_err(c[atoms], golden["settle_crd"], s["box"])
        vg = _rel_rms(v[atoms], golden["settle_vel"])
        print("covid SETTLE vs reference: crd %.3e A, vel rel RMS %.3e" % (eg, vg))
        assert eg < 5e-5
        assert vg < 2e-4
        assert float(p[0]) == pytest.approx(float(golden["summary_settle_pressure"]), rel=1e-4)
    with pytest.raises(SpongeError):
        case.fused(st)


def test_md_step_graph_matches_eager(torch, oracle_lib):
    """The NVE step (force, then the fused leap-frog + SETTLE launch) captured in one CUDA graph
    behind the force part gives the eager step's bits, through list rebuilds (every 3 steps) and
    the pruned list's renewals; the rigid waters keep their geometry."""
    from sponge_b200 import NonbondedEngine, Settle, constrain_pairs_from_bonds, sponge_io
    from sponge_b200 import systems as sysmod
    s = sysmod.config0()
    a, b, r, mass = sponge_io.bonds_and_masses(s)
    pi, pj, pr = constrain_pairs_from_bonds(a, b, r, mass)
    n = len(mass)
    dt = float(np.float32(np.float32(0.0005) * np.float32(20.455)))
    m64 = mass.astype(np.float64)
    inv = torch.tensor(np.divide(1.0, m64, out=np.zeros_like(m64), where=m64 != 0)
                       .astype(np.float32), device="cuda")
    m_t = torch.tensor(mass, device="cuda")
    engines, vels, settles = [], [], []
    for _ in range(2):
        eng = NonbondedEngine(s, refresh_interval=3)
        eng.update_list(forced=1)
        vel = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        st = Settle(n, pi, pj, pr, mass, dt)
        eng.md_step(st, inv, m_t, vel)
        engines.append(eng)
        vels.append(vel)
        settles.append(st)
    eager, graphed = engines
    graphed.capture_md_graph(settles[1], inv, m_t, vels[1])
    for _ in range(7):
        eager.update_list()
        eager.md_step(settles[0], inv, m_t, vels[0])
        graphed.md_step_graph()
    torch.cuda.synchronize()
    assert np.array_equal(eager.crd.cpu().numpy(), graphed.crd.cpu().numpy())
    assert np.array_equal(vels[0].cpu().numpy(), vels[1].cpu().numpy())
    c = graphed.crd.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(c))
    d = H.distances(c, s["box"], pi, pj)
    assert np.abs(d - pr).max() < 5e-5
