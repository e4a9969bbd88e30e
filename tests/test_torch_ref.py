"""The FP64 torch restatement used for reference gradients, pinned to the C oracle.

* energies and forces of oracle/torch_ref.py agree with oracle.cpp (itself pinned to the
  reference's CUDA output) on the config-0 and config-3 systems; the only difference is the
  float rounding of the x12 / x6 table scaling the module (and the C oracle) applies;
* its autograd gradient of a loss on energy and forces (double backward through F = -dE/dx)
  agrees with central finite differences on a small box.
"""

import numpy as np
import pytest

from sponge_b200 import systems

torch = pytest.importorskip("torch")


def _setup(sys, oracle_lib):
    from oracle import torch_ref
    uc = oracle_lib.crd_to_uint(oracle_lib.periodic_map(sys["crd"], sys["box"]), sys["box"])
    m = torch_ref.EnergyModel(sys, uc)
    x = m.positions(uc)
    q = torch.tensor(sys["charge"].astype(np.float64))
    A = torch.tensor(sys["lj_A"].astype(np.float64))
    B = torch.tensor(sys["lj_B"].astype(np.float64))
    return uc, m, x, q, A, B


@pytest.mark.parametrize("name", ["config0", "config3"])
def test_torch_reference_matches_oracle(name, oracle_lib):
    sys = getattr(systems, name)()
    uc, m, x, q, A, B = _setup(sys, oracle_lib)
    ref = oracle_lib.reference_energies(sys, uc=uc)
    x.requires_grad_(True)
    e, parts = m.energy(x, q, A, B, parts=True)
    (g,) = torch.autograd.grad(e, x)
    F = -g.numpy()
    for k in ("e_direct", "e_corr", "e_self", "e_rec"):
        assert abs(float(parts[k].detach()) - ref[k]) <= 1e-10 * abs(ref[k]) + 1e-9, k
    # LJ terms differ only by the float rounding of A*12, B*6 in the module's tables
    for k in ("e_lj", "e_lrc"):
        assert abs(float(parts[k].detach()) - ref[k]) <= 2e-6 * abs(ref[k]), k
    err = np.sqrt(((F - ref["f_total"]) ** 2).sum() / (ref["f_total"] ** 2).sum())
    assert err < 1e-7, err


def test_torch_reference_gradient_matches_finite_differences(oracle_lib):
    sys = systems.small_water()
    uc, m, x, q, A, B = _setup(sys, oracle_lib)
    rng = np.random.default_rng(3)
    Ft = torch.tensor(rng.normal(0, 1.0, (len(sys["charge"]), 3)))

    def loss(x, q, A, B, create_graph):
        e, F = m.energy_forces(x, q, A, B, create_graph=create_graph)
        return ((F - Ft) ** 2).mean() + 0.1 * (e + 100.0) ** 2

    xs, qs, As = x.clone().requires_grad_(True), q.clone().requires_grad_(True), \
        A.clone().requires_grad_(True)
    L = loss(xs, qs, As, B, True)
    L.backward()
    h = 1e-4
    checks = [("x", (5, 1)), ("x", (17, 2)), ("q", 3), ("q", 40), ("A", 0)]
    for what, k in checks:
        step = h * (1e-3 * float(A[0]) if what == "A" else 1.0)
        vals = []
        for s in (1.0, -1.0):
            xx, qq, AA = x.clone(), q.clone(), A.clone()
            {"x": xx, "q": qq, "A": AA}[what][k] += s * step
            vals.append(float(loss(xx, qq, AA, B, False).detach()))
        fd = (vals[0] - vals[1]) / (2 * step)
        got = float({"x": xs.grad, "q": qs.grad, "A": As.grad}[what][k])
        assert abs(got - fd) <= 1e-5 * max(abs(fd), 1e-8), (what, k, got, fd)
