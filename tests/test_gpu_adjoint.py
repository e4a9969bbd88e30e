"""GPU parity of the adjoint kernels on the force-field fitting workload (config-3 system).

Loss over 16 seeded configurations c:
    L = 1/16 sum_c [ mean((F_c - F*_c)^2) + 0.1 (E_c - E*_c)^2 ]
with targets E*, F* from the same system evaluated with per-type sigma/epsilon and per-atom
charges perturbed by 5% Gaussian noise. Gradients with respect to positions, per-atom charges
and per-type sigma/epsilon come from the adjoint torch.autograd.Function in FP32 (CUDA kernels
through the C ABI). They are checked against
  * the FP64 reference gradient (oracle/torch_ref.py, autograd through the forces) over all 16
    configurations: relative L2 error <= 1e-4 per parameter group;
  * central finite differences (step 1e-4) of the FP64 loss for a seeded sample of parameters
    (loss over the first 4 configurations): relative L2 error <= 1e-4 per group.
Types with epsilon = 0 (water H) carry no LJ gradient and are left out of the sigma/epsilon
groups.
"""

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
FD_STEP = 1e-4
E_WEIGHT = 0.1


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def fit(oracle_lib):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sponge_b200
    sponge_b200.lib()
    from sponge_b200.adjoint import NonbondedModel, lj_tables
    s, frames, target = systems.config3_fit()
    model = NonbondedModel(s)
    sig_t = torch.tensor(target["lj_sigma"], dtype=torch.float64)
    eps_t = torch.tensor(target["lj_eps"], dtype=torch.float64)
    At, Bt = lj_tables(sig_t, eps_t)
    qt = torch.tensor(target["charge"], device="cuda")
    tgt = []
    with torch.no_grad():
        for c in frames:
            E, F = model(torch.tensor(c, device="cuda"), qt, At.float(), Bt.float())
            tgt.append((float(E.item()), F.detach().clone()))
    # fixed-point coordinates of each frame, as the modules quantise them
    uc = [oracle_lib.crd_to_uint(oracle_lib.periodic_map(c, s["box"]), s["box"]) for c in frames]
    fitted = np.array([t for t in range(s["n_types"]) if s["lj_eps"][t] > 0])
    return dict(torch=torch, s=s, frames=frames, target=tgt, model=model, uc=uc, fitted=fitted)


def gpu_grads(fit, idx):
    torch = fit["torch"]
    from sponge_b200.adjoint import lj_tables
    s = fit["s"]
    model = fit["model"]
    sig = torch.tensor(s["lj_sigma"], dtype=torch.float64, requires_grad=True)
    eps = torch.tensor(s["lj_eps"], dtype=torch.float64, requires_grad=True)
    q = torch.tensor(s["charge"], device="cuda", requires_grad=True)
    A, B = lj_tables(sig, eps)
    crds = []
    L = 0.0
    for c in idx:
        x = torch.tensor(fit["frames"][c], device="cuda", requires_grad=True)
        crds.append(x)
        E, F = model(x, q, A.float(), B.float())
        Et, Ft = fit["target"][c]
        L = L + ((F - Ft) ** 2).mean() + E_WEIGHT * (E - Et) ** 2
    L = L / len(idx)
    L.backward()
    return dict(L=float(L.item()), x=[t.grad.detach().cpu().numpy() for t in crds],
                q=q.grad.detach().cpu().numpy(), sig=sig.grad.numpy(), eps=eps.grad.numpy())


class RefLoss:
    """FP64 torch loss over a set of configurations (the same targets as the GPU loss)."""

    def __init__(self, fit, idx):
        import oracle.torch_ref as tr
        torch = fit["torch"]
        self.torch = torch
        self.fit = fit
        self.idx = list(idx)
        s = fit["s"]
        self.models = {c: tr.EnergyModel(s, fit["uc"][c]) for c in self.idx}
        self.x0 = {c: self.models[c].positions(fit["uc"][c]) for c in self.idx}
        self.tgt = {c: (fit["target"][c][0],
                        fit["target"][c][1].detach().cpu().double()) for c in self.idx}

    def params(self):
        torch = self.torch
        s = self.fit["s"]
        return dict(sig=torch.tensor(s["lj_sigma"], dtype=torch.float64),
                    eps=torch.tensor(s["lj_eps"], dtype=torch.float64),
                    q=torch.tensor(s["charge"].astype(np.float64)),
                    x={c: self.x0[c].clone() for c in self.idx})

    def loss(self, p, create_graph=False, frames=None):
        from sponge_b200.adjoint import lj_tables
        A, B = lj_tables(p["sig"], p["eps"])
        L = 0.0
        for c in (frames if frames is not None else self.idx):
            E, F = self.models[c].energy_forces(p["x"][c], p["q"], A, B,
                                                create_graph=create_graph)
            Et, Ft = self.tgt[c]
            L = L + ((F - Ft) ** 2).mean() + E_WEIGHT * (E - Et) ** 2
        return L / len(self.idx)


def test_adjoint_matches_fp64_reference_gradient(fit):
    idx = list(range(len(fit["frames"])))
    g = gpu_grads(fit, idx)
    ref = RefLoss(fit, idx)
    p = ref.params()
    for k in ("sig", "eps", "q"):
        p[k].requires_grad_(True)
    for c in idx:
        p["x"][c].requires_grad_(True)
    L = ref.loss(p, create_graph=True)
    L.backward()
    Lr = float(L.detach())
    assert abs(g["L"] - Lr) <= 1e-4 * abs(Lr)
    f = fit["fitted"]
    errs = {
        "positions": rel_l2(np.concatenate([a.ravel() for a in g["x"]]),
                            np.concatenate([p["x"][c].grad.numpy().ravel() for c in idx])),
        "charges": rel_l2(g["q"], p["q"].grad.numpy()),
        "sigma": rel_l2(g["sig"][f], p["sig"].grad.numpy()[f]),
        "epsilon": rel_l2(g["eps"][f], p["eps"].grad.numpy()[f]),
    }
    print("adjoint vs FP64 reference gradient (rel L2):", errs)
    for k, v in errs.items():
        assert v <= GRAD_TOL, (k, v)


def test_adjoint_matches_central_finite_differences(fit):
    idx = [0, 1, 2, 3]
    g = gpu_grads(fit, idx)
    ref = RefLoss(fit, idx)
    rng = np.random.default_rng(31)
    n = len(fit["s"]["charge"])
    f = fit["fitted"]
    picks = {
        "positions": [(int(a), int(d)) for a, d in zip(rng.choice(n, 4, replace=False),
                                                        rng.integers(0, 3, 4))],
        "charges": [int(a) for a in rng.choice(n, 4, replace=False)],
        "sigma": [int(t) for t in rng.choice(f, 4, replace=False)],
        "epsilon": [int(t) for t in rng.choice(f, 4, replace=False)],
    }

    def fd(mutate, frames=None):
        vals = []
        for sgn in (1.0, -1.0):
            p = ref.params()
            mutate(p, sgn * FD_STEP)
            vals.append(float(ref.loss(p, frames=frames).detach()))
        return (vals[0] - vals[1]) / (2 * FD_STEP)

    errs = {}
    got, want = [], []
    for a, d in picks["positions"]:
        def m(p, h, a=a, d=d):
            p["x"][0][a, d] += h
        want.append(fd(m, frames=[0]))
        got.append(g["x"][0][a, d])
    errs["positions"] = rel_l2(got, want)
    for key, pk in (("charges", "q"), ("sigma", "sig"), ("epsilon", "eps")):
        got, want = [], []
        for t in picks[key]:
            def m(p, h, t=t, pk=pk):
                p[pk][t] += h
            want.append(fd(m))
            got.append(g[pk][t])
        errs[key] = rel_l2(got, want)
    print("adjoint vs central finite differences (rel L2):", errs)
    for k, v in errs.items():
        assert v <= GRAD_TOL, (k, v)


def test_adjoint_zero_cotangent_and_linearity(fit):
    """dL/dp is linear in the cotangents: g(2 gE, 2 gF) = 2 g(gE, gF); zero cotangents give zero."""
    torch = fit["torch"]
    model = fit["model"]
    s = fit["s"]
    from sponge_b200.adjoint import lj_tables
    A, B = lj_tables(torch.tensor(s["lj_sigma"]), torch.tensor(s["lj_eps"]))
    x = torch.tensor(fit["frames"][0], device="cuda")
    q = torch.tensor(s["charge"], device="cuda")
    model._forward(x, q, A.float(), B.float())
    gen = torch.Generator(device="cuda").manual_seed(5)
    gF = torch.randn((model.n, 3), device="cuda", generator=gen)
    g1 = [t.cpu().numpy() for t in model._backward(torch.tensor(0.7), gF)]
    g2 = [t.cpu().numpy() for t in model._backward(torch.tensor(1.4), 2 * gF)]
    g0 = [t.cpu().numpy() for t in model._backward(torch.tensor(0.0), torch.zeros_like(gF))]
    for a, b, z in zip(g1, g2, g0):
        assert np.allclose(2 * a, b, rtol=1e-5, atol=1e-7 * np.abs(b).max())
        assert np.abs(z).max() == 0.0
