"""GPU parity of the FEP/TI path (soft-core LJ + PME with lambda-dependent charges) against the
FP64 oracle, on FEP boxes at several lambda values.

Tolerances: forces relative RMS <= 1e-5 against FP64; dU/dlambda and its parts within 1e-5 of
the sum of the parts' magnitudes; the fused step against the module sequence to float rounding
of the final conversion (1e-6) and bit-identical run to run; the batched step (one launch per
stage over all boxes, and the per-box graph branches) identical to the boxes stepped one at a
time.
"""

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
DUDL_TOL = 1e-5


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


BOXES = {
    "w600_l0": lambda: systems.fep_box(600, 0.0, 71),
    "w600_l04": lambda: systems.fep_box(600, 0.4, 72),
    "w900_l1": lambda: systems.fep_box(900, 1.0, 73),
    "config4_box1": lambda: systems.config4(1),
}

PART_KEYS = ("dhdl_lj", "dhdl_direct", "cross_rec", "cross_self", "cross_corr", "dhdl_lrc")


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sponge_b200
    sponge_b200.lib()
    return torch


@pytest.fixture(scope="module", params=list(BOXES))
def fep(request, cuda, oracle_lib):
    from sponge_b200.fep import FepEngine
    s = BOXES[request.param]()
    eng = FepEngine(s)
    eng.update_list(forced=1)
    eng.to_uint()
    cuda.cuda.synchronize()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.fep_reference(s, uc=uc)
    return request.param, s, eng, ref


def test_fep_step_forces_and_dudl(fep, cuda):
    name, s, eng, ref = fep
    runs = []
    for _ in range(2):
        eng.frc.zero_()
        eng.step()
        cuda.cuda.synchronize()
        runs.append((eng.frc.cpu().numpy().astype(np.float64), float(eng.dudl.item())))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1] == runs[1][1]
    err = rel_rms(runs[0][0], ref["f_total"])
    scale = sum(abs(ref[k]) for k in PART_KEYS)
    print("%s: force rel RMS %.2e, dU/dl %.6f vs %.6f (scale %.1f)" %
          (name, err, runs[0][1], ref["dU"], scale))
    assert err < FORCE_TOL
    assert abs(runs[0][1] - ref["dU"]) <= DUDL_TOL * scale


def test_dudl_parts_through_module_calls(fep):
    name, s, eng, ref = fep
    parts = eng.dudl_parts()
    scale = sum(abs(ref[k]) for k in PART_KEYS)
    for k in PART_KEYS:
        assert abs(parts[k] - ref[k]) <= DUDL_TOL * scale, (k, parts[k], ref[k])


def test_module_sequence_matches_fused_step(fep, cuda):
    name, s, eng, ref = fep
    eng.frc.zero_()
    eng.forces_modules()
    a = eng.frc.cpu().numpy().astype(np.float64)
    eng.frc.zero_()
    eng.step(want_dudl=False)
    b = eng.frc.cpu().numpy().astype(np.float64)
    assert rel_rms(a, ref["f_total"]) < FORCE_TOL
    assert rel_rms(b, a) < 1e-6


def test_soft_core_energies(fep, cuda):
    name, s, eng, ref = fep
    torch = cuda
    n = eng.n
    ae = torch.zeros(n, dtype=torch.float32, device="cuda")
    av = torch.zeros(n, dtype=torch.float32, device="cuda")
    ad = torch.zeros(n, dtype=torch.float32, device="cuda")
    eng.frc.zero_()
    eng.sc.LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
        n, eng.uint_crd, eng.charge, eng.frc, eng.nl, eng.pme.beta, 1, ae, 1, av, ad)
    e_sum = float(ae.double().sum())
    d_sum = float(ad.double().sum())
    scale = abs(ref["e_lj"]) + abs(ref["e_direct"])
    assert abs(d_sum - ref["e_direct"]) <= 1e-5 * scale
    assert abs(e_sum - ref["e_lj"] - ref["e_direct"]) <= 1e-5 * scale


@pytest.mark.parametrize("name", ["w600_l04", "config4_box1"])
def test_plain_form_matches_oracle(name, cuda, oracle_lib):
    from sponge_b200 import FORM_PLAIN
    from sponge_b200.fep import FepEngine
    s = BOXES[name]()
    eng = FepEngine(s, form=FORM_PLAIN)
    eng.update_list(forced=1)
    eng.to_uint()
    uc = eng.uint_crd.cpu().numpy().view(np.uint32)
    ref = oracle_lib.fep_reference(s, uc=uc)
    eng.frc.zero_()
    eng.forces_modules()
    assert rel_rms(eng.frc.cpu().numpy(), ref["f_total"]) < FORCE_TOL
    parts = eng.dudl_parts()
    scale = sum(abs(ref[k]) for k in PART_KEYS)
    for k in ("dhdl_lj", "dhdl_direct", "dhdl_lrc"):
        assert abs(parts[k] - ref[k]) <= DUDL_TOL * scale, (k, parts[k], ref[k])


def _batch_boxes():
    # three boxes share the 30^3 grid (one batched FFT group of plane kernels), the 2600-water
    # box runs the pass-by-pass register transforms (a batched group without the plane kernel)
    # and the 1700-water box the generic stage kernels (its own FFT launches); the last box has
    # too many perturbed atoms for the split form and runs the soft-core cluster kernel
    many = systems.fep_box(500, 0.3, 106)
    many["mask"] = np.asarray(many["mask"]).copy()
    many["mask"][:300] = 1  # 280 water atoms join the 20 solute atoms in the perturbed group
    return [systems.fep_box(n, lam, 100 + k) for k, (n, lam) in
            enumerate([(500, 0.0), (1700, 0.2), (800, 0.5), (2600, 0.8), (650, 1.0)])] + [many]


def test_split_form_chosen(cuda):
    from sponge_b200.fep import FepEngine
    boxes = _batch_boxes()
    assert FepEngine(boxes[0]).sc.split_form == (True, 20)
    split, npert = FepEngine(boxes[-1]).sc.split_form
    assert not split and npert == 300


@pytest.mark.parametrize("mode", ["kernels", "streams"])
def test_batched_graph_matches_single_boxes(cuda, mode):
    import sponge_b200
    from sponge_b200.fep import FepBatch
    batch = FepBatch(_batch_boxes(), mode=mode)
    batch.engines[1].pme.set_fft_variant(sponge_b200.FFT_GENERIC)
    batch.engines[3].pme.set_fft_variant(sponge_b200.FFT_LINES)
    batch.rebuild()
    # one box at a time, eagerly
    for e in batch.engines:
        e.frc.zero_()
        e.step()
    cuda.cuda.synchronize()
    single = [(e.frc.cpu().numpy().copy(), float(e.dudl.item())) for e in batch.engines]
    counts = (1, 2, 5)
    if mode == "kernels":
        best = batch.tune(candidates=(2, 1), reps=2)
        assert best[0] in (1, 2)
        counts = (2, 1)
        batch.capture(1)
        # the force clear, pack, spread, gather, finalize, self sums, dU/dlambda; the packed
        # pair kernel and the soft-core search and evaluation of the split boxes, the soft-core
        # cluster kernel of the other; the FFTs: 3 for the plane group, 5 for the pass-by-pass
        # group, 5 for the generic box
        assert batch.launches == 7 + 4 + 3 + 5 + 5, batch.launches
    else:
        best = batch.tune(candidates=(1, 2, 5), reps=2)
        assert best[0] in (1, 2, 5)
    for n in counts:  # sub-batches (kernels) or streams (per-box branches)
        batch.capture(n)
        for rep in range(2):  # the replay leaves every accumulator clear for the next one
            if rep:
                batch.rebuild()  # the captured rebuild of all lists: the same lists again
            batch.graph.replay()
            cuda.cuda.synchronize()
            for e, (f, d) in zip(batch.engines, single):
                assert np.array_equal(e.frc.cpu().numpy(), f), n
                assert float(e.dudl.item()) == d, n


def test_batch_refuses_changed_box(cuda):
    import sponge_b200
    from sponge_b200 import FepBatchStep
    from sponge_b200.fep import FepEngine
    engines = [FepEngine(s) for s in _batch_boxes()[:2]]
    for e in engines:
        e.update_list(forced=1)
        e.to_uint()
    dudl = cuda.zeros(2, dtype=cuda.float64, device="cuda")
    b = FepBatchStep([(e.nl, e.sc, e.pme, e.uint_crd, e.charge, e.excl, e.frc, dudl[k:k + 1])
                      for k, e in enumerate(engines)])
    b.step()
    cuda.cuda.synchronize()
    assert float(dudl[0].item()) != 0.0
    engines[1].sc.set_lambda(0.7)
    with pytest.raises(sponge_b200.SpongeError, match="create the batch again"):
        b.step()


def test_batch_beyond_one_pair_launch(cuda):
    """98 windows: the packed pair kernel carries at most 96 windows' descriptors per launch, so
    the batch issues two; every window still gets the bits of its own step."""
    from sponge_b200.fep import FepBatch
    boxes = [systems.fep_box(500, k / 97.0, 300 + k) for k in range(98)]
    batch = FepBatch(boxes)
    batch.rebuild()
    for e in batch.engines:
        e.frc.zero_()
        e.step()
    cuda.cuda.synchronize()
    single = [(e.frc.cpu().numpy().copy(), float(e.dudl.item())) for e in batch.engines]
    batch.capture(1)
    # the force clear, pack, spread, gather, finalize, self sums, dU/dlambda; two packed pair
    # launches; the soft-core search and evaluation; the three FFT stages of the one grid size
    assert batch.launches == 7 + 2 + 2 + 3, batch.launches
    batch.graph.replay()
    cuda.cuda.synchronize()
    for e, (f, d) in zip(batch.engines, single):
        assert np.array_equal(e.frc.cpu().numpy(), f)
        assert float(e.dudl.item()) == d


def test_batch_forces_only(cuda):
    """Without dU/dlambda outputs the batch runs the force-only kernels: the forces are the
    bits of each window's own force-only step; a batch asking dU/dlambda of only some windows is
    refused."""
    import sponge_b200
    from sponge_b200 import FepBatchStep
    from sponge_b200.fep import FepEngine
    engines = [FepEngine(s) for s in _batch_boxes()[:3] + _batch_boxes()[-1:]]
    for e in engines:
        e.update_list(forced=1)
        e.to_uint()
    single = []
    for e in engines:
        e.frc.zero_()
        e.step(want_dudl=False)
        cuda.cuda.synchronize()
        single.append(e.frc.cpu().numpy().copy())
    b = FepBatchStep([(e.nl, e.sc, e.pme, e.uint_crd, e.charge, e.excl, e.frc, None)
                      for e in engines])
    for e in engines:
        e.frc.zero_()
    b.step()
    cuda.cuda.synchronize()
    for e, f in zip(engines, single):
        assert np.array_equal(e.frc.cpu().numpy(), f)
    with pytest.raises(sponge_b200.SpongeError):
        FepBatchStep([(e.nl, e.sc, e.pme, e.uint_crd, e.charge, e.excl, e.frc,
                       e.dudl if k == 0 else None) for k, e in enumerate(engines)])
