"""The pruned pair list (sb_nl_set_prune) on the GPU.

The packed pair kernel walks only the entries with a pair within cutoff + buffer at the last
prune, each with its mask reduced to the slots within that radius and the entries of a cluster
sorted by the slot pairs they use (a batch skips the slot pairs none of its entries uses).
Checked on the 3,000-atom water box (rc 8 A, skin 2 A, buffer 0.5 A):

* at the coordinates of the build, the pruned walk evaluates the same pairs as the full walk:
  forces agree per atom to FP32 rounding of the i-atom sums (a single missing pair near the
  cut-off would move its atoms' forces by ~1e-4 of the RMS force), energies to 1e-6;
* a launch that prunes and one that walks the list an earlier launch pruned give the same bits;
* after every atom moves by up to 0.2 A (below half the buffer, no new prune) and then by up to
  0.6 A (above it: the coordinate packing requests a prune), with the full list kept, the forces
  still match the full walk and the FP64 oracle at the new coordinates, although pairs that were
  beyond cutoff + buffer at the last prune are now inside the cut-off.
"""

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = pytest.mark.gpu

ALL = ("direct", "lrc", "excluded", "reciprocal")


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def _forces(eng, need_energy=0, need_virial=0):
    eng.reset()
    eng.forces(need_energy=need_energy, need_virial=need_virial, parts=ALL)
    return eng.frc.cpu().numpy().astype(np.float64)


def _max_rel(a, b):
    """Largest per-atom force difference over the RMS force."""
    d = np.sqrt(((a - b) ** 2).sum(1)).max()
    return float(d / np.sqrt((b ** 2).sum(1).mean()))


def _pair(s, buffer):
    from sponge_b200 import NonbondedEngine
    eng = NonbondedEngine(s, prune_buffer=buffer, prune_interval=0)
    eng.update_list(forced=1)
    eng.to_uint()
    return eng


def test_pruned_walk_matches_full_walk(torch):
    s = systems.config0()
    full, pruned = _pair(s, 0.0), _pair(s, 0.5)
    fa = _forces(full, 1, 1)
    fb = _forces(pruned, 1, 1)   # this launch prunes
    fc = _forces(pruned, 1, 1)   # this one walks the list the previous launch built
    assert np.array_equal(fb, fc)
    err = _max_rel(fb, fa)
    print("pruned vs full walk: max per-atom difference / RMS force %.2e" % err)
    assert err < 1e-5
    assert pruned.potential() == pytest.approx(full.potential(), rel=1e-6)
    assert pruned.virial() == pytest.approx(full.virial(), rel=1e-6)
    f0 = _forces(pruned)
    assert np.array_equal(f0, _forces(pruned))


def test_moved_atoms_keep_every_pair(torch, oracle_lib):
    s = systems.config0()
    full, pruned = _pair(s, 0.0), _pair(s, 0.5)
    _forces(pruned)  # prune at the build coordinates
    x0 = full.crd.cpu().numpy().astype(np.float64)
    box = np.asarray(s["box"], np.float64)
    rng = np.random.default_rng(5)
    n = x0.shape[0]
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    frac = rng.uniform(0.0, 1.0, size=(n, 1)) ** (1.0 / 3.0)
    rc, rb = float(s["cutoff"]), float(s["cutoff"]) + 0.5
    for amp in (0.2, 0.6):
        x1 = np.mod(x0 + amp * frac * u, box).astype(np.float32)
        x1 = np.where(x1 >= box.astype(np.float32), np.float32(0.0), x1)
        for eng in (full, pruned):
            eng.crd.copy_(torch.from_numpy(x1))
            eng.to_uint()
        uc = pruned.uint_crd.cpu().numpy().view(np.uint32)
        t = dict(s, crd=x1)
        keys = oracle_lib.pairs(uc, t, "cells")
        i, j = keys // n, keys % n

        def dist(x):
            d = x[j] - x[i]
            d -= box * np.round(d / box)
            return np.sqrt((d ** 2).sum(1))
        entered = int(((dist(x1.astype(np.float64)) < rc) & (dist(x0) > rb)).sum())
        fa = _forces(full)
        fb = _forces(pruned)
        err = _max_rel(fb, fa)
        ref = oracle_lib.reference_energies(t, uc=uc)["f_total"]
        rms = float(np.sqrt(((fb - ref) ** 2).sum() / (ref ** 2).sum()))
        print("moved up to %.1f A: %d pairs entered from beyond rc + buffer; max per-atom "
              "difference / RMS force %.2e; rel RMS vs FP64 %.2e" % (amp, entered, err, rms))
        if amp > 0.5:
            assert entered > 0
        else:
            assert entered == 0
        assert err < 1e-5
        assert rms < 1e-5
