"""Generates the soft-core golden fixtures of this directory by running the REFERENCE's own CUDA
modules: LJ_SOFT_CORE (SPONGE/Lennard_Jones_force/LJ_soft_core.cu) over the reference's
NEIGHBOR_LIST, and TI_CORE's PME cross terms (SPONGE/TI_core/TI_core.cu:670-730) over the
reference's Particle_Mesh_Ewald, through oracle/ref_harness/sc_harness.cu.

Run on a machine with a GPU after building the harness (make -C oracle/ref_harness):

    python tests/golden/make_golden_fep.py

One FEP box (600 waters + a 20-atom solute that vanishes in lambda, soft core alpha 0.5, p 1,
sigma 3 A; sponge_b200.systems.fep_box, regenerated from its seed by the tests) at lambda 0, 0.4
and 1: the soft-core force with energy and virial requested (float32, as the reference writes
it), its per-atom energy / LJ virial / direct Coulomb energy, the energies and dH/dlambda parts
the reference prints, and its pair list as a count plus the keys that differ from the oracle's.
"""

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle.ref_harness import run as refrun  # noqa: E402
from sponge_b200 import systems  # noqa: E402

N_WATER = 600
SEED = 1004077
LAMBDAS = (0.0, 0.4, 1.0)


def case(lam):
    return systems.fep_box(N_WATER, lam, SEED, name="fep_w%d_l%g" % (N_WATER, lam))


def path_for(lam):
    return os.path.join(HERE, "reference_fep_l%s.npz" % ("%g" % lam).replace(".", "p"))


def main():
    for lam in LAMBDAS:
        s = case(lam)
        uc = oracle.crd_to_uint(oracle.periodic_map(s["crd"], s["box"]), s["box"])
        keys = oracle.pairs(uc, s, "cells")
        r = refrun.run_softcore(s, uc, keys)
        ref_pairs = r["pairs"]
        out = dict(
            lam=np.float64(lam), frc=r["frc"], ae=r["ae"], av=r["av"], adir=r["adir"],
            n_pairs=np.int64(ref_pairs.size),
            pairs_sha256=hashlib.sha256(np.sort(ref_pairs).tobytes()).hexdigest(),
            pairs_only_ref=np.setdiff1d(ref_pairs, keys),
            pairs_only_oracle=np.setdiff1d(keys, ref_pairs),
            capacities=np.array(r["capacities"], np.int64))
        for k, v in r["summary"].items():
            out["summary_" + k] = np.float64(v)
        np.savez_compressed(path_for(lam), **out)
        print("wrote", path_for(lam), "pairs", ref_pairs.size, "oracle", keys.size)


if __name__ == "__main__":
    main()
