"""Generates the golden fixtures of this directory by running the REFERENCE's own CUDA modules.

Run on a machine with a GPU after building the harness (make -C oracle/ref_harness):

    python tests/golden/make_golden.py

For each seeded system (sponge_b200.systems) the reference harness (oracle/ref_harness) drives
SPONGE's unchanged NEIGHBOR_LIST, LENNARD_JONES_INFORMATION and Particle_Mesh_Ewald once and
the outputs are stored compactly: forces of one evaluation (float32, as the reference writes
them), the reference's energies by part, virial and potential sums, and its pair list (in full
for the small system, as a count plus the keys within 1e-4 A^2 of the list threshold otherwise).
The systems themselves are regenerated from their seeds by the tests, so only outputs are stored.
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

CASES = {
    "small": lambda: systems.small_water(),
    "config0": systems.config0,
    "config1": systems.config1,
    "config3": systems.config3,
}


def main(names=None):
    for name in names or CASES:
        s = CASES[name]()
        uc = oracle.crd_to_uint(oracle.periodic_map(s["crd"], s["box"]), s["box"])
        keys = oracle.pairs(uc, s, "cells")
        r = refrun.run(s, uc, keys)
        ref_pairs = r["pairs"]
        out = dict(
            name=name,
            frc=r["frc"],
            frc_plain=r["frc_plain"],
            n_pairs=np.int64(ref_pairs.size),
            pairs_sha256=hashlib.sha256(np.sort(ref_pairs).tobytes()).hexdigest(),
            capacities=np.array(r["capacities"], np.int64),
        )
        if name == "small":
            out["pairs"] = ref_pairs
        else:
            # keys that differ from the oracle's pinned criterion (boundary pairs)
            out["pairs_only_ref"] = np.setdiff1d(ref_pairs, keys)
            out["pairs_only_oracle"] = np.setdiff1d(keys, ref_pairs)
        for k, v in r["summary"].items():
            out["summary_" + k] = np.float64(v)
        path = os.path.join(HERE, "reference_%s.npz" % name)
        np.savez_compressed(path, **out)
        print("wrote", path, "pairs", ref_pairs.size, "oracle", keys.size)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
