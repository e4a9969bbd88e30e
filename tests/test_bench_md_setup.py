"""The bench's MD set-up on the CPU: the degrees of freedom its thermostat targets.

The equilibration rescales the velocities to 0.5 * ndof * kB * T; for the 96,000-atom box
(31,000 rigid waters, three distance constraints each) that is 194,997 degrees of freedom, for
the 1,000,512-atom box (333,504 rigid waters) 2,001,021. The constraint pairs are counted from
the systems' own bonds, as the bench counts them.
"""

import numpy as np

import bench
from sponge_b200 import constrain_pairs_from_bonds, sponge_io, systems


def test_degrees_of_freedom_formula():
    assert bench.md_degrees_of_freedom(3, 3) == 3            # one rigid water
    assert bench.md_degrees_of_freedom(96000, 93000) == 194997
    assert bench.md_degrees_of_freedom(1000512, 1000512) == 2001021


def test_constraints_of_the_bench_box():
    s = systems.config1()
    ba, bb, br, mass = sponge_io.bonds_and_masses(s)
    pi, pj, pr = constrain_pairs_from_bonds(ba, bb, br, mass)
    assert len(pi) == 93000  # three per rigid water
    ndof = bench.md_degrees_of_freedom(len(np.asarray(s["charge"])), len(pi))
    assert ndof == 194997
