"""FP64 CPU oracle for SPONGE's nonbonded hot path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
this package. It is the checker: the product library (``sponge_b200``) never calls it and has no
CPU fallback.
"""

from .oracle import *  # noqa: F401,F403
