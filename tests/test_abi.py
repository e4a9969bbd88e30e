"""The C-ABI library loads on a machine without a GPU and exports every declared symbol."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sponge_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"SB_API\s+(?:const\s+char\s*\*|int)\s+(sb_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    from sponge_b200 import build
    return build.build()


def test_header_declares_the_module_api():
    names = declared_symbols()
    for must in ("sb_nl_create", "sb_nl_update", "sb_lj_pme_direct_force",
                 "sb_pme_reciprocal_force", "sb_pme_excluded_force", "sb_pme_get_energy",
                 "sb_nonbonded_step", "sb_nl_atom_group"):
        assert must in names


def test_library_exports_every_declared_symbol(libpath):
    L = ctypes.CDLL(libpath)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_no_undeclared_exports(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True)
    exported = {l.split()[-1] for l in out.stdout.splitlines() if " T " in l}
    sb = {e for e in exported if e.startswith("sb_")}
    assert sb == set(declared_symbols())


def test_version_and_error_without_gpu(libpath):
    L = ctypes.CDLL(libpath)
    assert L.sb_version() >= 100
    L.sb_last_error.restype = ctypes.c_char_p
    # argument validation happens before any device work
    L.sb_nl_create.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                               ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                               ctypes.c_void_p]
    assert L.sb_nl_create(0, None, 10.0, 2.0, 0, 0.5, 800, 0, None) == 1
    assert b"invalid" in L.sb_last_error()


def test_python_mirror_refuses_without_cuda():
    import torch
    import sponge_b200
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sponge_b200.SpongeError):
        sponge_b200.NeighborList(10, [10, 10, 10], 3.0, 1.0)
