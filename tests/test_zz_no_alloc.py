"""GPU test of sb_pme_get_energy_noalloc, the allocation-free PME energy query.

sb_pme_get_energy allocates (and frees) a throwaway force array on every call. Callers that
cannot allocate device memory at that point -- a host program whose GPU memory is all owned by
its own pool allocator, or a tight driver loop that cannot afford cudaFree's device-wide wait --
use sb_pme_get_energy_noalloc, which takes that array from a fixed block of the library's device
memory (up to 131072 atoms). This file checks, through the C ABI, that it returns the same energy
parts as sb_pme_get_energy on two calls in a row (energies within 1e-5 relative, the energy
tolerance of the other GPU tests), that further calls leave the device's free memory unchanged,
and that it refuses what it cannot do without allocating. It is collected last so that a run
stopping at the first failure has already run every other test; it creates its own modules and
passes alone or after the other tests.
"""

import ctypes

import numpy as np
import pytest

from sponge_b200 import systems

pytestmark = pytest.mark.gpu

ENERGY_TOL = 1e-5
MAX_ATOMS = 131072


def _parts(fn, eng, which):
    from sponge_b200 import _box3, _ptr, _stream
    e = ctypes.c_float()
    p = (ctypes.c_double * 5)()
    st = fn(eng.pme.handle, eng.nl.handle, _ptr(eng.uint_crd), _ptr(eng.charge),
            _box3(eng.scaler), _ptr(eng.excl_start), _ptr(eng.excl_list), _ptr(eng.excl_numbers),
            int(which), ctypes.byref(e), p, _stream(None))
    return st, e.value, np.array(list(p))


@pytest.fixture(scope="module")
def engine():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sponge_b200
    sponge_b200.lib()
    from sponge_b200 import NonbondedEngine
    eng = NonbondedEngine(systems.config0())
    eng.update_list(forced=1)
    eng.to_uint()
    torch.cuda.synchronize()
    return eng


def test_noalloc_energy_matches_allocating_query(engine):
    import sponge_b200
    L = sponge_b200.lib()
    eng = engine
    eng.nl.d_nl  # the DIRECT part reads the list's ATOM_GROUP export: materialise it once
    for which in range(5):
        st, e_ref, p_ref = _parts(L.sb_pme_get_energy, eng, which)
        assert st == 0, L.sb_last_error()
        for call in range(2):  # two calls in a row share the same static block
            st, e, p = _parts(L.sb_pme_get_energy_noalloc, eng, which)
            assert st == 0, L.sb_last_error()
            assert abs(e - e_ref) <= ENERGY_TOL * max(abs(e_ref), 1e-30), (which, call, e, e_ref)
            nz = p_ref != 0
            assert np.all(np.abs(p[nz] - p_ref[nz]) <= ENERGY_TOL * np.abs(p_ref[nz])), \
                (which, call, p, p_ref)
            assert np.all(p[~nz] == 0), (which, call, p)


def test_noalloc_leaves_device_memory_unchanged(engine):
    """The property the entry point exists for: after its first call on the device, further
    calls take no device memory (free memory as the driver reports it does not move)."""
    import torch
    import sponge_b200
    from sponge_b200 import PME_TOTAL
    L = sponge_b200.lib()
    eng = engine
    eng.nl.d_nl
    st, _, _ = _parts(L.sb_pme_get_energy_noalloc, eng, PME_TOTAL)
    assert st == 0, L.sb_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        st, _, _ = _parts(L.sb_pme_get_energy_noalloc, eng, PME_TOTAL)
        assert st == 0, L.sb_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_refuses_what_would_allocate():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sponge_b200
    from sponge_b200 import PME_DIRECT, PME_RECIPROCAL, NonbondedEngine, ParticleMeshEwald
    L = sponge_b200.lib()
    # a fresh list has no ATOM_GROUP export yet: DIRECT must be refused, not allocated
    eng = NonbondedEngine(systems.small_water())
    eng.update_list(forced=1)
    eng.to_uint()
    st, _, _ = _parts(L.sb_pme_get_energy_noalloc, eng, PME_DIRECT)
    assert st == 5 and b"sb_nl_atom_group" in L.sb_last_error()
    # more atoms than the static block holds
    big = ParticleMeshEwald(MAX_ATOMS + 1, eng.box, 5.0, 1e-5, (16, 16, 16))
    from sponge_b200 import _box3, _ptr, _stream
    st = L.sb_pme_get_energy_noalloc(big.handle, None, _ptr(eng.uint_crd), _ptr(eng.charge),
                                     _box3(eng.scaler), None, None, None, PME_RECIPROCAL, None,
                                     None, _stream(None))
    assert st == 1 and b"maximum" in L.sb_last_error()
    big.Clear()
    # a list of another system (another atom count) is refused before any launch
    other = NonbondedEngine(systems.small_water(n_side=3))
    other.update_list(forced=1)
    other.nl.d_nl
    st = L.sb_pme_get_energy_noalloc(eng.pme.handle, other.nl.handle, _ptr(eng.uint_crd),
                                     _ptr(eng.charge), _box3(eng.scaler), None, None, None,
                                     PME_DIRECT, None, None, _stream(None))
    assert st == 1 and b"holds" in L.sb_last_error()
