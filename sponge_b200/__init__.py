"""sponge_b200: B200-native nonbonded hot path of SPONGE behind its module API.

Python mirror of the three SPONGE module structs, calling the C ABI of libsponge_b200.so
(include/sponge_b200.h) with torch CUDA tensors as device memory:

* ``NeighborList``      <- NEIGHBOR_LIST              (SPONGE/neighbor_list/neighbor_list.cuh:44-106)
* ``LennardJones``      <- LENNARD_JONES_INFORMATION  (SPONGE/Lennard_Jones_force/Lennard_Jones_force.cuh:41-149)
* ``ParticleMeshEwald`` <- Particle_Mesh_Ewald        (SPONGE/PME_force/PME_force.cuh:25-123)

Method names, argument meaning and accumulation semantics (+= into forces, per-atom energies
and the single-float virial/potential) are the reference's. There is no CPU path: every call
needs the compiled library and a CUDA device, and fails loudly otherwise.

Coordinates in fixed point are held in torch.int32 tensors carrying the uint32 bit pattern
(torch has no general uint32 arithmetic); shape [N, 3].
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libsponge_b200.so")
_LIB = None

FORM_FIXED = 0
FORM_PLAIN = 1

PME_TOTAL, PME_DIRECT, PME_RECIPROCAL, PME_CORRECTION, PME_SELF = range(5)

FFT_AUTO, FFT_GENERIC, FFT_LINES = range(3)

STATUS_LIST_OVERFLOW = 1
STATUS_COLUMN_OVERFLOW = 2
STATUS_ATOMGROUP_OVERFLOW = 4

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float

# name -> argtypes (restype int unless stated)
_SIGS = {
    "sb_version": [],
    "sb_last_error": [],
    "sb_nl_create": [_i, _vp, _f, _f, _i, _f, _i, _i, _vp],
    "sb_nl_destroy": [_vp],
    "sb_nl_update": [_vp, _vp, _vp, _vp, _vp, _i, _i, _vp],
    "sb_nl_update_volume": [_vp, _vp],
    "sb_nl_atom_group": [_vp, _vp, _vp],
    "sb_nl_pair_count": [_vp, _vp, _vp],
    "sb_nl_export_pairs": [_vp, _vp, ctypes.c_int64, _vp, _vp],
    "sb_nl_status": [_vp, _vp, _vp],
    "sb_nl_set_prune": [_vp, _f, _i],
    "sb_nl_uint_crd": [_vp, _vp],
    "sb_lj_create": [_i, _i, _vp, _vp, _vp, _f, _vp, _i, _vp],
    "sb_lj_destroy": [_vp],
    "sb_lj_pme_direct_force": [_vp, _vp, _i, _vp, _vp, _vp, _f, _i, _vp, _i, _vp, _vp, _vp],
    "sb_lj_long_range_correction": [_vp, _i, _vp, _i, _vp, _vp],
    "sb_lj_get_energy": [_vp, _vp, _vp, _vp, _vp],
    "sb_lj_update_volume": [_vp, _vp],
    "sb_lj_long_range_factor": [_vp, _vp],
    "sb_lj_set_kernel_variant": [_vp, _i],
    "sb_lj_tune": [_vp, _vp, _vp, _vp, _f, _vp, _vp],
    "sb_pme_create": [_i, _vp, _f, _f, _i, _i, _i, _i, _vp],
    "sb_pme_destroy": [_vp],
    "sb_pme_info": [_vp, _vp, _vp],
    "sb_pme_set_fft_variant": [_vp, _i],
    "sb_nonbonded_set_overlap": [_vp, _i],
    "sb_pme_atom_energy_arrays": [_vp, _vp, _vp],
    "sb_pme_excluded_force": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_pme_reciprocal_force": [_vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp],
    "sb_pme_get_energy": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp],
    "sb_pme_get_energy_noalloc": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp],
    "sb_pme_update_box": [_vp, _vp],
    "sb_pme_bc_table": [_vp, _vp],
    "sb_nonbonded_step": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp,
                          _vp, _vp, _vp],
    "sb_crd_to_uint_crd": [_i, _vp, _vp, _vp, _vp],
    "sb_nonbonded_force": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp,
                           _vp, _vp],
    "sb_lj_set_tables": [_vp, _vp, _vp],
    "sb_adjoint_create": [_vp, _vp, _vp, _vp],
    "sb_adjoint_destroy": [_vp],
    "sb_adjoint_backward": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp,
                            _vp, _vp, _vp, _vp],
    "sb_sc_create": [_i, _i, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _f, _vp, _f, _f, _f,
                     _f, _f, _i, _vp],
    "sb_sc_destroy": [_vp],
    "sb_sc_set_lambda": [_vp, _f],
    "sb_sc_pme_direct_force": [_vp, _vp, _i, _vp, _vp, _vp, _f, _i, _vp, _i, _vp, _vp, _vp],
    "sb_sc_long_range_correction": [_vp, _i, _vp, _i, _vp, _vp],
    "sb_sc_dh_dlambda": [_vp, _vp, _vp, _vp, _f, _vp, _vp],
    "sb_pme_ti_cross": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_fep_step": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_sc_split_form": [_vp, _vp, _vp],
    "sb_fep_batch_create": [_i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_fep_batch_step": [_vp, _vp],
    "sb_fep_batch_launches": [_vp],
    "sb_fep_batch_destroy": [_vp],
    "sb_nb14_create": [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_nb14_destroy": [_vp],
    "sb_nb14_force": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_nb14_energy": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "sb_vsite_create": [_i, _i, _vp, _vp, _vp, _vp],
    "sb_vsite_destroy": [_vp],
    "sb_vsite_coordinate_refresh": [_vp, _vp, _vp, _vp, _vp],
    "sb_vsite_force_redistribute": [_vp, _vp, _vp, _vp, _vp],
    "sb_settle_create": [_i, _i, _vp, _vp, _vp, _vp, _f, _f, _vp],
    "sb_settle_destroy": [_vp],
    "sb_settle_info": [_vp, _vp, _vp, _vp],
    "sb_settle_remember": [_vp, _vp, _vp, _vp],
    "sb_settle_apply": [_vp, _vp, _vp, _vp, _vp, _i, _vp, _vp],
    "sb_md_leap_frog": [_i, _vp, _vp, _vp, _vp, _vp, _f, _vp],
    "sb_md_nve_settle_step": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp],
}


class SpongeError(RuntimeError):
    pass


def library_path():
    return _LIBPATH


def lib():
    """Load libsponge_b200.so (built in-tree by ``python -m sponge_b200.build``)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIBPATH):
            raise SpongeError("libsponge_b200.so is not built: run `python -m sponge_b200.build`")
        L = ctypes.CDLL(_LIBPATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.sb_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def _check(status):
    if status != 0:
        msg = lib().sb_last_error()
        raise SpongeError("sponge_b200 error %d: %s" % (status, msg.decode() if msg else ""))


def _require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise SpongeError("sponge_b200 needs a CUDA device; there is no CPU path")
    return torch


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise SpongeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise SpongeError("expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream if isinstance(stream, int) else stream.cuda_stream


def _box3(box):
    return (ctypes.c_float * 3)(*[float(v) for v in np.broadcast_to(np.asarray(box, np.float64), 3)])


class DeviceArray:
    """Zero-copy view of library-owned device memory (``torch.as_tensor(x, device='cuda')``)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


def crd_to_uint_crd(crd, box, out=None, stream=None):
    """Crd_To_Uint_Crd with the quarter coefficient (SPONGE/common.cu:264-287)."""
    torch = _require_cuda()
    n = crd.shape[0]
    if out is None:
        out = torch.empty((n, 3), dtype=torch.int32, device=crd.device)
    _check(lib().sb_crd_to_uint_crd(n, _box3(box), _ptr(crd), _ptr(out), _stream(stream)))
    return out


class NeighborList:
    """NEIGHBOR_LIST. ``Neighbor_List_Update`` wraps ``crd`` into the box in place on rebuilds."""

    CONDITIONAL_UPDATE, FORCED_UPDATE = 0, 1
    CONDITIONAL_CHECK, FORCED_CHECK = 0, 1

    def __init__(self, atom_numbers, box_length, cutoff, skin, refresh_interval=0,
                 skin_permit=0.5, max_neighbor_numbers=800, form=FORM_FIXED):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        self.cutoff, self.skin = float(cutoff), float(skin)
        self.box_length = np.asarray(box_length, np.float32)
        self.max_neighbor_numbers = int(max_neighbor_numbers)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_nl_create(self.atom_numbers, _box3(box_length), self.cutoff, self.skin,
                                  int(refresh_interval), float(skin_permit),
                                  self.max_neighbor_numbers, int(form), ctypes.byref(self.handle)))

    def Neighbor_List_Update(self, crd, excluded_list_start=None, excluded_list=None,
                             excluded_numbers=None, forced_update=0, forced_check=0, stream=None):
        _check(lib().sb_nl_update(self.handle, _ptr(crd), _ptr(excluded_list_start),
                                  _ptr(excluded_list), _ptr(excluded_numbers), int(forced_update),
                                  int(forced_check), _stream(stream)))

    def Update_Volume(self, box_length):
        self.box_length = np.asarray(box_length, np.float32)
        _check(lib().sb_nl_update_volume(self.handle, _box3(box_length)))

    @property
    def d_nl(self):
        """Device address of the ATOM_GROUP[N] compatibility list (materialised on demand)."""
        p = ctypes.c_void_p()
        _check(lib().sb_nl_atom_group(self.handle, ctypes.byref(p), _stream(None)))
        return p.value

    def pair_count(self):
        c = ctypes.c_int64()
        _check(lib().sb_nl_pair_count(self.handle, ctypes.byref(c), _stream(None)))
        return c.value

    def export_pairs(self):
        """Half pair set as sorted int64 keys i*N + j (i < j)."""
        n = self.pair_count()
        keys = np.empty(max(n, 1), np.int64)
        c = ctypes.c_int64()
        _check(lib().sb_nl_export_pairs(self.handle, keys.ctypes.data, n, ctypes.byref(c),
                                        _stream(None)))
        return keys[:c.value]

    def status(self):
        f = ctypes.c_int()
        _check(lib().sb_nl_status(self.handle, ctypes.byref(f), _stream(None)))
        return f.value

    def set_prune(self, prune_buffer, prune_interval=0):
        """Pruned pair list for the packed pair kernel (sb_nl_set_prune; 0 turns it off)."""
        _check(lib().sb_nl_set_prune(self.handle, float(prune_buffer), int(prune_interval)))

    def uint_crd(self):
        torch = _require_cuda()
        p = ctypes.c_void_p()
        _check(lib().sb_nl_uint_crd(self.handle, ctypes.byref(p)))
        return torch.as_tensor(DeviceArray(p.value, (self.atom_numbers, 3), "<i4"), device="cuda")

    def Clear(self):
        if self.handle:
            lib().sb_nl_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


class LennardJones:
    """LENNARD_JONES_INFORMATION. ``LJ_A``/``LJ_B`` are the lower-triangular tables already
    multiplied by 12 and 6 (h_LJ_A / h_LJ_B of the reference)."""

    def __init__(self, atom_numbers, atom_type_numbers, LJ_A, LJ_B, atom_LJ_type, cutoff,
                 box_length, form=FORM_FIXED):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        self.atom_type_numbers = int(atom_type_numbers)
        self.h_LJ_A = np.ascontiguousarray(LJ_A, np.float32)
        self.h_LJ_B = np.ascontiguousarray(LJ_B, np.float32)
        self.h_atom_LJ_type = np.ascontiguousarray(atom_LJ_type, np.int32)
        self.cutoff = float(cutoff)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_lj_create(self.atom_numbers, self.atom_type_numbers,
                                  self.h_LJ_A.ctypes.data, self.h_LJ_B.ctypes.data,
                                  self.h_atom_LJ_type.ctypes.data, self.cutoff,
                                  _box3(box_length), int(form), ctypes.byref(self.handle)))

    @property
    def long_range_factor(self):
        f = ctypes.c_float()
        _check(lib().sb_lj_long_range_factor(self.handle, ctypes.byref(f)))
        return f.value

    def LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(self, atom_numbers, uint_crd, charge, frc,
                                                        nl, pme_beta, need_atom_energy=0,
                                                        atom_energy=None, need_virial=0,
                                                        atom_lj_virial=None,
                                                        atom_direct_pme_energy=None,
                                                        stream=None):
        _check(lib().sb_lj_pme_direct_force(self.handle, nl.handle, int(atom_numbers),
                                            _ptr(uint_crd), _ptr(charge), _ptr(frc),
                                            float(pme_beta), int(need_atom_energy),
                                            _ptr(atom_energy), int(need_virial),
                                            _ptr(atom_lj_virial), _ptr(atom_direct_pme_energy),
                                            _stream(stream)))

    def Long_Range_Correction(self, need_pressure, d_virial, need_potential, d_potential,
                              stream=None):
        _check(lib().sb_lj_long_range_correction(self.handle, int(need_pressure), _ptr(d_virial),
                                                 int(need_potential), _ptr(d_potential),
                                                 _stream(stream)))

    def Get_Energy(self, uint_crd, nl, stream=None):
        e = ctypes.c_float()
        _check(lib().sb_lj_get_energy(self.handle, nl.handle, _ptr(uint_crd), ctypes.byref(e),
                                      _stream(stream)))
        return e.value

    def Update_Volume(self, box_length):
        _check(lib().sb_lj_update_volume(self.handle, _box3(box_length)))

    def set_kernel_variant(self, atoms_per_lane):
        """Pair-kernel shape: 8 or 4 i atoms per lane, 2 for eight atoms per lane on packed
        FP32x2 slot pairs (the default), or 1 for the compacted kernel (one in-cutoff pair per
        lane); a tuning knob with the same results to FP32 rounding."""
        _check(lib().sb_lj_set_kernel_variant(self.handle, int(atoms_per_lane)))

    def tune(self, nl, uint_crd, charge, pme_beta, stream=None):
        """Time each pair-kernel shape on the current list and keep the fastest."""
        c = ctypes.c_int()
        _check(lib().sb_lj_tune(self.handle, nl.handle, _ptr(uint_crd), _ptr(charge),
                                float(pme_beta), ctypes.byref(c), _stream(stream)))
        return c.value

    def Clear(self):
        if self.handle:
            lib().sb_lj_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


class ParticleMeshEwald:
    """Particle_Mesh_Ewald. ``fft`` entries <= 0 pick the size as Get_Fft_Patameter does."""

    TOTAL, DIRECT, RECIPROCAL, CORRECTION, SELF = range(5)

    def __init__(self, atom_numbers, box_length, cutoff, tolerance=1e-5, fft=(-1, -1, -1),
                 form=FORM_FIXED):
        torch = _require_cuda()
        self.atom_numbers = int(atom_numbers)
        self.box_length = np.asarray(box_length, np.float32)
        self.handle = ctypes.c_void_p()
        f = [int(v) if v is not None else -1 for v in (fft if fft is not None else (-1, -1, -1))]
        _check(lib().sb_pme_create(self.atom_numbers, _box3(box_length), float(cutoff),
                                   float(tolerance), f[0], f[1], f[2], int(form),
                                   ctypes.byref(self.handle)))
        b = ctypes.c_float()
        k = (ctypes.c_int * 3)()
        _check(lib().sb_pme_info(self.handle, ctypes.byref(b), k))
        self.beta = b.value
        self.fftx, self.ffty, self.fftz = k[0], k[1], k[2]
        pd, pc = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().sb_pme_atom_energy_arrays(self.handle, ctypes.byref(pd), ctypes.byref(pc)))
        self.d_direct_atom_energy = torch.as_tensor(
            DeviceArray(pd.value, (self.atom_numbers,), "<f4"), device="cuda")
        self.d_correction_atom_energy = torch.as_tensor(
            DeviceArray(pc.value, (self.atom_numbers,), "<f4"), device="cuda")

    def scaler(self):
        return (np.float32(1.0) / np.float32(4294967296.0)) * self.box_length

    def set_fft_variant(self, variant):
        """FFT kernel family of the fixed-point form: FFT_AUTO (register line transforms where
        the axis size has one, with the y and x passes fused per kz plane for square planes; the
        default), FFT_LINES (the register transforms pass by pass: the same bits as FFT_AUTO) or
        FFT_GENERIC (stage kernels only); a fixed rule, same results to FP32 rounding.
        Synchronises."""
        _check(lib().sb_pme_set_fft_variant(self.handle, int(variant)))

    def set_overlap(self, on):
        """Fixed-form fused force: run the exclusion correction and the reciprocal grid chain on
        a side stream concurrently with the pair kernel (default on; same forces either way)."""
        _check(lib().sb_nonbonded_set_overlap(self.handle, int(bool(on))))

    def PME_Excluded_Force_With_Atom_Energy(self, uint_crd, scaler, charge, excluded_list_start,
                                            excluded_list, excluded_numbers, frc, atom_energy,
                                            stream=None):
        _check(lib().sb_pme_excluded_force(self.handle, _ptr(uint_crd), _box3(scaler),
                                           _ptr(charge), _ptr(excluded_list_start),
                                           _ptr(excluded_list), _ptr(excluded_numbers),
                                           _ptr(frc), _ptr(atom_energy), _stream(stream)))

    def PME_Reciprocal_Force_With_Energy_And_Virial(self, uint_crd, charge, force, need_virial=0,
                                                    need_energy=0, d_virial=None,
                                                    d_potential=None, stream=None):
        _check(lib().sb_pme_reciprocal_force(self.handle, _ptr(uint_crd), _ptr(charge),
                                             _ptr(force), int(need_virial), int(need_energy),
                                             _ptr(d_virial), _ptr(d_potential), _stream(stream)))

    def Get_Energy(self, uint_crd, charge, nl, scaler, excluded_list_start, excluded_list,
                   excluded_numbers, which_part=0, parts=False, stream=None):
        e = ctypes.c_float()
        p = (ctypes.c_double * 5)()
        _check(lib().sb_pme_get_energy(self.handle, nl.handle if nl is not None else None,
                                       _ptr(uint_crd), _ptr(charge), _box3(scaler),
                                       _ptr(excluded_list_start), _ptr(excluded_list),
                                       _ptr(excluded_numbers), int(which_part), ctypes.byref(e),
                                       p, _stream(stream)))
        if parts:
            return e.value, dict(zip(("total", "direct", "reciprocal", "correction", "self"),
                                     list(p)))
        return e.value

    def Update_Box_Length(self, box_length):
        self.box_length = np.asarray(box_length, np.float32)
        _check(lib().sb_pme_update_box(self.handle, _box3(box_length)))

    Update_Volume = Update_Box_Length

    def Clear(self):
        if self.handle:
            lib().sb_pme_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


def nonbonded_step(nl, lj, pme, crd, uint_crd, charge, excl, frc, need_energy=0, need_virial=0,
                   atom_energy=None, atom_virial=None, d_virial=None, d_potential=None,
                   stream=None):
    """One MD step's nonbonded forces through the fused C entry point (sb_nonbonded_step)."""
    es, el, en = excl
    _check(lib().sb_nonbonded_step(nl.handle, lj.handle, pme.handle, _ptr(crd), _ptr(uint_crd),
                                   _ptr(charge), _ptr(es), _ptr(el), _ptr(en), _ptr(frc),
                                   int(need_energy), int(need_virial), _ptr(atom_energy),
                                   _ptr(atom_virial), _ptr(d_virial), _ptr(d_potential),
                                   _stream(stream)))


def nonbonded_force(nl, lj, pme, uint_crd, charge, excl, frc, need_energy=0, need_virial=0,
                    atom_energy=None, atom_virial=None, d_virial=None, d_potential=None,
                    stream=None):
    """The force part of a step with the list as it stands (sb_nonbonded_force); capturable
    in a CUDA graph."""
    es, el, en = excl
    _check(lib().sb_nonbonded_force(nl.handle, lj.handle, pme.handle, _ptr(uint_crd),
                                    _ptr(charge), _ptr(es), _ptr(el), _ptr(en), _ptr(frc),
                                    int(need_energy), int(need_virial), _ptr(atom_energy),
                                    _ptr(atom_virial), _ptr(d_virial), _ptr(d_potential),
                                    _stream(stream)))


from .engine import NonbondedEngine  # noqa: E402,F401


class SoftCore:
    """LJ_SOFT_CORE (SPONGE/Lennard_Jones_force/LJ_soft_core.cuh:42-159). Tables are the
    lower-triangular A/B coefficients of each end state already multiplied by 12 and 6."""

    def __init__(self, atom_numbers, LJ_AA, LJ_AB, LJ_BA, LJ_BB, atom_LJ_type_A, atom_LJ_type_B,
                 mask, charge_B_A, cutoff, box_length, lambda_lj, alpha=0.5, p=1.0, sigma=3.0,
                 sigma_min=0.0, form=FORM_FIXED, n_types_A=None, n_types_B=None):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        f32, i32 = np.float32, np.int32
        self.h = [np.ascontiguousarray(x, t) for x, t in
                  ((LJ_AA, f32), (LJ_AB, f32), (LJ_BA, f32), (LJ_BB, f32),
                   (atom_LJ_type_A, i32), (atom_LJ_type_B, i32), (mask, i32), (charge_B_A, f32))]
        ntA = int(n_types_A) if n_types_A is not None else int(self.h[4].max()) + 1
        ntB = int(n_types_B) if n_types_B is not None else int(self.h[5].max()) + 1
        self.lambda_lj = float(lambda_lj)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_sc_create(self.atom_numbers, ntA, self.h[0].ctypes.data,
                                  self.h[1].ctypes.data, ntB, self.h[2].ctypes.data,
                                  self.h[3].ctypes.data, self.h[4].ctypes.data,
                                  self.h[5].ctypes.data, self.h[6].ctypes.data,
                                  self.h[7].ctypes.data, float(cutoff), _box3(box_length),
                                  self.lambda_lj, float(alpha), float(p), float(sigma),
                                  float(sigma_min), int(form), ctypes.byref(self.handle)))

    @property
    def split_form(self):
        """(uses the split form, perturbed atom count) of the fused FEP step."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib().sb_sc_split_form(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return bool(a.value), int(b.value)

    def set_lambda(self, lambda_lj):
        self.lambda_lj = float(lambda_lj)
        _check(lib().sb_sc_set_lambda(self.handle, self.lambda_lj))

    def LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
            self, atom_numbers, uint_crd, charge, frc, nl, pme_beta, need_atom_energy=0,
            atom_energy=None, need_virial=0, atom_lj_virial=None, atom_direct_pme_energy=None,
            stream=None):
        _check(lib().sb_sc_pme_direct_force(self.handle, nl.handle, int(atom_numbers),
                                            _ptr(uint_crd), _ptr(charge), _ptr(frc),
                                            float(pme_beta), int(need_atom_energy),
                                            _ptr(atom_energy), int(need_virial),
                                            _ptr(atom_lj_virial), _ptr(atom_direct_pme_energy),
                                            _stream(stream)))

    def Long_Range_Correction(self, need_pressure, d_virial, need_potential, d_potential,
                              stream=None):
        _check(lib().sb_sc_long_range_correction(self.handle, int(need_pressure), _ptr(d_virial),
                                                 int(need_potential), _ptr(d_potential),
                                                 _stream(stream)))

    def Get_Partial_H_Partial_Lambda(self, uint_crd, charge, nl, pme_beta, stream=None):
        """(LJ, direct Coulomb, long-range correction) parts of dH/dlambda (FP64)."""
        h = (ctypes.c_double * 3)()
        _check(lib().sb_sc_dh_dlambda(self.handle, nl.handle, _ptr(uint_crd), _ptr(charge),
                                      float(pme_beta), h, _stream(stream)))
        return tuple(h)

    def Clear(self):
        if self.handle:
            lib().sb_sc_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


def pme_ti_cross(pme, uint_crd, charge, charge_B_A, excl, stream=None):
    """TI_CORE::Get_Cross_PME_Partial_H_Partial_Lambda: (reciprocal, self, correction)."""
    h = (ctypes.c_double * 3)()
    es, el, en = excl
    _check(lib().sb_pme_ti_cross(pme.handle, _ptr(uint_crd), _ptr(charge), _ptr(charge_B_A),
                                 _ptr(es), _ptr(el), _ptr(en), h, _stream(stream)))
    return tuple(h)


class FepBatchStep:
    """sb_fep_batch_*: the fused FEP step of many boxes in one launch per stage. ``boxes`` is a
    list of (nl, sc, pme, uint_crd, charge, (excl_start, excl_list, excl_numbers), frc, dudl),
    dudl a 1-element float64 CUDA tensor receiving the box's dU/dlambda (None in every box for
    forces only). The tensors must outlive the batch (their device addresses are stored at
    creation)."""

    def __init__(self, boxes):
        n = len(boxes)
        arr = lambda: (_vp * n)()
        nls, scs, pmes, uc, q, es, el, en, frc, du = (arr() for _ in range(10))
        want = boxes[0][7] is not None
        for k, (nl, sc, pme, u, c, excl, f, d) in enumerate(boxes):
            if (d is not None) != want:
                raise SpongeError("dudl must be given for every box or for none")
            nls[k], scs[k], pmes[k] = nl.handle, sc.handle, pme.handle
            uc[k], q[k], frc[k], du[k] = _ptr(u), _ptr(c), _ptr(f), _ptr(d)
            es[k], el[k], en[k] = (_ptr(t) for t in excl)
        self._keep = boxes
        h = _vp()
        _check(lib().sb_fep_batch_create(n, nls, scs, pmes, uc, q, es, el, en, frc,
                                         du if want else None, ctypes.byref(h)))
        self.handle = h

    @property
    def launches(self):
        return int(lib().sb_fep_batch_launches(self.handle))

    def step(self, stream=None):
        _check(lib().sb_fep_batch_step(self.handle, _stream(stream)))

    def __del__(self):
        if getattr(self, "handle", None):
            lib().sb_fep_batch_destroy(self.handle)
            self.handle = None


def fep_step(nl, sc, pme, uint_crd, charge, excl, frc, dudl=None, stream=None):
    """One FEP force evaluation (forces += into frc) with dU/dlambda into the device double
    ``dudl`` (a 1-element float64 CUDA tensor, optional)."""
    es, el, en = excl
    _check(lib().sb_fep_step(nl.handle, sc.handle, pme.handle, _ptr(uint_crd), _ptr(charge),
                             _ptr(es), _ptr(el), _ptr(en), _ptr(frc), _ptr(dudl),
                             _stream(stream)))


def nb14_pair_tables(atom_a, atom_b, lj_scale, lj_A, lj_B, lj_type):
    """Per-pair A (x12) and B (x6) of the 1-4 pairs as NON_BOND_14::Initial builds them
    (SPONGE/nb14/nb14.cu:203-217): lj_scale times the LJ tables' entry of the pair's types
    (lower-triangle index max(ti,tj)(max+1)/2 + min). lj_A / lj_B are the LJ module's tables
    already scaled by 12 and 6."""
    ta = np.asarray(lj_type, np.int64)[np.asarray(atom_a, np.int64)]
    tb = np.asarray(lj_type, np.int64)[np.asarray(atom_b, np.int64)]
    hi, lo = np.maximum(ta, tb), np.minimum(ta, tb)
    k = hi * (hi + 1) // 2 + lo
    scale = np.asarray(lj_scale, np.float32)
    return ((scale * np.asarray(lj_A, np.float32)[k]).astype(np.float32),
            (scale * np.asarray(lj_B, np.float32)[k]).astype(np.float32))


class NonBond14:
    """NON_BOND_14 from arrays (pair atoms, per-pair A/B as nb14_pair_tables gives them, Coulomb
    scale factors)."""

    def __init__(self, atom_numbers, atom_a, atom_b, A, B, cf_scale):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        a = np.ascontiguousarray(atom_a, np.int32)
        b = np.ascontiguousarray(atom_b, np.int32)
        A = np.ascontiguousarray(A, np.float32)
        B = np.ascontiguousarray(B, np.float32)
        cf = np.ascontiguousarray(cf_scale, np.float32)
        self.nb14_numbers = int(a.size)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_nb14_create(self.atom_numbers, self.nb14_numbers, a.ctypes.data,
                                    b.ctypes.data, A.ctypes.data, B.ctypes.data, cf.ctypes.data,
                                    ctypes.byref(self.handle)))

    def Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial(self, uint_crd, charge, scaler, frc,
                                                             atom_energy=None, atom_virial=None,
                                                             stream=None):
        _check(lib().sb_nb14_force(self.handle, _ptr(uint_crd), _ptr(charge), _box3(scaler),
                                   _ptr(frc), _ptr(atom_energy), _ptr(atom_virial),
                                   _stream(stream)))

    def Get_14_LJ_Energy(self, uint_crd, scaler, stream=None):
        e = ctypes.c_double()
        _check(lib().sb_nb14_energy(self.handle, _ptr(uint_crd), None, _box3(scaler),
                                    ctypes.byref(e), None, _stream(stream)))
        return e.value

    def Get_14_CF_Energy(self, uint_crd, charge, scaler, stream=None):
        e = ctypes.c_double()
        _check(lib().sb_nb14_energy(self.handle, _ptr(uint_crd), _ptr(charge), _box3(scaler),
                                    None, ctypes.byref(e), _stream(stream)))
        return e.value

    def Clear(self):
        if self.handle:
            lib().sb_nb14_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


class VirtualAtoms:
    """VIRTUAL_INFORMATION from arrays: ``types`` [V], ``atoms`` [V, 4] (virtual atom, from_1,
    from_2, from_3; unused parents may be anything in range), ``params`` [V, 2] as the
    virtual_atom_in_file line gives them."""

    def __init__(self, atom_numbers, types, atoms, params):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        t = np.ascontiguousarray(types, np.int32)
        a = np.ascontiguousarray(atoms, np.int32).reshape(-1, 4)
        p = np.ascontiguousarray(params, np.float32).reshape(-1, 2)
        self.virtual_numbers = int(t.size)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_vsite_create(self.atom_numbers, self.virtual_numbers, t.ctypes.data,
                                     a.ctypes.data, p.ctypes.data, ctypes.byref(self.handle)))

    def Coordinate_Refresh(self, uint_crd, scaler, crd, stream=None):
        _check(lib().sb_vsite_coordinate_refresh(self.handle, _ptr(uint_crd), _box3(scaler),
                                                 _ptr(crd), _stream(stream)))

    def Force_Redistribute(self, uint_crd, scaler, frc, stream=None):
        _check(lib().sb_vsite_force_redistribute(self.handle, _ptr(uint_crd), _box3(scaler),
                                                 _ptr(frc), _stream(stream)))

    def Clear(self):
        if self.handle:
            lib().sb_vsite_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass


TIME_CONVERSION = 20.455  # SPONGE's internal time unit per ps (CONSTANT_TIME_CONVERTION)


def constrain_pairs_from_bonds(bond_a, bond_b, bond_r, mass, constrain_mass=3.3):
    """CONSTRAIN::Add_HBond_To_Constrain_Pair (SPONGE/constrain/constrain.cu:81-112): the bonds
    with an atom lighter than ``constrain_mass`` (and heavier than 0), in bond order.
    Returns (i, j, r)."""
    a = np.asarray(bond_a, np.int64)
    b = np.asarray(bond_b, np.int64)
    m = np.asarray(mass, np.float32)
    ma, mb = m[a], m[b]
    keep = ((ma < constrain_mass) & (ma > 0)) | ((mb < constrain_mass) & (mb > 0))
    return (a[keep].astype(np.int32), b[keep].astype(np.int32),
            np.asarray(bond_r, np.float32)[keep])


def md_leap_frog(atom_numbers, inverse_mass, frc, vel, crd, dt, acc=None, stream=None):
    """MD_INFORMATION::NVE_iteration::Leap_Frog: acc = F/m, vel += dt acc, crd += dt vel
    (dt in SPONGE's internal unit, TIME_CONVERSION per ps)."""
    _check(lib().sb_md_leap_frog(int(atom_numbers), _ptr(inverse_mass), _ptr(frc), _ptr(vel),
                                 _ptr(crd), _ptr(acc), float(dt), _stream(stream)))


class Settle:
    """SETTLE over CONSTRAIN's pair list (see constrain_pairs_from_bonds): rigid triangles and
    rigid pairs; ``dt`` in SPONGE's internal unit; ``exp_gamma`` 1 for NVE."""

    def __init__(self, atom_numbers, pair_i, pair_j, pair_r, mass, dt, exp_gamma=1.0):
        _require_cuda()
        self.atom_numbers = int(atom_numbers)
        i = np.ascontiguousarray(pair_i, np.int32)
        j = np.ascontiguousarray(pair_j, np.int32)
        r = np.ascontiguousarray(pair_r, np.float32)
        m = np.ascontiguousarray(mass, np.float32)
        self.handle = ctypes.c_void_p()
        _check(lib().sb_settle_create(self.atom_numbers, int(i.size), i.ctypes.data,
                                      j.ctypes.data, r.ctypes.data, m.ctypes.data, float(dt),
                                      float(exp_gamma), ctypes.byref(self.handle)))
        t, p, rest = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().sb_settle_info(self.handle, ctypes.byref(t), ctypes.byref(p),
                                    ctypes.byref(rest)))
        self.triangle_numbers, self.pair_numbers, self.remaining_pairs = t.value, p.value, rest.value

    def Remember_Last_Coordinates(self, uint_crd, scaler, stream=None):
        _check(lib().sb_settle_remember(self.handle, _ptr(uint_crd), _box3(scaler),
                                        _stream(stream)))

    def Do_SETTLE(self, mass, crd, box_length, vel, need_pressure=0, pressure=None, stream=None):
        _check(lib().sb_settle_apply(self.handle, _ptr(mass), _ptr(crd), _box3(box_length),
                                     _ptr(vel), int(need_pressure), _ptr(pressure),
                                     _stream(stream)))

    def nve_step(self, uint_crd, scaler, inverse_mass, mass, frc, vel, crd, box_length,
                 acc=None, need_pressure=0, pressure=None, stream=None):
        """Remember + leap-frog + SETTLE in one launch (the same bits as the three calls)."""
        _check(lib().sb_md_nve_settle_step(self.handle, _ptr(uint_crd), _box3(scaler),
                                           _ptr(inverse_mass), _ptr(mass), _ptr(frc), _ptr(vel),
                                           _ptr(crd), _ptr(acc), _box3(box_length),
                                           int(need_pressure), _ptr(pressure), _stream(stream)))

    def Clear(self):
        if self.handle:
            lib().sb_settle_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass
