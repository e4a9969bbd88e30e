"""ctypes wrappers around ``liboracle.so`` (built from ``oracle.cpp`` by ``oracle/Makefile``).

Test infrastructure only: see the package docstring. Each wrapper names the reference code it
restates; the C++ file carries the full citations.
"""

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


def build(force=False):
    """Compile liboracle.so with the committed Makefile (g++ only)."""
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(so):
            build()
        L = ctypes.CDLL(so)
        L.orc_periodic_map.argtypes = [ctypes.c_int, _f32p, _f32p]
        L.orc_crd_to_uint.argtypes = [ctypes.c_int, _f32p, _f32p, _u32p]
        L.orc_get_beta.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_get_beta.restype = ctypes.c_float
        L.orc_fft_size.argtypes = [ctypes.c_float]
        L.orc_fft_size.restype = ctypes.c_int
        L.orc_bspline_moduli.argtypes = [ctypes.c_int, _f64p]
        pairfn = [ctypes.c_int, _u32p, _f32p, ctypes.c_float, ctypes.c_float, _i32p, _i32p,
                  _i32p, _i64p, ctypes.c_long, ctypes.c_int]
        for f in (L.orc_pairs_bruteforce, L.orc_pairs_cells):
            f.argtypes = pairfn
            f.restype = ctypes.c_long
        L.orc_direct.argtypes = [ctypes.c_int, _u32p, _f32p, _i32p, _f32p, _f32p, _f32p,
                                 ctypes.c_float, ctypes.c_double, _i64p, ctypes.c_long, _f64p,
                                 _f64p, _f64p, ctypes.c_int]
        L.orc_lrc_factor.argtypes = [ctypes.c_int, _i32p, ctypes.c_int, _f32p, ctypes.c_float]
        L.orc_lrc_factor.restype = ctypes.c_double
        L.orc_excluded.argtypes = [ctypes.c_int, _u32p, _f32p, _f32p, ctypes.c_double, _i32p,
                                   _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_self_energy.argtypes = [ctypes.c_int, _f32p, ctypes.c_double, ctypes.c_double]
        L.orc_self_energy.restype = ctypes.c_double
        L.orc_fft3.argtypes = [_f64p, _i32p, ctypes.c_int, ctypes.c_int]
        L.orc_pme.argtypes = [ctypes.c_int, _u32p, _f32p, _f32p, _i32p, ctypes.c_double, _f64p,
                              _f64p, ctypes.c_void_p, ctypes.c_int]
        L.orc_ewald_recip.argtypes = [ctypes.c_int, _u32p, _f32p, _f32p, ctypes.c_double,
                                      ctypes.c_int, _f64p, _f64p, ctypes.c_int]
        L.orc_nonbonded.argtypes = [ctypes.c_int, _u32p, _f32p, _i32p, _f32p, _f32p, _f32p,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_double, _i32p,
                                    _i32p, _i32p, _i32p, _f64p, _f64p, ctypes.c_int]
        L.orc_nonbonded.restype = ctypes.c_long
        L.orc_softcore.argtypes = [ctypes.c_int, _u32p, _f32p, _f32p, _i32p, _i32p, _i32p,
                                   _f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_float,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, _i64p,
                                   ctypes.c_long, _f64p, _f64p]
        L.orc_ti_cross.argtypes = [ctypes.c_int, _u32p, _f32p, _f32p, _f32p, _i32p,
                                   ctypes.c_double, _i32p, _i32p, _i32p, _f64p]
        L.orc_nb14.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _f32p, _f32p, _i32p, _i32p,
                               _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f64p]
        L.orc_vsite.argtypes = [ctypes.c_int, _i32p, _i32p, _f32p, _i32p, ctypes.c_int, _u32p,
                                _f32p, ctypes.c_int, _f64p, _f64p]
        L.orc_nve_settle.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f32p, _f32p,
                                     _u32p, _f32p, ctypes.c_double, ctypes.c_double, _f64p,
                                     _f64p, _f64p, _f64p, _f64p]
        L.orc_threads.restype = ctypes.c_int
        L.orc_set_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def threads():
    return lib().orc_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


def periodic_map(crd, box):
    """Crd_Periodic_Map (SPONGE/common.cu:299-352); returns a wrapped copy."""
    c = np.ascontiguousarray(crd, np.float32).copy()
    lib().orc_periodic_map(c.shape[0], c.reshape(-1), np.ascontiguousarray(box, np.float32))
    return c


def crd_to_uint(crd, box):
    """Crd_To_Uint_Crd with the quarter coefficient (SPONGE/common.cu:264-287)."""
    c = np.ascontiguousarray(crd, np.float32)
    out = np.empty((c.shape[0], 3), np.uint32)
    lib().orc_crd_to_uint(c.shape[0], c.reshape(-1), np.ascontiguousarray(box, np.float32),
                          out.reshape(-1))
    return out


def get_beta(cutoff, tolerance=1e-5):
    """Get_Beta (SPONGE/PME_force/PME_force.cu:71-100)."""
    return float(lib().orc_get_beta(cutoff, tolerance))


def fft_size(length):
    """Get_Fft_Patameter (SPONGE/common.cu:513-534)."""
    return int(lib().orc_fft_size(length))


def bspline_moduli(K):
    out = np.empty(K, np.float64)
    lib().orc_bspline_moduli(K, out)
    return out


def _excl(sys):
    return (np.ascontiguousarray(sys["excl_start"], np.int32),
            np.ascontiguousarray(sys["excl_numbers"], np.int32),
            np.ascontiguousarray(sys["excl_list"], np.int32) if len(sys["excl_list"])
            else np.zeros(1, np.int32))


def pairs(uc, sys, method="cells", cap=None, nthreads=0):
    """Half pair set {i<j} as sorted int64 keys i*N+j under the pinned FP32 criterion."""
    n = uc.shape[0]
    if cap is None:
        cap = max(1024, n * 800)
    out = np.empty(cap, np.int64)
    es, en, el = _excl(sys)
    f = lib().orc_pairs_bruteforce if method == "brute" else lib().orc_pairs_cells
    cnt = f(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
            np.ascontiguousarray(sys["box"], np.float32), sys["cutoff"], sys["skin"],
            es, en, el, out, cap, nthreads)
    if cnt > cap:
        return pairs(uc, sys, method, cap=int(cnt) + 16, nthreads=nthreads)
    return out[:cnt].copy()


def scaled_tables(sys):
    """h_LJ_A * 12 and h_LJ_B * 6 in float, as the LJ module stores them (Lennard_Jones_force.cu:1092-1098)."""
    A12 = (np.asarray(sys["lj_A"], np.float32) * np.float32(12.0)).astype(np.float32)
    B6 = (np.asarray(sys["lj_B"], np.float32) * np.float32(6.0)).astype(np.float32)
    return A12, B6


def direct(uc, sys, pair_keys, beta, nthreads=0):
    """LJ + Ewald direct force/energies/virial over a pair set in FP64.

    Returns (frc [N,3] f64, atom_energy [N] f64, dict(e_lj, e_direct, virial_lj, n_in_cutoff))."""
    n = uc.shape[0]
    A12, B6 = scaled_tables(sys)
    frc = np.zeros(3 * n, np.float64)
    ae = np.zeros(n, np.float64)
    out = np.zeros(4, np.float64)
    pk = np.ascontiguousarray(pair_keys, np.int64)
    if pk.size == 0:
        pk = np.zeros(1, np.int64)
        npairs = 0
    else:
        npairs = pk.size
    lib().orc_direct(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                     np.ascontiguousarray(sys["charge"], np.float32),
                     np.ascontiguousarray(sys["lj_type"], np.int32), A12, B6,
                     np.ascontiguousarray(sys["box"], np.float32), sys["cutoff"], beta, pk,
                     npairs, frc, ae, out, nthreads)
    return frc.reshape(n, 3), ae, dict(e_lj=out[0], e_direct=out[1], virial_lj=out[2],
                                       n_in_cutoff=int(out[3]))


def lrc_factor(sys):
    _, B6 = scaled_tables(sys)
    return float(lib().orc_lrc_factor(len(sys["lj_type"]),
                                      np.ascontiguousarray(sys["lj_type"], np.int32),
                                      int(sys["n_types"]), B6, sys["cutoff"]))


def excluded(uc, sys, beta):
    """Exclusion correction (SPONGE/PME_force/PME_force.cu:620-695)."""
    n = uc.shape[0]
    frc = np.zeros(3 * n, np.float64)
    ae = np.zeros(n, np.float64)
    out = np.zeros(1, np.float64)
    es, en, el = _excl(sys)
    lib().orc_excluded(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                       np.ascontiguousarray(sys["charge"], np.float32),
                       np.ascontiguousarray(sys["box"], np.float32), beta, es, en, el, frc, ae,
                       out)
    return frc.reshape(n, 3), ae, float(out[0])


def self_energy(sys, beta):
    box = np.asarray(sys["box"], np.float64)
    return float(lib().orc_self_energy(len(sys["charge"]),
                                       np.ascontiguousarray(sys["charge"], np.float32), beta,
                                       float(box[0] * box[1] * box[2])))


def fft3(grid, sign):
    """Unnormalised 3D FFT (sign -1 forward, +1 inverse) of a complex128 grid."""
    g = np.ascontiguousarray(grid, np.complex128).copy()
    K = np.array(g.shape, np.int32)
    lib().orc_fft3(g.view(np.float64).reshape(-1), K, int(sign), 0)
    return g


def pme(uc, sys, beta, fft=None, want_grid=False, nthreads=0):
    """SPME reciprocal force and energy in FP64. Returns (frc [N,3], E_rec[, Q grid])."""
    n = uc.shape[0]
    K = np.array(fft if fft is not None else sys["fft"], np.int32)
    frc = np.zeros(3 * n, np.float64)
    out = np.zeros(1, np.float64)
    grid = np.zeros(int(K.prod()), np.float64) if want_grid else None
    lib().orc_pme(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                  np.ascontiguousarray(sys["charge"], np.float32),
                  np.ascontiguousarray(sys["box"], np.float32), K, beta, frc, out,
                  grid.ctypes.data if grid is not None else None, nthreads)
    if want_grid:
        return frc.reshape(n, 3), float(out[0]), grid.reshape(tuple(K))
    return frc.reshape(n, 3), float(out[0])


def ewald_recip(uc, sys, beta, kmax, nthreads=0):
    """Classic Ewald reciprocal sum (no grid): converged reference for the SPME method error."""
    n = uc.shape[0]
    frc = np.zeros(3 * n, np.float64)
    out = np.zeros(1, np.float64)
    lib().orc_ewald_recip(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                          np.ascontiguousarray(sys["charge"], np.float32),
                          np.ascontiguousarray(sys["box"], np.float32), beta, kmax, frc, out,
                          nthreads)
    return frc.reshape(n, 3), float(out[0])


def nonbonded(uc, sys, beta, nthreads=0):
    """Whole FP64 evaluation (cell list + direct + exclusions + SPME): the CPU baseline.

    Returns (frc [N,3], dict of energies, pair count)."""
    n = uc.shape[0]
    A12, B6 = scaled_tables(sys)
    frc = np.zeros(3 * n, np.float64)
    out = np.zeros(7, np.float64)
    es, en, el = _excl(sys)
    npairs = lib().orc_nonbonded(n, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                                 np.ascontiguousarray(sys["charge"], np.float32),
                                 np.ascontiguousarray(sys["lj_type"], np.int32), A12, B6,
                                 np.ascontiguousarray(sys["box"], np.float32), sys["cutoff"],
                                 sys["skin"], beta, np.array(sys["fft"], np.int32), es, en, el,
                                 frc, out, nthreads)
    if npairs < 0:
        raise MemoryError("oracle pair buffer allocation failed")
    keys = ("e_lj", "e_direct", "e_corr", "e_rec", "e_self", "virial_lj", "n_in_cutoff")
    return frc.reshape(n, 3), dict(zip(keys, out.tolist())), int(npairs)


def reference_energies(sys, uc=None, nthreads=0):
    """All FP64 quantities for a system in one call (convenience for tests)."""
    if uc is None:
        uc = crd_to_uint(periodic_map(sys["crd"], sys["box"]), sys["box"])
    beta = get_beta(sys["cutoff"], sys["tolerance"])
    pk = pairs(uc, sys, nthreads=nthreads)
    fd, ae, d = direct(uc, sys, pk, beta, nthreads)
    fe, aee, ecorr = excluded(uc, sys, beta)
    fr, erec = pme(uc, sys, beta, nthreads=nthreads)
    box = np.asarray(sys["box"], np.float64)
    V = float(box.prod())
    f = lrc_factor(sys)
    res = dict(beta=beta, pairs=pk, uc=uc, f_direct=fd, f_excl=fe, f_rec=fr,
               e_lj=d["e_lj"], e_direct=d["e_direct"], virial_lj=d["virial_lj"],
               n_in_cutoff=d["n_in_cutoff"], e_corr=ecorr, e_rec=erec,
               e_self=self_energy(sys, beta), lrc_factor=f, e_lrc=f / V, virial_lrc=6 * f / V)
    res["f_total"] = fd + fe + fr
    return res


# ---------------------------------------------------------------------------------------------
# FEP / TI (soft-core LJ, LJ_soft_core.cu; PME cross terms, TI_core.cu:670-730)
# ---------------------------------------------------------------------------------------------
def fep_tables(sys):
    """Scaled (x12, x6) lower-triangular tables of the A and B states."""
    f32 = np.float32
    A12 = (np.asarray(sys["lj_A"], f32) * f32(12.0)).astype(f32)
    B6 = (np.asarray(sys["lj_B"], f32) * f32(6.0)).astype(f32)
    A12b = (np.asarray(sys["lj_A_B"], f32) * f32(12.0)).astype(f32)
    B6b = (np.asarray(sys["lj_B_B"], f32) * f32(6.0)).astype(f32)
    return A12, B6, A12b, B6b


def sc_sigma6(sys):
    return float(sys["sc_sigma"]) ** 6, float(sys["sc_sigma_min"]) ** 6


def softcore(uc, sys, pair_keys, beta, lam=None, charge=None):
    """Soft-core LJ + direct Coulomb at lambda over a half pair set in FP64.

    Returns (frc [N,3], dict(e_lj, e_direct, dhdl_lj, dhdl_direct))."""
    n = uc.shape[0]
    lam = sys["lam"] if lam is None else lam
    q = np.ascontiguousarray(sys["charge"] if charge is None else charge, np.float32)
    AA, AB, BA, BB = fep_tables(sys)
    s6, s6m = sc_sigma6(sys)
    pk = np.ascontiguousarray(pair_keys, np.int64)
    npairs = pk.size
    if npairs == 0:
        pk = np.zeros(1, np.int64)
    frc = np.zeros(3 * n, np.float64)
    out = np.zeros(4, np.float64)
    lib().orc_softcore(n, np.ascontiguousarray(uc, np.uint32).reshape(-1), q,
                       np.ascontiguousarray(sys["dq"], np.float32),
                       np.ascontiguousarray(sys["lj_type"], np.int32),
                       np.ascontiguousarray(sys["lj_type_B"], np.int32),
                       np.ascontiguousarray(sys["mask"], np.int32), AA, AB, BA, BB,
                       np.ascontiguousarray(sys["box"], np.float32), sys["cutoff"], beta, lam,
                       sys["sc_alpha"], sys["sc_p"], s6, s6m, pk, npairs, frc, out)
    return frc.reshape(n, 3), dict(e_lj=out[0], e_direct=out[1], dhdl_lj=out[2],
                                   dhdl_direct=out[3])


def ti_cross(uc, sys, beta, charge=None):
    """PME cross terms of dH/dlambda: reciprocal sum dq_i phi_i, self, exclusion correction."""
    n = uc.shape[0]
    q = np.ascontiguousarray(sys["charge"] if charge is None else charge, np.float32)
    es, en, el = _excl(sys)
    out = np.zeros(3, np.float64)
    lib().orc_ti_cross(n, np.ascontiguousarray(uc, np.uint32).reshape(-1), q,
                       np.ascontiguousarray(sys["dq"], np.float32),
                       np.ascontiguousarray(sys["box"], np.float32),
                       np.array(sys["fft"], np.int32), beta, es, en, el, out)
    return dict(rec=out[0], self=out[1], corr=out[2])


def fep_lrc(sys, lam=None):
    """LJ long-range correction of the soft-core module: the factor at lambda (B6 mixed
    linearly between the states, LJ_soft_core.cu:85-120) and its lambda derivative
    (:123-156), both times -(2 pi/3)/rc^3/6; energy = factor/V."""
    lam = sys["lam"] if lam is None else lam
    _, B6a, _, B6b = fep_tables(sys)
    ta = np.asarray(sys["lj_type"], np.int64)
    tb = np.asarray(sys["lj_type_B"], np.int64)
    combos, cnt = np.unique(np.stack([ta, tb], 1), axis=0, return_counts=True)
    a = combos[:, 0]
    b = combos[:, 1]

    def tri(x, y):
        M = np.maximum(x, y)
        m = np.minimum(x, y)
        return M * (M + 1) // 2 + m
    w = np.outer(cnt, cnt).astype(np.float64)
    sa = (w * B6a[tri(a[:, None], a[None, :])].astype(np.float64)).sum()
    sb = (w * B6b[tri(b[:, None], b[None, :])].astype(np.float64)).sum()
    kappa = -2.0 / 3.0 * np.pi / float(sys["cutoff"]) ** 3 / 6.0
    return kappa * ((1.0 - lam) * sa + lam * sb), kappa * (sb - sa)


def fep_reference(sys, uc=None, lam=None):
    """FP64 forces, potential energy U(lambda) and dU/dlambda of an FEP box (soft-core LJ +
    direct, exclusion correction, self, SPME reciprocal, long-range correction) with the
    charges at lambda."""
    lam = sys["lam"] if lam is None else lam
    if uc is None:
        uc = crd_to_uint(periodic_map(sys["crd"], sys["box"]), sys["box"])
    q = ((1.0 - lam) * np.asarray(sys["charge_A"], np.float64) +
         lam * np.asarray(sys["charge_B"], np.float64)).astype(np.float32)
    sq = dict(sys)
    sq["charge"] = q
    beta = get_beta(sys["cutoff"], sys["tolerance"])
    pk = pairs(uc, sys)
    fs, p = softcore(uc, sys, pk, beta, lam=lam, charge=q)
    fe, _, ecorr = excluded(uc, sq, beta)
    fr, erec = pme(uc, sq, beta)
    eself = self_energy(sq, beta)
    V = float(np.prod(np.asarray(sys["box"], np.float64)))
    flrc, flrc_ti = fep_lrc(sys, lam)
    x = ti_cross(uc, sys, beta, charge=q)
    U = p["e_lj"] + p["e_direct"] + ecorr + eself + erec + flrc / V
    dU = p["dhdl_lj"] + p["dhdl_direct"] + x["rec"] + x["self"] + x["corr"] + flrc_ti / V
    return dict(uc=uc, beta=beta, pairs=pk, charge=q, f_total=fs + fe + fr, f_sc=fs, U=U,
                dU=dU, e_lj=p["e_lj"], e_direct=p["e_direct"], e_corr=ecorr, e_self=eself,
                e_rec=erec, e_lrc=flrc / V, dhdl_lj=p["dhdl_lj"], dhdl_direct=p["dhdl_direct"],
                cross_rec=x["rec"], cross_self=x["self"], cross_corr=x["corr"],
                dhdl_lrc=flrc_ti / V)


def nb14(uc, box, charge, atom_a, atom_b, A, B, cf):
    """1-4 pairs in FP64 (SPONGE/nb14/nb14.cu:92-170). A, B per pair (x12, x6).
    Returns (frc [N,3], atom_energy [N], atom_virial [N], e_lj, e_cf)."""
    n = uc.shape[0]
    a = np.ascontiguousarray(atom_a, np.int32)
    frc = np.zeros(3 * n, np.float64)
    ae = np.zeros(n, np.float64)
    av = np.zeros(n, np.float64)
    out = np.zeros(2, np.float64)
    lib().orc_nb14(n, a.size, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                   np.ascontiguousarray(charge, np.float32), np.ascontiguousarray(box, np.float32),
                   a, np.ascontiguousarray(atom_b, np.int32), np.ascontiguousarray(A, np.float32),
                   np.ascontiguousarray(B, np.float32), np.ascontiguousarray(cf, np.float32), frc,
                   ae, av, out)
    return frc.reshape(n, 3), ae, av, float(out[0]), float(out[1])


def vsite_levels(n, types, atoms):
    """Level of each virtual-atom record: one above its highest parent (virtual_atoms.cu:
    246-290), iterated to a fixed point so that the record order does not matter."""
    npar = {0: 1, 1: 2, 2: 3, 3: 3}
    atoms = np.asarray(atoms, np.int64).reshape(-1, 4)
    level = np.zeros(n, np.int64)
    for _ in range(len(types) + 1):
        changed = False
        for r, t in enumerate(types):
            lv = max(level[atoms[r, k]] for k in range(1, npar[int(t)] + 1)) + 1
            if level[atoms[r, 0]] != lv:
                level[atoms[r, 0]] = lv
                changed = True
        if not changed:
            break
    return np.array([level[atoms[r, 0]] for r in range(len(types))], np.int32)


def vsite(uc, box, types, atoms, params, crd=None, frc=None):
    """Virtual atoms in FP64: with ``crd`` [N,3], returns the refreshed coordinates
    (Coordinate_Refresh); with ``frc`` [N,3], returns the redistributed forces
    (Force_Redistribute)."""
    n = uc.shape[0]
    t = np.ascontiguousarray(types, np.int32)
    a = np.ascontiguousarray(atoms, np.int32).reshape(-1)
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    lv = vsite_levels(n, t, a)
    ml = int(lv.max()) if lv.size else 0
    mode = 0 if crd is not None else 1
    c = np.ascontiguousarray(crd if crd is not None else np.zeros((n, 3)), np.float64).reshape(-1).copy()
    f = np.ascontiguousarray(frc if frc is not None else np.zeros((n, 3)), np.float64).reshape(-1).copy()
    lib().orc_vsite(t.size, t, a, p, lv, ml, np.ascontiguousarray(uc, np.uint32).reshape(-1),
                    np.ascontiguousarray(box, np.float32), mode, c, f)
    return (c if mode == 0 else f).reshape(n, 3)


def nve_settle(uc, box, pair_i, pair_j, pair_r, mass, dt, frc, crd, vel, exp_gamma=1.0):
    """One NVE leap-frog step with SETTLE in FP64 (SPONGE/MD_core/MD_core.cu:13-32,
    SPONGE/constrain/SETTLE.cu). Returns (crd, vel, acc, constraint virial, triangles, pairs)."""
    n = uc.shape[0]
    c = np.ascontiguousarray(crd, np.float64).reshape(-1).copy()
    v = np.ascontiguousarray(vel, np.float64).reshape(-1).copy()
    a = np.zeros(3 * n, np.float64)
    out = np.zeros(3, np.float64)
    i = np.ascontiguousarray(pair_i, np.int32)
    lib().orc_nve_settle(n, i.size, i, np.ascontiguousarray(pair_j, np.int32),
                         np.ascontiguousarray(pair_r, np.float32),
                         np.ascontiguousarray(mass, np.float32),
                         np.ascontiguousarray(uc, np.uint32).reshape(-1),
                         np.ascontiguousarray(box, np.float32), float(dt), float(exp_gamma),
                         np.ascontiguousarray(frc, np.float64).reshape(-1), c, v, a, out)
    return (c.reshape(n, 3), v.reshape(n, 3), a.reshape(n, 3), float(out[0]), int(out[1]),
            int(out[2]))
