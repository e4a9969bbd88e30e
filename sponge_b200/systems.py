"""Seeded synthetic systems for the nonbonded hot path (water boxes, solute, FEP boxes).

Everything is generated: there is no dataset. A system is a plain dict of numpy arrays in the
units and layouts SPONGE's modules consume:

* ``crd``      float32 [N,3]   Angstrom, inside [0, box)
* ``charge``   float32 [N]     already multiplied by 18.2223, so q_i q_j / r is kcal/mol
                               (SPONGE stores charges this way, ``MD_core/MD_core.cu:1051-1080``)
* ``lj_type``  int32   [N]
* ``lj_A``, ``lj_B`` float32 [T(T+1)/2]  lower-triangular A = 4 eps sigma^12, B = 4 eps sigma^6
                               as written in an ``LJ_in_file`` (unscaled; the module multiplies by
                               12 and 6 on read, ``Lennard_Jones_force/Lennard_Jones_force.cu:1092-1098``)
* ``excl_start``, ``excl_numbers``, ``excl_list`` int32  exclusion CSR with j > i only
                               (``MD_core/MD_core.cu:308-351``)
* ``box``      float32 [3]
* ``cutoff``, ``skin``, ``fft`` (3 ints or None), ``tolerance``

Water model: rigid 3-site, r_OH = 0.9572 A, angle HOH = 104.52 deg, q_O = -0.834 e,
q_H = +0.417 e, LJ on O only (sigma = 3.15061 A, eps = 0.1521 kcal/mol). O sits on a cubic
lattice with +-0.3 A uniform jitter and a uniformly random orientation (uniform quaternion).
"""

import numpy as np

CHARGE_UNIT = 18.2223
R_OH = 0.9572
THETA_HOH = np.deg2rad(104.52)
Q_O = -0.834
Q_H = 0.417
SIGMA_O = 3.15061
EPS_O = 0.1521


def _random_rotations(rng, n):
    """Uniform random rotation matrices from uniform unit quaternions (Shoemake)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a = np.sqrt(1 - u1)
    b = np.sqrt(u1)
    w = a * np.sin(2 * np.pi * u2)
    x = a * np.cos(2 * np.pi * u2)
    y = b * np.sin(2 * np.pi * u3)
    z = b * np.cos(2 * np.pi * u3)
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _water_sites(rng, o_pos):
    """O, H1, H2 positions for waters whose O atoms are at ``o_pos`` [n,3] (float64)."""
    n = o_pos.shape[0]
    half = THETA_HOH / 2
    local = np.array([[0.0, 0.0, 0.0],
                      [R_OH * np.sin(half), 0.0, R_OH * np.cos(half)],
                      [-R_OH * np.sin(half), 0.0, R_OH * np.cos(half)]])
    R = _random_rotations(rng, n)
    sites = o_pos[:, None, :] + np.einsum('nij,kj->nki', R, local)
    return sites.reshape(n * 3, 3)


def _lattice(n_side, spacing):
    g = (np.arange(n_side) + 0.5) * spacing
    X, Y, Z = np.meshgrid(g, g, g, indexing='ij')
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _lj_tables(sigmas, epss):
    """Lower-triangular A/B tables (pair index max*(max+1)/2+min) with geometric mixing.

    Types with eps == 0 give A = B = 0 with every partner."""
    t = len(sigmas)
    npair = t * (t + 1) // 2
    A = np.zeros(npair, dtype=np.float64)
    B = np.zeros(npair, dtype=np.float64)
    for i in range(t):
        for j in range(i + 1):
            s = np.sqrt(sigmas[i] * sigmas[j])
            e = np.sqrt(epss[i] * epss[j])
            k = i * (i + 1) // 2 + j
            A[k] = 4 * e * s ** 12
            B[k] = 4 * e * s ** 6
    return A.astype(np.float32), B.astype(np.float32)


def _water_exclusions(n_water, first_atom=0, n_total=None):
    """Exclusion CSR for waters stored O,H1,H2 consecutively from ``first_atom``."""
    if n_total is None:
        n_total = first_atom + 3 * n_water
    numbers = np.zeros(n_total, dtype=np.int32)
    lists = []
    for w in range(n_water):
        o = first_atom + 3 * w
        numbers[o] = 2
        numbers[o + 1] = 1
        lists.append((o + 1, o + 2, o + 2))
    flat = np.array(lists, dtype=np.int32).ravel() if lists else np.zeros(0, np.int32)
    # CSR in atom order: O -> [H1, H2], H1 -> [H2], H2 -> []
    start = np.zeros(n_total, dtype=np.int32)
    start[1:] = np.cumsum(numbers)[:-1]
    return start, numbers, flat


def _finish(crd, charge_e, lj_type, sig, eps, excl, box, cutoff, skin, fft, tolerance=1e-5,
            name=""):
    box = np.asarray(box, dtype=np.float32)
    crd = np.mod(crd, box.astype(np.float64)).astype(np.float32)
    crd = np.where(crd >= box, np.float32(0.0), crd).astype(np.float32)
    A, B = _lj_tables(sig, eps)
    start, numbers, lst = excl
    return dict(
        name=name,
        crd=np.ascontiguousarray(crd, dtype=np.float32),
        charge=(np.asarray(charge_e, np.float64) * CHARGE_UNIT).astype(np.float32),
        lj_type=np.asarray(lj_type, np.int32),
        n_types=len(sig),
        lj_A=A, lj_B=B,
        lj_sigma=np.asarray(sig, np.float64), lj_eps=np.asarray(eps, np.float64),
        excl_start=start.astype(np.int32), excl_numbers=numbers.astype(np.int32),
        excl_list=lst.astype(np.int32),
        box=box, cutoff=float(cutoff), skin=float(skin),
        fft=None if fft is None else tuple(int(v) for v in fft),
        tolerance=float(tolerance),
    )


def water_box(n_side, spacing, box, seed, remove=0, cutoff=8.0, skin=2.0, fft=None, name=""):
    """Cubic lattice water box; ``remove`` random lattice sites are dropped."""
    rng = np.random.default_rng(seed)
    sites = _lattice(n_side, spacing)
    if remove:
        keep = np.sort(rng.choice(sites.shape[0], sites.shape[0] - remove, replace=False))
        sites = sites[keep]
    nw = sites.shape[0]
    o = sites + rng.uniform(-0.3, 0.3, size=sites.shape)
    crd = _water_sites(rng, o)
    q = np.tile([Q_O, Q_H, Q_H], nw)
    t = np.tile([0, 1, 1], nw)
    return _finish(crd, q, t, [SIGMA_O, 1.0], [EPS_O, 0.0], _water_exclusions(nw),
                   [box] * 3, cutoff, skin, fft, name=name)


def config0(seed=1000):
    """1,000 waters in a 31.04 A cube; rc 8, skin 2, PME 32^3."""
    return water_box(10, 3.104, 31.04, seed, cutoff=8.0, skin=2.0, fft=(32, 32, 32),
                     name="water3k_pme32")


def _solvated(n_solute, radius, n_water, box, n_side, seed, cutoff, skin, fft,
              solute_q_sigma=0.4, n_types=20, min_dist=2.2, clear=2.6, name="",
              center=None, neutral=True):
    rng = np.random.default_rng(seed)
    if center is None:
        center = np.full(3, box / 2)
    # random sequential addition inside a sphere, min pair distance min_dist (cell-accelerated)
    pts = []
    cell = min_dist
    grid = {}
    tries = 0
    while len(pts) < n_solute:
        tries += 1
        if tries > 500 * n_solute:
            raise RuntimeError("solute placement did not converge")
        p = rng.uniform(-radius, radius, 3)
        if p @ p > radius * radius:
            continue
        key = tuple(np.floor(p / cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        d = p - q
                        if d @ d < min_dist * min_dist:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pts.append(p)
            grid.setdefault(key, []).append(p)
    solute = np.array(pts) + center
    # water O candidates on a lattice, away from the solute
    sites = _lattice(n_side, box / n_side)
    d = sites[:, None, :] - solute[None, :, :]
    d -= box * np.round(d / box)
    # chunked min-distance to keep memory bounded
    keep = np.ones(sites.shape[0], dtype=bool)
    for s in range(0, sites.shape[0], 4096):
        dd = sites[s:s + 4096, None, :] - solute[None, :, :]
        dd -= box * np.round(dd / box)
        keep[s:s + 4096] = (np.einsum('ijk,ijk->ij', dd, dd) >= clear * clear).all(axis=1)
    del d
    sites = sites[keep]
    if sites.shape[0] < n_water:
        raise RuntimeError("not enough water sites")
    pick = np.sort(rng.choice(sites.shape[0], n_water, replace=False))
    o = sites[pick] + rng.uniform(-0.3, 0.3, size=(n_water, 3))
    wcrd = _water_sites(rng, o)
    # solute types and charges
    sig = list(rng.uniform(2.5, 4.0, n_types))
    eps = list(rng.uniform(0.05, 0.25, n_types))
    stype = rng.integers(0, n_types, n_solute) + 2
    sq = rng.normal(0.0, solute_q_sigma, n_solute)
    if neutral:
        sq -= sq.mean()
    crd = np.concatenate([solute, wcrd])
    q = np.concatenate([sq, np.tile([Q_O, Q_H, Q_H], n_water)])
    t = np.concatenate([stype, np.tile([0, 1, 1], n_water)])
    excl = _water_exclusions(n_water, first_atom=n_solute, n_total=n_solute + 3 * n_water)
    return _finish(crd, q, t, [SIGMA_O, 1.0] + sig, [EPS_O, 0.0] + eps, excl,
                   [box] * 3, cutoff, skin, fft, name=name)


def config1(seed=1001):
    """96,000 atoms: 3,000 solute atoms (20 LJ types) in a 25 A sphere + 31,000 waters in a
    98.6 A cube; rc 10, skin 2, PME 96^3."""
    return _solvated(3000, 25.0, 31000, 98.6, 33, seed, 10.0, 2.0, (96, 96, 96),
                     name="solvated96k_pme96")


def config2(seed=1002):
    """1,000,512 atoms: 333,504 waters (70^3 lattice minus 9,496 sites) in a 215.3 A cube;
    rc 10, skin 2, PME 216^3."""
    return water_box(70, 215.3 / 70, 215.3, seed, remove=9496, cutoff=10.0, skin=2.0,
                     fft=(216, 216, 216), name="water1m_pme216")


def config3(seed=1003):
    """The config-0 box (31.04 A, 1,000 waters) with 200 solute atoms of 20 types in a
    10.5 A sphere: 3,200 atoms, rc 8, skin 2, PME 32^3 (differentiation case)."""
    return _solvated(200, 10.5, 1000, 31.04, 12, seed, 8.0, 2.0, (32, 32, 32),
                     name="water_solute3k_pme32")


def config3_fit(n_frames=16, seed=1003, jitter=0.05, noise=0.05):
    """Force-field fitting workload on the config-3 system.

    Returns (system, frames, target) where ``frames`` are ``n_frames`` seeded configurations
    (the base coordinates with independent Gaussian displacements of ``jitter`` A per
    coordinate, wrapped into the box) and ``target`` holds the parameter set the target
    energies and forces are computed with: per-type sigma/epsilon and per-atom charges each
    multiplied by (1 + ``noise`` N(0, 1)), seeded."""
    s = config3(seed)
    rng = np.random.default_rng(seed + 5000)
    box = np.asarray(s["box"], np.float64)
    frames = []
    for _ in range(n_frames):
        c = s["crd"].astype(np.float64) + rng.normal(0.0, jitter, s["crd"].shape)
        c = np.mod(c, box)
        c = np.where(c >= box, 0.0, c)
        frames.append(c.astype(np.float32))
    sig = s["lj_sigma"] * (1.0 + noise * rng.normal(size=s["lj_sigma"].shape))
    eps = s["lj_eps"] * (1.0 + noise * rng.normal(size=s["lj_eps"].shape))
    q = s["charge"].astype(np.float64) * (1.0 + noise * rng.normal(size=s["charge"].shape))
    target = dict(lj_sigma=sig, lj_eps=eps, charge=q.astype(np.float32))
    return s, frames, target


WATER_VOLUME = 18.01528 / (0.997 * 0.602214076)  # A^3 per molecule at 0.997 g/cm^3


def fft_smooth(n, even=True):
    """Smallest 2-3-5-smooth integer >= n (an FFT-friendly grid size), even by default (the
    real-to-complex transform along z halves the last size)."""
    k = max(int(n), 2 if even else 1)
    while True:
        if even and k % 2:
            k += 1
            continue
        m = k
        for f in (2, 3, 5):
            while m % f == 0:
                m //= f
        if m == 1:
            return k
        k += 1


def fep_box(n_water, lam, seed, n_solute=20, q_sigma=0.3, cutoff=9.0, skin=2.0, alpha=0.5,
            p=1.0, sigma=3.0, sigma_min=0.0, name=""):
    """A water box at 0.997 g/cm^3 holding a perturbed solute of ``n_solute`` atoms for FEP/TI.

    The solute (20 LJ types as in the 96k-atom system, charges N(0, q_sigma) e, not neutralised)
    is fully coupled in state A and vanishes in state B: B-state LJ type ``n_types`` has no LJ
    and B-state charges are zero, so the charges at ``lam`` are (1 - lam) q_A. Waters are
    unperturbed. Soft-core parameters follow LJ_SOFT_CORE::Initial's keys (alpha, p, sigma,
    sigma_min; LJ_soft_core.cu:1420-1610). PME grid ~1 A, even and 2-3-5-smooth."""
    L = float((n_water * WATER_VOLUME) ** (1.0 / 3.0))
    k = fft_smooth(int(np.ceil(L)))
    n_side = int(np.ceil((n_water * 1.12) ** (1.0 / 3.0)))
    s = _solvated(n_solute, 4.5, n_water, L, n_side, seed, cutoff, skin, (k, k, k),
                  solute_q_sigma=q_sigma, name=name, neutral=False)
    nt = int(s["n_types"])
    n = len(s["charge"])
    mask = np.zeros(n, np.int32)
    mask[:n_solute] = 1
    type_b = s["lj_type"].copy()
    type_b[:n_solute] = nt
    A_b, B_b = _lj_tables(list(s["lj_sigma"]) + [1.0], list(s["lj_eps"]) + [0.0])
    q_a = s["charge"].astype(np.float32)
    q_b = q_a.copy()
    q_b[:n_solute] = 0.0
    s.update(
        lj_type_B=type_b.astype(np.int32), n_types_B=nt + 1, lj_A_B=A_b, lj_B_B=B_b, mask=mask,
        charge_A=q_a, charge_B=q_b,
        charge=((1.0 - lam) * q_a.astype(np.float64) + lam * q_b).astype(np.float32),
        dq=(q_b.astype(np.float64) - q_a).astype(np.float32),
        lam=float(lam), sc_alpha=float(alpha), sc_p=float(p), sc_sigma=float(sigma),
        sc_sigma_min=float(sigma_min))
    return s


def config4(box_index, n_boxes=48, seed=1004):
    """Box ``box_index`` of the batched FEP/TI workload: water counts U[500, 8000] (seeded),
    lambda = box_index / (n_boxes - 1), rc 9 A, skin 2 A."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(500, 8001, n_boxes)
    lam = box_index / (n_boxes - 1) if n_boxes > 1 else 0.0
    return fep_box(int(counts[box_index]), lam, seed * 1000 + box_index,
                   name="fep%02d_w%d" % (box_index, counts[box_index]))


def small_water(n_side=4, spacing=3.104, seed=7, cutoff=5.0, skin=1.0, fft=(16, 16, 16)):
    """A tiny water box for fast parity tests (n_side^3 waters)."""
    return water_box(n_side, spacing, n_side * spacing, seed, cutoff=cutoff, skin=skin,
                     fft=fft, name="water_small")


CONFIGS = {0: config0, 1: config1, 2: config2, 3: config3}
