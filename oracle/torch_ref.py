"""FP64 torch restatement of the nonbonded energy, for gradient checks (test infrastructure only).

The energy is the sum the forward modules compute, written as a differentiable function of
positions, per-atom charges and the LJ tables so that torch autograd gives FP64 reference
gradients of any loss on energies and forces (forces = -dE/dx with ``create_graph=True``):

* LJ + Ewald direct over the half pair list inside the cutoff:
  E = A12/12 r^-12 - B6/6 r^-6 + q_i q_j erfc(beta r)/r   (Lennard_Jones_force.cu:166-293)
* exclusion correction  E = -q_i q_j erf(beta r)/r          (PME_force.cu:620-695)
* self + neutralising    E = -beta/sqrt(pi) sum q^2 - pi/(2 beta^2 V) (sum q)^2  (:758-762)
* smooth PME reciprocal  E = 1/2 <Q, theta>, theta = IFFT(BC FFT(Q)), 4th-order B-splines
  on the exact grid coordinate (:367-421, :253-286, :722-773)
* LJ long-range correction E = f/V, f = -(2 pi/3)/rc^3 sum_ab n_a n_b B6_ab/6 (:1119-1130)

Positions are the fixed-point coordinates dequantised exactly (x = u L / 2^32), the minimum
image is taken modulo the box, and the in-cutoff pair set is frozen at construction (the FP32
criterion of the list kernels, applied to the base coordinates) so that the function is smooth
for finite differences. It agrees with the C oracle (oracle.cpp) to FP64 rounding on energies
and forces.
"""

import math

import numpy as np
import torch

from . import oracle as _o


def tri_index(a, b):
    """Lower-triangular pair-table index of types a, b (Lennard_Jones_force.cu:106-112)."""
    M = np.maximum(a, b)
    m = np.minimum(a, b)
    return M * (M + 1) // 2 + m


def bc_half(K, box, beta):
    """Green's function x B-spline moduli on the real-FFT half spectrum [K0, K1, K2//2+1]."""
    B = [_o.bspline_moduli(int(k)) for k in K]
    L = np.asarray(box, np.float64)
    V = float(L.prod())
    kx = np.arange(K[0])
    ky = np.arange(K[1])
    kz = np.arange(K[2] // 2 + 1)
    mx = np.where(kx > K[0] // 2, K[0] - kx, kx).astype(np.float64)
    my = np.where(ky > K[1] // 2, K[1] - ky, ky).astype(np.float64)
    mz = kz.astype(np.float64)
    m2 = (mx[:, None, None] / L[0]) ** 2 + (my[None, :, None] / L[1]) ** 2 + \
        (mz[None, None, :] / L[2]) ** 2
    m2[0, 0, 0] = 1.0
    bc = B[0][kx][:, None, None] * B[1][ky][None, :, None] * B[2][kz][None, None, :] * \
        np.exp(-math.pi ** 2 * m2 / beta ** 2) / (math.pi * m2 * V)
    bc[0, 0, 0] = 0.0
    return bc


def _bspline(f):
    """4th-order B-spline weights w_k(f), k = 0..3, stacked on the last axis."""
    f2 = f * f
    f3 = f2 * f
    return torch.stack([f3 / 6.0,
                        -0.5 * f3 + 0.5 * f2 + 0.5 * f + 1.0 / 6.0,
                        0.5 * f3 - f2 + 2.0 / 3.0,
                        -f3 / 6.0 + 0.5 * f2 - 0.5 * f + 1.0 / 6.0], dim=-1)


class EnergyModel:
    """Differentiable FP64 nonbonded energy of one system topology."""

    def __init__(self, sys, uc):
        """``uc``: [N, 3] uint32 fixed-point coordinates fixing the in-cutoff pair set."""
        self.sys = sys
        self.n = n = len(sys["charge"])
        self.box = np.asarray(sys["box"], np.float32)
        self.L = torch.tensor(self.box.astype(np.float64), dtype=torch.float64)
        self.beta = float(_o.get_beta(sys["cutoff"], sys["tolerance"]))
        self.K = tuple(int(k) for k in sys["fft"])
        self.rc = float(sys["cutoff"])
        uc = np.ascontiguousarray(uc, np.uint32).reshape(n, 3)
        keys = _o.pairs(uc, sys)
        i = (keys // n).astype(np.int64)
        j = (keys % n).astype(np.int64)
        # FP32 in-cutoff criterion of the pair kernels on the base coordinates
        s = (np.float32(1.0 / 4294967296.0) * self.box).astype(np.float32)
        d = ((uc[j] - uc[i]).view(np.int32).astype(np.float32) * s).astype(np.float32)
        r2 = ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32) +
              d[:, 2] * d[:, 2]).astype(np.float32)
        keep = r2 < np.float32(self.rc * self.rc)
        self.pi = torch.from_numpy(i[keep])
        self.pj = torch.from_numpy(j[keep])
        t = np.asarray(sys["lj_type"], np.int64)
        self.ptype = torch.from_numpy(tri_index(t[i[keep]], t[j[keep]]))
        es, en, el = (np.asarray(sys["excl_start"]), np.asarray(sys["excl_numbers"]),
                      np.asarray(sys["excl_list"]))
        ei = np.repeat(np.arange(n), en)
        ej = np.concatenate([el[es[a]:es[a] + en[a]] for a in range(n)]) if en.sum() else \
            np.zeros(0, np.int64)
        self.ei = torch.from_numpy(ei.astype(np.int64))
        self.ej = torch.from_numpy(np.asarray(ej, np.int64))
        nt = int(sys["n_types"])
        self.nt = nt
        cnt = np.bincount(t, minlength=nt).astype(np.float64)
        a, b = np.meshgrid(np.arange(nt), np.arange(nt), indexing="ij")
        self.lrc_w = torch.from_numpy(cnt[a] * cnt[b])
        self.lrc_idx = torch.from_numpy(tri_index(a, b).astype(np.int64))
        self.bc = torch.from_numpy(bc_half(self.K, self.box, self.beta))
        self.V = float(np.prod(self.box.astype(np.float64)))
        self._off = torch.arange(4)

    def positions(self, uc):
        """Exact dequantisation x = u L / 2^32 of fixed-point coordinates (FP64)."""
        u = torch.from_numpy(np.asarray(uc, np.uint32).reshape(-1, 3).astype(np.float64))
        return u * (self.L / 4294967296.0)

    def _min_image(self, d):
        return d - self.L * torch.round(d / self.L)

    def energy(self, x, q, A, B, parts=False):
        """x [N,3] A, q [N] (scaled charges), A/B lower-triangular tables as in the LJ file."""
        L = self.L
        beta = self.beta
        # LJ + Ewald direct
        d = self._min_image(x[self.pi] - x[self.pj])
        r2 = (d * d).sum(-1)
        r = torch.sqrt(r2)
        ri6 = 1.0 / (r2 * r2 * r2)
        A12 = 12.0 * A[self.ptype]
        B6 = 6.0 * B[self.ptype]
        e_lj = ((A12 / 12.0 * ri6 - B6 / 6.0) * ri6).sum()
        e_dir = (q[self.pi] * q[self.pj] * torch.special.erfc(beta * r) / r).sum()
        # exclusion correction
        de = self._min_image(x[self.ei] - x[self.ej])
        re = torch.sqrt((de * de).sum(-1))
        e_corr = -(q[self.ei] * q[self.ej] * torch.erf(beta * re) / re).sum()
        # self + neutralising
        e_self = -beta / math.sqrt(math.pi) * (q * q).sum() - \
            0.5 * math.pi / (beta * beta * self.V) * q.sum() ** 2
        # reciprocal
        K = torch.tensor(self.K, dtype=torch.float64)
        u = x * (K / L)
        base = torch.floor(u).detach()
        fr = u - base
        w = _bspline(fr)  # [N, 3, 4]
        Ki = torch.tensor(self.K, dtype=torch.int64)
        idx = torch.remainder(base.to(torch.int64)[:, :, None] - self._off[None, None, :],
                              Ki[None, :, None])  # [N, 3, 4]
        flat = (idx[:, 0, :, None, None] * self.K[1] + idx[:, 1, None, :, None]) * self.K[2] + \
            idx[:, 2, None, None, :]
        val = q[:, None, None, None] * w[:, 0, :, None, None] * w[:, 1, None, :, None] * \
            w[:, 2, None, None, :]
        G = self.K[0] * self.K[1] * self.K[2]
        Q = torch.zeros(G, dtype=torch.float64).index_add(0, flat.reshape(-1), val.reshape(-1))
        Q = Q.reshape(self.K)
        theta = torch.fft.irfftn(torch.fft.rfftn(Q) * self.bc, s=self.K) * G
        e_rec = 0.5 * (Q * theta).sum()
        # LJ long-range correction
        B6sq = 6.0 * B[self.lrc_idx]
        e_lrc = (self.lrc_w * B6sq).sum() * (-2.0 / 3.0 * math.pi / self.rc ** 3 / 6.0) / self.V
        e = e_lj + e_dir + e_corr + e_self + e_rec + e_lrc
        if parts:
            return e, dict(e_lj=e_lj, e_direct=e_dir, e_corr=e_corr, e_self=e_self,
                           e_rec=e_rec, e_lrc=e_lrc)
        return e

    def energy_forces(self, x, q, A, B, create_graph=False):
        """(E, F) with F = -dE/dx; ``create_graph`` keeps F differentiable."""
        if not x.requires_grad:
            x = x.requires_grad_(True)
        e = self.energy(x, q, A, B)
        (g,) = torch.autograd.grad(e, x, create_graph=create_graph)
        return e, -g
