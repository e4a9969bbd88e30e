"""Differentiable nonbonded energy and forces for force-field fitting.

``NonbondedModel(system)(crd, charge, lj_A, lj_B)`` returns ``(E, F)``: the nonbonded potential
energy (FP64 scalar tensor: LJ + long-range correction + Ewald direct + exclusion correction +
self + reciprocal, summed as MD_core sums it) and the forces (float32 [N, 3]) of one
configuration, evaluated by the fixed-point CUDA modules. It is a ``torch.autograd.Function``:
the backward pass calls the hand-written adjoint kernels (``sb_adjoint_backward``), which return
the Jacobian-vector products of (E, F) with the loss cotangents with respect to positions,
per-atom charges and the LJ tables, in one pass over the neighbor list plus a transposed PME
spread/gather that recomputes the charge grid. ``lj_tables(sigma, epsilon)`` maps per-type
sigma/epsilon to the tables (geometric mixing) in torch, so their gradients follow by autograd.

Arguments: ``crd`` [N, 3] float32 (A), ``charge`` [N] float32 in the modules' scaled units
(e x 18.2223), ``lj_A`` / ``lj_B`` the lower-triangular tables of A = 4 eps sigma^12 and
B = 4 eps sigma^6 as the LJ file holds them (the module stores them x12 and x6).
"""

import ctypes

import numpy as np

from . import FORM_FIXED, SpongeError, _check, _ptr, _require_cuda, _stream, lib
from .engine import NonbondedEngine


def lj_tables(sigma, epsilon):
    """Lower-triangular A, B (pair index max*(max+1)/2 + min) from per-type sigma/epsilon with
    geometric mixing; types with epsilon 0 give zero entries (and zero gradients)."""
    import torch
    nt = sigma.shape[0]
    idx = torch.tril_indices(nt, nt, device=sigma.device)
    a, b = idx[0], idx[1]  # a >= b, ordered as max*(max+1)/2 + min
    s = torch.sqrt(sigma[a] * sigma[b])
    pe = epsilon[a] * epsilon[b]
    pos = pe > 0
    e = torch.where(pos, torch.sqrt(torch.where(pos, pe, torch.ones_like(pe))),
                    torch.zeros_like(pe))
    s6 = s ** 6
    return 4.0 * e * s6 * s6, 4.0 * e * s6


def _tri_from_square(g, nt):
    """Gradient of a symmetric lower-triangular table from the square [a][b] gradient."""
    import torch
    sym = g + g.t() - torch.diag(torch.diagonal(g))
    idx = torch.tril_indices(nt, nt, device=g.device)
    return sym[idx[0], idx[1]]


class _NonbondedFunction:
    """Holder of the autograd.Function class (built lazily so that importing needs no torch)."""
    cls = None


def _function():
    if _NonbondedFunction.cls is not None:
        return _NonbondedFunction.cls
    import torch

    class NonbondedFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, crd, charge, lj_A, lj_B, model):
            key = model._forward(crd, charge, lj_A, lj_B)
            E = model.energy_tensor()
            F = model.eng.frc.clone()
            ctx.model = model
            ctx.key = key
            ctx.save_for_backward(crd.detach().clone(), charge.detach().clone(),
                                  lj_A.detach().clone(), lj_B.detach().clone())
            return E, F

        @staticmethod
        def backward(ctx, gE, gF):
            crd, charge, A, B = ctx.saved_tensors
            model = ctx.model
            if model._key != ctx.key:
                model._forward(crd, charge, A, B, force_eval=False)
            g_crd, g_q, g_A, g_B = model._backward(gE, gF)
            return (g_crd.to(crd.device, crd.dtype), g_q.to(charge.device, charge.dtype),
                    g_A.to(A.device, A.dtype), g_B.to(B.device, B.dtype), None)

    _NonbondedFunction.cls = NonbondedFunction
    return NonbondedFunction


class NonbondedModel:
    """One system topology (atom types, exclusions, box, cutoff, grid) on one GPU."""

    def __init__(self, system, max_neighbor_numbers=1200):
        torch = _require_cuda()
        self.torch = torch
        self.eng = NonbondedEngine(system, form=FORM_FIXED, refresh_interval=0,
                                   max_neighbor_numbers=max_neighbor_numbers)
        self.n = self.eng.n
        self.nt = int(system["n_types"])
        self.handle = ctypes.c_void_p()
        _check(lib().sb_adjoint_create(self.eng.nl.handle, self.eng.lj.handle,
                                       self.eng.pme.handle, ctypes.byref(self.handle)))
        dev = self.eng.frc.device
        self.g_crd = torch.zeros(3 * self.n, dtype=torch.float64, device=dev)
        self.g_q = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self.g_lj = torch.zeros(2 * self.nt * self.nt, dtype=torch.float64, device=dev)
        self._tables = None
        self._key = None
        self._count = 0

    def __call__(self, crd, charge, lj_A, lj_B):
        return _function().apply(crd, charge, lj_A, lj_B, self)

    # -- internals ---------------------------------------------------------------------------
    def _set_tables(self, lj_A, lj_B):
        A12 = (lj_A.detach().to("cpu", self.torch.float32) * 12.0).numpy().astype(np.float32)
        B6 = (lj_B.detach().to("cpu", self.torch.float32) * 6.0).numpy().astype(np.float32)
        if self._tables is not None and np.array_equal(self._tables[0], A12) and \
                np.array_equal(self._tables[1], B6):
            return
        A12 = np.ascontiguousarray(A12)
        B6 = np.ascontiguousarray(B6)
        _check(lib().sb_lj_set_tables(self.eng.lj.handle, A12.ctypes.data, B6.ctypes.data))
        self._tables = (A12, B6)

    def _forward(self, crd, charge, lj_A, lj_B, force_eval=True):
        eng = self.eng
        if tuple(crd.shape) != (self.n, 3) or tuple(charge.shape) != (self.n,):
            raise SpongeError("NonbondedModel: crd must be [N, 3] and charge [N]")
        self._set_tables(lj_A, lj_B)
        eng.crd.copy_(crd.detach().to(eng.crd.device, self.torch.float32))
        eng.charge.copy_(charge.detach().to(eng.charge.device, self.torch.float32))
        eng.update_list(forced=1)
        eng.to_uint()
        if force_eval:
            eng.reset()
            eng.forces(need_energy=1)
        self._count += 1
        self._key = self._count
        return self._key

    def energy_tensor(self):
        eng = self.eng
        return eng.atom_energy.double().sum() + eng.d_potential.double()[0]

    def _backward(self, gE, gF):
        torch = self.torch
        eng = self.eng
        ge = 0.0 if gE is None else float(gE.detach().double().item())
        if gF is None:
            gf = torch.zeros((self.n, 3), dtype=torch.float32, device=eng.frc.device)
        else:
            gf = gF.detach().to(eng.frc.device, torch.float32).contiguous()
        _check(lib().sb_adjoint_backward(
            self.handle, eng.nl.handle, eng.lj.handle, eng.pme.handle, _ptr(eng.uint_crd),
            _ptr(eng.charge), _ptr(eng.excl_start), _ptr(eng.excl_list),
            _ptr(eng.excl_numbers), ctypes.c_double(ge), _ptr(gf), _ptr(self.g_crd),
            _ptr(self.g_q), _ptr(self.g_lj), _stream(None)))
        nt = self.nt
        gA = _tri_from_square(self.g_lj[:nt * nt].view(nt, nt), nt) * 12.0
        gB = _tri_from_square(self.g_lj[nt * nt:].view(nt, nt), nt) * 6.0
        return self.g_crd.view(self.n, 3).clone(), self.g_q.clone(), gA, gB

    def close(self):
        if self.handle:
            lib().sb_adjoint_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
