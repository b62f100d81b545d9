"""torch.autograd wrapper of the B200 J/K build.

``direct_jk_ad(basis, density, coords)`` returns (J, K) differentiable with
respect to the density and the nuclear coordinates:

* density: J and K are self-adjoint linear maps on (nonsymmetric) AO
  densities, so dL/dD = J(dL/dJ) + K(dL/dK) -- the reference's
  ``_density_transpose`` (src/gradscf/integrals/backends/native/jk.py:385-391);
* coordinates: the J/K coordinate VJP kernel (b200jk_direct_jk_geom_vjp;
  reference csrc/direct_jk_geometry.cc:122-182) gives one row per shell
  centre; each centre follows its nucleus, so the rows are summed onto the
  nuclei (the chain rule the reference applies through parameters.centers).

A geometry-specific plan is built for the coordinates of each forward call
(cached by table contents).  Screening (cutoff > 0) is allowed for both
derivatives here, unlike the reference, which rejects a screened coordinate
derivative (backends/native/jk.py:358-361); cutoff 0 reproduces it exactly.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi
from .basis import BasisParameters, pack
from .jk import cached_plan


class BasisContext:
    """Static basis data: topology, parameters and the nucleus of every shell."""

    def __init__(self, topology, parameters: BasisParameters, shell_atoms, *, cutoff=0.0,
                 precision="fp64", fp32_cut=1e-6):
        self.topology = topology
        self.parameters = parameters
        self.shell_atoms = np.asarray(shell_atoms)
        self.cutoff = float(cutoff)
        self.precision = precision
        self.fp32_cut = fp32_cut

    def plan_for(self, coords: np.ndarray, device):
        par = self.parameters.with_coordinates(coords, self.shell_atoms)
        atm, bas, env = pack(self.topology, par)
        return cached_plan(atm, bas, env, cart=self.topology.cart, cutoff=self.cutoff, device=device), bas


def _jk(plan, d, hermi, precision, fp32_cut):
    n = plan.nao[0]
    flat = d.reshape(-1, n * n).contiguous()
    out = plan.jk_packed(flat, hermi=hermi, precision=precision, fp32_cut=fp32_cut)
    return out[0].reshape(d.shape), out[1].reshape(d.shape)


class _DirectJK(torch.autograd.Function):
    @staticmethod
    def forward(ctx, density, coords, basis):
        coords_np = coords.detach().to("cpu", torch.float64).numpy()
        plan, bas = basis.plan_for(coords_np, density.device)
        d = density.detach().contiguous()
        hermi = bool(torch.equal(d, d.transpose(-1, -2)))
        j, k = _jk(plan, d, hermi, basis.precision, basis.fp32_cut)
        ctx.save_for_backward(d)
        ctx.plan, ctx.bas, ctx.basis = plan, bas, basis
        ctx.natom = coords.shape[0]
        return j, k

    @staticmethod
    def backward(ctx, gj, gk):
        (d,) = ctx.saved_tensors
        plan, basis = ctx.plan, ctx.basis
        gj = torch.zeros_like(d) if gj is None else gj.contiguous()
        gk = torch.zeros_like(d) if gk is None else gk.contiguous()
        grad_d = grad_c = None
        if ctx.needs_input_grad[0]:
            jj, _ = _jk(plan, gj, False, basis.precision, basis.fp32_cut)
            _, kk = _jk(plan, gk, False, basis.precision, basis.fp32_cut)
            grad_d = jj + kk
        if ctx.needs_input_grad[1]:
            n = plan.nao[0]
            nb = d.numel() // (n * n)
            natm = plan.natm[0]
            g = torch.zeros((natm, 3), dtype=torch.float64, device=d.device)
            cot = torch.stack([gj.reshape(nb, n * n), gk.reshape(nb, n * n)]).contiguous()
            dd = d.reshape(nb, n * n).contiguous()
            with torch.cuda.device(d.device):
                st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
                _capi.check(_capi.lib().b200jk_direct_jk_geom_vjp(
                    plan._h, ctypes.c_void_p(dd.data_ptr()), nb, ctypes.c_void_p(cot.data_ptr()), 1, 1,
                    ctypes.c_void_p(g.data_ptr()), st))
            plan.reduce_shards(g)
            rows = torch.as_tensor(ctx.bas[:, 0].astype(np.int64), device=d.device)
            owner = torch.as_tensor(basis.shell_atoms.astype(np.int64), device=d.device)
            grad_c = torch.zeros((ctx.natom, 3), dtype=torch.float64, device=d.device)
            grad_c.index_add_(0, owner, g[rows])
        return grad_d, grad_c, None


def direct_jk_ad(basis: BasisContext, density: torch.Tensor, coords: torch.Tensor):
    """Differentiable (J, K) of a (..., n, n) density at nuclear `coords` (natom, 3), Bohr."""
    return _DirectJK.apply(density, coords, basis)
