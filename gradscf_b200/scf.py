"""Restricted Hartree-Fock on the B200 J/K build (the caller of the hot path).

Follows the reference caller's arithmetic (src/gradscf/scf/rks.py:305-321,
src/gradscf/scf/energy.py:23-31):
  * incremental J/K: J(D) = J_last + J(D - D_last), same for K;
  * F = h + J - K/2,  E = tr(D h) + tr(D J)/2 - tr(D K)/4 + E_nuc,
    D = 2 C_occ C_occ^T.
DIIS extrapolation (commutator F D S - S D F) and the generalised eigenproblem
stay FP64 in torch on the device.  The one-electron integrals and all J/K
builds go through the C ABI.  ``precision="split"`` runs quartets with
Q_ij Q_kl max|dD| < fp32_cut in FP32 (FP64 J/K accumulation).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _capi
from .basis import nuclear_repulsion, nuclear_repulsion_gradient, pack, prepare_basis
from .jk import DEFAULT_FP32_CUT, DirectJKPlan


@dataclass
class SCFResult:
    energy: float
    converged: bool
    cycles: int
    density: torch.Tensor
    mo_energy: torch.Tensor
    mo_coeff: torch.Tensor
    nocc: int
    jk_ms: list = field(default_factory=list)       # device time of each J/K build
    energies: list = field(default_factory=list)


class Molecule:
    """A molecule with its basis, libcint tables and a device J/K plan."""

    def __init__(self, atom, basis, *, unit="Angstrom", cart=False, schwarz_cut=1e-12,
                 device=None, charge=0):
        self.topology, self.parameters, self.shell_atoms = prepare_basis(atom, basis, unit=unit,
                                                                         cart=cart)
        self.atm, self.bas, self.env = pack(self.topology, self.parameters)
        self.cart = bool(cart)
        self.charges = np.asarray(self.topology.nuclear_charges, dtype=np.float64)
        self.coords = np.asarray(self.parameters.nuclear_coords, dtype=np.float64)
        self.nelectron = int(self.charges.sum()) - int(charge)
        self.plan = DirectJKPlan([(self.atm, self.bas, self.env)], cart=cart, cutoff=schwarz_cut,
                                 device=device)
        self.device = self.plan.device
        self.nao = self.plan.nao[0]
        self.e_nuc = nuclear_repulsion(self.charges, self.coords)

    def int1e(self, which):
        n = self.nao
        out = torch.empty((n, n), dtype=torch.float64, device=self.device)
        code = {"ovlp": 0, "kin": 1, "nuc": 2}[which]
        with torch.cuda.device(self.device):
            st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            _capi.check(_capi.lib().b200jk_int1e(self.plan._h, code, ctypes.c_void_p(out.data_ptr()), st))
        return out

    def jk(self, density, *, precision="fp64", fp32_cut=DEFAULT_FP32_CUT, hermi=True):
        return self.plan.jk(density, hermi=hermi, precision=precision, fp32_cut=fp32_cut)


def _solve(f, x):
    e, c = torch.linalg.eigh(x.T @ f @ x)
    return e, x @ c


def rhf(mol: Molecule, *, conv_tol=1e-10, conv_tol_grad=None, max_cycle=100, precision="fp64",
        fp32_cut=DEFAULT_FP32_CUT, incremental=True, diis_space=8, density0=None, timing=True):
    """Run RHF; returns SCFResult (energy in Hartree)."""
    dev = mol.device
    s = mol.int1e("ovlp")
    h = mol.int1e("kin") + mol.int1e("nuc")
    w, v = torch.linalg.eigh(s)
    x = v / torch.sqrt(w)
    nocc = mol.nelectron // 2
    if conv_tol_grad is None:
        conv_tol_grad = float(np.sqrt(conv_tol))
    if density0 is None:
        e, c = _solve(h, x)
        d = 2.0 * c[:, :nocc] @ c[:, :nocc].T
    else:
        d = torch.as_tensor(density0, dtype=torch.float64, device=dev)
    d_last = torch.zeros_like(d)
    j = torch.zeros_like(d)
    k = torch.zeros_like(d)
    hist_f, hist_e = [], []
    e_old = None
    energies, jk_ms = [], []
    converged = False
    stream = torch.cuda.current_stream(dev)
    for cycle in range(1, max_cycle + 1):
        delta = d - d_last if incremental else d
        if timing:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
        dj, dk = mol.jk(delta, precision=precision, fp32_cut=fp32_cut)
        if timing:
            ev1.record(stream)
            jk_ms.append((ev0, ev1))
        if incremental:
            j, k = j + dj, k + dk
        else:
            j, k = dj, dk
        d_last = d
        f = h + j - 0.5 * k
        energy = (torch.sum(d * h) + 0.5 * torch.sum(d * j) - 0.25 * torch.sum(d * k)).item() + mol.e_nuc
        energies.append(energy)
        err = f @ d @ s - s @ d @ f
        err_o = x.T @ err @ x
        gnorm = torch.linalg.norm(err_o).item()
        if e_old is not None and abs(energy - e_old) < conv_tol and gnorm < conv_tol_grad:
            converged = True
            break
        hist_f.append(f)
        hist_e.append(err_o)
        hist_f, hist_e = hist_f[-diis_space:], hist_e[-diis_space:]
        if len(hist_f) > 1:
            m = len(hist_f)
            b = -torch.ones((m + 1, m + 1), dtype=torch.float64, device=dev)
            b[m, m] = 0.0
            for a in range(m):
                for c_ in range(a, m):
                    b[a, c_] = b[c_, a] = torch.sum(hist_e[a] * hist_e[c_])
            rhs = torch.zeros(m + 1, dtype=torch.float64, device=dev)
            rhs[m] = -1.0
            coef = torch.linalg.solve(b, rhs)[:m]
            f = sum(cf * fi for cf, fi in zip(coef, hist_f))
        mo_e, c = _solve(f, x)
        d = 2.0 * c[:, :nocc] @ c[:, :nocc].T
        e_old = energy
    # final orbitals of the converged Fock matrix
    f = h + j - 0.5 * k
    mo_e, c = _solve(f, x)
    torch.cuda.synchronize(dev)
    times = [a.elapsed_time(b) for a, b in jk_ms] if timing else []
    return SCFResult(energy=energies[-1], converged=converged, cycles=cycle, density=d,
                     mo_energy=mo_e, mo_coeff=c, nocc=nocc, jk_ms=times, energies=energies)


def rhf_gradient(mol: Molecule, res: SCFResult):
    """Nuclear gradient dE/dR (natom, 3) of a converged RHF result.

    One-electron terms (D-weighted h derivatives incl. the operator
    derivative, W-weighted overlap derivatives) and the two-electron J/K
    coordinate VJP with cotangents J* = D/2, K* = -D/4, then the centre
    rows folded onto their nuclei, plus the nuclear repulsion gradient.
    """
    dev = mol.device
    d = res.density
    c, e, nocc = res.mo_coeff, res.mo_energy, res.nocc
    wmat = 2.0 * (c[:, :nocc] * e[:nocc]) @ c[:, :nocc].T
    natm = mol.atm.shape[0]
    g1 = torch.zeros((natm, 3), dtype=torch.float64, device=dev)
    g2 = torch.zeros((natm, 3), dtype=torch.float64, device=dev)
    lib = _capi.lib()
    with torch.cuda.device(dev):
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        dd = d.contiguous()
        ww = wmat.contiguous()
        _capi.check(lib.b200jk_int1e_grad(mol.plan._h, ctypes.c_void_p(dd.data_ptr()),
                                          ctypes.c_void_p(ww.data_ptr()), ctypes.c_void_p(g1.data_ptr()), st))
        cot = torch.stack([d / 2.0, -d / 4.0]).reshape(2, 1, -1).contiguous()
        _capi.check(lib.b200jk_direct_jk_geom_vjp(mol.plan._h, ctypes.c_void_p(dd.data_ptr()), 1,
                                                  ctypes.c_void_p(cot.data_ptr()), 1, 1,
                                                  ctypes.c_void_p(g2.data_ptr()), st))
    g = (g1 + g2).cpu().numpy()
    nnuc = len(mol.charges)
    out = g[:nnuc].copy()
    for s, a in enumerate(mol.shell_atoms):
        out[a] += g[mol.bas[s, 0]]
    return out + nuclear_repulsion_gradient(mol.charges, mol.coords)
