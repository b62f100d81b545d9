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
from .jk import DEFAULT_FP32_CUT, PRECISIONS, DirectJKPlan


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
        fp32_cut=DEFAULT_FP32_CUT, incremental=True, diis_space=8, density0=None, timing=True,
        fixed_cycles=None, on_jk=None, use_graph=False):
    """Run RHF; returns SCFResult (energy in Hartree).

    fixed_cycles: run exactly that many iterations (no convergence stop).
    use_graph: replay one CUDA-graph-captured J/K build per iteration.
    on_jk(cycle, delta): optional callback before each J/K build (e.g. to
    flush L2 or toggle profiling); its work is outside the timed build.
    """
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
    graph = None
    if use_graph:
        from .jk import JKGraph
        graph = JKGraph(mol.plan, 1, hermi=1, precision=precision, fp32_cut=fp32_cut)
    n = mol.nao
    ncyc = fixed_cycles if fixed_cycles is not None else max_cycle
    for cycle in range(1, ncyc + 1):
        delta = d - d_last if incremental else d
        if on_jk is not None:
            on_jk(cycle, delta)
        if timing:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
        if graph is not None:
            o = graph.run(delta)
            dj, dk = o[0, 0].reshape(n, n), o[1, 0].reshape(n, n)
        else:
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
            if fixed_cycles is None:
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
    if graph is not None:
        graph.close()
    times = [a.elapsed_time(b) for a, b in jk_ms] if timing else []
    return SCFResult(energy=energies[-1], converged=converged, cycles=cycle, density=d,
                     mo_energy=mo_e, mo_coeff=c, nocc=nocc, jk_ms=times, energies=energies)


def rhf_gradient(mol: Molecule, res: SCFResult, *, precision="fp64", fp32_cut=DEFAULT_FP32_CUT):
    """Nuclear gradient dE/dR (natom, 3) of a converged RHF result.

    One-electron terms (D-weighted h derivatives incl. the operator
    derivative, W-weighted overlap derivatives) and the two-electron J/K
    coordinate VJP with cotangents J* = D/2, K* = -D/4, then the centre
    rows folded onto their nuclei, plus the nuclear repulsion gradient.
    precision="split" runs the VJP's small-bound quartets in FP32
    (b200jk_direct_jk_geom_vjp_precision).
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
        _capi.check(lib.b200jk_direct_jk_geom_vjp_precision(
            mol.plan._h, ctypes.c_void_p(dd.data_ptr()), 1, ctypes.c_void_p(cot.data_ptr()), 1, 1,
            PRECISIONS[precision], float(fp32_cut), ctypes.c_void_p(g2.data_ptr()), st))
    mol.plan.reduce_shards(g2)   # sharded plan: sum the ranks' two-electron parts
    g = (g1 + g2).cpu().numpy()
    nnuc = len(mol.charges)
    out = g[:nnuc].copy()
    for s, a in enumerate(mol.shell_atoms):
        out[a] += g[mol.bas[s, 0]]
    return out + nuclear_repulsion_gradient(mol.charges, mol.coords)


def uhf_jk(mol: Molecule, density_a, density_b, *, with_k=True, precision="fp64",
           fp32_cut=DEFAULT_FP32_CUT):
    """Open-shell J/K as the reference's UKS caller builds them
    (src/gradscf/scf/uks.py:255-265): one build of the stacked (D_a, D_b)
    batch; J = J(D_a) + J(D_b), K_a = K(D_a), K_b = K(D_b).  Without K one
    build of D_a + D_b.  Returns (D_tot, J, K_a, K_b)."""
    d_tot = density_a + density_b
    if not with_k:
        j, _ = mol.plan.jk(d_tot, with_k=False, hermi=True, precision=precision, fp32_cut=fp32_cut)
        z = torch.zeros_like(j)
        return d_tot, j, z, z
    j, k = mol.plan.jk(torch.stack((density_a, density_b)), hermi=True, precision=precision,
                       fp32_cut=fp32_cut)
    return d_tot, j.sum(0), k[0], k[1]


@dataclass
class UHFResult:
    energy: float
    converged: bool
    cycles: int
    density_a: torch.Tensor
    density_b: torch.Tensor
    energies: list = field(default_factory=list)


def uhf(mol: Molecule, *, spin=0, conv_tol=1e-10, max_cycle=100, precision="fp64",
        fp32_cut=DEFAULT_FP32_CUT, diis_space=8):
    """Unrestricted Hartree-Fock on the batched (nb = 2) J/K build:
    F_s = h + J - K_s, E = tr(D_tot h) + tr(D_tot J)/2 - (tr(D_a K_a) + tr(D_b K_b))/2
    + E_nuc, with D_s = C_s,occ C_s,occ^T and spin = n_alpha - n_beta.
    DIIS on the stacked alpha/beta commutators; core guess."""
    dev = mol.device
    s = mol.int1e("ovlp")
    h = mol.int1e("kin") + mol.int1e("nuc")
    w, v = torch.linalg.eigh(s)
    x = v / torch.sqrt(w)
    na = (mol.nelectron + spin) // 2
    nb = mol.nelectron - na
    if na - nb != spin or na < 0 or nb < 0:
        raise ValueError("spin is incompatible with the electron count")
    _, c = _solve(h, x)
    da = c[:, :na] @ c[:, :na].T
    db = c[:, :nb] @ c[:, :nb].T
    hist_f, hist_e, energies = [], [], []
    e_old = None
    converged = False
    cycle = 0
    for cycle in range(1, max_cycle + 1):
        dt, j, ka, kb = uhf_jk(mol, da, db, precision=precision, fp32_cut=fp32_cut)
        fa, fb = h + j - ka, h + j - kb
        energy = (torch.sum(dt * h) + 0.5 * torch.sum(dt * j)
                  - 0.5 * (torch.sum(da * ka) + torch.sum(db * kb))).item() + mol.e_nuc
        energies.append(energy)
        err = torch.stack([x.T @ (fa @ da @ s - s @ da @ fa) @ x, x.T @ (fb @ db @ s - s @ db @ fb) @ x])
        gnorm = torch.linalg.norm(err).item()
        if e_old is not None and abs(energy - e_old) < conv_tol and gnorm < np.sqrt(conv_tol):
            converged = True
            break
        hist_f.append(torch.stack([fa, fb]))
        hist_e.append(err)
        hist_f, hist_e = hist_f[-diis_space:], hist_e[-diis_space:]
        f2 = torch.stack([fa, fb])
        if len(hist_f) > 1:
            m = len(hist_f)
            bm = -torch.ones((m + 1, m + 1), dtype=torch.float64, device=dev)
            bm[m, m] = 0.0
            for i in range(m):
                for k_ in range(i, m):
                    bm[i, k_] = bm[k_, i] = torch.sum(hist_e[i] * hist_e[k_])
            rhs = torch.zeros(m + 1, dtype=torch.float64, device=dev)
            rhs[m] = -1.0
            coef = torch.linalg.solve(bm, rhs)[:m]
            f2 = sum(cf * fi for cf, fi in zip(coef, hist_f))
        _, ca = _solve(f2[0], x)
        _, cb = _solve(f2[1], x)
        da = ca[:, :na] @ ca[:, :na].T
        db = cb[:, :nb] @ cb[:, :nb].T
        e_old = energy
    return UHFResult(energy=energies[-1], converged=converged, cycles=cycle, density_a=da, density_b=db,
                     energies=energies)


class MoleculeBatch:
    """Independent molecules sharing one device plan (packed per-molecule blocks)."""

    def __init__(self, atoms, basis, *, unit="Angstrom", cart=False, schwarz_cut=1e-12, device=None):
        self.mols = []
        tables = []
        for atom in atoms:
            top, par, sa = prepare_basis(atom, basis, unit=unit, cart=cart)
            atm, bas, env = pack(top, par)
            charges = np.asarray(top.nuclear_charges, dtype=np.float64)
            coords = np.asarray(par.nuclear_coords, dtype=np.float64)
            self.mols.append(dict(atm=atm, bas=bas, env=env, charges=charges, coords=coords,
                                  nelectron=int(charges.sum()), e_nuc=nuclear_repulsion(charges, coords)))
            tables.append((atm, bas, env))
        self.plan = DirectJKPlan(tables, cart=cart, cutoff=schwarz_cut, device=device)
        self.device = self.plan.device
        self.nao = self.plan.nao
        self.offsets = self.plan.offsets

    def int1e(self, which):
        out = torch.empty((self.plan.packed_size,), dtype=torch.float64, device=self.device)
        code = {"ovlp": 0, "kin": 1, "nuc": 2}[which]
        with torch.cuda.device(self.device):
            st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            _capi.check(_capi.lib().b200jk_int1e(self.plan._h, code, ctypes.c_void_p(out.data_ptr()), st))
        return out

    def block(self, packed, m):
        n = self.nao[m]
        return packed[self.offsets[m]:self.offsets[m] + n * n].view(n, n)


def rhf_batch(batch: MoleculeBatch, *, conv_tol=1e-10, max_cycle=60, precision="fp64",
              fp32_cut=DEFAULT_FP32_CUT, diis_space=8, timing=True, use_graph=False,
              fixed_cycles=None, density0=None):
    """RHF of every molecule of the batch, vectorised over molecules of equal
    (nao, nocc): batched Fock/energy/DIIS/eigh in torch, and ONE packed J/K
    build (optionally a replayed CUDA graph) per iteration for all molecules.

    Returns (energies ndarray, densities list, jk_ms list, cycles, converged ndarray).
    """
    dev = batch.device
    plan = batch.plan
    s_all, h_all = batch.int1e("ovlp"), batch.int1e("kin") + batch.int1e("nuc")
    nm = len(batch.mols)
    keys = {}
    for m in range(nm):
        keys.setdefault((batch.nao[m], batch.mols[m]["nelectron"] // 2), []).append(m)
    groups = []
    for (n, nocc), ms in keys.items():
        base = torch.as_tensor([batch.offsets[m] for m in ms], device=dev, dtype=torch.int64)
        idx = base[:, None] + torch.arange(n * n, device=dev)[None, :]
        S = s_all[idx].view(-1, n, n)
        H = h_all[idx].view(-1, n, n)
        w, v = torch.linalg.eigh(S)
        X = v / torch.sqrt(w)[:, None, :]
        if density0 is None:
            e, c = torch.linalg.eigh(X.transpose(1, 2) @ H @ X)
            C = X @ c
            D = 2.0 * C[:, :, :nocc] @ C[:, :, :nocc].transpose(1, 2)
        else:
            D = torch.stack([density0[m] for m in ms]).to(dev)
        enuc = torch.as_tensor([batch.mols[m]["e_nuc"] for m in ms], device=dev, dtype=torch.float64)
        groups.append(dict(ms=ms, n=n, nocc=nocc, idx=idx, S=S, H=H, X=X, D=D, enuc=enuc, hf=[], he=[],
                           e_old=None, done=torch.zeros(len(ms), dtype=torch.bool, device=dev),
                           energy=torch.zeros(len(ms), dtype=torch.float64, device=dev)))
    packed = plan.packed_size
    d_last = torch.zeros(packed, dtype=torch.float64, device=dev)
    jk = torch.zeros((2, packed), dtype=torch.float64, device=dev)
    graph = None
    if use_graph:
        from .jk import JKGraph
        graph = JKGraph(plan, 1, hermi=1, precision=precision, fp32_cut=fp32_cut)
    jk_ms = []
    stream = torch.cuda.current_stream(dev)
    tol_grad = float(np.sqrt(conv_tol))
    ncyc = fixed_cycles if fixed_cycles is not None else max_cycle
    cycle = 0
    for cycle in range(1, ncyc + 1):
        d_packed = torch.zeros(packed, dtype=torch.float64, device=dev)
        for g in groups:
            d_packed[g["idx"].reshape(-1)] = g["D"].reshape(-1)
        delta = (d_packed - d_last).reshape(1, -1)
        if timing:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
        out = graph.run(delta) if graph is not None else plan.jk_packed(
            delta.contiguous(), hermi=1, precision=precision, fp32_cut=fp32_cut, check=False)
        if timing:
            ev1.record(stream)
            jk_ms.append((ev0, ev1))
        jk += out[:, 0]
        d_last = d_packed
        all_done = True
        for g in groups:
            n = g["n"]
            J = jk[0][g["idx"]].view(-1, n, n)
            K = jk[1][g["idx"]].view(-1, n, n)
            D, H, S, X = g["D"], g["H"], g["S"], g["X"]
            F = H + J - 0.5 * K
            en = (D * H).sum((1, 2)) + 0.5 * (D * J).sum((1, 2)) - 0.25 * (D * K).sum((1, 2)) + g["enuc"]
            err = X.transpose(1, 2) @ (F @ D @ S - S @ D @ F) @ X
            gn = torch.linalg.norm(err, dim=(1, 2))
            if g["e_old"] is not None:
                g["done"] = g["done"] | (((en - g["e_old"]).abs() < conv_tol) & (gn < tol_grad))
            g["energy"] = en
            g["e_old"] = en
            if not bool(g["done"].all()):
                all_done = False
            g["hf"].append(F)
            g["he"].append(err)
            del g["hf"][:-diis_space], g["he"][:-diis_space]
            k_ = len(g["hf"])
            if k_ > 1:
                E = torch.stack(g["he"], 1)                       # (G, k, n, n)
                Bm = -torch.ones((E.shape[0], k_ + 1, k_ + 1), dtype=torch.float64, device=dev)
                Bm[:, :k_, :k_] = torch.einsum("gaij,gbij->gab", E, E)
                Bm[:, k_, k_] = 0.0
                rhs = torch.zeros((E.shape[0], k_ + 1), dtype=torch.float64, device=dev)
                rhs[:, k_] = -1.0
                coef = torch.linalg.solve(Bm, rhs)[:, :k_]
                F = torch.einsum("gk,gkij->gij", coef, torch.stack(g["hf"], 1))
            e, c = torch.linalg.eigh(X.transpose(1, 2) @ F @ X)
            C = X @ c
            g["D"] = 2.0 * C[:, :, :g["nocc"]] @ C[:, :, :g["nocc"]].transpose(1, 2)
        if all_done and fixed_cycles is None:
            break
    torch.cuda.synchronize(dev)
    if graph is not None:
        graph.close()
    energies = np.zeros(nm)
    converged = np.zeros(nm, dtype=bool)
    densities = [None] * nm
    for g in groups:
        en = g["energy"].cpu().numpy()
        dn = g["done"].cpu().numpy()
        for i, m in enumerate(g["ms"]):
            energies[m] = en[i]
            converged[m] = dn[i]
            densities[m] = g["D"][i]
    times = [a.elapsed_time(b) for a, b in jk_ms] if timing else []
    return energies, densities, times, cycle, converged


def replica_shard(costs, rank, world):
    """The molecules of a batch that rank `rank` of `world` runs when a batch
    of independent molecules runs as replicas (no collective on the data
    path): contiguous cost-balanced blocks (b200jk_partition_items).  Returns
    the molecule indices."""
    owner = _capi.partition_items(np.asarray(costs, dtype=np.int64), world)
    return np.nonzero(owner == rank)[0]


def gather_replicas(ids, values, count, group=None):
    """Every rank's per-molecule results (molecule ids -> values) gathered on
    every rank into one array of `count` (one host all-gather at the end)."""
    import torch.distributed as dist
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, ([int(i) for i in ids], [float(v) for v in values]), group=group)
    out = np.full(count, np.nan)
    for pid, pval in parts:
        out[pid] = pval
    return out


def fragment_guess(mol: Molecule, fragments, basis, *, unit="Angstrom"):
    """Block-diagonal guess density from converged RHF densities of the
    fragments (consecutive atoms of `mol`, in order), all solved in one
    batched J/K plan."""
    batch = MoleculeBatch(fragments, basis, unit=unit, cart=mol.cart, device=mol.device)
    _, ds, _, _, _ = rhf_batch(batch, conv_tol=1e-8, timing=False)
    d0 = torch.zeros((mol.nao, mol.nao), dtype=torch.float64, device=mol.device)
    o = 0
    for d in ds:
        n = d.shape[0]
        d0[o:o + n, o:o + n] = d
        o += n
    if o != mol.nao:
        raise ValueError("fragments do not cover the molecule's basis")
    return d0
