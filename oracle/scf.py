"""CPU ORACLE -- test infrastructure only: numpy RHF energy and gradient on
libcint integrals (oracle/_ref/libcint_ref.so via oracle/__init__.py).

The SCF follows the reference caller's arithmetic:
  F = h + J - K/2,  E = tr(D h) + tr(D J)/2 - tr(D K)/4 + E_nuc
(src/gradscf/scf/energy.py:23-31), with D = 2 C_occ C_occ^T.
The gradient is the standard RHF expression; its two-electron part is the
reference's geometry VJP (csrc/direct_jk_geometry.cc:122-182) with cotangents
J* = D/2, K* = -D/4, and its one-electron part uses libcint's int1e_ip*
blocks the way the reference's geometry products do.
"""
from __future__ import annotations

import numpy as np

from . import direct_jk, direct_jk_geometry_vjp, int1e, int1e_ip


def _nuclear_repulsion(charges, coords):
    e = 0.0
    for i in range(len(charges)):
        for j in range(i):
            e += charges[i] * charges[j] / np.linalg.norm(coords[i] - coords[j])
    return e


def rhf(atm, bas, env, nelectron, charges, coords, *, cart, conv_tol=1e-12, max_cycle=100,
        cutoff=0.0, workers=8, density0=None):
    """Plain DIIS RHF.  Returns dict(energy, density, mo_energy, mo_coeff, ...)."""
    s = int1e(atm, bas, env, "ovlp", cart=cart)
    h = int1e(atm, bas, env, "kin", cart=cart) + int1e(atm, bas, env, "nuc", cart=cart)
    e_nuc = _nuclear_repulsion(charges, coords)
    nocc = nelectron // 2
    w, v = np.linalg.eigh(s)
    x = v / np.sqrt(w)
    def solve(f):
        e, c = np.linalg.eigh(x.T @ f @ x)
        return e, x @ c
    if density0 is None:
        e, c = solve(h)
        d = 2.0 * c[:, :nocc] @ c[:, :nocc].T
    else:
        d = density0
    hist_f, hist_e = [], []
    e_old = 0.0
    for cycle in range(max_cycle):
        j, k = direct_jk(atm, bas, env, d, cart=cart, cutoff=cutoff, workers=workers)
        f = h + j - 0.5 * k
        energy = np.sum(d * h) + 0.5 * np.sum(d * j) - 0.25 * np.sum(d * k) + e_nuc
        err = f @ d @ s - s @ d @ f
        hist_f.append(f); hist_e.append(err)
        hist_f, hist_e = hist_f[-8:], hist_e[-8:]
        if len(hist_f) > 1:
            m = len(hist_f)
            b = -np.ones((m + 1, m + 1)); b[m, m] = 0.0
            for i in range(m):
                for jj in range(m):
                    b[i, jj] = np.sum(hist_e[i] * hist_e[jj])
            rhs = np.zeros(m + 1); rhs[m] = -1.0
            coef = np.linalg.solve(b, rhs)[:m]
            f = sum(cf * fi for cf, fi in zip(coef, hist_f))
        mo_e, c = solve(f)
        d_new = 2.0 * c[:, :nocc] @ c[:, :nocc].T
        if abs(energy - e_old) < conv_tol and np.max(np.abs(err)) < np.sqrt(conv_tol) * 1e-3:
            d = d_new
            break
        e_old, d = energy, d_new
    j, k = direct_jk(atm, bas, env, d, cart=cart, cutoff=cutoff, workers=workers)
    f = h + j - 0.5 * k
    energy = np.sum(d * h) + 0.5 * np.sum(d * j) - 0.25 * np.sum(d * k) + e_nuc
    mo_e, c = solve(f)
    return dict(energy=energy, density=d, mo_energy=mo_e, mo_coeff=c, nocc=nocc, hcore=h,
                overlap=s, cycles=cycle + 1)


def rhf_gradient(atm, bas, env, result, charges, coords, shell_atoms, *, cart, workers=8):
    """d E_RHF / d R_nuclei, shape (natom, 3)."""
    d = result["density"]
    c, e, nocc = result["mo_coeff"], result["mo_energy"], result["nocc"]
    wmat = 2.0 * (c[:, :nocc] * e[:nocc]) @ c[:, :nocc].T
    natom = len(charges)
    n = d.shape[0]
    ao = np.zeros(len(bas) + 1, dtype=int)
    for s in range(len(bas)):
        l, nc = int(bas[s, 1]), int(bas[s, 3])
        ao[s + 1] = ao[s] + nc * (((l + 1) * (l + 2) // 2) if cart else 2 * l + 1)
    ao_atom = np.zeros(n, dtype=int)
    for s in range(len(bas)):
        ao_atom[ao[s]:ao[s + 1]] = shell_atoms[s]
    ipovlp = int1e_ip(atm, bas, env, "ipovlp", cart=cart)
    h1 = -(int1e_ip(atm, bas, env, "ipkin", cart=cart) + int1e_ip(atm, bas, env, "ipnuc", cart=cart))
    grad = np.zeros((natom, 3))
    for a in range(natom):
        rows = ao_atom == a
        vrinv = -charges[a] * int1e_ip(atm, bas, env, "iprinv", cart=cart, atom=a)
        vrinv[:, rows] += h1[:, rows]
        hd = vrinv + vrinv.transpose(0, 2, 1)
        grad[a] += np.einsum("xij,ij->x", hd, d)
        sd = np.zeros_like(ipovlp)
        sd[:, rows] = -ipovlp[:, rows]
        sd = sd + sd.transpose(0, 2, 1)
        grad[a] -= np.einsum("xij,ij->x", sd, wmat)
    cot = np.stack([d[None] / 2.0, -d[None] / 4.0])
    genv = direct_jk_geometry_vjp(atm, bas, env, d[None], cot, cart=cart, workers=workers)
    for s in range(len(bas)):
        ptr = atm[bas[s, 0], 1]
        grad[shell_atoms[s]] += genv[ptr:ptr + 3]
    for i in range(natom):
        for j in range(natom):
            if i != j:
                r = coords[i] - coords[j]
                grad[i] -= charges[i] * charges[j] * r / np.linalg.norm(r) ** 3
    return grad


def uhf(atm, bas, env, nalpha, nbeta, charges, coords, *, cart, conv_tol=1e-12, max_cycle=100,
        workers=8):
    """Plain DIIS UHF on stacked (D_a, D_b) direct J/K builds, as the
    reference's UKS caller builds them (src/gradscf/scf/uks.py:255-265):
    J = J(D_a) + J(D_b), K_s = K(D_s), F_s = h + J - K_s,
    E = tr(D_tot h) + tr(D_tot J)/2 - (tr(D_a K_a) + tr(D_b K_b))/2 + E_nuc."""
    s = int1e(atm, bas, env, "ovlp", cart=cart)
    h = int1e(atm, bas, env, "kin", cart=cart) + int1e(atm, bas, env, "nuc", cart=cart)
    e_nuc = _nuclear_repulsion(charges, coords)
    w, v = np.linalg.eigh(s)
    x = v / np.sqrt(w)

    def solve(f):
        e, c = np.linalg.eigh(x.T @ f @ x)
        return e, x @ c

    _, c = solve(h)
    da, db = c[:, :nalpha] @ c[:, :nalpha].T, c[:, :nbeta] @ c[:, :nbeta].T
    hist_f, hist_e = [], []
    e_old = None
    for cycle in range(max_cycle):
        j, k = direct_jk(atm, bas, env, np.stack([da, db]), cart=cart, workers=workers)
        jt = j.sum(0)
        fa, fb = h + jt - k[0], h + jt - k[1]
        dt = da + db
        energy = np.sum(dt * h) + 0.5 * np.sum(dt * jt) - 0.5 * (np.sum(da * k[0]) + np.sum(db * k[1])) + e_nuc
        err = np.stack([x.T @ (fa @ da @ s - s @ da @ fa) @ x, x.T @ (fb @ db @ s - s @ db @ fb) @ x])
        if e_old is not None and abs(energy - e_old) < conv_tol and np.linalg.norm(err) < np.sqrt(conv_tol):
            return dict(energy=energy, density_a=da, density_b=db, cycles=cycle + 1)
        hist_f.append(np.stack([fa, fb])); hist_e.append(err)
        hist_f, hist_e = hist_f[-8:], hist_e[-8:]
        f2 = np.stack([fa, fb])
        if len(hist_f) > 1:
            m = len(hist_f)
            bm = -np.ones((m + 1, m + 1)); bm[m, m] = 0.0
            for i in range(m):
                for jj in range(m):
                    bm[i, jj] = np.sum(hist_e[i] * hist_e[jj])
            rhs = np.zeros(m + 1); rhs[m] = -1.0
            coef = np.linalg.solve(bm, rhs)[:m]
            f2 = sum(cf * fi for cf, fi in zip(coef, hist_f))
        _, ca = solve(f2[0]); _, cb = solve(f2[1])
        da, db = ca[:, :nalpha] @ ca[:, :nalpha].T, cb[:, :nbeta] @ cb[:, :nbeta].T
        e_old = energy
    return dict(energy=energy, density_a=da, density_b=db, cycles=max_cycle)
