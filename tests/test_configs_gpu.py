"""Parity at the benchmark workloads: the CUDA path against the CPU oracle on
the systems the throughput numbers are quoted on, so the scale-dependent code
paths (long ket runs cut into work items, heavy-item splitting, grouped
contraction buckets, the per-item FP32 boundary search, batched molecules)
meet the oracle at full size.

Workloads (seeded generator of gradscf_b200/workloads.py):
  * (H2O)32 cc-pVDZ, 768 functions, seed 1, Schwarz cut 1e-12: J/K of the
    fragment-guess density and of the first SCF iteration's increment dD;
  * (H2O)16 6-31G*, seed 2: RHF forces against the oracle gradient;
  * the batch of 256 uneven clusters (sizes from seed 3, cluster m from seed
    1000 + m): one batched plan, per-cluster J/K of a seeded subset;
  * the first 8 waters of the (H2O)64 cc-pVTZ cluster (seed 4): f shells.

Tolerances: FP64 J/K 1e-10 max-abs against the oracle (the reference's
libcint J/K); split precision 1e-8 Ha in the two-electron energy
E2 = tr(D J)/2 - tr(D K)/4 assembled from each side's J/K at the same
density; forces 1e-6 Ha/Bohr.  The oracle runs on every host core.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import oracle  # noqa: E402
import oracle.scf as OS  # noqa: E402
from gradscf_b200 import _capi, scf  # noqa: E402
from gradscf_b200 import basis as B  # noqa: E402
from gradscf_b200 import workloads as W  # noqa: E402
from gradscf_b200.jk import DirectJKPlan  # noqa: E402

WORKERS = os.cpu_count() or 1
FP32_CUT = 1e-6


def _fragments(spec, n):
    atoms = spec.split("; ")
    return ["; ".join(atoms[3 * i:3 * i + 3]) for i in range(n)]


def _e2(d, j, k):
    return 0.5 * float(np.sum(d * j)) - 0.25 * float(np.sum(d * k))


def _split_stats(plan):
    lib = _capi.lib()
    nc = _capi.NCLASS
    arrs = [(ctypes.c_int64 * nc)() for _ in range(4)]
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(lib.b200jk_plan_split_stats(plan._h, st, *arrs))
    q64, q32 = (int(np.frombuffer(a, dtype=np.int64).sum()) for a in arrs[:2])
    return q64, q32


@pytest.fixture(scope="module")
def c1():
    """(H2O)32 cc-pVDZ: fragment-guess density D0, first-iteration dD, and the
    oracle's J/K of both (one oracle call: each ERI is evaluated once for
    both densities)."""
    spec = W.water_cluster(32, 1)
    mol = scf.Molecule(spec, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    assert mol.nao == 768
    d0 = scf.fragment_guess(mol, _fragments(spec, 32), "cc-pvdz")
    res = scf.rhf(mol, fixed_cycles=1, density0=d0, timing=False)
    d0n = d0.cpu().numpy()
    dd = res.density.cpu().numpy() - d0n
    dens = np.stack([d0n, dd])
    j_or, k_or = oracle.direct_jk(mol.atm, mol.bas, mol.env, dens, cart=False, cutoff=1e-12,
                                  workers=WORKERS)
    return mol, dens, j_or, k_or


def test_c1_fp64_jk_matches_oracle(c1):
    mol, dens, j_or, k_or = c1
    n = mol.nao
    out = mol.plan.jk_packed(torch.as_tensor(dens.reshape(2, -1), device=mol.device), hermi=1)
    out = out.cpu().numpy().reshape(2, 2, n, n)
    for b in range(2):
        ej = np.abs(out[0, b] - j_or[b]).max()
        ek = np.abs(out[1, b] - k_or[b]).max()
        assert ej < 1e-10 and ek < 1e-10, (b, ej, ek)


def test_c1_split_energy_matches_oracle(c1):
    mol, dens, j_or, k_or = c1
    n = mol.nao
    plan = mol.plan
    parts = []
    fp32_share = []
    for b in range(2):
        x = torch.as_tensor(dens[b].reshape(1, -1), device=mol.device)
        o = plan.jk_packed(x, hermi=1, precision="split", fp32_cut=FP32_CUT).cpu().numpy()
        parts.append(o.reshape(2, n, n))
        q64, q32 = _split_stats(plan)
        fp32_share.append(q32 / (q32 + q64))
    # the increment's build runs mostly in FP32, as in the benchmark's SCF
    assert fp32_share[1] > 0.9, fp32_share
    # full density: E2(D0) from split J/K vs from the oracle's J/K
    d0, dd = dens
    e_gpu = _e2(d0, parts[0][0], parts[0][1])
    e_ref = _e2(d0, j_or[0], k_or[0])
    assert abs(e_gpu - e_ref) < 1e-8, (e_gpu, e_ref)
    # the next iteration's energy from incremental builds J(D0) + J(dD)
    d1 = d0 + dd
    j1, k1 = parts[0][0] + parts[1][0], parts[0][1] + parts[1][1]
    e_gpu = _e2(d1, j1, k1)
    e_ref = _e2(d1, j_or[0] + j_or[1], k_or[0] + k_or[1])
    assert abs(e_gpu - e_ref) < 1e-8, (e_gpu, e_ref)
    # element-wise error of the FP32-heavy increment build (reported bound)
    assert np.abs(parts[1][0] - j_or[1]).max() < 1e-6
    assert np.abs(parts[1][1] - k_or[1]).max() < 1e-6


def test_c2_forces_match_oracle_gradient():
    spec = W.water_cluster(16, 2)
    mol = scf.Molecule(spec, "6-31g*", cart=False, schwarz_cut=1e-12)
    assert mol.nao == 288
    d0 = scf.fragment_guess(mol, _fragments(spec, 16), "6-31g*")
    res = scf.rhf(mol, conv_tol=1e-11, conv_tol_grad=1e-8, density0=d0, timing=False)
    assert res.converged
    g_gpu = scf.rhf_gradient(mol, res)
    ref = dict(density=res.density.cpu().numpy(), mo_coeff=res.mo_coeff.cpu().numpy(),
               mo_energy=res.mo_energy.cpu().numpy(), nocc=res.nocc)
    g_ref = OS.rhf_gradient(mol.atm, mol.bas, mol.env, ref, mol.charges, mol.coords, mol.shell_atoms,
                            cart=False, workers=WORKERS)
    err = np.abs(g_gpu - g_ref).max()
    assert err < 1e-6, err
    # split-precision SCF: its forces agree with the FP64 ones to the same bar
    mol32 = scf.Molecule(spec, "6-31g*", cart=False, schwarz_cut=1e-12)
    res32 = scf.rhf(mol32, conv_tol=1e-11, conv_tol_grad=1e-8, density0=d0, precision="split",
                    timing=False)
    assert res32.converged
    assert abs(res32.energy - res.energy) < 1e-8
    assert np.abs(scf.rhf_gradient(mol32, res32) - g_ref).max() < 1e-6


def test_c3_batched_plan_subset_matches_oracle():
    sizes = W.batch_sizes(256, 3)
    specs = [W.water_cluster(int(nw), 1000 + m) for m, nw in enumerate(sizes)]
    tabs = []
    for s in specs:
        top, par, _ = B.prepare_basis(s, "cc-pvdz", cart=False)
        tabs.append(B.pack(top, par))
    plan = DirectJKPlan(tabs, cart=False, cutoff=1e-12)
    # one seeded PSD density per cluster, packed
    packed = np.zeros(plan.packed_size)
    dens = []
    for m, n in enumerate(plan.nao):
        d = W.psd_density(n, 5 * int(sizes[m]), 2000 + m)
        dens.append(d)
        packed[plan.offsets[m]:plan.offsets[m] + n * n] = d.ravel()
    x = torch.as_tensor(packed.reshape(1, -1), device=plan.device)
    out64 = plan.jk_packed(x, hermi=1).cpu().numpy()
    out32 = plan.jk_packed(x, hermi=1, precision="split", fp32_cut=FP32_CUT).cpu().numpy()
    # a seeded subset of 16 clusters of at most 10 waters (oracle time)
    small = [m for m in range(256) if sizes[m] <= 10]
    pick = np.random.default_rng(3).choice(small, size=16, replace=False)
    assert max(sizes[pick]) >= 6
    for m in pick:
        n = plan.nao[m]
        atm, bas, env = tabs[m]
        j0, k0 = oracle.direct_jk(atm, bas, env, dens[m], cart=False, cutoff=1e-12, workers=WORKERS)
        sl = slice(plan.offsets[m], plan.offsets[m] + n * n)
        j, k = out64[0, 0, sl].reshape(n, n), out64[1, 0, sl].reshape(n, n)
        assert np.abs(j - j0).max() < 1e-10 and np.abs(k - k0).max() < 1e-10, m
        js, ks = out32[0, 0, sl].reshape(n, n), out32[1, 0, sl].reshape(n, n)
        assert abs(_e2(dens[m], js, ks) - _e2(dens[m], j0, k0)) < 1e-8, m


def test_c4_cc_pvtz_subset_matches_oracle():
    # the first 8 waters of the (H2O)64 cc-pVTZ cluster: f shells on O, d on H
    atoms = W.water_cluster(64, 4).split("; ")[:24]
    mol = scf.Molecule("; ".join(atoms), "cc-pvtz", cart=False, schwarz_cut=1e-12)
    n = mol.nao
    assert n == 464
    d = W.psd_density(n, 40, 4)
    j0, k0 = oracle.direct_jk(mol.atm, mol.bas, mol.env, d, cart=False, cutoff=1e-12, workers=WORKERS)
    x = torch.as_tensor(d.reshape(1, -1), device=mol.device)
    o64 = mol.plan.jk_packed(x, hermi=1).cpu().numpy().reshape(2, n, n)
    assert np.abs(o64[0] - j0).max() < 1e-10 and np.abs(o64[1] - k0).max() < 1e-10
    o32 = mol.plan.jk_packed(x, hermi=1, precision="split", fp32_cut=FP32_CUT).cpu().numpy().reshape(2, n, n)
    assert abs(_e2(d, o32[0], o32[1]) - _e2(d, j0, k0)) < 1e-8
