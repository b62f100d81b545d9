"""One-electron integrals, the J/K coordinate VJP and RHF energy/forces on
the GPU against the oracle and the reference's published G01 record."""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import ctypes  # noqa: E402

import oracle  # noqa: E402
from oracle import scf as oscf  # noqa: E402
from gradscf_b200 import _capi  # noqa: E402
from gradscf_b200 import scf as S  # noqa: E402
from gradscf_b200.jk import DirectJKPlan  # noqa: E402
from tests.gpu_util import WATER, tables  # noqa: E402


@pytest.mark.parametrize("basis,cart", [("6-31g*", True), ("6-31g*", False), ("cc-pvtz", False),
                                        ("cc-pvdz", True)])
def test_one_electron_matrices_vs_oracle(basis, cart):
    mol = S.Molecule(WATER, basis, cart=cart)
    for which in ("ovlp", "kin", "nuc"):
        ref = oracle.int1e(mol.atm, mol.bas, mol.env, which, cart=cart)
        got = mol.int1e(which).cpu().numpy()
        assert np.abs(got - ref).max() < 1e-11, which


def _vjp(plan, d, cot, with_j=True, with_k=True):
    n = d.shape[-1]
    natm = plan.natm[0]
    g = torch.zeros((natm, 3), dtype=torch.float64, device="cuda")
    dd = torch.as_tensor(d, device="cuda").reshape(-1, n * n).contiguous()
    cc = torch.as_tensor(cot, device="cuda").reshape(-1, n * n).contiguous()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(_capi.lib().b200jk_direct_jk_geom_vjp(plan._h, ctypes.c_void_p(dd.data_ptr()), dd.shape[0],
                                                      ctypes.c_void_p(cc.data_ptr()), int(with_j), int(with_k),
                                                      ctypes.c_void_p(g.data_ptr()), st))
    return g.cpu().numpy()


@pytest.mark.parametrize("basis,cart,omega", [("6-31g*", False, 0.0), ("6-31g*", True, 0.0),
                                              ("cc-pvdz", False, 0.0), ("6-31g*", False, 0.33),
                                              ("cc-pvtz", False, 0.0)])
def test_geometry_vjp_vs_oracle_nonsymmetric(basis, cart, omega):
    # omega > 0: the erf(omega r)/r derivative integrals (libcint env[8])
    top, par, sa, atm, bas, env = tables(WATER, basis, cart)
    env = np.array(env, dtype=np.float64, copy=True)
    env[8] = omega
    rng = np.random.default_rng(932)
    n = top.nao
    d = rng.normal(size=(2, n, n))
    cot = rng.normal(size=(2, 2, n, n))
    plan = DirectJKPlan([(atm, bas, env)], cart=cart, cutoff=0.0)
    got = _vjp(plan, d, cot)
    ref_env = oracle.direct_jk_geometry_vjp(atm, bas, env, d, cot, cart=cart, workers=8)
    ref = np.stack([ref_env[atm[i, 1]:atm[i, 1] + 3] for i in range(len(atm))])
    assert np.abs(got - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())
    # translation sum rule
    assert np.abs(got.sum(0)).max() < 1e-9 * max(1.0, np.abs(ref).max())


def test_g01_water_rhf_energy_and_forces(golden_dir):
    rec = json.loads((golden_dir / "g01_water_rhf.json").read_text())
    atom = "; ".join(f"{s} {x} {y} {z}" for s, (x, y, z) in zip(rec["symbols"], rec["coordinates_bohr"]))
    mol = S.Molecule(atom, rec["basis"], unit="Bohr", cart=rec["cart"], schwarz_cut=0.0)
    res = S.rhf(mol, conv_tol=1e-13, conv_tol_grad=1e-9)
    assert res.converged
    assert abs(res.energy - rec["energy_hartree"]) < 1e-9
    grad = S.rhf_gradient(mol, res)
    np.testing.assert_allclose(grad, rec["gradient_hartree_per_bohr"], atol=1e-8)


def test_water_cc_pvdz_rhf_fp64_vs_oracle_and_split():
    mol = S.Molecule(WATER, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    res = S.rhf(mol, conv_tol=1e-10)
    ref = oscf.rhf(mol.atm, mol.bas, mol.env, 10, mol.charges, mol.coords, cart=False,
                   conv_tol=1e-12, cutoff=1e-12)
    assert res.converged and abs(res.energy - ref["energy"]) < 1e-9
    split = S.rhf(mol, conv_tol=1e-10, precision="split")
    assert split.converged and abs(split.energy - res.energy) < 1e-8


@pytest.mark.parametrize("precision,use_graph", [("fp64", False), ("split", True)])
def test_batched_rhf_matches_single_molecule_rhf(precision, use_graph):
    # uneven batch: two clusters of equal size share a vectorised group
    from gradscf_b200 import workloads as W
    specs = [W.water_cluster(n, 1000 + i) for i, n in enumerate((1, 3, 2, 3))]
    batch = S.MoleculeBatch(specs, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    en, ds, ms, cycles, conv = S.rhf_batch(batch, conv_tol=1e-10, precision=precision, use_graph=use_graph)
    assert conv.all() and len(ms) == cycles
    for m, spec in enumerate(specs):
        mol = S.Molecule(spec, "cc-pvdz", cart=False, schwarz_cut=1e-12)
        ref = S.rhf(mol, conv_tol=1e-10, precision=precision)
        assert abs(en[m] - ref.energy) < 1e-8, (m, en[m], ref.energy)
        assert ds[m].shape == (mol.nao, mol.nao)


def test_uhf_doublet_on_stacked_alpha_beta_builds_vs_oracle():
    # the reference's UKS caller (scf/uks.py:255-265) stacks (D_a, D_b) into
    # one nb = 2 direct J/K call; here the GPU UHF of the water cation
    # (doublet, cc-pVDZ) against the oracle's UHF on the same stacked builds
    from oracle import scf as OS
    mol = S.Molecule(WATER, "cc-pvdz", cart=False, schwarz_cut=0.0, charge=1)
    res = S.uhf(mol, spin=1, conv_tol=1e-11)
    assert res.converged
    na = (mol.nelectron + 1) // 2
    ref = OS.uhf(mol.atm, mol.bas, mol.env, na, mol.nelectron - na, mol.charges, mol.coords, cart=False,
                 conv_tol=1e-12)
    assert abs(res.energy - ref["energy"]) < 1e-8
    # one stacked build against the oracle's at the converged densities
    da, db = res.density_a, res.density_b
    dt, j, ka, kb = S.uhf_jk(mol, da, db)
    j0, k0 = oracle.direct_jk(mol.atm, mol.bas, mol.env, np.stack([da.cpu().numpy(), db.cpu().numpy()]),
                              cart=False, workers=8)
    assert np.abs(j.cpu().numpy() - j0.sum(0)).max() < 1e-10
    assert np.abs(ka.cpu().numpy() - k0[0]).max() < 1e-10 and np.abs(kb.cpu().numpy() - k0[1]).max() < 1e-10


def test_split_precision_vjp_matches_fp64():
    # (H2O)3 cc-pVTZ (f shells: every VJP kernel family), converged RHF density:
    # the FP64 slice alone (cut 0) is the FP64 VJP; FP32 slices stay close
    from gradscf_b200 import workloads as W
    mol = S.Molecule(W.water_cluster(3, 2), "cc-pvtz", cart=False, schwarz_cut=1e-12)
    res = S.rhf(mol, conv_tol=1e-9)
    g64 = S.rhf_gradient(mol, res)
    g0 = S.rhf_gradient(mol, res, precision="split", fp32_cut=0.0)
    assert np.abs(g0 - g64).max() < 1e-12
    for cut, tol in ((1e-6, 1e-8), (1e-3, 1e-6)):
        gs = S.rhf_gradient(mol, res, precision="split", fp32_cut=cut)
        err = np.abs(gs - g64).max()
        assert 0.0 < err < tol, (cut, err)
