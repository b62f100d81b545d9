"""CUDA-graph replay, the torch.autograd wrapper and RHF forces on the GPU.

Density derivatives follow the reference test
tests/integrals/test_native_direct_parallel.py:105-129 (loss 0.7 sum J^2 +
0.3 sum K^2 against the full-ERI einsum, atol 2e-9); coordinate derivatives
are checked against the oracle's restatement of the reference geometry VJP
and central finite differences (step 1e-4 Bohr, as
tests/integrals/test_direct_geometry_response.py:83-89).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import oracle  # noqa: E402
from gradscf_b200 import basis as B  # noqa: E402
from gradscf_b200 import scf as S  # noqa: E402
from gradscf_b200 import workloads as W  # noqa: E402
from gradscf_b200.autograd import BasisContext, direct_jk_ad  # noqa: E402
from gradscf_b200.jk import JKGraph  # noqa: E402
from tests.gpu_util import WATER  # noqa: E402


def test_graph_replay_matches_eager_build():
    mol = S.Molecule(W.water_cluster(3, 1), "cc-pvdz", cart=False)
    n = mol.nao
    for precision in ("fp64", "split"):
        graph = JKGraph(mol.plan, 1, precision=precision)
        for seed in (1, 2):
            d = torch.as_tensor(W.psd_density(n, 15, seed), device="cuda")
            ref = mol.plan.jk_packed(d.reshape(1, -1), hermi=1, precision=precision).clone()
            got = graph.run(d).clone()
            assert (got - ref).abs().max().item() < 1e-11
        graph.close()


def test_rhf_with_graph_matches_eager():
    mol = S.Molecule(W.water_cluster(2, 1), "cc-pvdz", cart=False)
    a = S.rhf(mol, conv_tol=1e-10)
    b = S.rhf(mol, conv_tol=1e-10, use_graph=True)
    assert abs(a.energy - b.energy) < 1e-10


def _ctx(atom, basis, cart, cutoff=0.0):
    top, par, sa = B.prepare_basis(atom, basis, cart=cart)
    return BasisContext(top, par, sa, cutoff=cutoff), top, par, sa


def test_density_gradient_matches_einsum_reference():
    ctx, top, par, sa = _ctx(WATER, "6-31g*", False)
    atm, bas, env = B.pack(top, par)
    eri = oracle.eri_s1(atm, bas, env, cart=False)
    rng = np.random.default_rng(804)
    d0 = rng.normal(size=(2, top.nao, top.nao))
    d = torch.tensor(d0, device="cuda", requires_grad=True)
    coords = torch.tensor(par.nuclear_coords, device="cuda")
    j, k = direct_jk_ad(ctx, d, coords)
    loss = 0.7 * (j ** 2).sum() + 0.3 * (k ** 2).sum()
    loss.backward()
    jr, kr = oracle.full_jk(eri, d0)
    # dL/dD = J(1.4 J) + K(0.6 K) (self-adjoint maps)
    gj, _ = oracle.full_jk(eri, 1.4 * jr)
    _, gk = oracle.full_jk(eri, 0.6 * kr)
    np.testing.assert_allclose(d.grad.cpu().numpy(), gj + gk, atol=2e-9, rtol=2e-10)


def test_coordinate_gradient_vs_oracle_vjp_and_finite_differences():
    atom = "O 0 0 0; H 0 0.7572 0.5865; H 0.05 -0.7572 0.5865"
    ctx, top, par, sa = _ctx(atom, "6-31g*", False)
    atm, bas, env = B.pack(top, par)
    n = top.nao
    rng = np.random.default_rng(932)
    d0 = rng.normal(size=(n, n))
    wj, wk = rng.normal(size=(2, n, n))
    coords0 = np.asarray(par.nuclear_coords)

    def loss_at(c, grad=False):
        coords = torch.tensor(c, device="cuda", requires_grad=grad)
        j, k = direct_jk_ad(ctx, torch.as_tensor(d0, device="cuda"), coords)
        loss = (torch.as_tensor(wj, device="cuda") * j).sum() + (torch.as_tensor(wk, device="cuda") * k).sum()
        if grad:
            loss.backward()
            return coords.grad.cpu().numpy()
        return loss.item()

    g = loss_at(coords0, grad=True)
    # oracle: env-sized VJP with cotangents (wj, wk), centre rows folded onto nuclei
    genv = oracle.direct_jk_geometry_vjp(atm, bas, env, d0[None], np.stack([wj[None], wk[None]]),
                                         cart=False, workers=8)
    ref = np.zeros_like(g)
    for s, a in enumerate(sa):
        p = atm[bas[s, 0], 1]
        ref[a] += genv[p:p + 3]
    np.testing.assert_allclose(g, ref, atol=1e-9 * max(1.0, np.abs(ref).max()))
    h = 1e-4
    for atom_i, axis in ((0, 2), (1, 1), (2, 0)):
        cp, cm = coords0.copy(), coords0.copy()
        cp[atom_i, axis] += h
        cm[atom_i, axis] -= h
        fd = (loss_at(cp) - loss_at(cm)) / (2 * h)
        assert abs(fd - g[atom_i, axis]) < 2e-7 * max(1.0, abs(fd))


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_rhf_forces_finite_differences_water_cluster(precision):
    # (H2O)4 6-31G* from the seeded generator; central differences with step
    # 1e-4 Bohr on 6 random coordinates (seed 2), tolerance 1e-6 Ha/Bohr.
    spec = W.water_cluster(4, 2)
    mol = S.Molecule(spec, "6-31g*", cart=False, schwarz_cut=1e-12)
    res = S.rhf(mol, conv_tol=1e-12, conv_tol_grad=1e-9, precision=precision)
    g = S.rhf_gradient(mol, res)
    natom = len(mol.charges)
    rng = np.random.default_rng(2)
    picks = [(int(rng.integers(natom)), int(rng.integers(3))) for _ in range(6)]
    coords = mol.coords.copy()
    syms = ["O", "H", "H"] * 4
    h = 1e-4

    def energy(c):
        atom = [(s, tuple(x)) for s, x in zip(syms, c)]
        m = S.Molecule(atom, "6-31g*", unit="Bohr", cart=False, schwarz_cut=1e-12)
        return S.rhf(m, conv_tol=1e-12, conv_tol_grad=1e-9, precision=precision, density0=res.density).energy

    for a, x in picks:
        cp, cm = coords.copy(), coords.copy()
        cp[a, x] += h
        cm[a, x] -= h
        fd = (energy(cp) - energy(cm)) / (2 * h)
        assert abs(fd - g[a, x]) < 1e-6, (a, x, fd, g[a, x])
    # translational invariance of the analytic gradient
    assert np.abs(g.sum(0)).max() < 1e-8
