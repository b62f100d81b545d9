"""The CPU oracle against the reference's own golden data (no GPU).

The oracle is libcint compiled from the reference sources plus a C
restatement of the reference's direct J/K driver; these tests pin it before
anything is compared with it.
"""
import json

import numpy as np
import pytest

import oracle
from oracle import scf
from gradscf_b200 import basis as B


def test_g01_water_energy_and_gradient(golden_dir):
    rec = json.loads((golden_dir / "g01_water_rhf.json").read_text())
    atom = "; ".join(f"{s} {x} {y} {z}" for s, (x, y, z) in zip(rec["symbols"], rec["coordinates_bohr"]))
    top, par, sa = B.prepare_basis(atom, rec["basis"], unit="Bohr", cart=rec["cart"])
    atm, bas, env = B.pack(top, par)
    charges = np.array(top.nuclear_charges, float)
    res = scf.rhf(atm, bas, env, 10, charges, par.nuclear_coords, cart=True, conv_tol=1e-13)
    assert abs(res["energy"] - rec["energy_hartree"]) < 1e-10
    g = scf.rhf_gradient(atm, bas, env, res, charges, par.nuclear_coords, sa, cart=True)
    np.testing.assert_allclose(g, rec["gradient_hartree_per_bohr"], atol=1e-9)


def test_h2_sto3g_direct_equals_einsum(golden_dir):
    rec = json.loads((golden_dir / "h2_sto3g_jk.json").read_text())
    top, par, _ = B.prepare_basis(rec["atom"], rec["basis"], cart=True)
    atm, bas, env = B.pack(top, par)
    j, k = oracle.direct_jk(atm, bas, env, np.array(rec["density"]), cart=True)
    np.testing.assert_allclose(j, rec["j"], atol=3e-12, rtol=3e-12)
    np.testing.assert_allclose(k, rec["k"], atol=3e-12, rtol=3e-12)


@pytest.mark.parametrize("cart", [False, True], ids=["sph", "cart"])
@pytest.mark.parametrize("workers", [1, 2, 4])
def test_general_contraction_direct_equals_einsum(golden_dir, cart, workers):
    rec = json.loads((golden_dir / "h2_general_jk.json").read_text())
    top, par, _ = B.prepare_basis(rec["atom"], rec["basis"], cart=cart)
    atm, bas, env = B.pack(top, par)
    sub = rec["cart" if cart else "sph"]
    j, k = oracle.direct_jk(atm, bas, env, np.array(sub["density"]), cart=cart, workers=workers)
    np.testing.assert_allclose(j, sub["j"], atol=2e-10, rtol=1e-10)
    np.testing.assert_allclose(k, sub["k"], atol=2e-10, rtol=1e-10)


def test_screening_is_linear_and_huge_cut_gives_zero(golden_dir):
    rec = json.loads((golden_dir / "h2_general_jk.json").read_text())
    top, par, _ = B.prepare_basis(rec["atom"], rec["basis"], cart=False)
    atm, bas, env = B.pack(top, par)
    rng = np.random.default_rng(803)
    d, t = rng.normal(size=(2, 4, top.nao, top.nao))
    a = oracle.direct_jk(atm, bas, env, d + 0.37 * t, cart=False, cutoff=1e-6)
    b = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-6)
    c = oracle.direct_jk(atm, bas, env, t, cart=False, cutoff=1e-6)
    for x, y, z in zip(a, b, c):
        np.testing.assert_allclose(x, y + 0.37 * z, atol=2e-10, rtol=1e-10)
    for x in oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e9):
        np.testing.assert_array_equal(x, 0.0)


def test_worker_partition_is_bitwise_reproducible():
    top, par, _ = B.prepare_basis("O 0 0 0; H 0 0.7572 0.5865; H 0 -0.7572 0.5865", "cc-pvdz", cart=False)
    atm, bas, env = B.pack(top, par)
    d = np.random.default_rng(802).normal(size=(2, top.nao, top.nao))
    first = oracle.direct_jk(atm, bas, env, d, cart=False, workers=4, cutoff=1e-12)
    again = oracle.direct_jk(atm, bas, env, d, cart=False, workers=4, cutoff=1e-12)
    for x, y in zip(first, again):
        np.testing.assert_array_equal(x, y)


def test_invalid_inputs_raise():
    top, par, _ = B.prepare_basis("H 0 0 0; H 0 0 0.74", "sto-3g", cart=True)
    atm, bas, env = B.pack(top, par)
    with pytest.raises(oracle.OracleError, match="Nonfinite"):
        oracle.direct_jk(atm, bas, env, np.full((2, 2), np.nan), cart=True)
    with pytest.raises(oracle.OracleError, match="workers"):
        oracle.direct_jk(atm, bas, env, np.eye(2), cart=True, workers=0)
    bad = bas.copy(); bad[0, 1] = 13
    with pytest.raises(oracle.OracleError, match="unsupported"):
        oracle.direct_jk(atm, bad, env, np.eye(2), cart=True)


@pytest.mark.parametrize("cart", [True, False], ids=["cart", "sph"])
def test_geometry_products_restatement_vs_finite_differences(cart):
    # the reference's geometry-response fixture: H2 at (0,0,0), (.2,-.1,.8)
    # Angstrom, 3-21G, nonsymmetric densities from seed 932
    # (tests/integrals/test_direct_geometry_response.py:14-24); plus water
    # 6-31G* for d shells.  Order 1 = d/du J/K, order 2 = d/dv of order 1,
    # the order-2 VJP = the gradient of <cot, order 1>, checked by central
    # differences of the oracle itself (step 1e-4 Bohr).
    for atom, basis in (("H 0 0 0; H .2 -.1 .8", "3-21g"),
                        ("O 0 0 0; H 0 0.7572 0.5865; H 0 -0.7572 0.5865", "6-31g*")):
        top, par, _ = B.prepare_basis(atom, basis, cart=cart)
        atm, bas, env = B.pack(top, par)
        n = top.nao
        rng = np.random.default_rng(932)
        d = rng.normal(size=(2, n, n))
        slots = (atm[:, 1][:, None] + np.arange(3)[None, :]).ravel()
        u = np.zeros(len(env))
        v = np.zeros(len(env))
        u[slots] = rng.normal(size=slots.size) * .17
        v[slots] = rng.normal(size=slots.size) * .11
        h = 1e-4
        jk = lambda e: oracle.direct_jk(atm, bas, e, d, cart=cart, workers=4)  # noqa: E731
        jvp1 = lambda e: oracle.direct_jk_geometry_product(atm, bas, e, d, u, order=1, cart=cart,  # noqa: E731
                                                            workers=4)
        j1, k1 = jvp1(env)
        (jp, kp), (jm, km) = jk(env + h * u), jk(env - h * u)
        np.testing.assert_allclose(j1, (jp - jm) / (2 * h), atol=2e-7, rtol=3e-7)
        np.testing.assert_allclose(k1, (kp - km) / (2 * h), atol=2e-7, rtol=3e-7)
        j2, k2 = oracle.direct_jk_geometry_product(atm, bas, env, d, u, v, order=2, cart=cart, workers=4)
        (jp, kp), (jm, km) = jvp1(env + h * v), jvp1(env - h * v)
        np.testing.assert_allclose(j2, (jp - jm) / (2 * h), atol=2e-7, rtol=3e-7)
        np.testing.assert_allclose(k2, (kp - km) / (2 * h), atol=2e-7, rtol=3e-7)
        cot = np.stack([np.cos(d), np.sin(d)])
        g = oracle.direct_jk_geometry_product(atm, bas, env, d, u, cot, order=2, cart=cart,
                                              transpose=True, workers=4)
        assert abs(g @ v - (np.sum(cot[0] * j2) + np.sum(cot[1] * k2))) < 1e-10
        assert np.all(g[np.setdiff1d(np.arange(len(env)), slots)] == 0.0)
