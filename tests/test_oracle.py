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
