"""Coordinate JVPs (order 1 and 2) and the order-2 VJP of J/K on the GPU
against the oracle's restatement of the reference's geometry products
(csrc/direct_jk_geometry.cc:8-99 over csrc/eri_geometry_entries.h:6-31 and
csrc/geometry_contraction.h:7-53, libcint's int2e_ip1 / ipip1 / ipvip1 /
ip1ip2), plus finite differences and the translation sum rule.

Tolerances follow the reference's geometry-response tests
(tests/integrals/test_direct_geometry_response.py:69,92-93): atol 3e-10 /
rtol 2e-10 against the oracle, 2e-7 against central differences (step 1e-4).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import oracle  # noqa: E402
from gradscf_b200 import jk as J  # noqa: E402
from tests.gpu_util import WATER, tables  # noqa: E402


def _directions(atm, env, seed):
    rng = np.random.default_rng(seed)
    slots = (atm[:, 1][:, None] + np.arange(3)[None, :]).ravel()
    u = np.zeros(len(env))
    v = np.zeros(len(env))
    u[slots] = rng.normal(size=slots.size) * .17
    v[slots] = rng.normal(size=slots.size) * .11
    return u, v


def _close(a, b, atol=3e-10, rtol=2e-10):
    a = a.cpu().numpy() if torch.is_tensor(a) else a
    np.testing.assert_allclose(a, b, atol=atol, rtol=rtol)


@pytest.mark.parametrize("atom,basis,cart", [("H 0 0 0; H .2 -.1 .8", "3-21g", True),
                                             (WATER, "6-31g*", False), (WATER, "6-31g*", True)],
                         ids=["h2-321g", "water-631gs-sph", "water-631gs-cart"])
def test_geometry_products_match_oracle(atom, basis, cart):
    top, par, sa, atm, bas, env = tables(atom, basis, cart)
    n = top.nao
    rng = np.random.default_rng(932)
    d = rng.normal(size=(2, n, n))                    # nonsymmetric, nb = 2
    u, v = _directions(atm, env, 933)
    # order 1
    j1, k1 = J.direct_jk_geometry_jvp(atm, bas, env, d, u, cart=cart)
    oj1, ok1 = oracle.direct_jk_geometry_product(atm, bas, env, d, u, order=1, cart=cart, workers=8)
    _close(j1, oj1)
    _close(k1, ok1)
    # order 2
    j2, k2 = J.direct_jk_geometry_jvp(atm, bas, env, d, u, v, cart=cart)
    oj2, ok2 = oracle.direct_jk_geometry_product(atm, bas, env, d, u, v, order=2, cart=cart, workers=8)
    _close(j2, oj2)
    _close(k2, ok2)
    # order-2 VJP with the reference test's cotangents (cos D, sin D)
    cot = (np.cos(d), np.sin(d))
    g = J.direct_jk_geometry_hvp(atm, bas, env, d, u, cot, cart=cart)
    og = oracle.direct_jk_geometry_product(atm, bas, env, d, u, np.stack(cot), order=2, cart=cart,
                                           transpose=True, workers=8)
    _close(g, og)
    # J or K alone
    jj, kz = J.direct_jk_geometry_jvp(atm, bas, env, d, u, v, cart=cart, with_k=False)
    _close(jj, oj2)
    assert torch.count_nonzero(kz) == 0


def test_geometry_products_finite_differences_and_sum_rule():
    top, par, sa, atm, bas, env = tables(WATER, "6-31g*", False)
    n = top.nao
    rng = np.random.default_rng(5)
    c = rng.normal(size=(n, 5)) / np.sqrt(n)
    d = c @ c.T
    u, v = _directions(atm, env, 6)
    h = 1e-4
    # order 2 = d/dv of order 1, order 1 = d/du of J/K (both on the GPU)
    jp, kp = J.direct_jk_geometry_jvp(atm, bas, env + h * v, d, u, cart=False)
    jm, km = J.direct_jk_geometry_jvp(atm, bas, env - h * v, d, u, cart=False)
    j2, k2 = J.direct_jk_geometry_jvp(atm, bas, env, d, u, v, cart=False)
    _close(j2, ((jp - jm) / (2 * h)).cpu().numpy(), atol=2e-7, rtol=3e-7)
    _close(k2, ((kp - km) / (2 * h)).cpu().numpy(), atol=2e-7, rtol=3e-7)
    jp, kp = J.direct_jk(atm, bas, env + h * u, d, cart=False)
    jm, km = J.direct_jk(atm, bas, env - h * u, d, cart=False)
    j1, k1 = J.direct_jk_geometry_jvp(atm, bas, env, d, u, cart=False)
    _close(j1, ((jp - jm) / (2 * h)).cpu().numpy(), atol=2e-7, rtol=3e-7)
    _close(k1, ((kp - km) / (2 * h)).cpu().numpy(), atol=2e-7, rtol=3e-7)
    # the order-2 VJP is the gradient of <cot, d(J,K)/du>: check along v
    cot = (np.cos(d), np.sin(d))
    g = J.direct_jk_geometry_hvp(atm, bas, env, d, u, cot, cart=False)

    def f(e):
        a, b = J.direct_jk_geometry_jvp(atm, bas, e, d, u, cart=False)
        return float(np.sum(cot[0] * a.cpu().numpy()) + np.sum(cot[1] * b.cpu().numpy()))

    np.testing.assert_allclose(g @ v, (f(env + h * v) - f(env - h * v)) / (2 * h), rtol=1e-6, atol=1e-9)
    # translation sum rule: moving every centre together changes nothing
    ones = np.zeros(len(env))
    ones[(atm[:, 1][:, None] + np.arange(3)[None, :]).ravel()] = 1.0
    for m in J.direct_jk_geometry_jvp(atm, bas, env, d, ones, cart=False):
        assert m.abs().max().item() < 3e-11
    for m in J.direct_jk_geometry_jvp(atm, bas, env, d, ones, v, cart=False):
        assert m.abs().max().item() < 3e-11


def test_geometry_products_reject_non_coordinate_directions():
    top, par, sa, atm, bas, env = tables(WATER, "sto-3g", True)
    d = np.eye(top.nao)
    u = np.zeros(len(env))
    u[int(bas[0, 5])] = 1.0                          # an exponent slot
    with pytest.raises(ValueError, match="coordinates only"):
        J.direct_jk_geometry_jvp(atm, bas, env, d, u, cart=True)
    with pytest.raises(ValueError, match="finite"):
        J.direct_jk_geometry_jvp(atm, bas, env, d, np.full(len(env), np.nan), cart=True)
