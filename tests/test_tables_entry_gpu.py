"""The reference-shaped entry point b200jk_direct_jk_tables, through the C ABI.

It takes the argument list of the reference's XLA handler GradSCFDirectJK
(csrc/direct_jk.cc:7-11, bound at :97-102): libcint atm/bas/env tables, a
(nb, n, n) density, a (with_j + with_k, nb, n, n) result, cart, cutoff,
workers, with_j, with_k.  Results are compared with the oracle at the FP64
bar (1e-10 max-abs); the handler's error returns are checked in its order
(workers, operator flags, tables, shapes, density values).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import oracle  # noqa: E402
from gradscf_b200 import _capi  # noqa: E402
from tests.gpu_util import WATER, tables  # noqa: E402


def _call(atm, bas, env, d, *, cart=False, cutoff=1e-12, workers=1, with_j=1, with_k=1, n=None, nops=None):
    atm = np.ascontiguousarray(atm, dtype=np.int32)
    bas = np.ascontiguousarray(bas, dtype=np.int32)
    env = np.ascontiguousarray(env, dtype=np.float64)
    dt = torch.as_tensor(d, device="cuda").contiguous()
    nb, nn = dt.shape[0], dt.shape[-1]
    nops = (int(bool(with_j)) + int(bool(with_k))) if nops is None else nops
    out = torch.full((max(nops, 1), nb, nn, nn), float("nan"), dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = _capi.lib().b200jk_direct_jk_tables(
        p(atm), atm.shape[0], p(bas), bas.shape[0], p(env), env.shape[0],
        ctypes.c_void_p(dt.data_ptr()), nb, nn if n is None else n, ctypes.c_void_p(out.data_ptr()),
        int(cart), ctypes.c_double(cutoff), int(workers), int(with_j), int(with_k), st)
    _capi.check(rc)
    return out.cpu().numpy()


@pytest.mark.parametrize("cart", [False, True], ids=["sph", "cart"])
def test_tables_entry_matches_oracle_nonsymmetric_batch(cart):
    top, par, sa, atm, bas, env = tables(WATER, "cc-pvdz", cart)
    n = top.nao
    rng = np.random.default_rng(11)
    d = rng.normal(size=(2, n, n)) * 0.1           # nonsymmetric, nb = 2
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=cart, cutoff=1e-12, workers=4)
    out = _call(atm, bas, env, d, cart=cart, workers=4)
    assert out.shape == (2, 2, n, n)
    assert np.abs(out[0] - j0).max() < 1e-10
    assert np.abs(out[1] - k0).max() < 1e-10
    # J only / K only: a one-operator result buffer, J before K as in the handler
    oj = _call(atm, bas, env, d, cart=cart, with_k=0)
    ok = _call(atm, bas, env, d, cart=cart, with_j=0)
    assert oj.shape[0] == 1 and ok.shape[0] == 1
    assert np.abs(oj[0] - j0).max() < 1e-10
    assert np.abs(ok[0] - k0).max() < 1e-10


def test_tables_entry_error_returns():
    top, par, sa, atm, bas, env = tables(WATER, "6-31g*", False)
    n = top.nao
    d = np.random.default_rng(12).normal(size=(1, n, n))
    with pytest.raises(_capi.InvalidArgument, match="workers must be positive"):
        _call(atm, bas, env, d, workers=0)
    with pytest.raises(_capi.InvalidArgument, match="at least one selected operator"):
        _call(atm, bas, env, d, with_j=0, with_k=0, nops=1)
    with pytest.raises(_capi.InvalidArgument, match="at least one selected operator"):
        _call(atm, bas, env, d, with_j=2)
    with pytest.raises(_capi.InvalidArgument, match="shape mismatch"):
        _call(atm, bas, env, d, n=n + 1)
    bad = np.array(env, copy=True)
    bad[8] = 1e300                                    # omega above sqrt(DBL_MAX)/2 (tables.h:44-45)
    with pytest.raises(_capi.InvalidArgument, match="omega exceeds"):
        _call(atm, bas, bad, d)
    bad = np.array(env, copy=True)
    bad[-1] = np.inf
    with pytest.raises(_capi.InvalidArgument, match="env must be finite"):
        _call(atm, bas, bad, d)
    dn = d.copy()
    dn[0, 3, 1] = np.nan
    with pytest.raises(_capi.InvalidArgument, match="Nonfinite density"):
        _call(atm, bas, env, dn)
    # the library stays usable after every refusal
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12)
    out = _call(atm, bas, env, d)
    assert np.abs(out[0] - j0).max() < 1e-10 and np.abs(out[1] - k0).max() < 1e-10
