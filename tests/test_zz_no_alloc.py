"""The allocation-free J/K entry point (b200jk_direct_jk_noalloc).

Some callers may not allocate device memory while they run: an XLA custom
call on a stream XLA owns, code inside CUDA stream capture, a process with a
fixed memory budget.  For them the library offers one entry point whose
scratch is a fixed static device array instead of memory allocated per call.
This test calls it through the C ABI twice in a row and compares both results
with the allocating entry point's, at the FP64 parity tolerance of the other
tests (1e-10 max-abs); it also checks that a call needing more scratch than
the fixed array is refused with a clear error.  The file name sorts last so a
run that stops at the first failure has already run every other test; it
also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

from gradscf_b200 import _capi  # noqa: E402
from gradscf_b200 import basis as B  # noqa: E402
from gradscf_b200 import workloads as W  # noqa: E402
from gradscf_b200.jk import DirectJKPlan  # noqa: E402


def _plan(nwater):
    top, par, _ = B.prepare_basis(W.water_cluster(nwater, 1), "cc-pvdz", cart=False)
    atm, bas, env = B.pack(top, par)
    return DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12), top.nao


def _noalloc(plan, d, hermi, precision=_capi.FP64, fp32_cut=1e-6, with_j=1, with_k=1):
    n2 = d.shape[1]
    out = torch.full((with_j + with_k, d.shape[0], n2), float("nan"), dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _capi.lib().b200jk_direct_jk_noalloc(plan._h, ctypes.c_void_p(d.data_ptr()), d.shape[0],
                                              ctypes.c_void_p(out.data_ptr()), with_j, with_k, int(hermi),
                                              precision, ctypes.c_double(fp32_cut), st)
    _capi.check(rc)
    _capi.check(_capi.lib().b200jk_check_status(plan._h, st))
    return out


def _cart_count(nwater):
    # raw Cartesian functions of the plan (every contraction column of every shell)
    top, par, _ = B.prepare_basis(W.water_cluster(nwater, 1), "cc-pvdz", cart=False)
    _, bas, _ = B.pack(top, par)
    return int(sum(int(r[3]) * (int(r[1]) + 1) * (int(r[1]) + 2) // 2 for r in bas))


def _scratch_doubles(cart_stride, nb, hermi, split, with_j, with_k):
    """The entry point's scratch need: effective densities (FP64, and FP32 in
    split mode), J and K accumulators, each region rounded up to 256 bytes."""
    r = lambda x: (x + 31) // 32 * 32  # noqa: E731
    ndm = nb if hermi else 2 * nb
    return (r(ndm * cart_stride) + (r((ndm * cart_stride + 1) // 2) if split else 0)
            + (r(nb * cart_stride) if with_j else 0) + (r(ndm * cart_stride) if with_k else 0))


@pytest.mark.parametrize("hermi", [1, 0])
def test_noalloc_matches_allocating_entry_point_twice(hermi):
    plan, n = _plan(4)
    rng = np.random.default_rng(7)
    c = rng.normal(size=(n, 20)) / np.sqrt(n)
    d = c @ c.T if hermi else rng.normal(size=(n, n)) * 0.05
    dt = torch.as_tensor(d.reshape(1, n * n), device="cuda").contiguous()
    ref = plan.jk_packed(dt, hermi=hermi).clone()
    for _ in range(2):
        got = _noalloc(plan, dt, hermi)
        assert torch.isfinite(got).all()
        assert (got - ref).abs().max().item() < 1e-10


def test_noalloc_split_precision_matches():
    plan, n = _plan(4)
    c = np.random.default_rng(8).normal(size=(n, 20)) / np.sqrt(n)
    dt = torch.as_tensor((c @ c.T).reshape(1, n * n), device="cuda").contiguous()
    ref = plan.jk_packed(dt, hermi=1, precision="split").clone()
    for _ in range(2):
        got = _noalloc(plan, dt, 1, precision=_capi.SPLIT)
        assert (got - ref).abs().max().item() < 1e-10


@pytest.mark.parametrize("with_j,with_k", [(1, 0), (0, 1)])
def test_noalloc_single_operator_matches(with_j, with_k):
    # only the selected accumulator is carved out of the array: the regions shift
    plan, n = _plan(4)
    d = np.random.default_rng(9).normal(size=(2, n, n)) * 0.05
    dt = torch.as_tensor(d.reshape(2, n * n), device="cuda").contiguous()
    ref = plan.jk_packed(dt, hermi=0, with_j=bool(with_j), with_k=bool(with_k)).clone()
    for _ in range(2):
        got = _noalloc(plan, dt, 0, with_j=with_j, with_k=with_k)
        assert got.shape == ref.shape
        assert (got - ref).abs().max().item() < 1e-10


def test_noalloc_split_precision_nonsymmetric_matches():
    # split mode with hermi = 0: twice the FP32 density region
    plan, n = _plan(4)
    d = np.random.default_rng(10).normal(size=(1, n, n)) * 0.05
    dt = torch.as_tensor(d.reshape(1, n * n), device="cuda").contiguous()
    ref = plan.jk_packed(dt, hermi=0, precision="split").clone()
    for _ in range(2):
        got = _noalloc(plan, dt, 0, precision=_capi.SPLIT)
        assert (got - ref).abs().max().item() < 1e-10


def test_noalloc_limit_boundary():
    # the largest batch that fits the fixed array runs; one more is refused
    plan, n = _plan(4)
    cs = _cart_count(4) ** 2
    limit = _capi.NOALLOC_SCRATCH_BYTES // 8
    nb = 1
    while _scratch_doubles(cs, nb + 1, 1, False, 1, 1) <= limit:
        nb += 1
    assert _scratch_doubles(cs, nb + 1, 1, False, 1, 1) > limit
    c = np.random.default_rng(11).normal(size=(nb, n, 6)) / np.sqrt(n)
    d = np.einsum("bik,bjk->bij", c, c)
    dt = torch.as_tensor(d.reshape(nb, n * n), device="cuda").contiguous()
    got = _noalloc(plan, dt, 1)
    ref = plan.jk_packed(dt, hermi=1)
    assert (got - ref).abs().max().item() < 1e-10
    over = torch.zeros((nb + 1, n * n), dtype=torch.float64, device="cuda")
    with pytest.raises(_capi.InvalidArgument, match="scratch"):
        _noalloc(plan, over, 1)


def test_noalloc_rejects_calls_beyond_the_fixed_scratch():
    plan, n = _plan(4)
    nb = _capi.NOALLOC_SCRATCH_BYTES // (8 * n * n) + 1
    d = torch.zeros((nb, n * n), dtype=torch.float64, device="cuda")
    with pytest.raises(_capi.InvalidArgument, match="scratch"):
        _noalloc(plan, d, 1)
