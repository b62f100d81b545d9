"""GPU direct J/K (C ABI, sm_100a kernels) against the CPU oracle.

Tolerances: the reference's own tests compare direct J/K with the full-ERI
einsum at atol 2e-10 / rtol 1e-10 (tests/integrals/test_native_direct_parallel.py:60)
and 3e-12 for H2/sto-3g (test_native_jk_dispatch.py:32); the FP64 bar of this
build is 1e-10 max-abs against the oracle.
"""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs CUDA")]

import oracle  # noqa: E402
from gradscf_b200 import jk as J  # noqa: E402
from gradscf_b200 import _capi  # noqa: E402
from tests.gpu_util import WATER, psd_density, tables  # noqa: E402


def gpu_jk(atm, bas, env, d, cart, cutoff=0.0, **kw):
    j, k = J.direct_jk(atm, bas, env, torch.as_tensor(d, device="cuda"), cart=cart, cutoff=cutoff, **kw)
    return j.cpu().numpy(), k.cpu().numpy()


def test_h2_sto3g_golden(golden_dir):
    rec = json.loads((golden_dir / "h2_sto3g_jk.json").read_text())
    top, par, sa, atm, bas, env = tables(rec["atom"], rec["basis"], True)
    j, k = gpu_jk(atm, bas, env, np.array(rec["density"]), True)
    np.testing.assert_allclose(j, rec["j"], atol=3e-12, rtol=3e-12)
    np.testing.assert_allclose(k, rec["k"], atol=3e-12, rtol=3e-12)


@pytest.mark.parametrize("cart", [False, True], ids=["sph", "cart"])
def test_general_contraction_nonsymmetric_batch_golden(golden_dir, cart):
    rec = json.loads((golden_dir / "h2_general_jk.json").read_text())
    top, par, sa, atm, bas, env = tables(rec["atom"], rec["basis"], cart)
    sub = rec["cart" if cart else "sph"]
    j, k = gpu_jk(atm, bas, env, np.array(sub["density"]), cart)
    np.testing.assert_allclose(j, sub["j"], atol=2e-10, rtol=1e-10)
    np.testing.assert_allclose(k, sub["k"], atol=2e-10, rtol=1e-10)


@pytest.mark.parametrize("basis,cart", [("cc-pvdz", False), ("6-31g*", True), ("6-31g*", False),
                                        ("cc-pvtz", False), ("cc-pvtz", True)])
def test_water_vs_oracle(basis, cart):
    top, par, sa, atm, bas, env = tables(WATER, basis, cart)
    d = psd_density(top.nao, 5, 0)
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=cart, workers=8)
    j, k = gpu_jk(atm, bas, env, d, cart)
    assert np.abs(j - j0).max() < 1e-10
    assert np.abs(k - k0).max() < 1e-10


def test_water_cc_pvdz_config0_screened():
    # Config: water cc-pVDZ (24 functions), Schwarz cut 1e-12, D = C C^T seed 0.
    top, par, sa, atm, bas, env = tables(WATER, "cc-pvdz", False)
    assert top.nao == 24
    d = psd_density(24, 5, 0)
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12)
    j, k = gpu_jk(atm, bas, env, d, False, cutoff=1e-12)
    assert np.abs(j - j0).max() < 1e-10 and np.abs(k - k0).max() < 1e-10


def test_water_dimer_nonsymmetric_screened():
    atom = WATER + "; O 2.9 0.1 0.2; H 3.4 0.8 0.5; H 3.5 -0.7 0.3"
    top, par, sa, atm, bas, env = tables(atom, "cc-pvdz", False)
    d = np.random.default_rng(807).normal(size=(3, top.nao, top.nao)) * 0.1
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12, workers=8)
    j, k = gpu_jk(atm, bas, env, d, False, cutoff=1e-12)
    assert np.abs(j - j0).max() < 1e-10 and np.abs(k - k0).max() < 1e-10


def test_with_j_with_k_selection_and_complex():
    top, par, sa, atm, bas, env = tables(WATER, "6-31g*", False)
    rng = np.random.default_rng(806)
    d = rng.normal(size=(top.nao, top.nao)) + 1j * rng.normal(size=(top.nao, top.nao))
    j0r, k0r = oracle.direct_jk(atm, bas, env, d.real, cart=False)
    j0i, k0i = oracle.direct_jk(atm, bas, env, d.imag, cart=False)
    j, k = J.direct_jk(atm, bas, env, torch.as_tensor(d, device="cuda"), cart=False, with_k=False)
    assert np.abs(j.cpu().numpy() - (j0r + 1j * j0i)).max() < 1e-10
    assert np.count_nonzero(k.cpu().numpy()) == 0
    j, k = J.direct_jk(atm, bas, env, torch.as_tensor(d, device="cuda"), cart=False, with_j=False)
    assert np.abs(k.cpu().numpy() - (k0r + 1j * k0i)).max() < 1e-10
    assert np.count_nonzero(j.cpu().numpy()) == 0


def test_screening_linear_and_huge_cut_zero():
    top, par, sa, atm, bas, env = tables(WATER, "cc-pvdz", False)
    rng = np.random.default_rng(803)
    d, t = rng.normal(size=(2, 4, top.nao, top.nao))
    a = gpu_jk(atm, bas, env, d + 0.37 * t, False, cutoff=1e-6)
    b = gpu_jk(atm, bas, env, d, False, cutoff=1e-6)
    c = gpu_jk(atm, bas, env, t, False, cutoff=1e-6)
    for x, y, z in zip(a, b, c):
        np.testing.assert_allclose(x, y + 0.37 * z, atol=2e-10, rtol=1e-10)
    for x in gpu_jk(atm, bas, env, d, False, cutoff=1e9):
        assert np.count_nonzero(x) == 0


def test_nonfinite_density_and_unsupported_inputs_raise():
    top, par, sa, atm, bas, env = tables(WATER, "sto-3g", True)
    d = np.full((top.nao, top.nao), np.nan)
    with pytest.raises(ValueError, match="Nonfinite"):
        gpu_jk(atm, bas, env, d, True)
    top, par, sa, atm, bas, env = tables("H 0 0 0; H 0 0 1", [[4, [1.0, 1.0]]], False)
    with pytest.raises(NotImplementedError):
        gpu_jk(atm, bas, env, np.eye(top.nao), False)
    bad = bas.copy(); bad[0, 2] = 0
    with pytest.raises(ValueError, match="unsupported"):
        J.DirectJKPlan([(atm, bad, env)], cart=False)


def test_split_precision_error_is_small():
    atom = WATER + "; O 2.9 0.1 0.2; H 3.4 0.8 0.5; H 3.5 -0.7 0.3"
    top, par, sa, atm, bas, env = tables(atom, "cc-pvdz", False)
    d = psd_density(top.nao, 10, 3)
    plan = J.cached_plan(atm, bas, env, cart=False, cutoff=1e-12)
    j64, k64 = plan.jk(torch.as_tensor(d, device="cuda"))
    j32, k32 = plan.jk(torch.as_tensor(d, device="cuda"), precision="split", fp32_cut=1e-6)
    ej = (j32 - j64).abs().max().item()
    ek = (k32 - k64).abs().max().item()
    assert ej < 1e-8 and ek < 1e-8
    de = 0.5 * torch.sum(torch.as_tensor(d, device="cuda") * ((j32 - j64) - 0.5 * (k32 - k64))).item()
    assert abs(de) < 1e-9


def test_batched_plan_matches_single_molecule_plans():
    mols = []
    for shift in (0.0, 0.3):
        atom = f"O 0 0 {shift}; H 0 0.7572 {0.5865 + shift}; H 0.1 -0.7572 {0.5865 - shift}"
        mols.append(tables(atom, "cc-pvdz", False))
    plan = J.DirectJKPlan([(m[3], m[4], m[5]) for m in mols], cart=False, cutoff=1e-12)
    ds = [psd_density(m[0].nao, 5, i) for i, m in enumerate(mols)]
    packed = torch.zeros((1, plan.packed_size), dtype=torch.float64, device="cuda")
    for m, d in enumerate(ds):
        packed[0, plan.offsets[m]:plan.offsets[m] + d.size] = torch.as_tensor(d.ravel(), device="cuda")
    out = plan.jk_packed(packed, hermi=1).cpu().numpy()
    for m, (mol, d) in enumerate(zip(mols, ds)):
        n = mol[0].nao
        j0, k0 = oracle.direct_jk(mol[3], mol[4], mol[5], d, cart=False, cutoff=1e-12)
        sl = slice(plan.offsets[m], plan.offsets[m] + n * n)
        assert np.abs(out[0, 0, sl].reshape(n, n) - j0).max() < 1e-10
        assert np.abs(out[1, 0, sl].reshape(n, n) - k0).max() < 1e-10


def test_quartet_count_matches_oracle():
    atom = WATER + "; O 2.9 0.1 0.2; H 3.4 0.8 0.5; H 3.5 -0.7 0.3"
    top, par, sa, atm, bas, env = tables(atom, "cc-pvdz", False)
    plan = J.cached_plan(atm, bas, env, cart=False, cutoff=1e-12)
    q = oracle.schwarz_bounds(atm, bas, env, cart=False)
    assert plan.quartets == oracle.count_quartets(q, 1e-12)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_sharded_partials_sum_to_full_build(precision):
    # the shards of a 3-way split, run one after another on this GPU, add up
    # to the unsharded build (the multi-GPU path sums them with one all-reduce)
    from gradscf_b200 import workloads as W
    top, par, sa, atm, bas, env = tables(W.water_cluster(3, 1), "cc-pvdz", False)
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    n = plan.nao[0]
    d = torch.as_tensor(psd_density(n, 15, 4), device="cuda").reshape(1, -1)
    full = plan.jk_packed(d, hermi=1, precision=precision).clone()
    acc = torch.zeros_like(full)
    nonempty = 0
    for r in range(3):
        plan.set_shard(r, 3)
        part = plan.jk_packed(d, hermi=1, precision=precision, reduce=False)
        nonempty += int(part.abs().max().item() > 0)
        acc += part
    plan.set_shard(0, 1)
    assert nonempty == 3
    assert (acc - full).abs().max().item() < 1e-11
    again = plan.jk_packed(d, hermi=1, precision=precision)
    assert (again - full).abs().max().item() < 1e-12


def test_autotune_keeps_results():
    # the tuner only changes how kets are cut into work items: results are unchanged
    from gradscf_b200 import workloads as W
    top, par, sa, atm, bas, env = tables(W.water_cluster(3, 1), "cc-pvdz", False)
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    n = plan.nao[0]
    d = torch.as_tensor(psd_density(n, 15, 6), device="cuda").reshape(1, -1)
    ref = {p_: plan.jk_packed(d, hermi=1, precision=p_).clone() for p_ in ("fp64", "split")}
    chosen = plan.autotune(d, precision="split", reps=1)
    assert chosen and set(chosen.values()) <= {32, 64, 128}
    for p_ in ("fp64", "split"):
        got = plan.jk_packed(d, hermi=1, precision=p_)
        assert (got - ref[p_]).abs().max().item() < 1e-11


@pytest.mark.parametrize("basis,cart", [("6-31g*", False), ("6-31g*", True), ("cc-pvdz", False)])
def test_long_range_omega_vs_oracle(basis, cart):
    # erf(omega r)/r integrals (libcint PTR_RANGE_OMEGA = env[8], as the
    # reference's get_jk sets it, plan.py:86-87): FP64 J/K to 1e-10 of the
    # oracle, screening bounds included; a nonsymmetric density as well
    top, par, sa, atm, bas, env = tables(WATER, basis, cart)
    env = np.array(env, dtype=np.float64, copy=True)
    env[8] = 0.33
    n = top.nao
    rng = np.random.default_rng(17)
    for d in (psd_density(n, 5, 3), rng.normal(size=(n, n))):
        j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=cart, cutoff=1e-12, workers=8)
        j, k = J.direct_jk(atm, bas, env, torch.as_tensor(d, device="cuda"), cart=cart, cutoff=1e-12)
        assert np.abs(j.cpu().numpy() - j0).max() < 1e-10
        assert np.abs(k.cpu().numpy() - k0).max() < 1e-10
    # the long-range integrals really differ from the Coulomb ones
    jf, _ = oracle.direct_jk(atm, bas, np.where(np.arange(env.size) == 8, 0.0, env), d, cart=cart,
                             cutoff=1e-12, workers=8)
    assert np.abs(jf - j0).max() > 1e-2
    js, ks = J.direct_jk(atm, bas, env, torch.as_tensor(psd_density(n, 5, 3), device="cuda"), cart=cart,
                         cutoff=1e-12, precision="split")
    j0, k0 = oracle.direct_jk(atm, bas, env, psd_density(n, 5, 3), cart=cart, cutoff=1e-12, workers=8)
    assert np.abs(js.cpu().numpy() - j0).max() < 1e-6 and np.abs(ks.cpu().numpy() - k0).max() < 1e-6


def test_prepare_jk_and_rsh_combination():
    # prepare_jk (backends/native/jk.py:118-162) binds the direct action;
    # rsh_jk = sr K(full) + (lr - sr) K(omega) with the full J (scf/rsh.py:62-85)
    from gradscf_b200 import basis as B
    top, par, sa = B.prepare_basis(WATER, "6-31g*", cart=False)
    provider = J.NativeDirectBasis(J.make_plan(top), par)
    d = torch.as_tensor(psd_density(top.nao, 5, 8), device="cuda")
    act = provider.prepare_jk(omega=0.4)
    jl, kl = act(d)
    j2, k2 = provider.get_jk(d, omega=0.4)
    assert (jl - j2).abs().max().item() < 1e-13 and (kl - k2).abs().max().item() < 1e-13
    jf, kf = provider.get_jk(d)
    jr, kr = J.rsh_jk(provider, d, (0.4, 0.65, 0.2))
    assert (jr - jf).abs().max().item() < 1e-14
    assert (kr - (0.2 * kf + 0.45 * kl)).abs().max().item() < 1e-12


def _pack_s8(eri):
    n = eri.shape[0]
    i, j = np.tril_indices(n)
    pairs = eri[i[:, None], j[:, None], i[None, :], j[None, :]]   # (np, np) s4
    a, b = np.tril_indices(pairs.shape[0])
    return pairs, pairs[a, b]


@pytest.mark.parametrize("basis,cart", [("6-31g*", False), ("6-31g*", True), ("cc-pvdz", False)])
def test_packed_eri_and_packed_jk_vs_oracle(basis, cart):
    # producer: csrc/packed_eri.cc (cut 0, s4 and s8); consumer: csrc/packed_jk.cc
    top, par, sa, atm, bas, env = tables(WATER, basis, cart)
    eri = oracle.eri_s1(atm, bas, env, cart=cart)
    s4_ref, s8_ref = _pack_s8(eri)
    s8 = J.packed_eri(atm, bas, env, cart=cart, aosym="s8")
    s4 = J.packed_eri(atm, bas, env, cart=cart, aosym="s4")
    assert s8.shape == s8_ref.shape and s4.shape == s4_ref.shape
    assert np.abs(s8.cpu().numpy() - s8_ref).max() < 1e-11
    assert np.abs(s4.cpu().numpy() - s4_ref).max() < 1e-11
    rng = np.random.default_rng(5)
    d = rng.normal(size=(2, top.nao, top.nao))
    jr, kr = oracle.full_jk(eri, d)
    for packed in (s8, s4):
        j, k = J.packed_jk(packed, torch.as_tensor(d, device="cuda"))
        np.testing.assert_allclose(j.cpu().numpy(), jr, atol=1e-10)
        np.testing.assert_allclose(k.cpu().numpy(), kr, atol=1e-10)
    jc, kc = J.build_jk_from_packed(s8, torch.complex(torch.as_tensor(d[0], device="cuda"),
                                                      torch.as_tensor(d[1], device="cuda")))
    np.testing.assert_allclose(jc.real.cpu().numpy(), jr[0], atol=1e-10)
    np.testing.assert_allclose(kc.imag.cpu().numpy(), kr[1], atol=1e-10)
    with pytest.raises(ValueError):
        J.packed_jk(s8[:-1], torch.as_tensor(d, device="cuda"))


def test_split_cc_pvtz_high_l_classes():
    # f shells on O, d on H: the FP32 tile path for kets up to f x f in split mode
    atom = "O 0 0 0; H 0 0.7572 0.5865; H 0 -0.7572 0.5865; O 2.9 0.1 0; H 3.5 0.8 0.3; H 3.4 -0.7 0.2"
    top, par, sa, atm, bas, env = tables(atom, "cc-pvtz", False)
    d = psd_density(top.nao, 10, 2)
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12, workers=8)
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    dd = torch.as_tensor(d, device="cuda").reshape(1, -1)
    for precision, tol in (("fp64", 1e-10), ("split", 1e-6)):
        out = plan.jk_packed(dd, hermi=1, precision=precision)
        n = top.nao
        assert np.abs(out[0, 0].reshape(n, n).cpu().numpy() - j0).max() < tol
        assert np.abs(out[1, 0].reshape(n, n).cpu().numpy() - k0).max() < tol


def test_simultaneous_calls_on_two_plans_keep_workspaces_separate():
    # tests/integrals/test_native_direct_parallel.py:73-88: two plans, two
    # host threads, each on its own stream; every result matches its oracle
    from concurrent.futures import ThreadPoolExecutor
    specs = (WATER, "H 0 0 0; H -0.2 0.3 1.8")
    ctx = []
    for atom in specs:
        top, par, sa, atm, bas, env = tables(atom, "6-31g*", False)
        plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
        d = np.random.default_rng(805).normal(size=(4, top.nao, top.nao))
        ctx.append((plan, atm, bas, env, d))

    def run(c, scale):
        plan, atm, bas, env, d = c
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            dd = torch.as_tensor(scale * d, device="cuda").reshape(4, -1)
            out = plan.jk_packed(dd, hermi=0, stream=stream)
            stream.synchronize()
            return out.cpu().numpy()

    for c in ctx:
        run(c, 1.0)  # plans and scratch initialised before the concurrent calls
    with ThreadPoolExecutor(max_workers=2) as ex:
        for scale in (1.0, 0.37):
            futs = [ex.submit(run, c, scale) for c in ctx]
            for f, (plan, atm, bas, env, d) in zip(futs, ctx):
                got = f.result()
                n = d.shape[-1]
                j0, k0 = oracle.direct_jk(atm, bas, env, scale * d, cart=False, cutoff=1e-12, workers=4)
                np.testing.assert_allclose(got[0].reshape(4, n, n), j0, atol=2e-10, rtol=1e-10)
                np.testing.assert_allclose(got[1].reshape(4, n, n), k0, atol=2e-10, rtol=1e-10)


def test_repeated_builds_agree_to_rounding():
    # the reference's fixed-worker reduction is bitwise reproducible
    # (test_native_direct_parallel.py:63-70); here J/K accumulate with
    # atomics on the GPU, so repeats agree to rounding, not bit for bit
    top, par, sa, atm, bas, env = tables(WATER, "cc-pvdz", False)
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    d = torch.as_tensor(np.random.default_rng(802).normal(size=(4, top.nao * top.nao)), device="cuda")
    first = plan.jk_packed(d, hermi=0).clone()
    for _ in range(3):
        again = plan.jk_packed(d, hermi=0)
        assert (again - first).abs().max().item() <= 1e-12 * max(1.0, first.abs().max().item())


def test_graph_survives_scratch_growth_and_refuses_stale_work_items():
    # a graph owns its scratch: a later build with more densities (which grows
    # the plan's scratch) leaves it valid; autotune rebuilds the work items,
    # after which the graph's launch is refused instead of replaying stale items
    from gradscf_b200 import workloads as W
    top, par, sa, atm, bas, env = tables(W.water_cluster(2, 1), "cc-pvdz", False)
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    n = plan.nao[0]
    d = psd_density(n, 10, 21)
    j0, k0 = oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12, workers=8)
    g = J.JKGraph(plan, 1, hermi=1)
    big = torch.as_tensor(np.stack([psd_density(n, 10, 22 + i) for i in range(3)]).reshape(3, -1),
                          device="cuda")
    plan.jk_packed(big, hermi=1)
    for _ in range(2):
        out = g.run(torch.as_tensor(d.reshape(1, -1), device="cuda")).cpu().numpy()
        assert np.abs(out[0, 0].reshape(n, n) - j0).max() < 1e-10
        assert np.abs(out[1, 0].reshape(n, n) - k0).max() < 1e-10
    plan.autotune(big[:1], precision="fp64", reps=1)
    with pytest.raises(_capi.InvalidArgument, match="recreate|create a new one"):
        g.launch()
    g.close()
    g = J.JKGraph(plan, 1, hermi=1)
    out = g.run(torch.as_tensor(d.reshape(1, -1), device="cuda")).cpu().numpy()
    assert np.abs(out[1, 0].reshape(n, n) - k0).max() < 1e-10
    g.close()


def test_bra_transfer_probe_variants_agree():
    # the recursion and the tensor-core GEMM form of the f x f bra transfer
    # compute the same map (b200jk_measure_bra_transfer)
    import ctypes
    ns = (ctypes.c_double * 2)()
    diff = ctypes.c_double()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(_capi.lib().b200jk_measure_bra_transfer(4096, 2, ns, ctypes.byref(diff), st))
    assert diff.value < 1e-12
    assert ns[0] > 0 and ns[1] > 0


def _border_stats(plan):
    import ctypes
    lib = _capi.lib()
    listed, overflow = ctypes.c_int64(), ctypes.c_int64()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(lib.b200jk_plan_border_stats(plan._h, st, ctypes.byref(listed), ctypes.byref(overflow)))
    return listed.value, overflow.value


@pytest.mark.parametrize("fp32_cut", [1e-9, 1e-6, 1e-4])
def test_split_fp64_flat_list_matches_fp64_build(fp32_cut):
    # (H2O)4 cc-pVDZ (generally contracted s shells: grouped buckets), a
    # small symmetric density (an SCF increment's scale, so the FP64 quartets
    # are the leading corners of the work items and run from the flat lists)
    # and a nonsymmetric one: the two slices of the split build together
    # against the FP64 build
    from gradscf_b200 import workloads as W
    top, par, sa, atm, bas, env = tables(W.water_cluster(4, 1), "cc-pvdz", False)
    n = top.nao
    rng = np.random.default_rng(7)
    d = np.stack([1e-3 * psd_density(n, 20, 5), 1e-3 * rng.standard_normal((n, n)) / n])
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    dd = torch.as_tensor(d.reshape(2, -1), device="cuda")
    ref = plan.jk_packed(dd, hermi=0).cpu().numpy()
    out = plan.jk_packed(dd, hermi=0, precision="split", fp32_cut=fp32_cut).cpu().numpy()
    listed, overflow = _border_stats(plan)
    assert listed > 0
    if fp32_cut == 1e-9:
        # more FP64 quartets than the lists hold: the items whose reservation
        # did not fit run their FP64 quartets on the bra-group path
        assert overflow > 0
    assert np.abs(out - ref).max() < 1e-9, np.abs(out - ref).max()
    # the symmetric density alone: J and K against the FP64 build
    ref1 = plan.jk_packed(dd[:1], hermi=1).cpu().numpy()
    out1 = plan.jk_packed(dd[:1], hermi=1, precision="split", fp32_cut=fp32_cut).cpu().numpy()
    assert np.abs(out1 - ref1).max() < 1e-9, np.abs(out1 - ref1).max()


def test_packed_jk_growing_batches_keep_shared_memory_limit():
    # the consumer's per-row exchange sums take 32 n nb bytes of shared memory:
    # a 60 KB call, then a 150 KB one in the same process (the kernel's
    # shared-memory limit is set once per device, for the largest size)
    top, par, sa, atm, bas, env = tables(WATER, "cc-pvtz", False)   # n = 58
    s8 = J.packed_eri(atm, bas, env, cart=False, aosym="s8")
    rng = np.random.default_rng(11)
    d = torch.as_tensor(rng.normal(size=(84, top.nao, top.nao)), device="cuda")
    j1, k1 = J.packed_jk(s8, d[:1])
    for nb in (33, 84):
        j, k = J.packed_jk(s8, d[:nb])
        assert torch.abs(j[0] - j1[0]).max().item() < 1e-12
        assert torch.abs(k[0] - k1[0]).max().item() < 1e-12
