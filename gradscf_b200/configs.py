"""Run the workload configurations of the J/K build and print one JSON record each.

    python -m gradscf_b200.configs c0|c2|c3|c4 [--quick]

c0  water cc-pVDZ (24 functions): FP64 RHF (Schwarz 1e-12, conv_tol 1e-10) and
    one J/K build of D = C C^T, C ~ N(0,1)/sqrt(24), 5 columns, seed 0.
c2  (H2O)16 6-31G* (seed 2): RHF forces in FP64 and split mode; central
    differences (step 1e-4 Bohr) on 6 random coordinates (seed 2).
c3  256 water clusters, N ~ U{1..24} (seed 3), cluster m from seed 1000+m,
    cc-pVDZ: one batched plan, one packed (graph-replayed) J/K build per SCF
    iteration for all clusters; aggregate quartets/s, FP64 vs split, and the
    per-cluster energy difference.
c4  (H2O)64 cc-pVTZ (3712 functions, seed 4): J/K builds in FP64 and split
    mode along an RHF SCF (fragment guess, 15 iterations) and one force.
prof  one small run of a kernel family for profiler captures (--case jk |
    grad | packed, --nwater, --basis).
tcprobe  the f x f bra transfer as the scalar recursion and as an FP64
    tensor-core GEMM, timed side by side.
Geometry generator and seeds: gradscf_b200/workloads.py.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import scf as S
from . import workloads as W


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _fragments(spec, n):
    atoms = spec.split("; ")
    return ["; ".join(atoms[3 * i:3 * i + 3]) for i in range(n)]


def run_c0():
    mol = S.Molecule(W.WATER, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    res = S.rhf(mol, conv_tol=1e-10)
    d = torch.as_tensor(W.psd_density(mol.nao, 5, 0), device=mol.device)
    for _ in range(3):
        mol.jk(d)
    e0, e1 = _events()
    e0.record()
    j, k = mol.jk(d)
    e1.record()
    torch.cuda.synchronize()
    return {"config": "c0", "nao": mol.nao, "rhf_energy_hartree": res.energy, "converged": res.converged,
            "cycles": res.cycles, "jk_ms_psd_density": e0.elapsed_time(e1), "quartets": mol.plan.quartets}


def run_c2(nwater=16, seed=2, npick=6):
    spec = W.water_cluster(nwater, seed)
    out = {"config": "c2", "system": f"(H2O){nwater} 6-31G* seed {seed}"}
    grads = {}
    syms = ["O", "H", "H"] * nwater
    for precision in ("fp64", "split"):
        mol = S.Molecule(spec, "6-31g*", cart=False, schwarz_cut=1e-12)
        d0 = S.fragment_guess(mol, _fragments(spec, nwater), "6-31g*")
        t0 = time.perf_counter()
        res = S.rhf(mol, conv_tol=1e-12, conv_tol_grad=1e-9, precision=precision, density0=d0)
        e0, e1 = _events()
        e0.record()
        g = S.rhf_gradient(mol, res, precision=precision)   # split: the split-precision VJP too
        e1.record()
        torch.cuda.synchronize()
        grads[precision] = g
        out[precision] = {"energy_hartree": res.energy, "cycles": res.cycles,
                          "gradient_ms": e0.elapsed_time(e1), "scf_s": time.perf_counter() - t0}
        rng = np.random.default_rng(seed)
        picks = [(int(rng.integers(len(mol.charges))), int(rng.integers(3))) for _ in range(npick)]
        h = 1e-4
        diffs = []
        for a, x in picks:
            vals = []
            for sgn in (1, -1):
                c = mol.coords.copy()
                c[a, x] += sgn * h
                m = S.Molecule([(s_, tuple(v)) for s_, v in zip(syms, c)], "6-31g*", unit="Bohr",
                               cart=False, schwarz_cut=1e-12)
                vals.append(S.rhf(m, conv_tol=1e-12, conv_tol_grad=1e-9, precision=precision,
                                  density0=res.density).energy)
            fd = (vals[0] - vals[1]) / (2 * h)
            diffs.append(abs(fd - g[a, x]))
        out[precision]["max_abs_fd_minus_analytic"] = float(max(diffs))
        out[precision]["net_force"] = float(np.abs(g.sum(0)).max())
    out["max_abs_force_split_minus_fp64"] = float(np.abs(grads["split"] - grads["fp64"]).max())
    return out


def run_c3(count=256, quick=False):
    import os
    sizes = W.batch_sizes(count=count, seed=3)
    if quick:
        sizes = sizes[:16]
    # several GPUs (torchrun): the clusters run as replicas, a cost-balanced
    # share per rank, energies gathered on the host at the end
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    mine = np.arange(len(sizes))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        mine = S.replica_shard((24 * np.asarray(sizes, dtype=np.int64)) ** 3, rank, world)
    all_sizes = sizes
    sizes = sizes[mine]
    specs = [W.water_cluster(int(nw), 1000 + int(m)) for m, nw in zip(mine, sizes)]
    batch = S.MoleculeBatch(specs, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    # fragment guess: every monomer of every cluster in one batched SCF
    monomers = [f for spec, nw in zip(specs, sizes) for f in _fragments(spec, int(nw))]
    mono = S.MoleculeBatch(monomers, "cc-pvdz", cart=False, schwarz_cut=1e-12)
    _, mds, _, _, _ = S.rhf_batch(mono, conv_tol=1e-9, timing=False)
    d0, pos = [], 0
    for nw in sizes:
        blocks = mds[pos:pos + int(nw)]
        pos += int(nw)
        d0.append(torch.block_diag(*blocks))
    out = {"config": "c3", "molecules": len(specs), "nao_min": int(min(batch.nao)),
           "nao_max": int(max(batch.nao)), "quartets_per_build": batch.plan.quartets}
    energies = {}
    for precision in ("fp64", "split"):
        en, _, ms, cycles, conv = S.rhf_batch(batch, conv_tol=1e-10, precision=precision, use_graph=True,
                                              density0=d0)
        energies[precision] = en
        steady = ms[1:] if len(ms) > 1 else ms
        out[precision] = {"cycles": cycles, "converged": int(conv.sum()),
                          "ms_per_build": float(np.mean(steady)),
                          "quartets_per_s": batch.plan.quartets / (np.mean(steady) * 1e-3)}
    out["split_speedup"] = out["fp64"]["ms_per_build"] / out["split"]["ms_per_build"]
    out["max_abs_dE_per_molecule_hartree"] = float(np.abs(energies["split"] - energies["fp64"]).max())
    if world > 1:
        import torch.distributed as dist
        n = len(all_sizes)
        e64 = S.gather_replicas(mine, energies["fp64"], n)
        e32 = S.gather_replicas(mine, energies["split"], n)
        t = torch.tensor([out["fp64"]["ms_per_build"], out["split"]["ms_per_build"]], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q = torch.tensor([out["quartets_per_build"]], dtype=torch.float64)
        dist.all_reduce(q)
        out = {"config": "c3", "ranks": world, "molecules": n, "scaling": "replicas",
               "quartets_per_build": int(q.item()),
               "fp64": {"ms_per_build_max_over_ranks": t[0].item(), "quartets_per_s": q.item() / (t[0].item() * 1e-3)},
               "split": {"ms_per_build_max_over_ranks": t[1].item(), "quartets_per_s": q.item() / (t[1].item() * 1e-3)},
               "max_abs_dE_per_molecule_hartree": float(np.nanmax(np.abs(e32 - e64))),
               "all_molecules_reported": bool(np.all(np.isfinite(e64)))}
        dist.destroy_process_group()
        if rank != 0:
            return None
    return out


def run_c4(nwater=64, seed=4, cycles=15, quick=False):
    if quick:
        nwater = 8
    spec = W.water_cluster(nwater, seed)
    t0 = time.perf_counter()
    mol = S.Molecule(spec, "cc-pvtz", cart=False, schwarz_cut=1e-12)
    plan_s = time.perf_counter() - t0
    d0 = S.fragment_guess(mol, _fragments(spec, nwater), "cc-pvtz")
    out = {"config": "c4", "nao": mol.nao, "quartets_per_build": mol.plan.quartets, "plan_s": plan_s}
    energies = {}
    for precision in ("fp64", "split"):
        res = S.rhf(mol, precision=precision, density0=d0, fixed_cycles=cycles, use_graph=True)
        energies[precision] = res.energy
        ms = res.jk_ms[1:]
        out[precision] = {"s_per_iter": float(np.mean(ms)) * 1e-3,
                          "quartets_per_s": mol.plan.quartets / (np.mean(ms) * 1e-3),
                          "energy_hartree": res.energy,
                          "last_iter_dE": abs(res.energies[-1] - res.energies[-2])}
        if precision == "split":
            e0, e1 = _events()
            e0.record()
            g = S.rhf_gradient(mol, res)
            e1.record()
            torch.cuda.synchronize()
            out["force_ms"] = e0.elapsed_time(e1)
            out["net_force"] = float(np.abs(g.sum(0)).max())
            # the same force with the split-precision coordinate VJP
            e0.record()
            gs = S.rhf_gradient(mol, res, precision="split")
            e1.record()
            torch.cuda.synchronize()
            out["force_split_vjp_ms"] = e0.elapsed_time(e1)
            out["force_split_vjp_max_abs_diff"] = float(np.abs(gs - g).max())
    out["split_speedup"] = out["fp64"]["s_per_iter"] / out["split"]["s_per_iter"]
    out["abs_dE_hartree"] = abs(energies["split"] - energies["fp64"])
    return out


def run_packed(nwater=4, seed=1, reps=5):
    """Packed-ERI producer and consumer on (H2O)n cc-pVDZ: s8 ERIs of every
    AO quartet (cut 0), then J/K of one density from them; the consumer
    streams the s8 array once (HBM roofline: bytes read / time)."""
    from . import basis as B
    from . import jk as J
    spec = W.water_cluster(nwater, seed)
    top, par, _ = B.prepare_basis(spec, "cc-pvdz", cart=False)
    atm, bas, env = B.pack(top, par)
    n = top.nao
    eri = J.packed_eri(atm, bas, env, cart=False, aosym="s8")
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(reps):
        eri = J.packed_eri(atm, bas, env, cart=False, aosym="s8")
    e1.record()
    torch.cuda.synchronize()
    t_eri = e0.elapsed_time(e1) / reps
    d = torch.as_tensor(W.psd_density(n, 5 * nwater, 0), device=eri.device)
    J.packed_jk(eri, d)
    e0.record()
    for _ in range(reps):
        J.packed_jk(eri, d)
    e1.record()
    torch.cuda.synchronize()
    t_jk = e0.elapsed_time(e1) / reps
    nbytes = eri.numel() * 8
    return {"config": "packed", "system": f"(H2O){nwater} cc-pVDZ", "nao": n, "s8_elements": eri.numel(),
            "producer_ms": t_eri, "consumer_ms": t_jk,
            "consumer_eri_read_gbs": nbytes / (t_jk * 1e-3) / 1e9}


def run_prof(case="jk", nwater=8, basis="cc-pvdz", seed=1):
    """One small run of a kernel family for profiler captures: `jk` one FP64
    and one split J/K build of (H2O)n (seeded PSD density), `grad` one
    coordinate VJP after them, `packed` the s8 producer and the consumer."""
    from . import basis as B
    from . import jk as J
    spec = W.water_cluster(nwater, seed)
    if case == "packed":
        return run_packed(nwater=nwater, seed=seed, reps=1)
    top, par, _ = B.prepare_basis(spec, basis, cart=False)
    atm, bas, env = B.pack(top, par)
    n = top.nao
    plan = J.DirectJKPlan([(atm, bas, env)], cart=False, cutoff=1e-12)
    d = torch.as_tensor(W.psd_density(n, 5 * nwater, 0), device=plan.device).reshape(1, -1)
    out = {"config": "prof", "case": case, "system": f"(H2O){nwater} {basis}", "nao": n}
    import ctypes
    from . import _capi
    lib = _capi.lib()
    nc = _capi.NCLASS
    q = (ctypes.c_int64 * nc)(); pq = (ctypes.c_int64 * nc)()
    _capi.check(lib.b200jk_plan_class_stats(plan._h, q, pq))
    out["class_quartets"] = {"({}{}|{}{})".format(*_capi.QUARTET_CLASSES[c]): [int(q[c]), int(pq[c])]
                             for c in range(nc) if q[c] > 0}
    for precision in ("fp64", "split"):
        plan.jk_packed(d, hermi=1, precision=precision)   # first use: kernel attributes, module load
        e0, e1 = _events()
        e0.record()
        plan.jk_packed(d, hermi=1, precision=precision)
        e1.record()
        torch.cuda.synchronize()
        out[f"{precision}_ms"] = e0.elapsed_time(e1)
        # per-class launch times of one more build (serial launches, CUDA events)
        lib.b200jk_plan_set_profiling(plan._h, 1)
        plan.jk_packed(d, hermi=1, precision=precision)
        ms64 = (ctypes.c_double * nc)(); ms32 = (ctypes.c_double * nc)(); nl = (ctypes.c_int32 * nc)()
        _capi.check(lib.b200jk_plan_profile(plan._h, ms64, ms32, nl))
        lib.b200jk_plan_set_profiling(plan._h, 0)
        cls = {}
        for c in range(nc):
            for tag, arr in (("f64", ms64), ("f32", ms32)):
                if arr[c] > 0:
                    cls["({}{}|{}{}){}".format(*_capi.QUARTET_CLASSES[c], tag)] = round(arr[c], 4)
        out[f"{precision}_class_ms"] = cls
    if case == "grad":
        g = torch.zeros((plan.natm[0], 3), dtype=torch.float64, device=plan.device)
        cot = torch.stack([d / 2.0, -d / 4.0]).contiguous()
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

        def vjp(precision=_capi.FP64):
            _capi.check(lib.b200jk_direct_jk_geom_vjp_precision(
                plan._h, ctypes.c_void_p(d.data_ptr()), 1, ctypes.c_void_p(cot.data_ptr()), 1, 1, precision,
                J.DEFAULT_FP32_CUT, ctypes.c_void_p(g.data_ptr()), st))
        vjp()   # first use
        e0, e1 = _events()
        e0.record()
        vjp()
        e1.record()
        torch.cuda.synchronize()
        out["vjp_ms"] = e0.elapsed_time(e1)
        g64 = g.clone()
        vjp(_capi.SPLIT)
        e0.record()
        vjp(_capi.SPLIT)
        e1.record()
        torch.cuda.synchronize()
        out["vjp_split_ms"] = e0.elapsed_time(e1)
        out["vjp_split_max_abs_diff"] = (g - g64).abs().max().item()
        # per-class launch times of one more VJP (serial launches, CUDA events)
        nc = _capi.NCLASS
        lib.b200jk_plan_set_profiling(plan._h, 1)
        vjp()
        ms64 = (ctypes.c_double * nc)(); ms32 = (ctypes.c_double * nc)(); nl = (ctypes.c_int32 * nc)()
        _capi.check(lib.b200jk_plan_profile(plan._h, ms64, ms32, nl))
        lib.b200jk_plan_set_profiling(plan._h, 0)
        out["vjp_class_ms"] = {"({}{}|{}{})".format(*_capi.QUARTET_CLASSES[c]): round(ms64[c], 4)
                               for c in range(nc) if ms64[c] > 0}
    plan.close()
    return out


def run_tcprobe(ncol=1 << 20, reps=20):
    """The tensor-core decision for the f x f bra transfer: the scalar
    recursion against the same linear map as a GEMM on the FP64 tensor cores
    (b200jk_measure_bra_transfer), ns per (root, axis, ket) column."""
    import ctypes
    from . import _capi
    ns = (ctypes.c_double * 2)()
    diff = ctypes.c_double()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(_capi.lib().b200jk_measure_bra_transfer(ncol, reps, ns, ctypes.byref(diff), st))
    return {"config": "tcprobe", "transfer": "f x f bra (16 outputs from 7 inputs per column), FP64",
            "columns": ncol, "reps": reps, "ns_per_column_recursion": ns[0], "ns_per_column_dmma_gemm": ns[1],
            "max_abs_diff": diff.value}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("config", choices=("c0", "c2", "c3", "c4", "packed", "prof", "tcprobe"))
    ap.add_argument("--quick", action="store_true", help="reduced size (smoke run)")
    ap.add_argument("--cycles", type=int, default=15, help="c4: SCF iterations per precision")
    ap.add_argument("--case", default="jk", choices=("jk", "grad", "packed"), help="prof: kernel family")
    ap.add_argument("--nwater", type=int, default=8, help="prof: cluster size")
    ap.add_argument("--basis", default="cc-pvdz", help="prof: basis set")
    a = ap.parse_args(argv)
    fn = {"c0": run_c0, "c2": run_c2, "c3": lambda: run_c3(quick=a.quick), "packed": run_packed,
          "c4": lambda: run_c4(cycles=a.cycles, quick=a.quick),
          "prof": lambda: run_prof(a.case, a.nwater, a.basis), "tcprobe": run_tcprobe}[a.config]
    if a.config == "c2" and a.quick:
        fn = lambda: run_c2(nwater=4)  # noqa: E731
    res = fn()
    if res is not None:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
