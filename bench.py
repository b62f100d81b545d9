"""Benchmark: direct J/K builds of an RHF SCF on the (H2O)32 / cc-pVDZ cluster.

Workload: the 768-function (H2O)32 cc-pVDZ cluster from the seeded
generator (seed 1), Schwarz cut 1e-12.  RHF from the core guess with DIIS;
each iteration builds J/K incrementally from dD = D - D_last as the
reference's SCF caller does (src/gradscf/scf/rks.py:305-321).

One step = one SCF iteration's complete J/K build (density transform, every
class-pair kernel, finalisation).  Per precision mode the SCF runs
exactly W + K iterations: W untimed, then K timed builds (CUDA events on the
launching stream; L2 flushed by a 512 MB write before each).  FP64 mode
evaluates every quartet in FP64; split mode evaluates quartets with
Q_ij Q_kl max|dD| < 1e-6 in FP32 (FP64 accumulation).  The energy
difference between the two runs after the same iterations is reported.

Headline `value`: ERI quartets/s of the split-precision builds (whole job over
all ranks).  Quartets = significant canonical contracted shell quartets of the
reference's shells (i>=j, k>=l, ij>=kl, Q_ij Q_kl >= 1e-12) -- every build
evaluates all of them.  `e2e` replays the K timed split builds through the
public API with the dD copied from pinned host memory and J/K copied back.

`--impl reference` times the reference's CPU path on the same workload:
libcint 6.1.3 compiled from the reference's sources, driven by the C
restatement of its direct J/K driver (oracle/_ref), with all host threads,
full J/K builds of the same (H2O)32 cc-pVDZ cluster (one step = one build;
as many as fit in about 150 s, at least one, after a warm-up build of the
water monomer).  The reference screens by Schwarz bounds only, so its build
time does not depend on the density's values.  The `cpu_baseline` object of
the GPU line is a bounded sample instead: one build of the first 8 waters.

Multi-GPU (torchrun): one J/K build is shared by the ranks (strong scaling):
each rank evaluates its cost-balanced block of every class pair's work items
(b200jk_plan_set_shard) and the partial J/K are summed by one NCCL
all-reduce inside every build; times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "J/K build s/iter & ERI quartets/s: split vs FP64 on B200 at |ΔE|≤1e-8 Ha"
WORKLOAD = "(H2O)32 cc-pVDZ direct J/K (768 sph AOs), Schwarz 1e-12, seed 1"
FP32_CUT = 1e-6
SAMPLE_WATERS = 8


def sample_workload():
    from gradscf_b200 import basis as B, workloads as W
    spec = "; ".join(W.water_cluster(32, 1).split("; ")[:3 * SAMPLE_WATERS])
    top, par, _ = B.prepare_basis(spec, "cc-pvdz", cart=False)
    atm, bas, env = B.pack(top, par)
    c = np.random.default_rng(1).normal(size=(top.nao, 5 * SAMPLE_WATERS)) / np.sqrt(top.nao)
    return top, atm, bas, env, 2.0 * c @ c.T


def cpu_reference_full(steps, budget_s=150.0):
    """The reference arm: full J/K builds of the benchmark cluster itself on
    every host core; returns (quartets/s, cores, sample, s per build, builds)."""
    import oracle
    from gradscf_b200 import basis as B, workloads as W
    cores = os.cpu_count() or 1
    top, par, _ = B.prepare_basis(W.WATER, "cc-pvdz", cart=False)   # warm-up: page in the library
    atm, bas, env = B.pack(top, par)
    oracle.direct_jk(atm, bas, env, W.psd_density(top.nao, 5, 0), cart=False, cutoff=1e-12, workers=cores)
    top, par, _ = B.prepare_basis(W.water_cluster(32, 1), "cc-pvdz", cart=False)
    atm, bas, env = B.pack(top, par)
    q = oracle.count_quartets(oracle.schwarz_bounds(atm, bas, env, cart=False), 1e-12)
    d = 2.0 * W.psd_density(top.nao, 160, 1)
    times = []
    t_start = time.perf_counter()
    while len(times) < max(1, steps):
        t0 = time.perf_counter()
        oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12, workers=cores)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start + times[-1] > budget_s:
            break
    sample = (f"{len(times)} full J/K build(s) of the seed-1 (H2O)32 cc-pVDZ cluster ({top.nao} sph AOs, "
              f"{q} significant quartets, the GPU arm's workload), Schwarz 1e-12, workers={cores}; "
              f"builds capped at what fits in {budget_s:.0f} s after one warm-up build of the water monomer")
    step_s = float(np.mean(times))
    return q / step_s, cores, sample, step_s, len(times)


def cpu_reference_run(steps, warmup):
    """Time the reference CPU path on the bounded sample; returns (q/s, cores, sample)."""
    import oracle
    top, atm, bas, env, d = sample_workload()
    q = oracle.count_quartets(oracle.schwarz_bounds(atm, bas, env, cart=False), 1e-12)
    cores = os.cpu_count() or 1
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        oracle.direct_jk(atm, bas, env, d, cart=False, cutoff=1e-12, workers=cores)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    sample = (f"one full J/K build of the first {SAMPLE_WATERS} waters of the seed-1 (H2O)32 "
              f"cluster ({top.nao} sph AOs, {q} significant quartets), cc-pVDZ, Schwarz 1e-12, "
              f"workers={cores}")
    return q / float(np.mean(times)), cores, sample, float(np.mean(times))


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) != 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[2:]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--nwater", type=int, default=32,
                    help="cluster size (profiling runs use a smaller case; the benchmark is 32)")
    ap.add_argument("--eager", action="store_true",
                    help="launch the J/K kernels one by one instead of replaying a captured CUDA graph")
    ap.add_argument("--class-times", action="store_true",
                    help="add every class pair's per-step kernel time (both modes) to the line")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline leg (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        value, cores, sample, step_s, nbuilds = cpu_reference_full(args.steps)
        line = {"metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": args.gpus,
                "steps": nbuilds, "warmup": 1, "ms_per_step": step_s * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOAD, "sample": sample},
                "cpu_baseline": {"value": value, "unit": "quartets/s", "cores": cores,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": value, "unit": "quartets/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    from gradscf_b200 import _capi, flop_model, scf, workloads
    from gradscf_b200.jk import JKGraph
    import ctypes

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    lib = _capi.lib()
    st_h = ctypes.c_void_p(stream.cuda_stream)

    spec = workloads.water_cluster(args.nwater, 1)
    mol = scf.Molecule(spec, "cc-pvdz", cart=False, schwarz_cut=1e-12, device=dev)
    atoms = spec.split("; ")
    frags = ["; ".join(atoms[3 * i:3 * i + 3]) for i in range(args.nwater)]
    d0 = scf.fragment_guess(mol, frags, "cc-pvdz")
    plan = mol.plan
    if world > 1:
        # one J/K build shared by the ranks: cost-balanced work-item shards,
        # partial J/K summed by an NCCL all-reduce inside every build
        plan.set_shard(rank, world)
    n = mol.nao
    quartets = plan.quartets
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    # autotune the register-path tile shape (kets per work item) on a
    # representative incremental dD: the last warm-up iteration's (untimed)
    tune_delta = []
    scf.rhf(mol, precision="split", fp32_cut=FP32_CUT, fixed_cycles=args.warmup + 1, density0=d0,
            on_jk=lambda c, dd: tune_delta.append(dd.clone()) if c == args.warmup + 1 else None)
    tuned = plan.autotune(tune_delta[0].reshape(1, -1), hermi=1, precision="split", fp32_cut=FP32_CUT)

    peaks = {}
    for name, flag in (("fp64", 1), ("fp32", 0)):
        v = ctypes.c_double()
        _capi.check(lib.b200jk_measure_fma_peak(flag, ctypes.byref(v), st_h))
        peaks[name] = v.value

    nc = _capi.NCLASS
    classes = _capi.QUARTET_CLASSES
    q = (ctypes.c_int64 * nc)(); pq = (ctypes.c_int64 * nc)()
    _capi.check(lib.b200jk_plan_class_stats(plan._h, q, pq))
    nclasspairs = sum(1 for c in range(nc) if q[c] > 0)
    W, K = args.warmup, args.steps
    total = W + K

    results, deltas = {}, {"fp64": [], "split": []}
    deltas_split = deltas["split"]
    clocks = ClockSampler(local)
    with clocks:
        for precision in ("fp64", "split"):
            acc = {"q64": np.zeros(nc), "q32": np.zeros(nc), "pq64": np.zeros(nc), "pq32": np.zeros(nc),
                   "maxdd": []}

            def read_split_stats():
                a_ = [(ctypes.c_int64 * nc)() for _ in range(4)]
                _capi.check(lib.b200jk_plan_split_stats(plan._h, st_h, *a_))
                for key, arr in zip(("q64", "q32", "pq64", "pq32"), a_):
                    acc[key] += np.frombuffer(arr, dtype=np.int64)

            def on_jk(cycle, delta, precision=precision):
                if cycle - 1 > W and precision == "split":
                    read_split_stats()          # stats of the previous (timed) build
                if cycle > W:
                    if cycle == W + 1:
                        if dist:
                            dist.barrier()
                        torch.cuda.synchronize()
                    acc["maxdd"].append(delta.abs().max().item())
                    deltas[precision].append(delta.detach().to("cpu").pin_memory())
                    flush.zero_()

            res = scf.rhf(mol, precision=precision, fp32_cut=FP32_CUT, fixed_cycles=total, on_jk=on_jk,
                          density0=d0, use_graph=not args.eager)
            torch.cuda.synchronize()
            if precision == "split":
                read_split_stats()
            if dist:
                dist.barrier()
            step_ms = float(np.mean(res.jk_ms[W:]))
            # per-class kernel times: the same K builds replayed with
            # per-launch events (kept out of the timed builds above)
            lib.b200jk_plan_set_profiling(plan._h, 1)
            dprof = torch.empty((1, n * n), dtype=torch.float64, device=dev)
            for delta in deltas[precision]:
                dprof.copy_(delta.reshape(1, n * n))
                flush.zero_()
                plan.jk_packed(dprof, hermi=1, precision=precision, fp32_cut=FP32_CUT, check=False)
            torch.cuda.synchronize()
            lib.b200jk_plan_set_profiling(plan._h, 0)
            ms64 = (ctypes.c_double * nc)(); ms32 = (ctypes.c_double * nc)(); nl = (ctypes.c_int32 * nc)()
            _capi.check(lib.b200jk_plan_profile(plan._h, ms64, ms32, nl))
            if dist:
                t = torch.tensor([step_ms], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                step_ms = t.item()
            results[precision] = {"ms": step_ms, "ms64": list(ms64), "ms32": list(ms32), "res": res,
                                  "acc": acc}
        # end-to-end through the public API: host dD in, host J/K out, every step
        hd = torch.empty((1, n * n), dtype=torch.float64, pin_memory=True)
        hout = torch.empty((2, 1, n * n), dtype=torch.float64, pin_memory=True)
        dd = torch.empty((1, n * n), dtype=torch.float64, device=dev)
        out = torch.empty((2, 1, n * n), dtype=torch.float64, device=dev)
        e2e = []
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        graph = None if args.eager else JKGraph(plan, 1, hermi=1, precision="split", fp32_cut=FP32_CUT)
        for delta in deltas_split:
            hd.copy_(delta.reshape(1, n * n))
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if graph is not None:
                graph.inp.copy_(hd, non_blocking=True)
                res_out = graph.launch()
            else:
                dd.copy_(hd, non_blocking=True)
                res_out = plan.jk_packed(dd, hermi=1, precision="split", fp32_cut=FP32_CUT, out=out, check=False)
            hout.copy_(res_out, non_blocking=True)
            e1.record(stream)
            e2e.append((e0, e1))
            stream.synchronize()   # the host reads this step's result before reusing hd / hout
        torch.cuda.synchronize()
        if graph is not None:
            graph.close()
        e2e_step = float(np.mean([a.elapsed_time(b) for a, b in e2e]))
        if dist:
            t = torch.tensor([e2e_step], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_step = t.item()

    qps = {p_: quartets / (results[p_]["ms"] * 1e-3) for p_ in results}
    r64, r32 = results["fp64"]["res"], results["split"]["res"]
    acc = results["split"]["acc"]

    # roofline of the dominant kernel over the timed split builds
    best, top = None, []
    for c in range(nc):
        for kind, msk, pqk, qk, peak in (("fp64", "ms64", "pq64", "q64", peaks["fp64"]),
                                         ("fp32", "ms32", "pq32", "q32", peaks["fp32"])):
            t = results["split"][msk][c]
            if t <= 0:
                continue
            fl = flop_model.class_flops(classes[c], acc[pqk][c], acc[qk][c])
            top.append({"class": "(%d%d|%d%d)" % classes[c], "prec": kind, "ms_per_step": round(t / K, 3),
                        "tflops": round(fl / (t * 1e-3) / 1e12, 3) if fl else 0.0})
            if best is None or t > best[0]:
                best = (t, c, kind, fl, peak)
    top.sort(key=lambda r: -r["ms_per_step"])
    t_ms, c, kind, flops, peak = best
    achieved = flops / (t_ms * 1e-3) / 1e12
    total_ms = sum(results["split"]["ms64"]) + sum(results["split"]["ms32"])
    roofline = {"bound": kind, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": f"jk class ({classes[c][0]}{classes[c][1]}|{classes[c][2]}{classes[c][3]}) {kind}",
                "share_of_step": t_ms / total_ms,
                "peak_source": f"measured {kind} FMA microkernel on this GPU (b200jk_measure_fma_peak)"}
    fl64 = sum(flop_model.class_flops(classes[c_], pq[c_], q[c_]) for c_ in range(nc))
    fp64_build = {"ms_per_build": results["fp64"]["ms"], "quartets_per_s": qps["fp64"],
                  "model_tflops": fl64 / (results["fp64"]["ms"] * 1e-3) / 1e12,
                  "frac_of_fp64_peak": fl64 / (results["fp64"]["ms"] * 1e-3) / 1e12 / peaks["fp64"]}
    nlaunch = ctypes.c_int64()
    _capi.check(lib.b200jk_plan_launches(plan._h, _capi.SPLIT, ctypes.byref(nlaunch)))
    gpu_launches = K * int(nlaunch.value)   # this library's kernels in the K timed split builds
    line = {"metric": METRIC, "value": qps["split"], "unit": "quartets/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": results["split"]["ms"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32/f64 split (f64 accumulation)", "data": "synthetic",
            "config": {"workload": WORKLOAD if args.nwater == 32 else f"(H2O){args.nwater} cc-pVDZ (profiling case)",
                       "step": "one RHF iteration's incremental J/K build (dD = D - D_last)",
                       "launch": "eager kernel launches" if args.eager else "one CUDA-graph replay per build",
                       "scf": f"fragment guess (converged monomer densities), DIIS(8), {W} untimed + {K} timed iterations per mode",
                       "quartets_per_build": quartets, "nao": n, "fp32_cut": FP32_CUT,
                       "l2": "flushed (512 MB write) before every timed build",
                       "autotuned_kets_per_item": tuned,
                       "parallelism": f"J/K work-item shards x{world} + NCCL all-reduce" if world > 1 else "single GPU"},
            "s_per_iter": {"split": results["split"]["ms"] * 1e-3, "fp64": results["fp64"]["ms"] * 1e-3},
            "fp64": fp64_build,
            "split_speedup_vs_fp64": results["fp64"]["ms"] / results["split"]["ms"],
            "energy": {"fp64_hartree": r64.energy, "split_hartree": r32.energy,
                       "abs_dE_hartree": abs(r32.energy - r64.energy),
                       "last_iter_dE_fp64": abs(r64.energies[-1] - r64.energies[-2])},
            "split_fraction_fp32_quartets": float(acc["q32"].sum() / max(1.0, acc["q32"].sum() + acc["q64"].sum())),
            "split_fraction_fp32_prim_quartets": float(acc["pq32"].sum() / max(1.0, acc["pq32"].sum() + acc["pq64"].sum())),
            "max_abs_dD_timed": [float(x) for x in acc["maxdd"]],
            "e2e": {"value": quartets / (e2e_step * 1e-3), "unit": "quartets/s",
                    "ms_per_step": e2e_step, "h2d_bytes_per_step": int(n * n * 8),
                    "d2h_bytes_per_step": int(2 * n * n * 8)},
            "roofline": roofline, "gpu_launches": gpu_launches, "clocks": clocks.summary(),
            "top_kernels_split_step": top[:8]}
    if args.class_times:
        def _ct(mode):
            out = {}
            for c_ in range(nc):
                for kind_, arr in (("f64", results[mode]["ms64"]), ("f32", results[mode]["ms32"])):
                    if arr[c_] > 0:
                        name = "({}{}|{}{})".format(*classes[c_])
                        out[f"{name}{kind_}"] = round(arr[c_] / K, 4)
            return out
        line["class_ms_per_step"] = {"split": _ct("split"), "fp64": _ct("fp64")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        value, cores, sample, _ = cpu_reference_run(1, 0)
        line["cpu_baseline"] = {"value": value, "unit": "quartets/s", "cores": cores,
                                "kind": "reference", "sample": sample}
    if rank == 0:
        print(json.dumps(line))
    plan.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
