#!/usr/bin/env python
"""LM iterations/s of the B200 Schur-complement LM engine on config 2.

Workload (config 2): 1,500 cameras with 9-parameter blocks on a 30x50 grid,
500,000 points each seen by k~U{2..12} grid-neighbour cameras (3.5 M
observations), N(0,1) px noise plus 1% outliers, seeded synthetic data
(seed 1236; no dataset is published for this path).  A "step" is one
LevenbergMarquardt outer iteration (nelson/LevenbergMarquardt.hpp:63-138):
computeIncrement + oplus + cost + gain ratio, then the Jacobian pass.

  value       mixed-precision LM iterations/s (device time, CUDA events on the
              library's stream), inputs resident in HBM; the FP64 GPU path is
              timed beside it and the final costs compared.
  e2e         the same metric through the C ABI with host buffers: each e2e step
              uploads cameras, points and observations from pinned memory,
              runs nl_lm_solve for the K iterations, downloads the parameters.
  roofline    the dominant kernel (the Cholesky trailing update of S).
  cpu_baseline the FP64 CPU oracle (OpenMP, all host cores) on a bounded sample
              (2 LM iterations at config 2; all K iterations at configs 0 / 1).
  oracle_parity the per-sub-iteration cost, damping and gain ratio of both GPU
              traces against that oracle sample's (bounds 1e-9 FP64, 1e-6 mixed).

--config 1 (or 0) runs the same measurement on that workload: config 1 is 200
9-parameter cameras, 50,000 points, 375 k observations (S 1,800 x 1,800).
--config 3 times the batched configuration (256 uneven problems in one
persistent launch).  The default config-2 run also carries compact config-1,
config-3 and 2D scan-alignment (device SingleSection) figures under
other_configs (--no-extras skips them).

--impl reference times the FP64 CPU oracle (the restatement of the reference's
CPU path) on the same workload; under torchrun only rank 0 runs it.
N > 1 GPUs run independent replicas of the problem (the path has no
cross-problem exchange); value is the total over ranks.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LM iters/s, mixed vs FP64 GPU at ≤1e-6 rel final-cost err; CPU ref beside"
UNIT = "LM iterations/s"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []  # (host time, csv line)
        self.t0 = self.t1 = None

    def start(self):
        """Start sampling every 20 ms; returns once the first sample is in (the
        timed region is short, so nvidia-smi must already be running)."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 5.0
            while not self.lines and time.perf_counter() < deadline:
                time.sleep(0.01)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def begin(self):
        self.t0 = time.perf_counter()

    def end(self):
        self.t1 = time.perf_counter()
        time.sleep(0.05)  # let the sample that covers the end arrive

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        t0 = self.t0 if self.t0 is not None else -1e30
        t1 = self.t1 if self.t1 is not None else 1e30
        inside = [ln for ts, ln in self.lines if t0 <= ts <= t1 + 0.03]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window_ms": round(1e3 * (t1 - t0), 1) if self.t0 is not None else None}


class Ranks:
    """The bench's N > 1 plumbing: one process per GPU, each solving its own
    replica of the problem (the path has no cross-problem exchange).  The only
    collectives are the barrier around a timed region and the max of the
    per-rank times; the reported rate is the whole job's: world x the units
    one rank processed / the slowest rank's time."""

    def __init__(self, world, backend, device, timeout_s=600):
        import torch
        self.torch, self.world, self.device, self.pg = torch, world, device, None
        if world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.pg = dist

    def barrier(self):
        if self.device.type == "cuda":
            self.torch.cuda.synchronize()
        if self.pg is not None:
            self.pg.barrier()

    def max(self, x):
        if self.pg is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def total_rate(self, units_per_rank, seconds):
        """Whole-job units/s from one rank's units and this rank's seconds
        (max over ranks taken here)."""
        return self.world * units_per_rank / self.max(seconds)

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None


def measured_peaks():
    """HBM copy bandwidth (GB/s) and dense BF16 throughput (TF/s, burst and
    sustained) of this pool's B200s, or the fallback figures."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm": d.get("hbm_gbs", 6650.0), "bf16": d.get("bf16_tflops", 1590.0),
                "bf16_sustained": d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0)), "src": "measured"}
    return {"hbm": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0, "src": "fallback"}


def fp64_gemm_peak(device):
    """Dense FP64 throughput of this GPU (TF/s): cuBLAS DGEMM through
    torch.matmul on 8192^3 (2 N^3 flop), best of 5, CUDA events.  The FP64
    pipe peak has no driver-measured figure, so the bench measures it here."""
    import torch
    n = 8192
    dev = torch.device("cuda", device)
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def workload_config(cfg, scale, prob, world):
    """The `config` object both arms print for the same workload."""
    s_bytes = (-(-prob.nc_var * prob.bc // 128) * 128) ** 2 * 4
    w_bytes = prob.ne * 112
    big = s_bytes + w_bytes > 126 * 2 ** 20
    return {"workload": f"config {cfg}: {prob.nc_var} cams ({prob.bc}-param) / {prob.np_var} pts / "
                        f"{prob.ne} obs, LevenbergMarquardt",
            "scale": scale, "parallelism": f"replicas x{world}",
            "l2": (f"inputs larger than L2 (S {s_bytes / 2**20:.0f} MiB + W {w_bytes / 2**20:.0f} MiB FP32)" if big
                   else f"working set {(s_bytes + w_bytes) / 2**20:.0f} MiB (S + W, FP32) is not larger than L2 "
                        f"and L2 is not flushed between LM iterations")}


def trace_parity(tr_gpu, tr_orc):
    """Largest relative differences of the per-sub-iteration records (chi2,
    mu, rho, |delta|^2) between a GPU trace and the oracle's, over the records
    both have while the oracle's cost is still falling."""
    n = min(len(tr_gpu), len(tr_orc))
    out = {"records": 0, "chi2": 0.0, "mu": 0.0, "rho": 0.0, "inc_sqnorm": 0.0}
    for k in range(n):
        a, b = tr_gpu[k], tr_orc[k]
        if b[2] < 0 or a[2] < 0:
            continue
        if k > 0 and abs(tr_orc[k, 2] - tr_orc[k - 1, 2]) < 1e-9 * tr_orc[k, 2]:
            break
        out["records"] += 1
        out["chi2"] = max(out["chi2"], abs(a[2] - b[2]) / abs(b[2]))
        if b[3] != 0:
            out["mu"] = max(out["mu"], abs(a[3] - b[3]) / abs(b[3]))
        if k > 0:
            out["rho"] = max(out["rho"], abs(a[4] - b[4]) / max(abs(b[4]), 1e-300))
        if b[5] > 0:
            out["inc_sqnorm"] = max(out["inc_sqnorm"], abs(a[5] - b[5]) / b[5])
    return out


def profiled_traffic():
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except ValueError:
            return None
    return None


def run_reference(args, rank, world):
    """--impl reference: the FP64 CPU oracle, rank 0 only."""
    if rank != 0:
        return
    from oracle.oracle import LMSettings, Oracle
    from nelson_b200.problems import make_config
    prob = make_config(args.config, args.scale)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    o = Oracle.from_ba(prob, threads=cores)
    for _ in range(args.warmup):  # warm-up: evaluation passes (page-in, thread pool)
        o.update(True)
    o.set_params(prob.cams, prob.pts)
    t0 = time.perf_counter()
    reason, tr, its, sub = o.lm_solve(LMSettings(maxNumIt=args.steps))
    dt = time.perf_counter() - t0
    its = max(its, 1)
    v = its / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / its,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded, config-{args.config} shapes; no public dataset)",
            "config": workload_config(args.config, args.scale, prob, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{its} LM iterations of config {args.config} in one oracle solve "
                                       f"(FP64 C++/OpenMP restatement; the reference itself cannot be built here)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "final_chi2": float(tr[-1, 2]), "reason": reason,
            "trace": [[float(x) for x in r[:5]] for r in tr]}
    print(json.dumps(line), flush=True)


def measure_batch(its, warmup, device, cpu=True, nprob=256):
    """Config 3: `nprob` independent uneven problems.  The product path is the
    persistent launch (nl_batch_lm_solve: one kernel, a device work queue, one
    CTA per problem; launch shape from nl_batch_autotune); the per-problem
    CUDA-graph path (nl_lm_solve_batch) is timed beside it.  problems/s over
    the batch (device time of the launch) and per-problem latency."""
    from nelson_b200 import native as N
    from nelson_b200.problems import make_batch
    probs = make_batch(nprob)
    # the handles carry structure and parameters; the persistent solve is FP64 whatever their precision
    hs = [N.BAProblemGPU.from_ba(p, precision=N.PREC_MIXED, device=device) for p in probs]
    b = N.PersistentBatch(hs)
    s = N.LMSettings(maxNumIt=its)

    def reset():
        for g, p in zip(hs, probs):
            g.set_params(p.cams, p.pts)

    nt, cps = b.autotune(s)
    for _ in range(warmup):
        reset()
        b.lm_solve(s)
    reset()
    clocks = Clocks(device)
    clocks.start()
    clocks.begin()
    reasons, chi2, iters, lat, solve_ms, dev_ms = b.lm_solve(s)
    clocks.end()
    ck = clocks.stop()
    # e2e: parameters uploaded from host buffers, the launch, results read back
    import ctypes as C
    L = N.load()
    t0 = time.perf_counter()
    for g, p in zip(hs, probs):
        assert L.nl_set_params(g.h, N._p(np.ascontiguousarray(p.cams)), N._p(np.ascontiguousarray(p.pts))) == 0
    b.lm_solve(s)
    outs = [g.get_params() for g in hs]
    e2e_s = time.perf_counter() - t0
    h2d = sum(p.cams.size + p.pts.size for p in probs) * 8
    d2h = sum(c.size + q.size for c, q in outs) * 8
    b.close()
    # the per-problem graph path on the same (mixed) handles, for comparison
    reset()
    N.lm_solve_batch(hs, s)
    reset()
    _, _, _, lat_g = N.lm_solve_batch(hs, s)
    for g in hs:
        g.close()
    out = {"metric": "problems/s (batched uneven problems, LM)", "value": nprob / (dev_ms / 1e3),
           "unit": "problems/s", "steps": its, "dtype": "f64",
           "config": {"workload": f"config 3: {nprob} problems, cams U{{8..64}} (6-param), pts U{{200..4000}}, "
                                  f"k~U{{3..8}}, {its} LM iterations each", "launch": "one persistent kernel",
                      "autotuned": {"threads": nt, "ctas_per_sm": cps}},
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
           "solve_ms": {"p50": float(np.percentile(solve_ms, 50)), "p99": float(np.percentile(solve_ms, 99))},
           "launch_ms": dev_ms,
           "e2e": {"value": nprob / e2e_s, "unit": "problems/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "step": "parameter upload + nl_batch_lm_solve + parameter download"},
           "graph_path": {"value": nprob / (float(lat_g.max()) / 1e3), "unit": "problems/s",
                          "note": "nl_lm_solve_batch: per-problem captured sub-iteration graphs interleaved over streams "
                                  "(mixed precision)"},
           "converged_or_stopped": {k: int(v) for k, v in zip(*np.unique(reasons, return_counts=True))},
           "clocks": ck, "cpu_baseline": None}
    if cpu:
        from oracle.oracle import LMSettings as OLM
        from oracle.oracle import Oracle
        cores = len(os.sched_getaffinity(0))
        t1 = time.perf_counter()
        nsample, worst = 0, 0.0
        while nsample < len(probs) and time.perf_counter() - t1 < 15.0:
            o = Oracle.from_ba(probs[nsample], threads=cores)
            o.lm_solve(OLM(maxNumIt=its))
            worst = max(worst, abs(o.chi2() - chi2[nsample]) / o.chi2())
            nsample += 1
        dt = time.perf_counter() - t1
        out["cpu_baseline"] = {"value": nsample / dt, "unit": "problems/s", "cores": cores, "kind": "port",
                               "sample": f"{nsample} of the {nprob} problems, {its} LM iterations each, one after "
                                         f"another (FP64 C++/OpenMP oracle, {dt:.1f} s)"}
        out["oracle_parity"] = {"problems_compared": nsample, "final_chi2_max_rel_err": worst, "bound": 1e-9,
                                "ok": bool(worst <= 1e-9)}
    return out


def measure_single(cfg, its, warmup, device):
    """A compact line for another single-problem configuration (config 1:
    the plain FP64 GPU path against the CPU reference): mixed and FP64 LM
    iterations/s (device time), the oracle's full K-iteration solve as the CPU
    baseline, and the per-sub-iteration parity of both GPU traces."""
    from nelson_b200 import native as N
    from nelson_b200.problems import make_config
    from oracle.oracle import LMSettings as OLM
    from oracle.oracle import Oracle
    prob = make_config(cfg)
    out = {"config": workload_config(cfg, 1.0, prob, 1)}
    traces = {}
    for name, prec in (("mixed", N.PREC_MIXED), ("fp64_gpu", N.PREC_FP64)):
        g = N.BAProblemGPU.from_ba(prob, precision=prec, device=device)
        g.lm_solve(N.LMSettings(maxNumIt=warmup), trace_cap=0)
        g.set_params(prob.cams, prob.pts)
        _, tr, it, _, rep = g.lm_solve(N.LMSettings(maxNumIt=its), trace_cap=4096, report=True)
        out[name] = {"value": max(it, 1) / (rep["device_ms"] / 1e3), "unit": UNIT, "final_chi2": rep["chi2"]}
        traces[name] = tr
        g.close()
    cores = len(os.sched_getaffinity(0))
    o = Oracle.from_ba(prob, threads=cores)
    t0 = time.perf_counter()
    _, tro, its_o, _ = o.lm_solve(OLM(maxNumIt=its))
    dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": max(its_o, 1) / dt, "unit": UNIT, "cores": cores, "kind": "port",
                           "sample": f"the full {its_o}-iteration LM solve (FP64 C++/OpenMP oracle, {dt:.1f} s)"}
    pm, pd = trace_parity(traces["mixed"], tro), trace_parity(traces["fp64_gpu"], tro)
    out["oracle_parity"] = {"records_compared": pd["records"],
                            "fp64_gpu": {k: pd[k] for k in ("chi2", "mu", "rho", "inc_sqnorm")},
                            "mixed": {k: pm[k] for k in ("chi2", "mu", "rho", "inc_sqnorm")},
                            "ok": bool(pd["chi2"] <= 1e-9 and pm["chi2"] <= 1e-6 and pd["records"] > 0)}
    out["fp64_gpu_vs_cpu"] = out["fp64_gpu"]["value"] / out["cpu_baseline"]["value"]
    return out


def measure_pose2d(device, cpu=True):
    """The device SingleSection (2D scan alignment with point-to-line edges,
    nl_pose2d_*): the reference test's problem solved to convergence, and a
    2,000-pose graph, FP64 and mixed.  solve_ms spans the whole LM solve on
    the library's stream (CUDA events; the host control between launches
    included).  The CPU baseline is the numpy FP64 oracle of the same solve
    (the full solve on the small problem, 3 LM iterations on the large one)."""
    from nelson_b200 import native as N
    from nelson_b200.problems import pose_graph_scene, scan_align_scene
    from oracle.pose2d import Pose2DOracle
    cores = len(os.sched_getaffinity(0))
    out = {}
    for key, prob, cpu_its in (("reference_problem", scan_align_scene(15, 3000, seed=5), 100),
                               ("pose_graph_2000", pose_graph_scene(2000, 500, 3000, 30, seed=7), 3)):
        npts = sum(len(prob.scans[i]) for i, _ in prob.edges)
        res = {"workload": f"{prob.name}: {len(prob.poses0)} variable poses + 1 fixed, {len(prob.edges)} edges, "
                           f"{npts} point-to-line residuals, AMD order, envelope solver",
               "edge_bytes_per_update": npts * 48}
        traces = {}
        for name, prec in (("fp64", N.PREC_FP64), ("mixed", N.PREC_MIXED)):
            g = N.Pose2DGPU.from_scan_align(prob, precision=prec, order="amd", device=device)
            g.set_solver_kind(N.SOLVER_ENVELOPE)
            g.lm_solve(N.LMSettings(maxNumIt=2), trace_cap=0)   # warm-up
            g.set_poses(prob.poses0)
            reason, tr, it = g.lm_solve()
            ms = g.last_report["device_ms"]
            chi2 = g.update(True)
            res[name] = {"solve_ms": ms, "iterations": it, "reason": reason, "lm_iters_per_s": max(it, 1) / (ms / 1e3),
                         "chi2_after": chi2, "chi2_below_1e-12": bool(chi2 < 1e-12)}
            traces[name] = tr
            g.close()
        if cpu:
            o = Pose2DOracle(prob)
            t0 = time.perf_counter()
            r_o, tro, it_o = o.lm_solve(maxNumIt=cpu_its)
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": max(it_o, 1) / dt, "unit": UNIT, "cores": cores, "kind": "port",
                                   "sample": f"{max(it_o, 1)} LM iteration(s), numpy FP64 oracle ({dt:.2f} s)"}
            n = min(len(tro), len(traces["fp64"]))
            rows = [k for k in range(n) if tro[k, 2] > 1e-9]
            rel = max((abs(traces["fp64"][k, 2] - tro[k, 2]) / tro[k, 2] for k in rows), default=None)
            res["oracle_parity"] = {"records_compared": len(rows), "fp64_chi2_max_rel_err": rel,
                                    "ok": bool(rel is not None and rel <= 1e-6)}
            res["fp64_vs_cpu"] = res["fp64"]["lm_iters_per_s"] / res["cpu_baseline"]["value"]
        out[key] = res
    return out


def run_batch(args, rank, world):
    """--config 3: the batched configuration as the bench line."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    ranks = Ranks(world, "nccl", torch.device("cuda", local))
    ranks.barrier()
    out = measure_batch(args.steps, args.warmup, local, cpu=(rank == 0 and not args.no_cpu_baseline))
    v = ranks.total_rate(256, 256 / out["value"])
    ranks.close()
    if rank == 0:
        out.update({"value": v, "n_gpus": world, "warmup": args.warmup, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded, config-3 generator)",
                    "gpu_launches": 1})
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-iters", type=int, default=0,
                    help="LM iterations of the CPU baseline sample (0: all K for configs 0 / 1, 2 for config 2)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the config-1 and config-3 figures of the default config-2 run")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    faulthandler.enable()  # a crash prints the Python stack of every thread to stderr
    rank, world, local = dist_env()

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.config == 3:
        run_batch(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    ranks = Ranks(world, "nccl", torch.device("cuda", local))

    from nelson_b200 import native as N
    from nelson_b200.problems import make_config

    prob = make_config(args.config, args.scale)
    gm = N.BAProblemGPU.from_ba(prob, precision=N.PREC_MIXED, device=local)
    gd = N.BAProblemGPU.from_ba(prob, precision=N.PREC_FP64, device=local)

    barrier = ranks.barrier
    max_over_ranks = ranks.max

    # ---- warm-up: W LM iterations on both paths ----
    for g in (gm, gd):
        g.lm_solve(N.LMSettings(maxNumIt=args.warmup), trace_cap=0)
        g.set_params(prob.cams, prob.pts)

    # ---- timed: K LM iterations, mixed (the product) then FP64 ----
    clocks = Clocks(local)
    clocks.start()
    launches0 = gm.kernel_launches()
    barrier()
    clocks.begin()
    r_m, tr_m, it_m, sub_m, rep_m = gm.lm_solve(N.LMSettings(maxNumIt=args.steps), trace_cap=4096, report=True)
    barrier()
    clocks.end()
    ck = clocks.stop()
    launches = gm.kernel_launches() - launches0
    r_d, tr_d, it_d, sub_d, rep_d = gd.lm_solve(N.LMSettings(maxNumIt=args.steps), trace_cap=4096, report=True)
    barrier()
    its_m = max(it_m, 1)
    its_d = max(it_d, 1)
    ms_m = max_over_ranks(rep_m["device_ms"])
    ms_d = max_over_ranks(rep_d["device_ms"])
    value = world * its_m / (ms_m / 1000.0)
    fp64_value = world * its_d / (ms_d / 1000.0)
    chi2_m, chi2_d = rep_m["chi2"], rep_d["chi2"]
    final_rel = abs(chi2_m - chi2_d) / abs(chi2_d)
    # per-iteration cost agreement of the accepted steps
    acc_m = [r[2] for r in tr_m if r[7] == 1 and r[2] > 0]
    acc_d = [r[2] for r in tr_d if r[7] == 1 and r[2] > 0]
    n = min(len(acc_m), len(acc_d))
    iter_rel = max((abs(a - b) / b for a, b in zip(acc_m[:n], acc_d[:n])), default=None)

    # ---- e2e: host buffers through the C ABI (pinned), K iterations per step ----
    cams_h = torch.from_numpy(np.ascontiguousarray(prob.cams)).pin_memory()
    pts_h = torch.from_numpy(np.ascontiguousarray(prob.pts)).pin_memory()
    obs_h = torch.from_numpy(np.ascontiguousarray(prob.obs)).pin_memory()
    cams_o = torch.empty_like(cams_h).pin_memory()
    pts_o = torch.empty_like(pts_h).pin_memory()
    L = N.load()
    import ctypes as C

    def vp(t):
        return C.c_void_p(t.data_ptr())

    e2e_steps = 1
    barrier()
    t0 = time.perf_counter()
    e2e_its = 0
    for _ in range(e2e_steps):
        assert L.nl_set_params(gm.h, vp(cams_h), vp(pts_h)) == 0
        assert L.nl_set_observations(gm.h, vp(obs_h), None) == 0
        rep = N.SolveReport()
        s = N.LMSettings(maxNumIt=args.steps)
        assert L.nl_lm_solve(gm.h, C.byref(s), C.byref(rep), None, 0) == 0
        assert L.nl_get_params(gm.h, vp(cams_o), vp(pts_o)) == 0
        e2e_its += max(rep.iterations, 1)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * e2e_its / e2e_s
    h2d = (cams_h.numel() + pts_h.numel() + obs_h.numel()) * 8
    d2h = (cams_o.numel() + pts_o.numel()) * 8

    # ---- the envelope solver (nl_set_solver_kind) on the same problem: the
    #      same increments, the tiles of S outside its Cholesky envelope skipped
    #      (a side measurement; the metric above is the dense solver's) ----
    envelope = {"note": "NL_SOLVER_ENVELOPE: tile-level profile Cholesky of the same S, camera order unchanged"}
    for name, g in (("mixed", gm), ("fp64", gd)):
        g.set_solver_kind(N.SOLVER_ENVELOPE)
        g.set_params(prob.cams, prob.pts)
        g.lm_solve(N.LMSettings(maxNumIt=1), trace_cap=0)
        g.set_params(prob.cams, prob.pts)
        barrier()
        _, _, it_e, _, rep_e = g.lm_solve(N.LMSettings(maxNumIt=args.steps), trace_cap=4096, report=True)
        barrier()
        envelope[name] = {"value": world * max(it_e, 1) / (max_over_ranks(rep_e["device_ms"]) / 1000.0),
                          "unit": UNIT, "final_chi2": rep_e["chi2"]}
        g.set_solver_kind(N.SOLVER_DENSE)
    envelope["speedup_vs_fp64_gpu"] = envelope["mixed"]["value"] / envelope["fp64"]["value"]
    envelope["final_chi2_equal_to_dense"] = envelope["mixed"]["final_chi2"] == chi2_m

    # ---- the FP64 comparison path: its trailing update against a measured DGEMM ----
    fp64_pipe = None
    if rank == 0:
        gd.set_params(prob.cams, prob.pts)
        gd.update(True)
        gd.compute_increment(0.0, 1e-3 * gd.max_abs_hdiag())
        p64 = gd.phase_times()
        dpk = fp64_gemm_peak(local)
        u64 = p64["update_ms"] * 1e-3
        a64 = p64["update_flop"] / u64 / 1e12 if u64 > 0 else None
        fp64_pipe = {"kernel": "cuBLAS DSYRK / DGEMM: the trailing update of the FP64 path's Cholesky",
                     "achieved_tflops": a64, "peak_tflops": dpk, "frac": (a64 / dpk) if a64 else None,
                     "peak_source": "measured here: torch.matmul float64 8192^3, best of 5, CUDA events",
                     "update_ms": p64["update_ms"], "factor_ms": p64["factor_ms"]}

    # ---- roofline of the dominant kernel: the trailing update of the factorisation ----
    peaks = measured_peaks()
    hbm, bf16 = peaks["hbm"], peaks["bf16_sustained"]
    gm.set_params(prob.cams, prob.pts)
    gm.update(True)
    mu = 1e-3 * gm.max_abs_hdiag()
    gm.compute_increment(0.0, mu)
    pt = gm.phase_times()
    # the factorisation's critical path, step by step (a separate call: timing
    # every step slows the factorisation itself)
    gm.set_timing_detail(True)
    gm.compute_increment(0.0, mu)
    ptd = gm.phase_times()
    gm.set_timing_detail(False)
    chain = {"factor_ms_timed_per_step": round(ptd["factor_ms"], 4), "panels": ptd["panels"],
             "diag_factor_ms": round(ptd["panel_ms"], 4), "row_tile_trsm_and_diag_update_ms": round(ptd["first_ms"], 4),
             "waits_ms": round(ptd["wait_ms"], 4)}
    # The trailing update is a rank-K update: K = 512 for the bulk of the
    # trailing matrix and the next group's columns (four panels per update),
    # K = 128 for the columns inside a group.  Every updated 128x128 FP32 tile
    # is read and written once per launch (128 KB: update_bytes) while the
    # BF16 hi/lo panels come from L2; the contraction runs as three BF16
    # products per FP32 multiply-add (hi*hi + hi*lo + lo*hi), i.e. 3 x
    # update_flop of tensor work.  At K = 512 that is 384 MMA flop per byte of
    # tile traffic, above the ridge of the measured peaks (~215), so the
    # update as a whole is tensor-bound; its roofline time is the larger of
    # the two lower bounds and both fractions are reported.
    alg_bytes = pt["update_bytes"]
    nlaunch = max(pt["update_launches"], 1)
    upd_s = pt["update_ms"] * 1e-3
    mma_flop = 3.0 * pt["update_flop"]
    t_hbm = alg_bytes / (hbm * 1e9)
    t_tc = mma_flop / (bf16 * 1e12)
    gbs = alg_bytes / upd_s / 1e9 if upd_s > 0 else None
    mma_tfl = mma_flop / upd_s / 1e12 if upd_s > 0 else None
    traffic = profiled_traffic()
    traffic_launch = None
    if traffic and traffic.get("bytes_per_tile_update"):
        traffic_launch = traffic["bytes_per_tile_update"] * (alg_bytes / (128 * 128 * 4 * 2)) / nlaunch
    tensor_bound = t_tc >= t_hbm
    roofline = {"bound": "tensor" if tensor_bound else "hbm",
                "kernel": "tc_syrk_kernel: Cholesky trailing update of S (tcgen05, split-BF16x3, K = 512 / 128)",
                "achieved": mma_tfl if tensor_bound else gbs,
                "peak": bf16 if tensor_bound else hbm,
                "unit": "TFLOP/s" if tensor_bound else "GB/s",
                "frac": ((mma_tfl / bf16) if tensor_bound else (gbs / hbm)) if upd_s > 0 else None,
                "peak_source": (f"{peaks['src']} sustained dense BF16 (the kernel runs inside a long step)"
                                if tensor_bound else f"{peaks['src']} HBM copy bandwidth"),
                "achieved_note": "BF16 MMA flops (3 per FP32 multiply-add of the n^3/3 trailing update) per second "
                                 "of summed update-launch time" if tensor_bound else
                                 "tile read-modify-write bytes per second of summed update-launch time",
                "roofline_ms": {"hbm": t_hbm * 1e3, "tensor": t_tc * 1e3, "launches_summed": upd_s * 1e3},
                "algorithmic_bytes_per_launch": alg_bytes / nlaunch,
                "algorithmic_flops_per_launch": pt["update_flop"] / nlaunch, "launches_per_factorisation": nlaunch,
                "traffic": traffic_launch,
                "traffic_source": (traffic or {}).get("source"),
                "hbm": {"achieved_gbs": gbs, "peak_gbs": hbm, "frac": (gbs / hbm) if gbs else None},
                "tensor": {"achieved_mma_tflops": mma_tfl, "peak_tflops": bf16,
                           "frac": (mma_tfl / bf16) if mma_tfl else None,
                           "achieved_fp32_tflops": pt["update_flop"] / upd_s / 1e12 if upd_s > 0 else None},
                "phases_ms": {k: round(v, 4) for k, v in pt.items()
                              if k.endswith("_ms") and k not in ("panel_ms", "wait_ms", "first_ms")},
                "critical_path": chain}

    # ---- CPU baseline: the FP64 oracle on a bounded sample ----
    # ... and its trace is the parity check of both GPU traces on this workload
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import LMSettings as OLM
        from oracle.oracle import Oracle
        cores = len(os.sched_getaffinity(0))
        o = Oracle.from_ba(prob, threads=cores)
        cpu_iters = args.cpu_iters if args.cpu_iters > 0 else {0: args.steps, 1: args.steps}.get(args.config, 2)
        t0 = time.perf_counter()
        _, tro, its_o, _ = o.lm_solve(OLM(maxNumIt=min(cpu_iters, args.steps)))
        dt = time.perf_counter() - t0
        cpu = {"value": max(its_o, 1) / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{max(its_o, 1)} LM iteration(s) of config {args.config} incl. the initial evaluation, "
                         f"FP64 C++/OpenMP oracle ({dt:.1f} s)"}
        pm, pd = trace_parity(tr_m, tro), trace_parity(tr_d, tro)
        parity = {"oracle_iterations": int(its_o), "records_compared": pd["records"],
                  "fp64_gpu": {k: pd[k] for k in ("chi2", "mu", "rho", "inc_sqnorm")},
                  "mixed": {k: pm[k] for k in ("chi2", "mu", "rho", "inc_sqnorm")},
                  "bounds": {"fp64_chi2": 1e-9, "mixed_chi2": 1e-6},
                  "ok": bool(pd["chi2"] <= 1e-9 and pm["chi2"] <= 1e-6 and pd["records"] > 0)}
        # the parameters after the oracle's iterations (outside every timed region)
        u_o, v_o = o.get_params()
        par = {}
        for name, g in (("fp64_gpu", gd), ("mixed", gm)):
            g.set_params(prob.cams, prob.pts)
            g.lm_solve(N.LMSettings(maxNumIt=int(its_o)), trace_cap=0)
            u_g, v_g = g.get_params()
            par[name] = {"cams_max_rel": float(np.abs(u_g - u_o).max() / np.abs(u_o).max()),
                         "pts_max_rel": float(np.abs(v_g - v_o).max() / np.abs(v_o).max())}
        parity["params_after_oracle_iterations"] = par

    # ---- the other configurations' headline figures, on rank 0 of a 1-GPU run ----
    others = None
    if rank == 0 and world == 1 and args.config == 2 and not args.no_extras:
        others = {"config1": measure_single(1, args.steps, 3, local),
                  "config3": measure_batch(10, 3, local, cpu=not args.no_cpu_baseline),
                  "pose2d": measure_pose2d(local, cpu=not args.no_cpu_baseline)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_m / its_m, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (FP64 refinement residual, solve accumulators, cost)",
                "data": f"synthetic (seeded, config-{args.config} shapes; no public dataset)",
                "config": workload_config(args.config, args.scale, prob, world),
                "fp64_gpu": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_d / its_d, "pipe": fp64_pipe},
                "speedup_vs_fp64_gpu": value / fp64_value,
                "final_cost_rel_err_vs_fp64": final_rel, "per_iter_cost_rel_err_vs_fp64": iter_rel,
                "oracle_parity": parity,
                "final_chi2": chi2_m, "reason": r_m, "subiterations": sub_m,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "step": f"upload + nl_lm_solve({args.steps} its) + download"},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "clocks": ck,
                "envelope_solver": envelope, "other_configs": others}
        print(json.dumps(line), flush=True)
    gm.close()
    gd.close()
    ranks.close()


if __name__ == "__main__":
    main()
