"""Benchmark: SILVAN progressive-sampling betweenness on one B200.

Workload (default): directed R-MAT, scale 20, edge factor 16, (a,b,c,d) =
(.57,.19,.19,.05), duplicates and self-loops removed, seed 2; eps 0.005,
delta 0.05, reference defaults otherwise (alpha 2.3, a 2, m_hat on).  The
graph is generated by this repository's seeded generator (the paper's
datasets are not available offline).

A step is one complete estimation (pass 1, empirical peeling, bounds, pass 2
up to the stopping decision) on the device-resident graph.  The metric is
paths/s: committed samples of both passes (void samples included, the
reference's unit) per second of the estimation window, i.e. the window the
reference reports as "Total time".  time-to-(eps,delta) is reported beside it.

  value   samples / device time of the K timed runs (CUDA events on the
          job's stream, device synchronised on both sides)
  e2e     the same through the C-ABI from host buffers: CSR upload, job
          creation, the run and the read-back of every estimate per step
  cpu_baseline / --impl reference
          the reference's own estimator (silvan/src/*.cpp with its LCG and
          OpenMP, its own flags) on the same graph, all host threads

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--config rmat20|ba10k] [--form batched|plain]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "rmat20": dict(workload="rmat20_directed_ef16_seed2", gen="rmat", scale=20, edge_factor=16,
                   seed=2, directed=True, eps=0.005, delta=0.05, k=0),
    "ba10k": dict(workload="ba_n10000_m5_seed1", gen="ba", n=10000, m=5, seed=1,
                  directed=False, eps=0.01, delta=0.05, k=0),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def make_graph(cfg):
    import silvan_b200 as sb
    if cfg["gen"] == "rmat":
        pairs = sb.rmat(cfg["scale"], cfg["edge_factor"], cfg["seed"], cfg["directed"])
    else:
        pairs = sb.barabasi_albert(cfg["n"], cfg["m"], cfg["seed"])
    return sb.HostGraph.from_pairs(pairs, cfg["directed"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def refbench_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsilvan_refbench.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.refbench_run.restype = C.c_int
    lib.refbench_run.argtypes = [C.c_uint32, C.c_int] + [C.c_void_p] * 4 + \
        [C.c_double, C.c_double, C.c_uint32, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int] + \
        [C.c_void_p] * 5 + [C.c_uint64]
    return lib


def reference_run(lib, csr, cfg, threads):
    tt, p1, p2, vis = C.c_double(), C.c_uint64(), C.c_uint64(), C.c_uint64()
    rc = lib.refbench_run(csr.n, int(csr.directed), csr.out_off.ctypes.data,
                          csr.out_adj.ctypes.data, csr.in_off.ctypes.data,
                          csr.in_adj.ctypes.data, cfg["eps"], cfg["delta"], cfg["k"], 2.3, 0,
                          2.0, 1, threads, C.byref(tt), C.byref(p1), C.byref(p2), C.byref(vis),
                          None, 0)
    if rc != 0:
        raise RuntimeError("reference run failed")
    return dict(total_time=tt.value, samples=p1.value + p2.value, vis=vis.value)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference_arm(args, cfg):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    lib = refbench_lib()
    if lib is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libsilvan_refbench.so was not built (needs the "
                          "reference sources at build time)"}))
        return 0
    hg = make_graph(cfg)
    csr = hg.csr()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_run(lib, csr, cfg, threads)
    runs = [reference_run(lib, csr, cfg, threads) for _ in range(args.steps)]
    samples = sum(r["samples"] for r in runs)
    t = sum(r["total_time"] for r in runs)
    val = samples / t
    print(json.dumps({
        "impl": "reference", "metric": "paths/sec", "value": val, "unit": "paths/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * t / len(runs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32/u64/f64", "data": "synthetic",
        "config": {"workload": cfg["workload"], "eps": cfg["eps"], "delta": cfg["delta"]},
        "time_to_guarantee_ms": 1000 * t / len(runs),
        "cpu_baseline": {"value": val, "unit": "paths/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(runs)} complete estimations (reference 'Total time' "
                                   f"window) on the benchmark graph"},
        "e2e": {"value": val, "unit": "paths/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rmat20", choices=sorted(CONFIGS))
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--slots", type=int, default=0,
                    help="sampler slots (0 = occupancy x SMs); small values bound the device "
                         "memory for profiler captures")
    ap.add_argument("--block", type=int, default=0, choices=[0, 128, 256, 512, 1024],
                    help="threads per sampler slot (0 = autotuned per graph and round)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference_arm(args, cfg)

    import numpy as np
    import torch
    import silvan_b200 as sb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    hg = make_graph(cfg)
    csr = hg.csr()
    g = sb.Graph.from_host(hg)
    seed0 = 1000 + 100 * rank

    def one_run(seed):
        job = sb.Probabilistic(g, cfg["eps"], cfg["delta"], k=cfg["k"], seed=seed,
                               form=args.form, slots=args.slots, block=args.block)
        res = job.run()
        del job
        return res

    for w in range(args.warmup):
        one_run(seed0 + w)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    results = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for s in range(args.steps):
            results.append(one_run(seed0 + args.warmup + s))
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    samples = sum(r["first_pass_samples"] + r["num_samples"] for r in results)
    t_dev = sum(r["time_device_s"] for r in results)
    launches = sum(r["kernel_launches"] for r in results)

    # e2e through the C-ABI from pinned host buffers: CSR upload, job
    # creation, the run and the read-back of every estimate, per step
    def pinned(a):
        t = torch.empty(a.shape, dtype={np.uint64: torch.int64, np.uint32: torch.int32}[
            a.dtype.type], pin_memory=True)
        v = t.numpy().view(a.dtype)
        v[...] = a
        return t, v

    keep = []
    pcsr = sb.CSR(csr.n, csr.directed, *[None] * 5, csr.n_components, csr.diameter)
    for f in ("out_off", "out_adj", "in_off", "in_adj", "cc"):
        t, v = pinned(getattr(csr, f))
        keep.append(t)
        setattr(pcsr, f, v)
    est_t = torch.empty(csr.n, dtype=torch.float64, pin_memory=True)
    e2e_t, e2e_samples = 0.0, 0
    h2d = int(csr.out_off.nbytes + csr.out_adj.nbytes + csr.cc.nbytes)
    if csr.directed:
        h2d += int(csr.in_off.nbytes + csr.in_adj.nbytes)
    d2h = csr.n * 8
    for s in range(0 if args.no_e2e else args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = sb.Graph.upload(pcsr, with_cc=True)
        job = sb.Probabilistic(g2, cfg["eps"], cfg["delta"], k=cfg["k"],
                               seed=seed0 + 50 + s, form=args.form, slots=args.slots,
                               block=args.block)
        r = job.run()
        job.get_centrality(out=est_t.numpy())
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t0
        e2e_samples += r["first_pass_samples"] + r["num_samples"]
        del job, g2

    # aggregate over ranks: total work / slowest rank
    vals = torch.tensor([samples, t_dev, e2e_samples, e2e_t], dtype=torch.float64, device="cuda")
    if pg:
        tot = vals.clone()
        mx = vals.clone()
        pg.all_reduce(tot)
        pg.all_reduce(mx, op=pg.ReduceOp.MAX)
        samples_all, t_max, e2e_s_all, e2e_t_max = tot[0].item(), mx[1].item(), tot[2].item(), \
            mx[3].item()
    else:
        samples_all, t_max, e2e_s_all, e2e_t_max = samples, t_dev, e2e_samples, e2e_t
    if rank == 0:
        peak, peak_kind = peaks()
        # roofline of the sampler kernel: algorithmic bytes per sample are
        # 8 B per scanned adjacency entry (neighbour id + visited-state probe),
        # 24 B per visited node (row offsets, sigma, state) and 4 B per
        # predecessor entry
        alg = sum(8 * r["vis_edges"] + 24 * r["ball_nodes"] + 4 * r["pred_entries"]
                  for r in results)
        t_samp = sum(r["time_sampling_s"] for r in results)
        achieved = alg / t_samp / 1e9 if t_samp > 0 else 0.0
        traffic = None
        tp = os.path.join(ROOT, "profiles", "sampler_traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                tj = json.load(f)
            if tj.get("workload") == cfg["workload"]:
                traffic = tj.get("bytes_per_launch")
        cpu = None
        if not args.no_cpu_baseline:
            lib = refbench_lib()
            if lib is not None:
                threads = os.cpu_count() or 1
                rr = reference_run(lib, csr, cfg, threads)
                cpu = {"value": rr["samples"] / rr["total_time"], "unit": "paths/s",
                       "cores": threads, "kind": "reference",
                       "sample": "one complete estimation of the benchmark graph by the "
                                 "reference's OpenMP build ('Total time' window)"}
        line = {
            "metric": "paths/sec", "value": samples_all / t_max, "unit": "paths/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64/f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "n": csr.n, "m": int(csr.out_off[-1]),
                       "eps": cfg["eps"], "delta": cfg["delta"], "form": args.form,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set above L2 (CSR 128 MB + per-slot state)",
                       "sampler_block": [r["sampler_block"] for r in results],
                       "sampler_launches_per_step": sum(r["sampler_launches"] for r in results)
                       / args.steps},
            "time_to_guarantee_ms": 1000 * t_max / args.steps,
            "samples_per_step": samples_all / max(1, world) / args.steps,
            "backtracked_paths_per_step": sum(r["backtracked_paths"] for r in results) /
                                          args.steps,
            "e2e": {"value": e2e_s_all / e2e_t_max if e2e_t_max > 0 else None,
                    "unit": "paths/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "sampler_kernel", "peak_kind": peak_kind},
            "breakdown_ms_per_step": {
                "sampler": 1000 * sum(r["time_sampling_s"] for r in results) / args.steps,
                "commit": 1000 * sum(r["time_apply_s"] for r in results) / args.steps,
                "total": 1000 * t_dev / args.steps},
            "work_per_step": {
                "vis_edges": sum(r["vis_edges"] for r in results) / args.steps,
                "ball_nodes": sum(r["ball_nodes"] for r in results) / args.steps,
                "pred_entries": sum(r["pred_entries"] for r in results) / args.steps,
                "checks": sum(r["checks"] for r in results) / args.steps},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
