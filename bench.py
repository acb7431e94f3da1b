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

Other workloads (--config): ba10k (Barabasi-Albert n = 10^4), grid2048 (top-10
on a 2048 x 2048 lattice with shortcuts), multigraph64 (64 graphs of uneven
size in one batched run), serve (a Poisson stream of requests on fresh R-MAT
graphs: p50/p99 latency and paths/s under continuous batching), ingest
(loading the R-MAT 20 edge list: device parse and CSR build).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--config rmat20|ba10k|grid2048|multigraph64|serve|ingest]
                       [--form batched|plain] [--block 0|128|256|512|1024]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # R-MAT scale 20: the headline configuration (batched vs plain)
    "rmat20": dict(kind="single", workload="rmat20_directed_ef16_seed2", gen="rmat", scale=20,
                   edge_factor=16, seed=2, directed=True, eps=0.005, delta=0.05, k=0),
    # Barabasi-Albert n = 10^4: the CPU-runnable case, checked against Brandes
    "ba10k": dict(kind="single", workload="ba_n10000_m5_seed1", gen="ba", n=10000, m=5, seed=1,
                  directed=False, eps=0.01, delta=0.05, k=0),
    # 2048 x 2048 grid, 5 % of edges deleted, 0.1 % shortcuts: top-10 relative
    # mode with single-path sampling (-s 0); the reference's default alpha
    # makes path counts explode on lattices (reported beside the line)
    "grid2048": dict(kind="single", workload="grid2048_del05_short001_seed3_top10", gen="grid",
                     side=2048, delete=0.05, shortcut=0.001, seed=3, directed=False, eps=0.1,
                     delta=0.05, k=10, alpha=0.0, alpha_given=True, cpu_samples=40000),
    # 64 graphs of uneven size (half ER mean degree 8, half BA 4 edges per
    # node, n log-uniform in [10^3, 2 * 10^6], seeds 100-163) in one batched run
    "multigraph64": dict(kind="multi", workload="64_graphs_er8_ba4_n1e3_2e6_seeds100_163",
                         eps=0.01, delta=0.05),
    # Poisson request stream of fresh R-MAT graphs (scale 10-20, directed
    # with probability 1/2, eps in {0.01, 0.005, 0.0025}, top-10 on 20 %);
    # --topk-eps-scale multiplies the top-10 requests' relative eps (at
    # relative eps 0.01 one scale-20 top-10 request alone needs over 4 * 10^7
    # samples)
    "serve": dict(kind="serve", workload="rmat_scale10_20_poisson_stream", delta=0.05),
    # Graph(filename) on the R-MAT 20 edge list: device parse + CSR build
    # (silvan_graph_load) against the host loader and the reference's own
    "ingest": dict(kind="ingest", workload="rmat20_directed_ef16_seed2_edge_list", scale=20,
                   edge_factor=16, seed=2, directed=True),
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
    elif cfg["gen"] == "grid":
        pairs = sb.grid(cfg["side"], cfg["delete"], cfg["shortcut"], cfg["seed"])
    else:
        pairs = sb.barabasi_albert(cfg["n"], cfg["m"], cfg["seed"])
    return sb.HostGraph.from_pairs(pairs, cfg["directed"])


def multigraph_sizes():
    """(node count, seed) of the 64 graphs of the multi-graph workload: even
    indices ER with mean degree 8, odd ones BA with 4 edges per node."""
    import math

    import numpy as np
    out = []
    for i in range(64):
        seed = 100 + i
        rng = np.random.default_rng(seed)
        out.append((int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e6))))), seed))
    return out


def multigraph_hosts():
    """The 64 graphs of the multi-graph workload."""
    import silvan_b200 as sb
    out = []
    for i, (n, seed) in enumerate(multigraph_sizes()):
        pairs = sb.erdos_renyi(n, 8.0, seed) if i % 2 == 0 else sb.barabasi_albert(n, 4, seed)
        out.append(sb.HostGraph.from_pairs(pairs, False))
    return out


def multigraph_ref_csrs(lib):
    """The same 64 graphs through the reference harness's generators."""
    return [RefCSR(lib, 1, n, 0, 0, 8.0, 0, seed, False) if i % 2 == 0 else
            RefCSR(lib, 0, n, 4, 0, 0, 0, seed, False)
            for i, (n, seed) in enumerate(multigraph_sizes())]


def job_kwargs(cfg):
    return dict(k=cfg.get("k", 0), alpha=cfg.get("alpha", 2.3),
                alpha_given=cfg.get("alpha_given", False))


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    polled every 5 ms from a thread (reads only), so that even a timed region
    of a few milliseconds gets samples."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.max_mhz = None
        self.stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            dev = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            idx = int(dev.split(",")[self.gpu]) if dev and dev.split(",")[0].isdigit() else self.gpu
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.t = None
        return self

    def _poll(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            self.stop.wait(0.005)

    def __exit__(self, *a):
        self.stop.set()
        if self.t:
            self.t.join(timeout=2)

    def summary(self):
        sm = [m for m, _ in self.samples]
        reasons = set()
        for _, r in self.samples:
            for nm, bit in self.REASONS.items():
                if r & bit:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "NVML, 5 ms"}


def refbench_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsilvan_refbench.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.refbench_graph_new.restype = C.c_void_p
    lib.refbench_graph_new.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                       C.c_double, C.c_uint64, C.c_int]
    lib.refbench_graph_info.argtypes = [C.c_void_p] * 4
    lib.refbench_graph_csr.argtypes = [C.c_void_p] * 5
    lib.refbench_graph_free.argtypes = [C.c_void_p]
    lib.refbench_run.restype = C.c_int
    lib.refbench_run.argtypes = [C.c_uint32, C.c_int] + [C.c_void_p] * 4 + \
        [C.c_double, C.c_double, C.c_uint32, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int] + \
        [C.c_void_p] * 5 + [C.c_uint64]
    lib.refbench_sample.restype = C.c_int
    lib.refbench_sample.argtypes = [C.c_uint32, C.c_int] + [C.c_void_p] * 4 + \
        [C.c_double, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


class RefCSR:
    """A benchmark graph built by the reference harness (no product library):
    the fields reference_run and reference_sample read."""

    def __init__(self, lib, kind, a, b, c, x, y, seed, directed):
        import numpy as np
        h = lib.refbench_graph_new(kind, a, b, c, x, y, seed, int(directed))
        if not h:
            raise RuntimeError("reference harness could not generate the graph")
        n, mo, mi = C.c_uint32(), C.c_uint64(), C.c_uint64()
        lib.refbench_graph_info(h, C.byref(n), C.byref(mo), C.byref(mi))
        self.n, self.directed = n.value, bool(directed)
        self.out_off = np.zeros(self.n + 1, np.uint64)
        self.out_adj = np.zeros(max(1, mo.value), np.uint32)
        self.in_off = np.zeros(self.n + 1, np.uint64) if directed else self.out_off
        self.in_adj = np.zeros(max(1, mi.value), np.uint32) if directed else self.out_adj
        lib.refbench_graph_csr(h, self.out_off.ctypes.data, self.out_adj.ctypes.data,
                               self.in_off.ctypes.data, self.in_adj.ctypes.data)
        lib.refbench_graph_free(h)
        self.out_adj = self.out_adj[:mo.value]
        self.in_adj = self.in_adj[:mi.value] if directed else self.out_adj


def ref_graph(lib, cfg):
    """The workload's graph through the reference harness's copy of the
    generators (the same seeded graphs as make_graph)."""
    if cfg["gen"] == "rmat":
        return RefCSR(lib, 2, cfg["scale"], cfg["edge_factor"], int(cfg["directed"]), 0, 0,
                      cfg["seed"], cfg["directed"])
    if cfg["gen"] == "grid":
        return RefCSR(lib, 3, cfg["side"], 0, 0, cfg["delete"], cfg["shortcut"], cfg["seed"],
                      False)
    return RefCSR(lib, 0, cfg["n"], cfg["m"], 0, 0, 0, cfg["seed"], cfg["directed"])


def csr_checksum(csr):
    """SHA-1 of the CSR rows (offsets as u64, then neighbours as u32; the
    in-rows too for directed graphs): both arms print it for their graph."""
    import hashlib

    import numpy as np
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(csr.out_off, np.uint64).tobytes())
    h.update(np.ascontiguousarray(csr.out_adj, np.uint32).tobytes())
    if csr.directed:
        h.update(np.ascontiguousarray(csr.in_off, np.uint64).tobytes())
        h.update(np.ascontiguousarray(csr.in_adj, np.uint32).tobytes())
    return h.hexdigest()[:16]


def reference_run(lib, csr, cfg, threads):
    tt, p1, p2, vis = C.c_double(), C.c_uint64(), C.c_uint64(), C.c_uint64()
    kw = job_kwargs(cfg)
    rc = lib.refbench_run(csr.n, int(csr.directed), csr.out_off.ctypes.data,
                          csr.out_adj.ctypes.data, csr.in_off.ctypes.data,
                          csr.in_adj.ctypes.data, cfg["eps"], cfg["delta"], kw["k"], kw["alpha"],
                          int(kw["alpha_given"]), 2.0, 1, threads, C.byref(tt), C.byref(p1),
                          C.byref(p2), C.byref(vis), None, 0)
    if rc != 0:
        raise RuntimeError("reference run failed")
    return dict(total_time=tt.value, samples=p1.value + p2.value, vis=vis.value)


def reference_sample(lib, csr, cfg, threads, count):
    """A bounded sample of the reference's per-sample routine (random_path)
    on all threads: samples per second of the parallel region."""
    sec, vis, paths = C.c_double(), C.c_uint64(), C.c_uint64()
    rc = lib.refbench_sample(csr.n, int(csr.directed), csr.out_off.ctypes.data,
                             csr.out_adj.ctypes.data, csr.in_off.ctypes.data,
                             csr.in_adj.ctypes.data, job_kwargs(cfg)["alpha"], threads, count,
                             C.byref(sec), C.byref(vis), C.byref(paths))
    if rc != 0:
        raise RuntimeError("reference sample failed")
    return dict(total_time=sec.value, samples=count, vis=vis.value)


def cpu_reference(lib, csr, cfg, threads):
    """The reference on the workload's graph, bounded to seconds: a whole
    estimation where one takes seconds, else a sample of random_path calls."""
    if cfg.get("cpu_samples"):
        r = reference_sample(lib, csr, cfg, threads, cfg["cpu_samples"])
        what = (f"{cfg['cpu_samples']} calls of the reference's random_path (its own LCG, "
                f"one sampler per OpenMP thread) on the benchmark graph; a whole estimation "
                f"takes minutes on the host")
    else:
        r = reference_run(lib, csr, cfg, threads)
        what = ("one complete estimation of the benchmark graph by the reference's OpenMP "
                "build ('Total time' window)")
    return r, what


def cpu_reference_stats(lib, csr, cfg, threads, runs=3, warmup=1):
    """cpu_reference after `warmup` untimed runs, `runs` times: the median
    rate and the spread, so that the CPU leg of the GPU arm and the
    reference arm measure the same thing the same way."""
    for _ in range(warmup):
        cpu_reference(lib, csr, cfg, threads)
    rates, what = [], ""
    for _ in range(runs):
        r, what = cpu_reference(lib, csr, cfg, threads)
        rates.append(r["samples"] / r["total_time"])
    return {"value": statistics.median(rates), "unit": "paths/s", "cores": threads,
            "kind": "reference", "runs": runs, "min": min(rates), "max": max(rates),
            "sample": f"median of {runs} x ({what}) after {warmup} untimed"}


def combine_replicas(pg, samples, t_dev, e2e_samples, e2e_t, device="cpu"):
    """Replicas on N ranks: total samples over all ranks, time of the slowest
    rank (the same for the end-to-end leg).  `pg` is torch.distributed (or
    None for one rank); every rank takes the same two collectives."""
    import torch
    if pg is None:
        return samples, t_dev, e2e_samples, e2e_t
    vals = torch.tensor([samples, t_dev, e2e_samples, e2e_t], dtype=torch.float64, device=device)
    tot = vals.clone()
    mx = vals.clone()
    pg.all_reduce(tot)
    pg.all_reduce(mx, op=pg.ReduceOp.MAX)
    return tot[0].item(), mx[1].item(), tot[2].item(), mx[3].item()


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
    if cfg["kind"] == "serve":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no request server; the serve line carries its "
                          "CPU baseline"}))
        return 0
    if cfg["kind"] == "ingest":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the ingest line carries the reference loader's time"}))
        return 0
    threads = os.cpu_count() or 1
    holder = {}
    if cfg["kind"] == "multi":
        csrs = multigraph_ref_csrs(lib)
        holder["what"] = "complete estimations of all 64 graphs, one by one"
        checksum = None

        def run():
            return [reference_run(lib, c, cfg, threads) for c in csrs]
    else:
        csr = ref_graph(lib, cfg)
        checksum = csr_checksum(csr)

        def run():
            r, holder["what"] = cpu_reference(lib, csr, cfg, threads)
            return [r]
    for _ in range(args.warmup):
        run()
    runs = [r for _ in range(args.steps) for r in run()]
    what = holder["what"]
    samples = sum(r["samples"] for r in runs)
    t = sum(r["total_time"] for r in runs)
    val = samples / t
    print(json.dumps({
        "impl": "reference", "metric": "paths/sec", "value": val, "unit": "paths/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32/u64/f64", "data": "synthetic",
        "config": dict({"workload": cfg["workload"], "eps": cfg.get("eps"), "delta": cfg["delta"],
                        "form": "reference OpenMP build", "parallelism": "host threads",
                        "csr_sha1_16": checksum},
                       **({} if cfg["kind"] == "multi" else job_kwargs(cfg))),
        "time_to_guarantee_ms": 1000 * t / args.steps,
        "cpu_baseline": {"value": val, "unit": "paths/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} x ({what})"},
        "e2e": {"value": val, "unit": "paths/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))
    return 0


def default_alpha_probe(sb, g, cfg):
    """The same job at the reference's default alpha (2.3, not given): on a
    lattice the multi-path count alpha * W exceeds the per-sample cap, which
    the library reports instead of looping for hours as the reference does."""
    t0 = time.perf_counter()
    try:
        job = sb.Probabilistic(g, cfg["eps"], cfg["delta"], k=cfg.get("k", 0), seed=7)
        res = job.run()
        out = {"status": "ok", "num_samples": res["num_samples"]}
    except sb.SilvanError as e:
        out = {"status": "error", "code": e.code, "message": str(e)}
    out.update(alpha=2.3, seconds=time.perf_counter() - t0)
    return out


def pinned_copy(torch, a):
    import numpy as np
    t = torch.empty(a.shape, dtype={np.uint64: torch.int64, np.uint32: torch.int32,
                                    np.float64: torch.float64}[a.dtype.type], pin_memory=True)
    v = t.numpy().view(a.dtype)
    v[...] = a
    return t, v


def pinned_csr(sb, torch, csr, keep):
    pcsr = sb.CSR(csr.n, csr.directed, *[None] * 5, csr.n_components, csr.diameter)
    for f in ("out_off", "out_adj", "in_off", "in_adj", "cc"):
        t, v = pinned_copy(torch, getattr(csr, f))
        keep.append(t)
        setattr(pcsr, f, v)
    return pcsr


def csr_bytes(csr):
    b = int(csr.out_off.nbytes + csr.out_adj.nbytes + csr.cc.nbytes)
    if csr.directed:
        b += int(csr.in_off.nbytes + csr.in_adj.nbytes)
    return b


def run_multi(args, cfg):
    """64 graphs of uneven size estimated together: every round draws the
    samples of all unfinished jobs in one persistent sampler launch."""
    rank, _, local = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    import torch
    import silvan_b200 as sb
    torch.cuda.set_device(local)
    hosts = multigraph_hosts()
    csrs = [h.csr() for h in hosts]
    graphs = [sb.Graph.from_host(h) for h in hosts]

    def jobs_for(gs, seed):
        return [sb.Probabilistic(g, cfg["eps"], cfg["delta"], seed=seed + i,
                                 block=args.block) for i, g in enumerate(gs)]

    for w in range(args.warmup):
        sb.run_batched(jobs_for(graphs, 10 * w))
    torch.cuda.synchronize()
    times, samples, results = [], 0, []
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            jobs = jobs_for(graphs, 1000 + 100 * s)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = sb.run_batched(jobs)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            samples += sum(r["first_pass_samples"] + r["num_samples"] for r in res)
            results.extend(res)
            del jobs
    t = sum(times)
    # e2e: upload of every CSR from pinned host memory, the batched run and
    # the read-back of every estimate, per step
    keep = []
    pcsrs = [pinned_csr(sb, torch, c, keep) for c in csrs]
    outs = [torch.empty(c.n, dtype=torch.float64, pin_memory=True) for c in csrs]
    e2e_t, e2e_samples = 0.0, 0
    for s in range(0 if args.no_e2e else args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gs = [sb.Graph.upload(pc, with_cc=True) for pc in pcsrs]
        jobs = jobs_for(gs, 5000 + 100 * s)
        res = sb.run_batched(jobs)
        for j, o in zip(jobs, outs):
            j.get_centrality(out=o.numpy())
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t0
        e2e_samples += sum(r["first_pass_samples"] + r["num_samples"] for r in res)
        del jobs, gs
    # the same jobs one after another (each with the whole GPU), for contrast
    seq_t, seq_samples = 0.0, 0
    # largest graph first, so that every job runs on the engine sized for it
    for i in sorted(range(len(graphs)), key=lambda i: -csrs[i].n):
        g = graphs[i]
        job = sb.Probabilistic(g, cfg["eps"], cfg["delta"], seed=1000 + i, block=args.block)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = job.run()
        torch.cuda.synchronize()
        seq_t += time.perf_counter() - t0
        seq_samples += r["first_pass_samples"] + r["num_samples"]
        del job
    cpu = None
    if not args.no_cpu_baseline:
        lib = refbench_lib()
        if lib is not None:
            threads = os.cpu_count() or 1
            rr = [reference_run(lib, c, cfg, threads) for c in csrs]
            cpu = {"value": sum(r["samples"] for r in rr) / sum(r["total_time"] for r in rr),
                   "unit": "paths/s", "cores": threads, "kind": "reference",
                   "seconds": sum(r["total_time"] for r in rr),
                   "sample": "complete estimations of all 64 graphs by the reference's "
                             "OpenMP build, one after another ('Total time' windows summed)"}
    alg = sum(8 * r["vis_edges"] + 24 * r["ball_nodes"] + 4 * r["pred_entries"] for r in results)
    print(json.dumps({
        "metric": "paths/sec", "value": samples / t, "unit": "paths/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32/u64/f64", "data": "synthetic",
        "config": {"workload": cfg["workload"], "graphs": len(graphs),
                   "nodes_total": int(sum(c.n for c in csrs)),
                   "edges_total": int(sum(int(c.out_off[-1]) for c in csrs) // 2),
                   "eps": cfg["eps"], "delta": cfg["delta"], "form": "batched multi-graph",
                   "timing": "host clock around the batched run, device synchronised on both "
                             "sides (the jobs run on the engine's own stream)",
                   "l2": "working set above L2"},
        "time_to_guarantee_ms": 1000 * t / args.steps,
        "one_by_one_ms": 1000 * seq_t, "one_by_one_paths_per_s": seq_samples / seq_t,
        "e2e": {"value": e2e_samples / e2e_t if e2e_t > 0 else None, "unit": "paths/s",
                "h2d_bytes_per_step": sum(csr_bytes(c) for c in csrs),
                "d2h_bytes_per_step": sum(c.n * 8 for c in csrs)},
        "roofline": {"bound": "hbm", "achieved": alg / 1e9 / sum(
                     r["time_sampling_s"] for r in results) if results[0]["time_sampling_s"]
                     else None, "peak": peaks()[0], "unit": "GB/s", "frac": None,
                     "traffic": None, "kernel": "sampler_kernel", "peak_kind": peaks()[1]},
        "cpu_baseline": cpu,
        "gpu_launches": sum(r["kernel_launches"] for r in results),
        "clocks": clk.summary(),
    }))
    return 0


def run_serve(args, cfg):
    """A Poisson stream of estimation requests on fresh graphs, served with
    continuous batching; latency is submission to result."""
    rank, _, local = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    import torch
    import silvan_b200 as sb
    torch.cuda.set_device(local)
    hosts = {}
    for scale in range(10, 21):
        for d in (0, 1):
            hosts[(scale, d)] = sb.HostGraph.from_pairs(
                sb.rmat(scale, 16, 500 + 2 * scale + d, bool(d)), bool(d))
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(args.requests):
        scale = int(rng.integers(10, 21))
        d = int(rng.integers(0, 2))
        eps = float(rng.choice([0.01, 0.005, 0.0025]))
        k = 10 if rng.random() < 0.2 else 0
        if k:
            eps *= args.topk_eps_scale
        reqs.append((scale, d, eps, k, float(rng.exponential(1.0 / args.rate))))
    srv = sb.Server(1 << 20, slots=args.slots)
    try:
        # warm-up: one request per graph class, one after another
        for key, hg in hosts.items():
            srv.wait(srv.submit(hg, 0.01, cfg["delta"], seed=1), 600)
        ids = [None] * len(reqs)
        t_first = time.perf_counter()

        def client():
            t_next = time.perf_counter()
            for i, (scale, d, eps, k, gap) in enumerate(reqs):
                t_next += gap
                dt = t_next - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[i] = srv.submit(hosts[(scale, d)], eps, cfg["delta"], k=k, seed=100 + i)

        with ClockSampler(local) as clk:
            th = threading.Thread(target=client)
            th.start()
            th.join()
            done = [srv.wait(rid, 600) for rid in ids]
            t_end = time.perf_counter()
        st = srv.stats()
    finally:
        srv.close()
    lat = np.array([r["latency_s"] for r in done]) * 1000
    samples = sum(r["first_pass_samples"] + r["num_samples"] for r in done)
    span = t_end - t_first
    p50, p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
    absolute = np.array([q[3] == 0 for q in reqs])
    classes = {}
    for name, mask in (("absolute", absolute), ("top10", ~absolute)):
        if mask.any():
            classes[name] = {"requests": int(mask.sum()),
                             "p50_ms": float(np.percentile(lat[mask], 50)),
                             "p99_ms": float(np.percentile(lat[mask], 99))}
    slo_ms = args.slo_ms
    print(json.dumps({
        "metric": "serve p99 latency", "value": p99, "unit": "ms", "n_gpus": 1,
        "steps": len(reqs), "warmup": len(hosts), "ms_per_step": float(lat.mean()),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32/u64/f64", "data": "synthetic",
        "config": {"workload": cfg["workload"], "requests": len(reqs),
                   "rate_per_s": args.rate, "delta": cfg["delta"],
                   "topk_eps": ("the drawn eps, as the workload states" if args.topk_eps_scale == 1
                                else f"{args.topk_eps_scale:g} x the drawn eps"),
                   "graphs": "22 pre-generated R-MAT graphs (scale 10-20 x directed or not), "
                             "each request uploads and estimates its own copy",
                   "latency": "host clock from submission to the finished result"},
        "p50_ms": p50, "p99_ms": p99, "max_ms": float(lat.max()), "by_mode": classes,
        "slowest": [{"scale": reqs[i][0], "directed": reqs[i][1], "eps": reqs[i][2],
                     "k": reqs[i][3], "ms": float(lat[i]),
                     "queued_ms": 1000 * done[i]["queued_s"],
                     "samples": done[i]["first_pass_samples"] + done[i]["num_samples"]}
                    for i in np.argsort(-lat)[:6]],
        "slo": {"p99_ms": slo_ms, "at_rate_per_s": args.rate, "met": p99 <= slo_ms},
        "paths_per_s": samples / span,
        "e2e": {"value": samples / span, "unit": "paths/s",
                "h2d_bytes_per_step": int(np.mean([csr_bytes(hosts[(r[0], r[1])].csr())
                                                   for r in reqs])),
                "d2h_bytes_per_step": int(np.mean([8 * hosts[(r[0], r[1])].csr().n
                                                   for r in reqs]))},
        "server": {"rounds": st["rounds"], "max_active": st["max_active"],
                   "slots": st["slots"],
                   "thread_s": {k: round(st[k + "_s"], 4) for k in
                                ("admit", "round", "commit", "finish")},
                   "longest_s": {k: round(st[k + "_max_s"], 4) for k in
                                 ("admit", "round", "commit", "finish")}},
        "gpu_launches": int(sum(r["kernel_launches"] for r in done)),
        "clocks": clk.summary(),
    }))
    return 0


def run_ingest(args, cfg):
    """Loading the benchmark graph from its 'u v' text file: the device
    ingest (parse and CSR on the GPU, components and diameter bound on the
    host copy), this library's host loader, and the reference's own loader
    (std::set insertion, silvan/src/Graph.cpp:37-90) once."""
    rank, _, local = dist_env()
    if rank != 0:
        return 0
    import tempfile

    import torch
    import silvan_b200 as sb
    torch.cuda.set_device(local)
    fd, path = tempfile.mkstemp(suffix=".txt")
    os.close(fd)
    try:
        sb.write_edge_list(path, sb.rmat(cfg["scale"], cfg["edge_factor"], cfg["seed"],
                                         cfg["directed"]))
        size = os.path.getsize(path)
        for _ in range(args.warmup):
            del_g = sb.Graph.load(path, cfg["directed"])
            del del_g
        dev, host = [], []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g = sb.Graph.load(path, cfg["directed"])
                torch.cuda.synchronize()
                dev.append(time.perf_counter() - t0)
                del g
        for _ in range(args.steps):
            t0 = time.perf_counter()
            h = sb.HostGraph.load(path, cfg["directed"])
            host.append(time.perf_counter() - t0)
            edges = int(h.info().m)
            del h
        ref_s = None
        if not args.no_cpu_baseline:
            try:
                from oracle.oracle import Ref, ref_available
                if ref_available():
                    t0 = time.perf_counter()
                    rg = Ref().graph(path, cfg["directed"])
                    ref_s = time.perf_counter() - t0
                    del rg
            except Exception:
                ref_s = None
    finally:
        os.unlink(path)
    t = sum(dev) / len(dev)
    print(json.dumps({
        "metric": "edge-list ingest", "value": size / t / 1e6, "unit": "MB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32",
        "data": "synthetic",
        "config": {"workload": cfg["workload"], "file_bytes": size, "edges": edges,
                   "includes": "file read, H2D, parse, CSR, read-back, host components and "
                               "diameter bound"},
        "host_loader_s": sum(host) / len(host),
        "reference_loader_s": ref_s,
        "cpu_baseline": {"value": size / ref_s / 1e6, "unit": "MB/s", "cores": 1,
                         "kind": "reference",
                         "sample": "one Graph(filename, directed) of the reference"}
        if ref_s else None,
        "clocks": clk.summary(),
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
    ap.add_argument("--plain-steps", type=int, default=3,
                    help="plain-form estimations on the first timed steps' seeds, for the "
                         "batched-over-plain ratio (0 = skip)")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests in the stream")
    ap.add_argument("--rate", type=float, default=4.0, help="serve: Poisson arrivals per second")
    ap.add_argument("--slo-ms", type=float, default=2500.0,
                    help="serve: stated p99 objective over all requests")
    ap.add_argument("--topk-eps-scale", type=float, default=1.0,
                    help="serve: top-10 requests use this multiple of the drawn eps as their "
                         "relative eps (1 = the workload as stated)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference_arm(args, cfg)
    if cfg["kind"] == "multi":
        return run_multi(args, cfg)
    if cfg["kind"] == "serve":
        return run_serve(args, cfg)
    if cfg["kind"] == "ingest":
        return run_ingest(args, cfg)

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
        job = sb.Probabilistic(g, cfg["eps"], cfg["delta"], seed=seed, form=args.form,
                               slots=args.slots, block=args.block, **job_kwargs(cfg))
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

    # The plain form (one launch sequence per 11-sample block, as the
    # reference's loop of Probabilistic.cpp:1054-1102 draws them) on the
    # first timed steps' seeds, after the timed region: the batched form's
    # speed-up on identical estimations.
    plain = None
    if args.form == "batched" and args.plain_steps > 0:
        bt, pt, same = 0.0, 0.0, True
        for s in range(min(args.plain_steps, args.steps)):
            job = sb.Probabilistic(g, cfg["eps"], cfg["delta"], seed=seed0 + args.warmup + s,
                                   form="plain", slots=args.slots, **job_kwargs(cfg))
            r = job.run()
            del job
            pt += r["time_device_s"]
            bt += results[s]["time_device_s"]
            same = same and r["num_samples"] == results[s]["num_samples"] and \
                r["vis_edges"] == results[s]["vis_edges"]
        k = min(args.plain_steps, args.steps)
        plain = {"plain_ms_per_estimation": 1000 * pt / k,
                 "batched_ms_per_estimation": 1000 * bt / k,
                 "batched_over_plain": pt / bt if bt > 0 else None, "estimations": k,
                 "same_results": same}

    # e2e through the C-ABI from pinned host buffers: CSR upload, job
    # creation, the run and the read-back of every estimate, per step
    keep = []
    pcsr = pinned_csr(sb, torch, csr, keep)
    est_t = torch.empty(csr.n, dtype=torch.float64, pin_memory=True)
    e2e_t, e2e_samples = 0.0, 0
    h2d = csr_bytes(csr)
    d2h = csr.n * 8
    for s in range(0 if args.no_e2e else args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = sb.Graph.upload(pcsr, with_cc=True)
        job = sb.Probabilistic(g2, cfg["eps"], cfg["delta"], **job_kwargs(cfg),
                               seed=seed0 + 50 + s, form=args.form, slots=args.slots,
                               block=args.block)
        r = job.run()
        job.get_centrality(out=est_t.numpy())
        torch.cuda.synchronize()
        e2e_t += time.perf_counter() - t0
        e2e_samples += r["first_pass_samples"] + r["num_samples"]
        del job, g2

    samples_all, t_max, e2e_s_all, e2e_t_max = combine_replicas(
        pg, samples, t_dev, e2e_samples, e2e_t, device="cuda")
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
        # DRAM bytes per launch: bytes per sample from an ncu capture of the
        # same kernel on this workload (profiles/), times samples per launch
        traffic = None
        tp = os.path.join(ROOT, "profiles", "sampler_traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                tj = json.load(f)
            launches_all = sum(r["sampler_launches"] for r in results)
            if tj.get("workload") == cfg["workload"] and launches_all:
                traffic = tj["dram_bytes_per_sample"] * samples / launches_all
        cpu = None
        if not args.no_cpu_baseline:
            lib = refbench_lib()
            if lib is not None:
                cpu = cpu_reference_stats(lib, csr, cfg, os.cpu_count() or 1)
        line = {
            "metric": "paths/sec", "value": samples_all / t_max, "unit": "paths/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64/f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "n": csr.n, "m": int(csr.out_off[-1]),
                       "csr_sha1_16": csr_checksum(csr),
                       "eps": cfg["eps"], "delta": cfg["delta"], "form": args.form,
                       **job_kwargs(cfg),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "working set above L2 (CSR + per-slot state)",
                       "sampler_block": [r["sampler_block"] for r in results],
                       "sampler_launches_per_step": sum(r["sampler_launches"] for r in results)
                       / args.steps,
                       "wide_levels_shared_per_step": sum(r["assisted_levels"] for r in results)
                       / args.steps,
                       "helper_tiles_per_step": sum(r["helper_tiles"] for r in results)
                       / args.steps},
            "time_to_guarantee_ms": 1000 * t_max / args.steps,
            "samples_per_step": samples_all / max(1, world) / args.steps,
            "samples_drawn_per_step": sum(r["samples_drawn"] for r in results) / args.steps,
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
        if plain is not None:
            line["plain_vs_batched"] = plain
        if cfg.get("alpha_given") and cfg.get("gen") == "grid":
            line["default_alpha_run"] = default_alpha_probe(sb, g, cfg)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
