"""silvan_b200 -- B200-native progressive-sampling betweenness estimation.

Python host side of the library: ctypes bindings of ``include/silvan.h``
mirroring the reference's interface (``Probabilistic(graph, flags).run(k,
delta, err)`` of silvan/include/Probabilistic.h:27-56 and the command line of
silvan/main.cpp).  Every estimate is computed by the CUDA kernels in
``libsilvan_b200.so``; there is no CPU path, and loading fails loudly when the
library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsilvan_b200.so")
CLI_PATH = os.path.join(PKG, "bin", "silvan")

OK = 0
E_BADARG, E_IO, E_PARSE, E_OOM, E_CUDA = -1, -2, -3, -4, -5
E_OVERFLOW, E_NP_CAP, E_TIMEOUT, E_CAPACITY, E_STATE, E_NOGPU = -6, -7, -8, -9, -10, -11
FORM_PLAIN, FORM_BATCHED = 0, 1
BACKTRACK_REFERENCE, BACKTRACK_SIGMA_WEIGHTED = 0, 1
TRIALS = 25

# Every function declared in include/silvan.h.
EXPORTS = [
    "silvan_params_default", "silvan_graph_load", "silvan_graph_upload", "silvan_graph_info",
    "silvan_graph_csr", "silvan_graph_destroy", "silvan_host_graph_load",
    "silvan_host_graph_from_pairs", "silvan_host_graph_info", "silvan_host_graph_csr",
    "silvan_host_graph_destroy", "silvan_graph_from_host", "silvan_job_create",
    "silvan_job_run", "silvan_read_estimates", "silvan_read_topk", "silvan_read_counters",
    "silvan_job_destroy", "silvan_run_rounds", "silvan_replay_samples", "silvan_generate",
    "silvan_graph_from_pairs", "silvan_last_error", "silvan_version", "silvan_job_result",
    "silvan_jobs_run_batched", "silvan_server_create", "silvan_server_submit",
    "silvan_server_poll", "silvan_server_wait", "silvan_server_estimates", "silvan_server_stats",
    "silvan_server_destroy", "silvan_replay_samples_noalloc", "silvan_exact_betweenness",
]

REQ_QUEUED, REQ_RUNNING, REQ_DONE = 1, 2, 3


class SilvanError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_components", C.c_uint32), ("m", C.c_uint64),
                ("diameter", C.c_uint32), ("directed", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("eps", C.c_double), ("delta", C.c_double), ("k", C.c_uint32),
                ("m_hat", C.c_int32), ("alpha", C.c_double), ("alpha_given", C.c_int32),
                ("form", C.c_int32), ("a", C.c_double), ("seed", C.c_uint64),
                ("verbose", C.c_double), ("np_cap", C.c_uint32), ("slots", C.c_uint32),
                ("threads", C.c_uint32), ("block", C.c_uint32),
                ("backtrack", C.c_uint32), ("assist_items", C.c_uint32),
                ("wait_polls", C.c_uint32), ("serial_checks", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("first_pass_samples", C.c_uint64), ("num_samples", C.c_uint64),
                ("vis_edges", C.c_uint64), ("void_samples", C.c_uint64),
                ("backtracked_paths", C.c_uint64), ("tau", C.c_uint32),
                ("diameter", C.c_uint32), ("iteration_index", C.c_int32),
                ("num_partitions", C.c_int32), ("stop_reason", C.c_int32),
                ("union_sample", C.c_uint32), ("numresults_topk", C.c_uint32),
                ("checks", C.c_uint32), ("omega", C.c_double),
                ("first_stopping_samples", C.c_double), ("last_stopping_samples", C.c_double),
                ("alpha_sp_sampling", C.c_double), ("eps_stop", C.c_double),
                ("eps_final_topk", C.c_double), ("sup_bcest", C.c_double),
                ("sup_emp_wimpy_var", C.c_double), ("max_num_samples", C.c_double),
                ("time_total_s", C.c_double), ("time_first_pass_s", C.c_double),
                ("time_sampling_s", C.c_double), ("time_apply_s", C.c_double),
                ("time_device_s", C.c_double), ("ball_nodes", C.c_uint64),
                ("pred_entries", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("sampler_launches", C.c_uint32), ("sampler_block", C.c_uint32),
                ("samples_drawn", C.c_uint64), ("assisted_levels", C.c_uint32),
                ("overlapped_checks", C.c_uint32), ("helper_tiles", C.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Status(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("void_samples", C.c_uint64), ("vis_edges", C.c_uint64),
                ("backtracked_paths", C.c_uint64), ("pass_", C.c_int32), ("done", C.c_int32)]


_lib = None


def load(path: str = LIB_PATH):
    """Loads the native library (building nothing; see silvan_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m silvan_b200.build`")
    lib = C.CDLL(path)
    P = C.c_void_p
    sig = {
        "silvan_params_default": (None, [P]),
        "silvan_graph_load": (C.c_int, [C.c_char_p, C.c_int, P]),
        "silvan_graph_upload": (C.c_int, [C.c_uint32, C.c_int, P, P, P, P, P, C.c_uint32,
                                          C.c_uint32, P]),
        "silvan_graph_info": (C.c_int, [P, P]),
        "silvan_graph_csr": (C.c_int, [P, P, P, P, P, P]),
        "silvan_graph_destroy": (C.c_int, [P]),
        "silvan_host_graph_load": (C.c_int, [C.c_char_p, C.c_int, P]),
        "silvan_host_graph_from_pairs": (C.c_int, [P, C.c_uint64, C.c_int, P]),
        "silvan_host_graph_info": (C.c_int, [P, P]),
        "silvan_host_graph_csr": (C.c_int, [P, P, P, P, P, P]),
        "silvan_host_graph_destroy": (C.c_int, [P]),
        "silvan_graph_from_host": (C.c_int, [P, P]),
        "silvan_graph_from_pairs": (C.c_int, [P, C.c_uint64, C.c_int, P]),
        "silvan_job_create": (C.c_int, [P, P, P]),
        "silvan_job_run": (C.c_int, [P, P, P]),
        "silvan_run_rounds": (C.c_int, [P, C.c_uint32, P, P]),
        "silvan_job_result": (C.c_int, [P, P]),
        "silvan_jobs_run_batched": (C.c_int, [P, C.c_uint32, C.c_uint64, P, P]),
        "silvan_read_estimates": (C.c_int, [P, P, C.c_uint32]),
        "silvan_read_topk": (C.c_int, [P, P, P, C.c_uint32, P]),
        "silvan_read_counters": (C.c_int, [P, P, P, P, P]),
        "silvan_job_destroy": (C.c_int, [P]),
        "silvan_replay_samples": (C.c_int, [P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double,
                                            C.c_uint32, P, P, P, P, P, P, P, C.c_uint64, P]),
        "silvan_generate": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                      C.c_double, C.c_uint64, P, C.c_uint64, P]),
        "silvan_server_create": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, P]),
        "silvan_server_submit": (C.c_int, [P, P, P, P]),
        "silvan_server_poll": (C.c_int, [P, C.c_uint64, P, P, P, P]),
        "silvan_server_wait": (C.c_int, [P, C.c_uint64, C.c_double]),
        "silvan_server_estimates": (C.c_int, [P, C.c_uint64, P, C.c_uint32, P, P, C.c_uint32, P]),
        "silvan_server_stats": (C.c_int, [P, P]),
        "silvan_server_destroy": (C.c_int, [P]),
        "silvan_replay_samples_noalloc": (C.c_int, [P, C.c_uint64, C.c_uint32, C.c_uint32,
                                                    C.c_double, C.c_uint32, P, P, P, P, P,
                                                    C.c_uint64, P, P]),
        "silvan_last_error": (C.c_char_p, []),
        "silvan_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc != OK:
        raise SilvanError(rc, load().silvan_last_error().decode())


# ---- synthetic workloads ----------------------------------------------------------

GEN_BA, GEN_ER, GEN_RMAT, GEN_GRID = 0, 1, 2, 3


def generate(kind, a=0, b=0, c=0, x=0.0, y=0.0, seed=1):
    """Edge pairs (uint32 array of shape (E, 2)) of a synthetic workload."""
    lib = load()
    cnt = C.c_uint64(0)
    rc = lib.silvan_generate(kind, a, b, c, x, y, seed, None, 0, C.byref(cnt))
    if rc not in (OK, E_CAPACITY):
        _check(rc)
    pairs = np.zeros((max(cnt.value, 1), 2), np.uint32)
    _check(lib.silvan_generate(kind, a, b, c, x, y, seed, _p(pairs), cnt.value, C.byref(cnt)))
    return pairs[:cnt.value]


def barabasi_albert(n, m, seed):
    return generate(GEN_BA, n, m, seed=seed)


def erdos_renyi(n, mean_degree, seed):
    return generate(GEN_ER, n, x=mean_degree, seed=seed)


def rmat(scale, edge_factor, seed, directed):
    return generate(GEN_RMAT, scale, edge_factor, int(directed), seed=seed)


def grid(side, delete_frac, shortcut_frac, seed):
    return generate(GEN_GRID, side, x=delete_frac, y=shortcut_frac, seed=seed)


def write_edge_list(path, pairs):
    with open(path, "w") as f:
        f.write("".join(f"{u} {v}\n" for u, v in pairs.tolist()))


# ---- graphs -------------------------------------------------------------------------


@dataclass
class CSR:
    n: int
    directed: bool
    out_off: np.ndarray
    out_adj: np.ndarray
    in_off: np.ndarray
    in_adj: np.ndarray
    cc: np.ndarray
    n_components: int
    diameter: int


class HostGraph:
    """Host-only ingest (Graph(filename, directed) + compute_cc +
    estimate_diameter of silvan/src/Graph.cpp) -- no device needed."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def load(cls, path, directed=False):
        h = C.c_void_p()
        _check(load().silvan_host_graph_load(str(path).encode(), int(directed), C.byref(h)))
        return cls(h)

    @classmethod
    def from_pairs(cls, pairs, directed=False):
        pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
        h = C.c_void_p()
        _check(load().silvan_host_graph_from_pairs(_p(pairs), len(pairs), int(directed),
                                                   C.byref(h)))
        return cls(h)

    def info(self):
        i = GraphInfo()
        _check(load().silvan_host_graph_info(self.h, C.byref(i)))
        return i

    def csr(self) -> CSR:
        i = self.info()
        n = i.n
        oo = np.zeros(n + 1, np.uint64)
        io = np.zeros(n + 1, np.uint64)
        load().silvan_host_graph_csr(self.h, _p(oo), None, _p(io), None, None)
        oa = np.zeros(max(int(oo[-1]), 1), np.uint32)
        ia = np.zeros(max(int(io[-1]), 1), np.uint32)
        cc = np.zeros(n, np.uint32)
        _check(load().silvan_host_graph_csr(self.h, _p(oo), _p(oa), _p(io), _p(ia), _p(cc)))
        return CSR(n, bool(i.directed), oo, oa[:int(oo[-1])], io, ia[:int(io[-1])], cc,
                   i.n_components, i.diameter)

    def __del__(self):
        try:
            if self.h:
                load().silvan_host_graph_destroy(self.h)
        except Exception:
            pass


class Graph:
    """A graph resident on the device (CSR + component ids)."""

    def __init__(self, handle):
        self.h = handle
        self._info = self.info()

    @classmethod
    def load(cls, path, directed=False):
        h = C.c_void_p()
        _check(load().silvan_graph_load(str(path).encode(), int(directed), C.byref(h)))
        return cls(h)

    @classmethod
    def from_pairs(cls, pairs, directed=False):
        pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
        h = C.c_void_p()
        _check(load().silvan_graph_from_pairs(_p(pairs), len(pairs), int(directed), C.byref(h)))
        return cls(h)

    @classmethod
    def from_host(cls, hg: HostGraph):
        h = C.c_void_p()
        _check(load().silvan_graph_from_host(hg.h, C.byref(h)))
        return cls(h)

    @classmethod
    def upload(cls, csr: CSR, with_cc=True):
        h = C.c_void_p()
        _check(load().silvan_graph_upload(
            csr.n, int(csr.directed), _p(csr.out_off), _p(csr.out_adj),
            _p(csr.in_off) if csr.directed else None, _p(csr.in_adj) if csr.directed else None,
            _p(csr.cc) if with_cc else None, csr.n_components, csr.diameter, C.byref(h)))
        return cls(h)

    def info(self):
        i = GraphInfo()
        _check(load().silvan_graph_info(self.h, C.byref(i)))
        return i

    @property
    def n(self):
        return self._info.n

    @property
    def diameter(self):
        return self._info.diameter

    def csr(self) -> CSR:
        i = self._info
        n = i.n
        oo = np.zeros(n + 1, np.uint64)
        io = np.zeros(n + 1, np.uint64)
        load().silvan_graph_csr(self.h, _p(oo), None, _p(io), None, None)
        oa = np.zeros(max(int(oo[-1]), 1), np.uint32)
        ia = np.zeros(max(int(io[-1]), 1), np.uint32)
        cc = np.zeros(n, np.uint32)
        _check(load().silvan_graph_csr(self.h, _p(oo), _p(oa), _p(io), _p(ia), _p(cc)))
        return CSR(n, bool(i.directed), oo, oa[:int(oo[-1])], io, ia[:int(io[-1])], cc,
                   i.n_components, i.diameter)

    def exact_betweenness(self):
        """Exact normalised betweenness of every node (Brandes on the device)."""
        out = np.zeros(self.n, np.float64)
        _check(load().silvan_exact_betweenness(self.h, _p(out), self.n))
        return out

    def replay(self, seed, first, count, alpha, np_cap=0):
        """Per-sample output of the device sampler for samples
        [first, first+count) (Sp_sampler::random_path, silvan/src/Sp_sampler.cpp:41)."""
        lib = load()
        pl = np.zeros(count, np.int32)
        npth = np.zeros(count, np.int32)
        vis = np.zeros(count, np.uint64)
        nent = np.zeros(count, np.uint32)
        st = np.zeros(count, np.int32)
        tot = C.c_uint64(0)
        cap = max(1 << 16, count * 32)
        while True:
            node = np.zeros(cap, np.uint32)
            cnt = np.zeros(cap, np.int32)
            rc = lib.silvan_replay_samples(self.h, seed, first, count, alpha, np_cap, _p(pl),
                                           _p(npth), _p(vis), _p(nent), _p(st), _p(node),
                                           _p(cnt), cap, C.byref(tot))
            if rc == E_CAPACITY and tot.value > cap:
                cap = int(tot.value)
                continue
            _check(rc)
            break
        e = int(tot.value)
        off = np.zeros(count + 1, np.int64)
        off[1:] = np.cumsum(nent.astype(np.int64))
        return dict(path_length=pl, num_paths=npth, vis_edges=vis, offsets=off,
                    nodes=node[:e].copy(), counts=cnt[:e].copy(), status=st)

    def __del__(self):
        try:
            if self.h:
                load().silvan_graph_destroy(self.h)
        except Exception:
            pass


class Probabilistic:
    """Mirror of the reference's estimator object (silvan/include/
    Probabilistic.h:27-56): construct with the graph and the binary's flags,
    call run(), read the centralities.

    Beyond the binary's flags: `seed` (the Philox key of the sample stream),
    `form` ("batched" or "plain"), `np_cap` (paths per sample), `slots` and
    `block` (sampler slots and threads per slot; 0 = chosen by the engine),
    `threads` (the divisor of union_sample; 1 = parity mode), `backtrack`
    ("reference", or "sigma" for path-count-weighted predecessors),
    `assist_items` (BFS levels of at least this many adjacency entries are
    expanded by several sampler CTAs; 0 = 128 x the CTA size while samples
    remain, 64 x once all are taken, 0xFFFFFFFF =
    never) and `wait_polls` (polls after which a wait between CTAs that
    share a level gives up and the job fails with E_TIMEOUT; 0 = default,
    0xFFFFFFFF = no polls, a hook for tests of that path) and
    `serial_checks` (evaluate each stopping-rule check before committing
    later samples, instead of overlapping the two).  Only `seed`,
    `backtrack` and, in top-k mode, `threads` change the results."""

    def __init__(self, graph: Graph, eps, delta, k=0, alpha=2.3, alpha_given=False, a=2.0,
                 m_hat=True, seed=42, form="batched", verbose=0.0, np_cap=0, slots=0,
                 threads=1, block=0, backtrack="reference", assist_items=0, wait_polls=0,
                 serial_checks=False):
        lib = load()
        p = Params()
        lib.silvan_params_default(C.byref(p))
        p.eps, p.delta, p.k = eps, delta, k
        p.alpha, p.alpha_given, p.a = alpha, int(alpha_given), a
        p.m_hat, p.seed, p.verbose = int(m_hat), seed, verbose
        p.form = FORM_PLAIN if form == "plain" else FORM_BATCHED
        p.np_cap, p.slots, p.threads, p.block = np_cap, slots, threads, block
        p.assist_items = assist_items
        p.wait_polls = wait_polls
        p.serial_checks = int(serial_checks)
        p.backtrack = {"reference": BACKTRACK_REFERENCE,
                       "sigma": BACKTRACK_SIGMA_WEIGHTED}[backtrack]
        self.graph = graph
        self.params = p
        h = C.c_void_p()
        _check(lib.silvan_job_create(graph.h, C.byref(p), C.byref(h)))
        self.h = h
        self.result = None

    def run(self, log=None):
        """Probabilistic::run: returns the result fields as a dict.  `log` may
        be an open file to receive the reference's status lines."""
        lib = load()
        res = Result()
        fp = None
        if log is not None:
            libc = C.CDLL(None)
            libc.fdopen.restype = C.c_void_p
            libc.fdopen.argtypes = [C.c_int, C.c_char_p]
            log.flush()
            fp = libc.fdopen(os.dup(log.fileno()), b"w")
        try:
            _check(lib.silvan_job_run(self.h, C.byref(res), fp))
        finally:
            if fp:
                libc.fflush(C.c_void_p(fp))
                libc.fclose.argtypes = [C.c_void_p]
                libc.fclose(fp)
        self.result = res.as_dict()
        return self.result

    def step(self, rounds=1):
        """Runs at most `rounds` rounds of the job's own schedule (silvan_run_rounds)."""
        st = Status()
        _check(load().silvan_run_rounds(self.h, rounds, C.byref(st), None))
        d = {f: getattr(st, f) for f, _ in Status._fields_}
        if st.done:
            res = Result()
            _check(load().silvan_job_result(self.h, C.byref(res)))
            self.result = res.as_dict()
        return d

    def get_centrality(self, out=None):
        """approx[v] / num_samples for every node (into `out` when given)."""
        n = self.graph.n
        if out is None:
            out = np.zeros(n, np.float64)
        _check(load().silvan_read_estimates(self.h, _p(out), n))
        return out

    def counters(self):
        n = self.graph.n
        approx = np.zeros(n, np.float64)
        wimpy = np.zeros(n, np.float64)
        mcrade = np.zeros(n * TRIALS, np.int64)
        part = np.zeros(n, np.int32)
        _check(load().silvan_read_counters(self.h, _p(approx), _p(wimpy), _p(mcrade), _p(part)))
        return dict(approx=approx, wimpy=wimpy, mcrade=mcrade.reshape(n, TRIALS),
                    partition_index=part)

    def topk(self):
        cap = max(1, (self.result or {}).get("numresults_topk", 0) + 1)
        nodes = np.zeros(cap, np.uint32)
        vals = np.zeros(cap, np.float64)
        cnt = C.c_uint32(0)
        _check(load().silvan_read_topk(self.h, _p(nodes), _p(vals), cap, C.byref(cnt)))
        return nodes[:cnt.value], vals[:cnt.value]

    def __del__(self):
        try:
            if getattr(self, "h", None):
                load().silvan_job_destroy(self.h)
        except Exception:
            pass


def run_batched(jobs, mem_budget=0):
    """Runs several jobs (same or different graphs) to completion with one
    persistent sampler launch per round for all unfinished jobs; returns each
    job's result dict (silvan_jobs_run_batched)."""
    lib = load()
    n = len(jobs)
    handles = (C.c_void_p * n)(*[j.h.value if isinstance(j.h, C.c_void_p) else j.h for j in jobs])
    res = (Result * n)()
    _check(lib.silvan_jobs_run_batched(handles, n, mem_budget, res, None))
    out = []
    for j, r in zip(jobs, res):
        j.result = r.as_dict()
        out.append(j.result)
    return out


class ServerStats(C.Structure):
    _fields_ = [("rounds", C.c_uint64), ("samples", C.c_uint64), ("max_active", C.c_uint64),
                ("queued", C.c_uint64), ("active", C.c_uint64), ("bytes_in_use", C.c_uint64),
                ("budget", C.c_uint64), ("slots", C.c_uint32), ("pad", C.c_uint32),
                ("admit_s", C.c_double), ("round_s", C.c_double), ("commit_s", C.c_double),
                ("finish_s", C.c_double), ("admit_max_s", C.c_double),
                ("round_max_s", C.c_double), ("commit_max_s", C.c_double),
                ("finish_max_s", C.c_double)]


class Server:
    """Estimation server with continuous batching (silvan_server_*): requests
    on graphs of different sizes are admitted by device-memory budget and
    served together, one persistent sampler launch per round."""

    def __init__(self, n_max, budget=0, slots=0):
        h = C.c_void_p()
        _check(load().silvan_server_create(n_max, budget, slots, C.byref(h)))
        self.h = h

    def submit(self, hg: HostGraph, eps, delta, k=0, alpha=2.3, alpha_given=False, a=2.0,
               m_hat=True, seed=42, np_cap=0):
        lib = load()
        p = Params()
        lib.silvan_params_default(C.byref(p))
        p.eps, p.delta, p.k = eps, delta, k
        p.alpha, p.alpha_given, p.a = alpha, int(alpha_given), a
        p.m_hat, p.seed, p.np_cap = int(m_hat), seed, np_cap
        rid = C.c_uint64()
        _check(lib.silvan_server_submit(self.h, hg.h, C.byref(p), C.byref(rid)))
        return rid.value

    def poll(self, rid):
        st = C.c_int32()
        res = Result()
        lat = C.c_double()
        qd = C.c_double()
        _check(load().silvan_server_poll(self.h, rid, C.byref(st), C.byref(res), C.byref(lat),
                                         C.byref(qd)))
        if st.value == REQ_DONE:
            return st.value, dict(res.as_dict(), latency_s=lat.value, queued_s=qd.value)
        return st.value, None

    def wait(self, rid, timeout_s=600.0):
        _check(load().silvan_server_wait(self.h, rid, timeout_s))
        return self.poll(rid)[1]

    def estimates(self, rid, n):
        out = np.zeros(n, np.float64)
        _check(load().silvan_server_estimates(self.h, rid, _p(out), n, None, None, 0, None))
        return out

    def stats(self):
        s = ServerStats()
        _check(load().silvan_server_stats(self.h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            load().silvan_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
