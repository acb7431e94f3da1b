"""Test infrastructure (oracle) -- never imported by the product.

ctypes bindings for the two CPU oracles built by ``oracle/Makefile``:

* ``Port``  -- ``_ref/liboracle.so``: the project's own single-threaded
  restatement of SILVAN's estimator (silvan_oracle.cpp) in parity mode.
* ``Ref``   -- ``_ref/libsilvan_ref.so``: the reference's own sources
  (silvan/src/*.cpp, unmodified) linked with the Philox stream and a small
  harness.  Only present where the reference sources were available at build
  time; the built library travels with the working tree.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_SO = os.path.join(REF_DIR, "liboracle.so")
REF_SO = os.path.join(REF_DIR, "libsilvan_ref.so")
REF_BIN = os.path.join(REF_DIR, "silvan")

T = 25  # Monte Carlo trials (silvan/include/Probabilistic.h:89)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RunResult(C.Structure):
    """Mirror of ``Result`` in silvan_oracle.cpp."""

    _fields_ = [
        ("graph_diameter", C.c_uint32),
        ("tau", C.c_uint32),
        ("first_pass_samples", C.c_uint64),
        ("num_samples", C.c_uint64),
        ("vis_edges", C.c_uint64),
        ("iteration_index", C.c_int32),
        ("num_partitions", C.c_int32),
        ("omega", C.c_double),
        ("first_stopping_samples", C.c_double),
        ("last_stopping_samples", C.c_double),
        ("alpha_sp_sampling", C.c_double),
        ("sup_bcest", C.c_double),
        ("sup_emp_wimpy_var", C.c_double),
        ("eps_final_topk", C.c_double),
        ("eps_stop", C.c_double),
        ("numresults_topk", C.c_uint32),
        ("union_sample", C.c_uint32),
        ("stop_reason", C.c_int32),
        ("zero_modulus", C.c_int32),
        ("checks", C.c_uint64),
    ]


class RefRunResult(C.Structure):
    """Mirror of ``RefRunResult`` in ref_harness.cpp."""

    _fields_ = [
        ("n", C.c_uint32),
        ("graph_diameter", C.c_uint32),
        ("num_samples", C.c_uint64),
        ("n_pairs", C.c_uint64),
        ("vis_edges", C.c_uint64),
        ("first_pass_samples", C.c_uint64),
        ("iteration_index", C.c_int32),
        ("num_partitions", C.c_int32),
        ("omega", C.c_double),
        ("first_stopping_samples", C.c_double),
        ("last_stopping_samples", C.c_double),
        ("alpha_sp_sampling", C.c_double),
        ("sup_bcest", C.c_double),
        ("sup_emp_wimpy_var", C.c_double),
        ("eps_final_topk", C.c_double),
        ("numresults_topk", C.c_uint32),
        ("union_sample", C.c_uint32),
        ("zero_modulus", C.c_int32),
        ("pad", C.c_int32),
    ]


@dataclass
class Replay:
    """Per-sample records of a replay: path_length, num_paths, vis_edges and
    the (node, count) path map of every sample (``offsets`` into nodes)."""

    path_length: np.ndarray
    num_paths: np.ndarray
    vis_edges: np.ndarray
    offsets: np.ndarray
    nodes: np.ndarray
    counts: np.ndarray
    zero_modulus: bool

    def sample(self, i):
        a, b = self.offsets[i], self.offsets[i + 1]
        return list(zip(self.nodes[a:b].tolist(), self.counts[a:b].tolist()))


def _replay(fn, handle, seed, first, count, alpha, cap=None):
    if cap is None:
        cap = max(1 << 16, count * 64)
    while True:
        pl = np.zeros(count, np.int32)
        npth = np.zeros(count, np.int32)
        vis = np.zeros(count, np.uint64)
        nent = np.zeros(count, np.uint32)
        node = np.zeros(cap, np.uint32)
        cnt = np.zeros(cap, np.int32)
        r = fn(handle, C.c_uint64(seed), C.c_uint32(first), C.c_uint32(count), C.c_double(alpha),
               _p(pl), _p(npth), _p(vis), _p(nent), _p(node), _p(cnt), C.c_uint64(cap))
        if r == -1:
            cap *= 4
            continue
        e = int(nent.sum())
        off = np.zeros(count + 1, np.int64)
        off[1:] = np.cumsum(nent.astype(np.int64))
        return Replay(pl, npth, vis, off, node[:e].copy(), cnt[:e].copy(), r == -2)


class Port:
    """The project's own CPU restatement (parity mode)."""

    def __init__(self, path=PORT_SO):
        lib = C.CDLL(path)
        lib.orc_graph_new.restype = C.c_void_p
        lib.orc_graph_new.argtypes = [C.c_uint32, C.c_int] + [C.c_void_p] * 5
        lib.orc_graph_free.argtypes = [C.c_void_p]
        lib.orc_replay.restype = C.c_int64
        lib.orc_replay.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double] + \
            [C.c_void_p] * 6 + [C.c_uint64]
        lib.orc_run.restype = C.c_int
        lib.orc_run.argtypes = [C.c_void_p, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                                C.c_double, C.c_int, C.c_double, C.c_int, C.c_uint64,
                                C.c_uint32, C.c_int, C.c_void_p]
        lib.orc_result_size.restype = C.c_uint64
        for f in ("orc_run_arrays", "orc_run_ranking", "orc_run_sp_lengths", "orc_run_partitions"):
            getattr(lib, f).restype = None
        lib.orc_brandes.restype = None
        lib.orc_brandes.argtypes = [C.c_void_p, C.c_void_p]
        assert lib.orc_result_size() == C.sizeof(RunResult)
        self.lib = lib

    def graph(self, n, directed, out_off, out_adj, in_off, in_adj, cc):
        out_off = np.ascontiguousarray(out_off, np.uint64)
        out_adj = np.ascontiguousarray(out_adj, np.uint32)
        in_off = np.ascontiguousarray(in_off if directed else out_off, np.uint64)
        in_adj = np.ascontiguousarray(in_adj if directed else out_adj, np.uint32)
        cc = np.ascontiguousarray(cc, np.uint32)
        h = self.lib.orc_graph_new(n, int(directed), _p(out_off), _p(out_adj), _p(in_off),
                                   _p(in_adj), _p(cc))
        return PortGraph(self, h, n)


class PortGraph:
    def __init__(self, port, h, n):
        self.port, self.h, self.n = port, h, n

    def __del__(self):
        try:
            self.port.lib.orc_graph_free(self.h)
        except Exception:
            pass

    def replay(self, seed, first, count, alpha):
        return _replay(self.port.lib.orc_replay, self.h, seed, first, count, alpha)

    def brandes(self):
        """Exact normalised betweenness of every node (the ground truth)."""
        out = np.zeros(self.n, np.float64)
        self.port.lib.orc_brandes(self.h, _p(out))
        return out

    def run(self, diameter, eps, delta, k=0, alpha=2.3, alpha_given=False, a=2.0, mhat=True,
            seed=42, threads=1, weighted=False):
        res = RunResult()
        lib = self.port.lib
        lib.orc_run(self.h, diameter, eps, delta, k, alpha, int(alpha_given), a, int(mhat), seed,
                    threads, int(weighted), C.byref(res))
        n = self.n
        out = {f: getattr(res, f) for f, _ in RunResult._fields_}
        approx = np.zeros(n, np.float64)
        wimpy = np.zeros(n, np.float64)
        mcrade = np.zeros(n * T, np.int64)
        part = np.zeros(n, np.int32)
        lib.orc_run_arrays(_p(approx), _p(wimpy), _p(mcrade), _p(part))
        rk_el = np.zeros(res.union_sample, np.uint32)
        rk_val = np.zeros(res.union_sample, np.float64)
        lib.orc_run_ranking(_p(rk_el), _p(rk_val))
        spl = np.zeros(diameter + 1, np.uint64)
        lib.orc_run_sp_lengths(_p(spl))
        pe = np.zeros(max(res.num_partitions, 1), np.float64)
        pid = np.zeros(max(res.num_partitions, 1), np.int32)
        lib.orc_run_partitions(_p(pe), _p(pid))
        out.update(approx=approx, wimpy=wimpy, mcrade=mcrade.reshape(n, T), partition_index=part,
                   ranking_elements=rk_el, ranking_values=rk_val, sp_lengths=spl,
                   epsilon_partition=pe[:res.num_partitions],
                   partition_ids=pid[:res.num_partitions])
        return out


def ref_available():
    return os.path.exists(REF_SO)


class Ref:
    """The reference's own sources with the Philox stream (see module doc)."""

    def __init__(self, path=REF_SO):
        lib = C.CDLL(path)
        lib.ref_graph_load.restype = C.c_void_p
        lib.ref_graph_load.argtypes = [C.c_char_p, C.c_int]
        lib.ref_graph_free.argtypes = [C.c_void_p]
        lib.ref_graph_nn.restype = C.c_uint32
        lib.ref_graph_nn.argtypes = [C.c_void_p]
        lib.ref_graph_ne.restype = C.c_uint64
        lib.ref_graph_ne.argtypes = [C.c_void_p]
        lib.ref_graph_csr.argtypes = [C.c_void_p] * 5
        lib.ref_graph_diameter.restype = C.c_uint32
        lib.ref_graph_diameter.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_replay.restype = C.c_int64
        lib.ref_replay.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double] + \
            [C.c_void_p] * 6 + [C.c_uint64]
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_double, C.c_uint32,
                                C.c_double, C.c_int, C.c_double, C.c_int, C.c_uint64, C.c_char_p,
                                C.c_double, C.c_void_p]
        lib.ref_last_stdout.restype = C.c_char_p
        self.lib = lib

    def graph(self, path, directed):
        return RefGraph(self, self.lib.ref_graph_load(path.encode(), int(directed)), directed)

    def run(self, path, directed, eps, delta, k=0, alpha=2.3, alpha_given=False, a=2.0, mhat=True,
            seed=42, output_file="", verbose=0.0):
        res = RefRunResult()
        lib = self.lib
        lib.ref_run(path.encode(), int(directed), eps, delta, k, alpha, int(alpha_given), a,
                    int(mhat), seed, output_file.encode(), verbose, C.byref(res))
        out = {f: getattr(res, f) for f, _ in RefRunResult._fields_}
        n = res.n
        approx = np.zeros(n, np.float64)
        wimpy = np.zeros(n, np.float64)
        mcrade = np.zeros(n * T, np.int64)
        part = np.zeros(n, np.int32)
        lib.ref_run_arrays(_p(approx), _p(wimpy), _p(mcrade), _p(part))
        rk_el = np.zeros(res.union_sample, np.uint32)
        rk_val = np.zeros(res.union_sample, np.float64)
        lib.ref_run_ranking(_p(rk_el), _p(rk_val))
        spl = np.zeros(res.graph_diameter + 1, np.uint64)
        lib.ref_run_sp_lengths(_p(spl))
        pe = np.zeros(max(res.num_partitions, 1), np.float64)
        pid = np.zeros(max(res.num_partitions, 1), np.int32)
        lib.ref_run_partitions(_p(pe), _p(pid))
        out.update(approx=approx, wimpy=wimpy, mcrade=mcrade.reshape(n, T), partition_index=part,
                   ranking_elements=rk_el, ranking_values=rk_val, sp_lengths=spl,
                   epsilon_partition=pe[:res.num_partitions],
                   partition_ids=pid[:res.num_partitions],
                   stdout=lib.ref_last_stdout().decode())
        return out


class RefGraph:
    def __init__(self, ref, h, directed):
        self.ref, self.h, self.directed = ref, h, directed
        self.n = ref.lib.ref_graph_nn(h)
        self.m = ref.lib.ref_graph_ne(h)

    def __del__(self):
        try:
            self.ref.lib.ref_graph_free(self.h)
        except Exception:
            pass

    def csr(self):
        n, m = self.n, self.m
        out_off = np.zeros(n + 1, np.uint64)
        out_adj = np.zeros(max(m, 1), np.uint32)
        in_off = np.zeros(n + 1, np.uint64)
        in_adj = np.zeros(max(m, 1), np.uint32)
        self.ref.lib.ref_graph_csr(self.h, _p(out_off), _p(out_adj), _p(in_off), _p(in_adj))
        return out_off, out_adj[:m], in_off, in_adj[:int(in_off[-1])]

    def diameter(self):
        cc = np.zeros(self.n, np.uint32)
        nc = np.zeros(1, np.uint32)
        d = self.ref.lib.ref_graph_diameter(self.h, _p(cc), _p(nc))
        return int(d), cc, int(nc[0])

    def replay(self, seed, first, count, alpha):
        return _replay(self.ref.lib.ref_replay, self.h, seed, first, count, alpha)
