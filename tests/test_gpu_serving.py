"""Serving with continuous batching: requests on graphs of different sizes,
submitted while others run, are admitted by device-memory budget and served
together; every result is the same as the request's stand-alone run (and as
the CPU oracle)."""
import threading
import time

import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix(sb, port, small_graphs):
    names = ["ba2k", "rmat11d", "er3k", "rmat11u", "ba2k", "rmat11d"]
    reqs = [(nm, 60 + i) for i, nm in enumerate(names)]
    # stand-alone: one job per request
    alone = {}
    for nm, seed in reqs:
        hg, csr, _ = small_graphs[nm]
        job = sb.Probabilistic(sb.Graph.from_host(hg), 0.03, 0.1, seed=seed)
        job.run()
        alone[(nm, seed)] = job.get_centrality()
    n_max = max(small_graphs[nm][1].n for nm, _ in reqs)
    srv = sb.Server(n_max)
    try:
        ids = {}
        for i, (nm, seed) in enumerate(reqs):
            ids[(nm, seed)] = srv.submit(small_graphs[nm][0], 0.03, 0.1, seed=seed)
            time.sleep(0.01 * (i % 3))  # arrivals while others run
        for key, rid in ids.items():
            res = srv.wait(rid, 300)
            est = srv.estimates(rid, small_graphs[key[0]][1].n)
            np.testing.assert_array_equal(est, alone[key])
            assert res["latency_s"] >= res["queued_s"] >= 0
        st = srv.stats()
        assert st["max_active"] >= 2  # requests really shared rounds
    finally:
        srv.close()
    # and the stand-alone result is the oracle's
    nm, seed = reqs[1]
    hg, csr, _ = small_graphs[nm]
    o = port_graph(port, csr).run(csr.diameter, 0.03, 0.1, seed=seed)
    np.testing.assert_array_equal(alone[(nm, seed)], o["approx"] / o["num_samples"])


def test_admission_respects_budget(sb, small_graphs):
    hg, csr, _ = small_graphs["rmat11d"]
    # a budget that fits about one request at a time
    srv = sb.Server(csr.n, budget=1)
    try:
        ids = [srv.submit(hg, 0.05, 0.1, seed=s) for s in range(3)]
        for rid in ids:
            srv.wait(rid, 300)
        assert srv.stats()["max_active"] == 1
    finally:
        srv.close()


def test_submit_from_threads(sb, small_graphs):
    hg, csr, _ = small_graphs["ba2k"]
    srv = sb.Server(csr.n)
    ids = []
    lock = threading.Lock()

    def client(seed):
        rid = srv.submit(hg, 0.05, 0.1, seed=seed)
        with lock:
            ids.append(rid)

    try:
        ts = [threading.Thread(target=client, args=(s,)) for s in range(8)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for rid in ids:
            assert srv.wait(rid, 300)["num_samples"] > 0
    finally:
        srv.close()


def test_mixed_stream_all_succeed(sb):
    """Requests of different sizes and modes arriving back to back: the
    uploader thread admits and uploads while the round thread captures and
    launches; every request must finish with its stand-alone result."""
    graphs = [sb.HostGraph.from_pairs(sb.rmat(s, 16, 70 + s, bool(s % 2)), bool(s % 2))
              for s in (11, 12, 13, 14, 15, 16)]
    reqs = []
    for i in range(18):
        hg = graphs[i % len(graphs)]
        k = 5 if i % 5 == 0 else 0
        eps = 0.1 if k else 0.02
        reqs.append((hg, eps, k, 300 + i))
    srv = sb.Server(1 << 16)
    try:
        ids = [srv.submit(hg, eps, 0.1, k=k, seed=seed) for hg, eps, k, seed in reqs]
        outs = []
        for rid, (hg, eps, k, seed) in zip(ids, reqs):
            res = srv.wait(rid, 600)
            outs.append((res, srv.estimates(rid, hg.info().n)))
    finally:
        srv.close()
    for (hg, eps, k, seed), (res, est) in zip(reqs[:6], outs[:6]):
        job = sb.Probabilistic(sb.Graph.from_host(hg), eps, 0.1, k=k, seed=seed)
        alone = job.run()
        assert res["num_samples"] == alone["num_samples"]
        np.testing.assert_array_equal(est, job.get_centrality())
