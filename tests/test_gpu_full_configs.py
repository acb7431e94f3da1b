"""Parity at the full sizes of the other benchmark configurations.

* The 2048 x 2048 grid (5 % of edges deleted, 0.1 % shortcuts, seed 3;
  4.2 M nodes, diameter bound about 260) with single-path sampling: the
  deep, narrow searches of about 85 levels per side, where the
  middle-predecessor searches of the backtrack (level scan and reverse scan)
  actually run.  Per-sample replay against the oracle over the first 1000
  samples and ranges spread over the first 10^6 indices.
* A whole top-10 estimation on a 128 x 128 grid of the same generator
  against the oracle: counters, schedule, ranking and eps_final_topk bit for
  bit (silvan/src/Probabilistic.cpp:587-687, Ranking_list.cpp:20-43).
* The 64 graphs of the multi-graph workload (ER mean degree 8 and BA with 4
  edges per node, n log-uniform in [10^3, 2 * 10^6], seeds 100-163) in one
  batched run: every job's result equals its stand-alone run."""
import math

import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu


def compare_replay(got, want, lo, hi):
    for f in ("path_length", "num_paths", "vis_edges"):
        np.testing.assert_array_equal(got[f], getattr(want, f), err_msg=f"{f} [{lo},{hi})")
    np.testing.assert_array_equal(got["offsets"], want.offsets)
    np.testing.assert_array_equal(got["nodes"], want.nodes)
    np.testing.assert_array_equal(got["counts"], want.counts)


@pytest.fixture(scope="module")
def grid2048(sb, port):
    hg = sb.HostGraph.from_pairs(sb.grid(2048, 0.05, 0.001, 3), False)
    csr = hg.csr()
    return csr, port_graph(port, csr), sb.Graph.from_host(hg)


def test_grid2048_replay(grid2048):
    csr, pg, g = grid2048
    assert csr.n == 2048 * 2048 and csr.diameter > 200
    got = g.replay(7, 0, 1000, 0.0)
    assert (got["status"] == 0).all()
    compare_replay(got, pg.replay(7, 0, 1000, 0.0), 0, 1000)
    # the searches are deep: long paths, many levels
    assert got["path_length"].max() > 50
    rng = np.random.default_rng(11)
    for first in sorted(rng.integers(1000, 1000000, size=8).tolist()):
        got = g.replay(7, first, 40, 0.0)
        compare_replay(got, pg.replay(7, first, 40, 0.0), first, first + 40)


def test_grid_top10_estimation_matches_oracle(sb, port):
    hg = sb.HostGraph.from_pairs(sb.grid(128, 0.05, 0.001, 3), False)
    csr = hg.csr()
    kw = dict(k=10, alpha=0.0, alpha_given=True)
    job = sb.Probabilistic(sb.Graph.from_host(hg), 0.1, 0.05, seed=5, **kw)
    res = job.run()
    o = port_graph(port, csr).run(csr.diameter, 0.1, 0.05, seed=5, **kw)
    for f in ("num_samples", "first_pass_samples", "vis_edges", "iteration_index",
              "num_partitions", "union_sample", "numresults_topk", "eps_final_topk",
              "stop_reason"):
        assert res[f] == o[f], (f, res[f], o[f])
    c = job.counters()
    for f in ("approx", "wimpy", "mcrade", "partition_index"):
        np.testing.assert_array_equal(c[f], o[f], err_msg=f)
    nodes, _ = job.topk()
    np.testing.assert_array_equal(nodes, o["ranking_elements"][:len(nodes)])


def multigraph64(sb):
    out = []
    for i in range(64):
        seed = 100 + i
        rng = np.random.default_rng(seed)
        n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e6)))))
        pairs = sb.erdos_renyi(n, 8.0, seed) if i % 2 == 0 else sb.barabasi_albert(n, 4, seed)
        out.append(sb.HostGraph.from_pairs(pairs, False))
    return out


def test_multigraph64_batched_equals_alone(sb):
    hosts = multigraph64(sb)
    graphs = [sb.Graph.from_host(h) for h in hosts]
    assert sum(g.n for g in graphs) > 2e7
    jobs = [sb.Probabilistic(g, 0.01, 0.05, seed=300 + i) for i, g in enumerate(graphs)]
    batched = sb.run_batched(jobs)
    small = set(sorted(range(64), key=lambda i: graphs[i].n)[:8])
    for i, g in enumerate(graphs):
        alone = sb.Probabilistic(g, 0.01, 0.05, seed=300 + i)
        r = alone.run()
        for f in ("num_samples", "first_pass_samples", "vis_edges", "iteration_index",
                  "num_partitions", "stop_reason", "omega", "eps_stop"):
            assert batched[i][f] == r[f], (i, f, batched[i][f], r[f])
        a, b = jobs[i].counters(), alone.counters()
        np.testing.assert_array_equal(a["approx"], b["approx"], err_msg=f"graph {i}")
        np.testing.assert_array_equal(a["wimpy"], b["wimpy"], err_msg=f"graph {i}")
        if i in small:
            np.testing.assert_array_equal(a["mcrade"], b["mcrade"], err_msg=f"graph {i}")
        del alone, a, b
