"""Whole-run parity: the device estimator in both forms must leave exactly
the counters, partitions, schedule and stopping decision of the CPU oracle
(Probabilistic::run in one-thread semantics, silvan/src/Probabilistic.cpp:
775-1139)."""
import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu

SCALARS = ["num_samples", "vis_edges", "iteration_index", "num_partitions", "omega",
           "first_stopping_samples", "last_stopping_samples", "alpha_sp_sampling",
           "union_sample"]


def run_both(sb, port, small_graphs, name, form, **kw):
    hg, csr, directed = small_graphs[name]
    g = sb.Graph.from_host(hg)
    job = sb.Probabilistic(g, form=form, **kw)
    res = job.run()
    cnt = job.counters()
    pg = port_graph(port, csr)
    okw = {k: v for k, v in kw.items() if k not in ("slots",)}
    o = pg.run(csr.diameter, okw.pop("eps"), okw.pop("delta"), **okw)
    return res, cnt, o, job


@pytest.mark.parametrize("form", ["batched", "plain"])
@pytest.mark.parametrize("name", ["ba2k", "rmat11d", "er3k"])
def test_run_matches_oracle(sb, port, small_graphs, name, form):
    res, cnt, o, _ = run_both(sb, port, small_graphs, name, form, eps=0.02, delta=0.1, seed=5)
    for f in SCALARS:
        assert res[f] == o[f], (f, res[f], o[f])
    assert res["first_pass_samples"] == o["first_pass_samples"]
    np.testing.assert_array_equal(cnt["approx"], o["approx"])
    np.testing.assert_array_equal(cnt["wimpy"], o["wimpy"])
    np.testing.assert_array_equal(cnt["mcrade"], o["mcrade"])
    np.testing.assert_array_equal(cnt["partition_index"], o["partition_index"])


def test_stepwise_equals_run(sb, port, small_graphs):
    hg, csr, directed = small_graphs["rmat11d"]
    g = sb.Graph.from_host(hg)
    a = sb.Probabilistic(g, 0.02, 0.1, seed=31)
    ra = a.run()
    b = sb.Probabilistic(g, 0.02, 0.1, seed=31)
    rounds = 0
    while not b.step(1)["done"]:
        rounds += 1
        assert rounds < 10000
    for f in SCALARS:
        assert b.result[f] == ra[f], f
    np.testing.assert_array_equal(a.counters()["approx"], b.counters()["approx"])
    np.testing.assert_array_equal(a.counters()["mcrade"], b.counters()["mcrade"])


def test_batched_jobs_match_alone(sb, port, small_graphs):
    """Multi-graph batching: jobs on different graphs sharing sampler launches
    give each job exactly its stand-alone (oracle) result."""
    names = ["ba2k", "rmat11d", "er3k", "rmat11u"]
    jobs, oracles = [], []
    for i, nm in enumerate(names):
        hg, csr, directed = small_graphs[nm]
        g = sb.Graph.from_host(hg)
        jobs.append(sb.Probabilistic(g, 0.02, 0.1, seed=40 + i))
        oracles.append(port_graph(port, csr).run(csr.diameter, 0.02, 0.1, seed=40 + i))
    results = sb.run_batched(jobs)
    for job, res, o in zip(jobs, results, oracles):
        for f in SCALARS:
            assert res[f] == o[f], f
        c = job.counters()
        np.testing.assert_array_equal(c["approx"], o["approx"])
        np.testing.assert_array_equal(c["mcrade"], o["mcrade"])
