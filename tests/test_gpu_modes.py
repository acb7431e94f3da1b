"""Whole-run parity in the estimator's other modes: top-k relative
approximation (silvan/src/Probabilistic.cpp:179-245,587-687 and
silvan/src/Ranking_list.cpp), m_hat off (-m), empirical peeling off (-a 0),
a given alpha (-s), single-path sampling on a lattice (-s 0), and every
sampler CTA size: the device run must leave exactly the oracle's counters,
schedule, stopping decision and ranking."""
import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu

SCALARS = ["num_samples", "vis_edges", "iteration_index", "num_partitions", "omega",
           "first_stopping_samples", "last_stopping_samples", "alpha_sp_sampling",
           "union_sample", "first_pass_samples", "stop_reason"]


def run_pair(sb, port, small_graphs, name, eps, delta, **kw):
    hg, csr, _ = small_graphs[name]
    job = sb.Probabilistic(sb.Graph.from_host(hg), eps, delta, **kw)
    res = job.run()
    okw = {k: v for k, v in kw.items() if k not in ("block", "slots", "form", "backtrack")}
    if "m_hat" in okw:
        okw["mhat"] = okw.pop("m_hat")
    if kw.get("backtrack") == "sigma":
        okw["weighted"] = True
    o = port_graph(port, csr).run(csr.diameter, eps, delta, **okw)
    return job, res, o


def assert_same_run(job, res, o):
    for f in SCALARS:
        assert res[f] == o[f], (f, res[f], o[f])
    c = job.counters()
    np.testing.assert_array_equal(c["approx"], o["approx"])
    np.testing.assert_array_equal(c["wimpy"], o["wimpy"])
    np.testing.assert_array_equal(c["mcrade"], o["mcrade"])
    np.testing.assert_array_equal(c["partition_index"], o["partition_index"])


@pytest.mark.parametrize("name,k,eps,extra", [
    ("ba2k", 5, 0.05, {}),
    ("rmat11d", 10, 0.1, {}),
    ("er3k", 8, 0.08, {"m_hat": False}),
    ("grid40", 10, 0.1, {"alpha": 0.0, "alpha_given": True}),
])
def test_topk_matches_oracle(sb, port, small_graphs, name, k, eps, extra):
    job, res, o = run_pair(sb, port, small_graphs, name, eps, 0.05, k=k, seed=21, **extra)
    assert_same_run(job, res, o)
    assert res["numresults_topk"] == o["numresults_topk"]
    assert res["eps_final_topk"] == o["eps_final_topk"]
    nodes, vals = job.topk()
    cnt = o["numresults_topk"]
    assert len(nodes) == cnt
    np.testing.assert_array_equal(nodes, o["ranking_elements"][:cnt])
    np.testing.assert_array_equal(vals, o["ranking_values"][:cnt] / o["num_samples"])


@pytest.mark.parametrize("name,kw", [
    ("ba2k", {"m_hat": False}),
    ("rmat11d", {"a": 0.0}),
    ("rmat11u", {"alpha": 3.0, "alpha_given": True}),
    ("er3k", {"a": 1.5, "m_hat": False}),
])
def test_absolute_options_match_oracle(sb, port, small_graphs, name, kw):
    job, res, o = run_pair(sb, port, small_graphs, name, 0.03, 0.1, seed=33, **kw)
    assert_same_run(job, res, o)


@pytest.mark.parametrize("block", [128, 256, 512, 1024])
def test_every_cta_size_gives_the_same_run(sb, port, small_graphs, block):
    """The autotuner may draw any round with any CTA size: each one must
    reproduce the oracle exactly."""
    job, res, o = run_pair(sb, port, small_graphs, "rmat11d", 0.02, 0.1, seed=9, block=block)
    assert res["sampler_block"] == block
    assert_same_run(job, res, o)


def test_plain_and_batched_topk_agree(sb, small_graphs):
    hg, _, _ = small_graphs["ba2k"]
    g = sb.Graph.from_host(hg)
    out = []
    for form in ("plain", "batched"):
        job = sb.Probabilistic(g, 0.05, 0.05, k=5, seed=4, form=form)
        res = job.run()
        out.append((res["num_samples"], job.topk(), job.get_centrality()))
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1][0], out[1][1][0])
    np.testing.assert_array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("name,extra", [
    ("ba2k", {}),
    ("rmat11d", {"block": 128}),
    ("grid40", {"alpha": 0.0, "alpha_given": True}),
    ("grid40", {"k": 10, "alpha": 0.0, "alpha_given": True}),
])
def test_sigma_weighted_backtrack_matches_oracle(sb, port, small_graphs, name, extra):
    """The sigma-weighted backtrack option (not the reference's rule) against
    the oracle's restatement of the same rule."""
    eps = 0.1 if extra.get("k") else 0.03
    job, res, o = run_pair(sb, port, small_graphs, name, eps, 0.1, seed=17, backtrack="sigma",
                           **extra)
    assert_same_run(job, res, o)
