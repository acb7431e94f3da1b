"""Wide BFS levels expanded by several CTAs (the sampler's help board): a
posted level is expanded tile by tile by its owner and by the CTAs that are
between samples or out of samples, with look-backs over the tiles in place
of the one-CTA tile order.  The level's queue order, predecessor keys,
counts, sigma and meeting list must be exactly those of the one-CTA
expansion (silvan/src/Sp_sampler.cpp:116-143), so whole runs must leave the
oracle's counters bit for bit; a threshold of one item posts every level
whenever an entry is free, which exercises entries taken, opened, joined and
handed on many times per launch."""
import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu

SCALARS = ["num_samples", "vis_edges", "iteration_index", "num_partitions", "omega",
           "first_stopping_samples", "last_stopping_samples", "alpha_sp_sampling",
           "union_sample", "first_pass_samples", "stop_reason", "void_samples",
           "backtracked_paths", "ball_nodes", "pred_entries"]
NEVER = 0xFFFFFFFF


def same_counters(ja, jb):
    a, b = ja.counters(), jb.counters()
    for f in ("approx", "wimpy", "mcrade", "partition_index"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.parametrize("name,block,form,items,extra", [
    ("rmat11d", 128, "batched", 1, {}),
    ("rmat11d", 1024, "batched", 1, {}),
    ("rmat11d", 512, "plain", 1, {}),
    ("rmat11u", 256, "batched", 64, {"alpha": 3.0, "alpha_given": True}),
    ("ba2k", 512, "batched", 1, {}),
    ("grid40", 128, "batched", 1, {"alpha": 0.0, "alpha_given": True}),
    ("er3k", 1024, "plain", 16, {"k": 8}),
])
def test_assisted_levels_match_oracle(sb, port, small_graphs, name, block, form, items, extra):
    hg, csr, _ = small_graphs[name]
    eps = 0.08 if extra.get("k") else 0.03
    job = sb.Probabilistic(sb.Graph.from_host(hg), eps, 0.1, seed=5, block=block, form=form,
                           assist_items=items, **extra)
    res = job.run()
    assert res["assisted_levels"] > 0
    o = port_graph(port, csr).run(csr.diameter, eps, 0.1, seed=5, **extra)
    for f in ("num_samples", "vis_edges", "iteration_index", "num_partitions", "omega",
              "first_stopping_samples", "last_stopping_samples", "alpha_sp_sampling",
              "union_sample", "first_pass_samples", "stop_reason"):
        assert res[f] == o[f], (f, res[f], o[f])
    c = job.counters()
    np.testing.assert_array_equal(c["approx"], o["approx"])
    np.testing.assert_array_equal(c["wimpy"], o["wimpy"])
    np.testing.assert_array_equal(c["mcrade"], o["mcrade"])
    if extra.get("k"):
        nodes, _ = job.topk()
        np.testing.assert_array_equal(nodes, o["ranking_elements"][:len(nodes)])


@pytest.mark.parametrize("scale,directed,items", [(15, True, 1), (16, True, 2048),
                                                  (15, False, 512)])
def test_assisted_and_alone_give_the_same_run(sb, scale, directed, items):
    """Larger R-MAT graphs, whose hub levels reach thousands of entries: the
    run with the help board and the run with every level on its own CTA
    agree in every counter and result field."""
    hg = sb.HostGraph.from_pairs(sb.rmat(scale, 16, scale, directed), directed)
    g = sb.Graph.from_host(hg)
    runs = []
    for ai in (items, NEVER):
        job = sb.Probabilistic(g, 0.01, 0.1, seed=3, assist_items=ai)
        res = job.run()
        runs.append((job, res))
    (ja, ra), (jb, rb) = runs
    assert ra["assisted_levels"] > 0 and ra["helper_tiles"] > 0
    assert rb["assisted_levels"] == 0 and rb["helper_tiles"] == 0
    for f in SCALARS:
        assert ra[f] == rb[f], (f, ra[f], rb[f])
    same_counters(ja, jb)


def test_replay_with_assisted_levels_matches_oracle(sb, port):
    """Per-sample records (path, path count, visited edges) of the replay hook
    while the help board is in use (the default threshold, on a graph whose
    hub levels pass it), against the oracle sample by sample."""
    hg = sb.HostGraph.from_pairs(sb.rmat(15, 16, 7, True), True)
    csr = hg.csr()
    g = sb.Graph.from_host(hg)
    got = g.replay(11, 0, 4000, 2.3)
    assert (got["status"] == 0).all()
    want = port_graph(port, csr).replay(11, 0, 4000, 2.3)
    for f in ("path_length", "num_paths", "vis_edges"):
        np.testing.assert_array_equal(got[f], getattr(want, f), err_msg=f)
    np.testing.assert_array_equal(got["offsets"], want.offsets)
    np.testing.assert_array_equal(got["nodes"], want.nodes)
    np.testing.assert_array_equal(got["counts"], want.counts)


def test_failed_shared_level_does_not_leak_into_later_jobs(sb, port, small_graphs):
    """Failure path of the help board.  With no polls allowed, every wait
    between the CTAs of a shared level gives up at once: the owner's level is
    marked failed while helpers may still be inside it, so records of its
    slot can be left half-written.  The job must fail with E_TIMEOUT, and the
    next jobs, which borrow the same pooled sampler engine (its slots and its
    board), must again match the oracle bit for bit with the board in use:
    the engine re-initialises the slots after such a launch and reopens the
    board entries that stayed closed.  The reference's own per-sample reset
    (silvan/src/Sp_sampler.cpp:226-231) is what these jobs rely on."""
    hg, csr, _ = small_graphs["rmat11d"]
    g = sb.Graph.from_host(hg)
    bad = sb.Probabilistic(g, 0.03, 0.1, seed=5, block=128, assist_items=1, wait_polls=NEVER)
    with pytest.raises(sb.SilvanError) as err:
        bad.run()
    assert err.value.code == sb.E_TIMEOUT
    del bad
    for seed, items in ((5, 1), (6, 0)):
        job = sb.Probabilistic(g, 0.03, 0.1, seed=seed, block=128, assist_items=items)
        res = job.run()
        if items == 1:
            assert res["assisted_levels"] > 0
        o = port_graph(port, csr).run(csr.diameter, 0.03, 0.1, seed=seed)
        for f in ("num_samples", "vis_edges", "iteration_index", "first_pass_samples",
                  "stop_reason"):
            assert res[f] == o[f], (seed, f, res[f], o[f])
        c = job.counters()
        for f in ("approx", "wimpy", "mcrade"):
            np.testing.assert_array_equal(c[f], o[f], err_msg=f"seed {seed}: {f}")
