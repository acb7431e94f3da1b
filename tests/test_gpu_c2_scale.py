"""Parity at the benchmark's full size: R-MAT scale 20, edge factor 16,
(.57, .19, .19, .05), seed 2, directed (1.05 M nodes, 16.1 M edges).

* Per-sample replay against the oracle: every sample of the first 10^4, then
  ranges spread over the first 10^6 sample indices.
* The whole estimation at eps 0.005 against the oracle's (counters, schedule
  and stopping decision bit for bit), and against the plain form.
* Size-independent invariants of the counters: wimpy <= approx and
  |mcrade| <= approx for every node (every update adds x in (0, 1], its
  square, and +-x truncated toward zero)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(sb, port):
    hg = sb.HostGraph.from_pairs(sb.rmat(20, 16, 2, True), True)
    csr = hg.csr()
    pg = port.graph(csr.n, True, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj, csr.cc)
    return hg, csr, pg, sb.Graph.from_host(hg)


def compare_replay(got, want, lo, hi):
    for f in ("path_length", "num_paths", "vis_edges"):
        np.testing.assert_array_equal(got[f], getattr(want, f), err_msg=f"{f} [{lo},{hi})")
    np.testing.assert_array_equal(got["offsets"], want.offsets)
    np.testing.assert_array_equal(got["nodes"], want.nodes)
    np.testing.assert_array_equal(got["counts"], want.counts)


def test_replay_first_ten_thousand(c2):
    _, _, pg, g = c2
    got = g.replay(42, 0, 10000, 2.3)
    assert (got["status"] == 0).all()
    compare_replay(got, pg.replay(42, 0, 10000, 2.3), 0, 10000)


def test_replay_spread_ranges(c2):
    _, _, pg, g = c2
    rng = np.random.default_rng(7)
    for first in sorted(rng.integers(10000, 1000000, size=10).tolist()):
        got = g.replay(42, first, 100, 2.3)
        compare_replay(got, pg.replay(42, first, 100, 2.3), first, first + 100)


def test_whole_estimation_matches_oracle_and_plain_form(sb, c2):
    _, csr, pg, g = c2
    fields = ["num_samples", "first_pass_samples", "vis_edges", "iteration_index",
              "num_partitions", "omega", "stop_reason", "alpha_sp_sampling"]
    job = sb.Probabilistic(g, 0.005, 0.05, seed=9)
    res = job.run()
    c = job.counters()
    o = pg.run(csr.diameter, 0.005, 0.05, seed=9)
    for f in fields:
        assert res[f] == o[f], f
    np.testing.assert_array_equal(c["approx"], o["approx"])
    np.testing.assert_array_equal(c["wimpy"], o["wimpy"])
    np.testing.assert_array_equal(c["mcrade"], o["mcrade"])
    np.testing.assert_array_equal(c["partition_index"], o["partition_index"])
    plain = sb.Probabilistic(g, 0.005, 0.05, seed=9, form="plain")
    rp = plain.run()
    assert rp["num_samples"] == res["num_samples"]
    np.testing.assert_array_equal(plain.counters()["mcrade"], c["mcrade"])
    # invariants
    assert (c["wimpy"] <= c["approx"]).all()
    assert (np.abs(c["mcrade"]) <= c["approx"][:, None] + 1e-6).all()
