"""Exact betweenness on the device (silvan_exact_betweenness): the same
values as the oracle's Brandes on the small graphs, deterministic, and the
ground truth of the (eps, delta) check on graphs too large for the CPU."""
import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["ba2k", "rmat11d", "er3k", "rmat11u", "grid40"])
def test_matches_oracle(sb, port, small_graphs, name):
    hg, csr, _ = small_graphs[name]
    g = sb.Graph.from_host(hg)
    got = g.exact_betweenness()
    want = port_graph(port, csr).brandes()
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-15)
    np.testing.assert_array_equal(got, g.exact_betweenness())  # no scheduling dependence


@pytest.mark.parametrize("directed", [True, False])
def test_guarantee_on_rmat13(sb, directed):
    """Estimates within eps of the exact values in at least 1 - delta of the
    runs (at most 1 miss in 10 at delta 0.05)."""
    eps, delta = 0.01, 0.05
    hg = sb.HostGraph.from_pairs(sb.rmat(13, 8, 31, directed), directed)
    g = sb.Graph.from_host(hg)
    bc = g.exact_betweenness()
    misses = 0
    for seed in range(10):
        job = sb.Probabilistic(g, eps, delta, seed=500 + seed)
        job.run()
        misses += int(np.abs(job.get_centrality() - bc).max() > eps)
    assert misses <= 1
