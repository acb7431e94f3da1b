"""Per-sample parity of the device sampler with the CPU oracle: for every
sample the path length, number of paths, edges visited and path map
(node -> count) must be identical (Sp_sampler::random_path,
silvan/src/Sp_sampler.cpp:41-238)."""
import numpy as np
import pytest

from conftest import SMALL_GRAPHS, port_graph

pytestmark = pytest.mark.gpu


def compare(a, b):
    for f in ("path_length", "num_paths", "vis_edges", "offsets", "nodes", "counts"):
        x, y = a[f], getattr(b, f)
        if not np.array_equal(np.asarray(x), np.asarray(y)):
            bad = np.nonzero(np.asarray(x)[: len(y)] != np.asarray(y)[: len(x)])[0]
            raise AssertionError(f"{f} differs first at {bad[:5]}")


# Lattices ask for astronomically many paths per sample at alpha > 0 (the
# reference does not finish on them, silvan/src/Sp_sampler.cpp:166-170), so the
# grid is replayed in single-path mode only.
CASES = [(n, a) for n in sorted(SMALL_GRAPHS) for a in (2.3, -1.0)
         if not (n.startswith("grid") and a > 0)]


@pytest.mark.parametrize("name,alpha", CASES)
def test_replay_matches_oracle(sb, port, small_graphs, name, alpha):
    hg, csr, directed = small_graphs[name]
    g = sb.Graph.from_host(hg)
    pg = port_graph(port, csr)
    a = g.replay(seed=7, first=0, count=2000, alpha=alpha)
    b = pg.replay(7, 0, 2000, alpha)
    assert not b.zero_modulus
    assert (a["status"] == 0).all()
    compare(a, b)


def test_replay_offsets_and_seeds(sb, port, small_graphs):
    hg, csr, _ = small_graphs["rmat11d"]
    g = sb.Graph.from_host(hg)
    pg = port_graph(port, csr)
    for seed, first in [(1, 0), (99, 123456), (2**40 + 3, 7)]:
        compare(g.replay(seed, first, 500, 2.3), pg.replay(seed, first, 500, 2.3))
