"""Device-side ingest (silvan_graph_load: the edge list parsed and the CSR
built on the GPU) must give exactly the graph of the host loader, which
follows the reference's Graph(filename, directed) (silvan/src/Graph.cpp:
37-90): the same n, rows, component ids and diameter bound on the golden
files, on the loader's edge cases (comments, re-inserted pairs, partial
lines, CR/LF, self-loops, duplicates, a missing final newline) and on a large
R-MAT file, and the same errors for unrepresentable ids."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)

FIELDS = ("out_off", "out_adj", "in_off", "in_adj", "cc")


def assert_same_graph(dev, host):
    assert dev.n == host.n
    assert dev.directed == host.directed
    assert dev.diameter == host.diameter
    assert dev.n_components == host.n_components
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(dev, f), getattr(host, f), err_msg=f)


@pytest.mark.parametrize("name", [k for k in MANIFEST if "_" not in k])
def test_golden_files(sb, name):
    m = MANIFEST[name]
    path = os.path.join(GOLDEN, m["graph"])
    assert_same_graph(sb.Graph.load(path, m["directed"]).csr(),
                      sb.HostGraph.load(path, m["directed"]).csr())


CASES = [
    "# c\n1 2\n2 1\n1 2\n3 3\n\n5 4\n",
    "junk\n1 2\n",
    "1 2\n3 x\n4\n",
    "0\t1\r\n  2 0\r\n#x\r\n",
    "7 7\n7 7\n1 0",
    "\n\n3 1\n",
    "+3 +1\n#\n\n2\t\t0\n",
    "5 1\n# 9 9\n  \n0 2 7\n",
]


@pytest.mark.parametrize("text", CASES)
@pytest.mark.parametrize("directed", [False, True])
def test_loader_edge_cases(sb, tmp_path, text, directed):
    p = tmp_path / "g.txt"
    p.write_text(text)
    assert_same_graph(sb.Graph.load(str(p), directed).csr(),
                      sb.HostGraph.load(str(p), directed).csr())


@pytest.mark.parametrize("text", ["1 2\n1 -2\n", "0 1\n4294967299 1\n", "1 2147483648\n"])
def test_unrepresentable_ids_same_error(sb, tmp_path, text):
    p = tmp_path / "g.txt"
    p.write_text(text)
    with pytest.raises(sb.SilvanError) as dev:
        sb.Graph.load(str(p))
    with pytest.raises(sb.SilvanError) as host:
        sb.HostGraph.load(str(p))
    assert dev.value.code == host.value.code == sb.E_PARSE
    assert str(dev.value) == str(host.value)


def test_missing_file(sb, tmp_path):
    with pytest.raises(sb.SilvanError) as e:
        sb.Graph.load(str(tmp_path / "none.txt"))
    assert e.value.code == sb.E_IO


@pytest.mark.parametrize("directed", [True, False])
def test_large_rmat_file(sb, tmp_path, directed):
    pairs = sb.rmat(15, 8, 21, directed)
    path = str(tmp_path / "r.txt")
    sb.write_edge_list(path, pairs)
    assert_same_graph(sb.Graph.load(path, directed).csr(), sb.HostGraph.load(path, directed).csr())


def test_estimation_on_device_loaded_graph(sb, tmp_path):
    """The device-loaded graph runs the estimator exactly as the host-loaded one."""
    path = os.path.join(GOLDEN, MANIFEST["rmat9d"]["graph"])
    d = MANIFEST["rmat9d"]["directed"]
    a = sb.Probabilistic(sb.Graph.load(path, d), 0.03, 0.1, seed=3)
    b = sb.Probabilistic(sb.Graph.from_host(sb.HostGraph.load(path, d)), 0.03, 0.1, seed=3)
    ra, rb = a.run(), b.run()
    assert ra["num_samples"] == rb["num_samples"]
    np.testing.assert_array_equal(a.get_centrality(), b.get_centrality())


@pytest.mark.parametrize("make", [
    lambda sb: sb.grid(64, 0.45, 0.0, 5),          # a lattice broken into many pieces
    lambda sb: sb.rmat(14, 4, 9, False),           # R-MAT with isolated ids
    lambda sb: sb.erdos_renyi(3000, 1.2, 4),       # near the percolation threshold
])
def test_undirected_components_on_the_device(sb, tmp_path, make):
    """Undirected graphs get their component numbers and diameter bound on
    the device (Tarjan's numbering is the order of the components' smallest
    ids); they must equal the host's restatement of the reference."""
    path = str(tmp_path / "u.txt")
    sb.write_edge_list(path, make(sb))
    dev = sb.Graph.load(path, False).csr()
    host = sb.HostGraph.load(path, False).csr()
    assert host.n_components > 10
    assert_same_graph(dev, host)


@pytest.mark.parametrize("make", [
    lambda sb: sb.rmat(14, 4, 9, True),            # thousands of components, shallow
    lambda sb: sb.rmat(12, 2, 3, True),            # sparse: many singleton components
    # a chain of 300 components with a few short cycles: deeper than the
    # device's passes, so the recursion ends on the host copy
    lambda sb: np.array([[i, i + 1] for i in range(300)] + [[5, 2], [100, 90], [250, 249]],
                        np.uint32),
])
def test_directed_bound_on_the_device(sb, tmp_path, make):
    """Directed graphs: the component numbers are the host's Tarjan order,
    and the diameter bound over them (pivots, eccentricities inside each
    component, the AllCCUpperBound recursion) is computed on the device; it
    must equal the host's restatement of the reference."""
    path = str(tmp_path / "d.txt")
    sb.write_edge_list(path, make(sb))
    dev = sb.Graph.load(path, True).csr()
    host = sb.HostGraph.load(path, True).csr()
    assert host.n_components > 10
    assert_same_graph(dev, host)
