"""Host ingest: edge-list parse with the reference loader's semantics
(silvan/src/Graph.cpp:37-90), CSR, Tarjan numbering and the AllCCUpperBound
diameter (silvan/src/Graph.cpp:109-316) -- against the golden fixtures and,
where present, the reference build itself.  No GPU needed."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)


@pytest.mark.parametrize("name", [k for k in MANIFEST if "_" not in k])
def test_ingest_matches_golden(sb, name):
    m = MANIFEST[name]
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    c = sb.HostGraph.load(os.path.join(GOLDEN, m["graph"]), m["directed"]).csr()
    assert c.n == int(g["n"])
    assert c.diameter == int(g["diameter"])
    assert c.n_components == int(g["n_components"])
    for f in ("out_off", "out_adj", "in_off", "in_adj", "cc"):
        np.testing.assert_array_equal(getattr(c, f), g[f], err_msg=f)


def csr_lists(c):
    return [c.out_adj[c.out_off[i]:c.out_off[i + 1]].tolist() for i in range(c.n)]


def load_text(sb, tmp_path, text, directed=False):
    p = tmp_path / "g.txt"
    p.write_text(text)
    return sb.HostGraph.load(str(p), directed).csr()


def test_comments_duplicates_selfloops(sb, tmp_path):
    c = load_text(sb, tmp_path, "# header\n1 2\n2 1\n1 2\n3 3\n\n5 4\n")
    # the empty line re-inserts the previous pair (3,3); ids 0..5 exist
    assert c.n == 6
    assert csr_lists(c) == [[], [2], [1], [3], [5], [4]]


def test_leading_bad_line_inserts_zero_pair(sb, tmp_path):
    # sscanf fails on the first line, so the initial (0, 0) is inserted
    c = load_text(sb, tmp_path, "junk\n1 2\n")
    assert csr_lists(c) == [[0], [2], [1]]


def test_partial_parse_keeps_previous_v(sb, tmp_path):
    c = load_text(sb, tmp_path, "1 2\n3 x\n", directed=True)
    assert csr_lists(c) == [[], [2], [], [2]]
    assert c.in_adj[c.in_off[2]:c.in_off[3]].tolist() == [1, 3]


def test_crlf_tabs_and_leading_space(sb, tmp_path):
    c = load_text(sb, tmp_path, "0\t1\r\n  2 0\r\n#x\r\n")
    assert csr_lists(c) == [[1, 2], [0], [0]]


@pytest.mark.parametrize("text", ["1 -2\n", "4294967299 1\n", "1 2147483648\n"])
def test_unrepresentable_ids_rejected(sb, tmp_path, text):
    with pytest.raises(sb.SilvanError) as e:
        load_text(sb, tmp_path, text)
    assert e.value.code == sb.E_PARSE


def test_missing_file(sb, tmp_path):
    with pytest.raises(sb.SilvanError) as e:
        sb.HostGraph.load(str(tmp_path / "none.txt"))
    assert e.value.code == sb.E_IO


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Ref, ref_available
    if not ref_available():
        pytest.skip("reference build not present")
    return Ref()


EDGE_CASES = [
    "# c\n1 2\n2 1\n1 2\n3 3\n\n5 4\n",
    "junk\n1 2\n",
    "1 2\n3 x\n4\n",
    "0\t1\r\n  2 0\r\n#x\r\n",
    "7 7\n7 7\n",
    "\n\n3 1\n",
]


@pytest.mark.parametrize("text", EDGE_CASES)
@pytest.mark.parametrize("directed", [False, True])
def test_loader_matches_reference(sb, ref, tmp_path, text, directed):
    p = tmp_path / "g.txt"
    p.write_text(text)
    c = sb.HostGraph.load(str(p), directed).csr()
    rg = ref.graph(str(p), directed)
    oo, oa, io, ia = rg.csr()
    D, cc, nc = rg.diameter()
    np.testing.assert_array_equal(c.out_off, oo)
    np.testing.assert_array_equal(c.out_adj, oa)
    np.testing.assert_array_equal(c.in_off, io)
    np.testing.assert_array_equal(c.in_adj, ia)
    np.testing.assert_array_equal(c.cc, cc)
    assert (c.diameter, c.n_components) == (D, nc)


@pytest.mark.parametrize("seed", range(6))
def test_scc_and_diameter_match_reference(sb, ref, tmp_path, seed):
    directed = seed % 2 == 0
    pairs = sb.rmat(9 + seed % 3, 3 + seed, 100 + seed, directed)
    p = str(tmp_path / "g.txt")
    sb.write_edge_list(p, pairs)
    c = sb.HostGraph.load(p, directed).csr()
    rg = ref.graph(p, directed)
    D, cc, nc = rg.diameter()
    np.testing.assert_array_equal(c.cc, cc)
    assert (c.diameter, c.n_components) == (D, nc)
