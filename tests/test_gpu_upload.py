"""silvan_graph_upload: a caller's CSR arrays (with components and diameter
bound) go to the device as they are, all copies in order on one stream, with
the offsets' narrowing, the row table and the row checks on a second stream.
A graph uploaded that way must run exactly like the same graph built from
the edge list (silvan/src/Graph.cpp:37-90), and malformed rows must come back
as SILVAN_E_BADARG: the checks clamp every offset to the entry count, so no
kernel reads past the adjacency array."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BADARG = -1


def same_runs(sb, g1, g2, **kw):
    runs = []
    for g in (g1, g2):
        job = sb.Probabilistic(g, 0.03, 0.1, seed=17, **kw)
        runs.append((job, job.run()))
    (ja, ra), (jb, rb) = runs
    for f in ("num_samples", "first_pass_samples", "vis_edges", "omega", "stop_reason",
              "diameter", "backtracked_paths"):
        assert ra[f] == rb[f], (f, ra[f], rb[f])
    ca, cb = ja.counters(), jb.counters()
    for f in ("approx", "wimpy", "mcrade"):
        np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)


@pytest.mark.parametrize("name", ["rmat11d", "ba2k", "grid40"])
def test_uploaded_csr_runs_like_the_host_graph(sb, small_graphs, name):
    hg, csr, _ = small_graphs[name]
    kw = {"alpha": 0.0, "alpha_given": True} if name == "grid40" else {}
    same_runs(sb, sb.Graph.from_host(hg), sb.Graph.upload(csr, with_cc=True), **kw)


def broken(csr, what):
    out_off = np.array(csr.out_off, dtype=np.uint64)
    out_adj = np.array(csr.out_adj, dtype=np.uint32)
    row = int(np.argmax(np.diff(out_off.astype(np.int64)) >= 2))  # a row with two entries
    b = int(out_off[row])
    if what == "unsorted":
        out_adj[b], out_adj[b + 1] = out_adj[b + 1], out_adj[b]
    elif what == "id_out_of_range":
        out_adj[b] = csr.n
    elif what == "offset_past_the_end":
        out_off[1] = out_off[-1] + 1000
    elif what == "offsets_decrease":
        out_off[row + 1] = out_off[row] - 1 if out_off[row] > 0 else out_off[row]
        out_off[row] = out_off[row] + 1
    return out_off, out_adj


@pytest.mark.parametrize("what", ["unsorted", "id_out_of_range", "offset_past_the_end",
                                  "offsets_decrease"])
def test_upload_rejects_malformed_rows(sb, small_graphs, what):
    _, csr, _ = small_graphs["rmat11d"]
    out_off, out_adj = broken(csr, what)
    bad = sb.CSR(csr.n, csr.directed, out_off, out_adj, np.array(csr.in_off, dtype=np.uint64),
                 np.array(csr.in_adj, dtype=np.uint32), np.array(csr.cc, dtype=np.uint32),
                 csr.n_components, csr.diameter)
    with pytest.raises(sb.SilvanError) as e:
        sb.Graph.upload(bad, with_cc=True)
    assert e.value.code == BADARG
    # the device is still usable, and a good upload still runs exactly
    hg, csr2, _ = small_graphs["ba2k"]
    same_runs(sb, sb.Graph.from_host(hg), sb.Graph.upload(csr2, with_cc=True))
