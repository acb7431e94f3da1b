"""The CPU oracle, pinned: Philox known answers, the committed golden
fixtures (outputs of the reference's own sources with the same stream) and,
where the reference build is present, fresh random cases against it."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLDEN, "manifest.json")) as f:
    MANIFEST = json.load(f)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def test_philox_known_answers(port):
    # Known-answer vectors of Philox4x32-10 from the Random123 distribution
    # (kat_vectors): zero counter/key, all-ones counter/key, digits of pi.
    f = port.lib.orc_philox4x32
    f.argtypes = [C.c_void_p] * 3
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for ctr, key, want in cases:
        c = np.array(ctr, np.uint32)
        k = np.array(key, np.uint32)
        o = np.zeros(4, np.uint32)
        f(c.ctypes.data, k.ctypes.data, o.ctypes.data)
        assert o.tolist() == want


def golden_port_graph(port, g, directed):
    return port.graph(int(g["n"]), directed, g["out_off"], g["out_adj"], g["in_off"], g["in_adj"],
                      g["cc"])


@pytest.mark.parametrize("name", [k for k in MANIFEST if "_" not in k])
@pytest.mark.parametrize("alpha,tag", [(2.3, "a23"), (-1.0, "am1")])
def test_port_replay_matches_golden(port, name, alpha, tag):
    m = MANIFEST[name]
    g = golden(name)
    pg = golden_port_graph(port, g, m["directed"])
    r = pg.replay(m["seed"], 0, m["replay"], alpha)
    for f in ("path_length", "num_paths", "vis_edges", "offsets", "nodes", "counts"):
        np.testing.assert_array_equal(getattr(r, f), g[f"{tag}_{f}"], err_msg=f)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_port_run_matches_golden(port, name):
    m = MANIFEST[name]
    g = golden(name)
    pg = golden_port_graph(port, g, m["directed"])
    run = dict(m["run"])
    o = pg.run(int(g["diameter"]), run.pop("eps"), run.pop("delta"), seed=m["seed"], **run)
    for f in ("approx", "wimpy", "mcrade", "partition_index", "ranking_elements",
              "ranking_values", "sp_lengths", "epsilon_partition", "partition_ids"):
        np.testing.assert_array_equal(o[f], g["run_" + f], err_msg=f)
    for f, v in m["scalars"].items():
        assert o[f] == v, f


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Ref, ref_available
    if not ref_available():
        pytest.skip("reference build not present")
    return Ref()


@pytest.mark.parametrize("seed", [3, 77, 2**33 + 5])
def test_port_matches_reference_sources(ref, port, sb, tmp_path, seed):
    # fresh graphs and seeds, both sampling modes, against the reference's code
    for kind, kw, directed in [("rmat", (10, 6, seed % 97, True), True),
                               ("ba", (800, 2, seed % 89), False)]:
        pairs = sb.rmat(*kw) if kind == "rmat" else sb.barabasi_albert(*kw)
        path = str(tmp_path / f"{kind}.txt")
        sb.write_edge_list(path, pairs)
        rg = ref.graph(path, directed)
        D, cc, nc = rg.diameter()
        oo, oa, io, ia = rg.csr()
        pg = port.graph(rg.n, directed, oo, oa, io, ia, cc)
        for alpha in (2.3, -1.0):
            a = rg.replay(seed, 1000, 400, alpha)
            b = pg.replay(seed, 1000, 400, alpha)
            for f in ("path_length", "num_paths", "vis_edges", "offsets", "nodes", "counts"):
                np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
        ra = ref.run(path, directed, 0.05, 0.1, seed=seed)
        rb = pg.run(D, 0.05, 0.1, seed=seed)
        for f in ("approx", "wimpy", "mcrade", "partition_index"):
            np.testing.assert_array_equal(ra[f], rb[f])


def _pair_dependencies(n, adj):
    """sum over ordered pairs (s, t) of sigma_st(v) / sigma_st by explicit
    BFS path counting from both ends (small graphs only)."""
    from collections import deque

    def bfs(s):
        dist = [-1] * n
        sig = [0] * n
        dist[s], sig[s] = 0, 1
        q = deque([s])
        while q:
            x = q.popleft()
            for y in adj[x]:
                if dist[y] < 0:
                    dist[y] = dist[x] + 1
                    q.append(y)
                if dist[y] == dist[x] + 1:
                    sig[y] += sig[x]
        return dist, sig

    radj = [[] for _ in range(n)]
    for x in range(n):
        for y in adj[x]:
            radj[y].append(x)
    fw = [bfs(s) for s in range(n)]

    def bfs_rev(t):
        dist = [-1] * n
        sig = [0] * n
        dist[t], sig[t] = 0, 1
        q = deque([t])
        while q:
            x = q.popleft()
            for y in radj[x]:
                if dist[y] < 0:
                    dist[y] = dist[x] + 1
                    q.append(y)
                if dist[y] == dist[x] + 1:
                    sig[y] += sig[x]
        return dist, sig

    bw = [bfs_rev(t) for t in range(n)]
    bc = np.zeros(n)
    for s in range(n):
        ds, ss = fw[s]
        for t in range(n):
            if t == s or ds[t] < 0:
                continue
            dt, st = bw[t]
            for v in range(n):
                if v in (s, t) or ds[v] < 0 or dt[v] < 0:
                    continue
                if ds[v] + dt[v] == ds[t]:
                    bc[v] += ss[v] * st[v] / ss[t]
    return bc / (n * (n - 1))


@pytest.mark.parametrize("directed", [False, True])
def test_brandes_matches_pair_enumeration(sb, port, directed):
    """The exact-betweenness ground truth of the (eps, delta) check."""
    pairs = sb.rmat(5, 3, 17, directed) if directed else sb.barabasi_albert(28, 2, 17)
    hg = sb.HostGraph.from_pairs(pairs, directed)
    csr = hg.csr()
    adj = [list(csr.out_adj[csr.out_off[u]:csr.out_off[u + 1]]) for u in range(csr.n)]
    want = _pair_dependencies(csr.n, adj)
    got = port.graph(csr.n, csr.directed, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj,
                     csr.cc).brandes()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15)
    # a path 0-1-2: the middle node lies on both ordered pairs (0,2), (2,0)
    p3 = sb.HostGraph.from_pairs(np.array([[0, 1], [1, 2]], np.uint32), False).csr()
    b3 = port.graph(p3.n, False, p3.out_off, p3.out_adj, p3.in_off, p3.in_adj, p3.cc).brandes()
    np.testing.assert_allclose(b3, [0, 1 / 3, 0])


def test_weighted_backtrack_restores_the_guarantee_on_a_lattice(sb, port):
    """On a lattice most pairs have many shortest paths.  The reference's
    backtrack (Sp_sampler.cpp:254-260 adds n_paths of the endpoint, 1, per
    predecessor) does not pick them uniformly, and its estimates miss exact
    betweenness by more than eps; the sigma-weighted option does not."""
    hg = sb.HostGraph.from_pairs(sb.grid(8, 0.0, 0.0, 1), False)
    csr = hg.csr()
    pg = port.graph(csr.n, False, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj, csr.cc)
    bc = pg.brandes()
    eps = 0.01
    for seed in range(3):
        kw = dict(seed=seed, alpha=0.0, alpha_given=True)
        ref = pg.run(csr.diameter, eps, 0.05, **kw)
        wtd = pg.run(csr.diameter, eps, 0.05, weighted=True, **kw)
        assert np.abs(ref["approx"] / ref["num_samples"] - bc).max() > eps
        assert np.abs(wtd["approx"] / wtd["num_samples"] - bc).max() <= eps
