"""silvan_replay_samples_noalloc is the sampler for callers that cannot let a
library allocate device memory: processes that already hold their whole
memory quota, or runtimes that give their libraries only buffers they
allocated themselves.  Its scratch is a fixed static device array shared by
every call, so it must return exactly what silvan_replay_samples returns,
call after call, on graphs of different sizes.  The caller supplies every
output as a device buffer (allocated here with torch, outside the entry
point).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def noalloc_replay(sb, g, seed, first, count, alpha, cap, allow_overflow=False):
    import torch

    dev = torch.device("cuda")
    pl = torch.zeros(count, dtype=torch.int32, device=dev)
    npth = torch.zeros(count, dtype=torch.int32, device=dev)
    vis = torch.zeros(count, dtype=torch.int64, device=dev)
    st = torch.zeros(count, dtype=torch.int32, device=dev)
    recs = torch.zeros(3 * cap, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    lib = sb.load()
    rc = lib.silvan_replay_samples_noalloc(
        g.h, seed, first, count, alpha, 0, C.c_void_p(pl.data_ptr()),
        C.c_void_p(npth.data_ptr()), C.c_void_p(vis.data_ptr()), C.c_void_p(st.data_ptr()),
        C.c_void_p(recs.data_ptr()), cap, C.c_void_p(cnt.data_ptr()), C.c_void_p(stream))
    assert rc == 0, lib.silvan_last_error()
    torch.cuda.synchronize()
    n_rec = int(cnt.item())
    assert allow_overflow or n_rec <= cap
    r = recs.cpu().numpy().view(np.uint32).reshape(-1, 3)[:min(n_rec, cap)]
    # placeholders of samples whose records did not fit (count 0)
    r = r[r[:, 2] != 0]
    order = np.lexsort((r[:, 0], r[:, 1]))  # by sample, then node
    r = r[order]
    nent = np.bincount(r[:, 1], minlength=count)
    off = np.zeros(count + 1, np.int64)
    off[1:] = np.cumsum(nent)
    return dict(path_length=pl.cpu().numpy(), num_paths=npth.cpu().numpy(),
                vis_edges=vis.cpu().numpy().astype(np.uint64), status=st.cpu().numpy(),
                offsets=off, nodes=r[:, 0].copy(), counts=r[:, 2].astype(np.int32))


def test_noalloc_matches_replay_on_consecutive_calls(sb, small_graphs):
    calls = [("rmat11d", 5, 0, 1500, 2.3), ("ba2k", 6, 777, 1200, 2.3),
             ("rmat11d", 7, 3000, 800, -1.0)]
    for name, seed, first, count, alpha in calls:
        hg = small_graphs[name][0]
        g = sb.Graph.from_host(hg)
        want = g.replay(seed, first, count, alpha)
        got = noalloc_replay(sb, g, seed, first, count, alpha, cap=1 << 20)
        for f in ("path_length", "num_paths", "vis_edges", "status", "offsets", "nodes",
                  "counts"):
            np.testing.assert_array_equal(got[f], want[f], err_msg=f"{name}: {f}")
        assert (got["status"] == 0).all()


def test_noalloc_rejects_oversize_requests(sb, small_graphs):
    hg = small_graphs["ba2k"][0]
    g = sb.Graph.from_host(hg)
    lib = sb.load()
    z = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.silvan_replay_samples_noalloc(g.h, 1, 0, 70000, 2.3, 0, z, z, z, z, z, 0, z, None)
    assert rc == sb.E_CAPACITY
    assert b"65536" in lib.silvan_last_error()


def test_noalloc_record_overflow_marks_only_the_samples_concerned(sb, small_graphs):
    """When the caller's record buffer is too small, the samples whose path
    maps did not fit report SILVAN_E_CAPACITY and leave no records; every
    other sample is exactly the regular replay's."""
    hg = small_graphs["rmat11d"][0]
    g = sb.Graph.from_host(hg)
    want = g.replay(5, 0, 1500, 2.3)
    total = int(want["offsets"][-1])
    got = noalloc_replay(sb, g, 5, 0, 1500, 2.3, cap=total // 3, allow_overflow=True)
    st = got["status"]
    full = np.flatnonzero(st == 0)
    cut = np.flatnonzero(st != 0)
    assert len(full) > 0 and len(cut) > 0
    assert (st[cut] == sb.E_CAPACITY).all()
    # every sample that lost its records had some to lose
    assert (np.diff(want["offsets"])[cut] > 0).all()
    np.testing.assert_array_equal(got["vis_edges"], want["vis_edges"])
    for i in full:
        a, b = got["offsets"][i], got["offsets"][i + 1]
        c, d = want["offsets"][i], want["offsets"][i + 1]
        np.testing.assert_array_equal(got["nodes"][a:b], want["nodes"][c:d])
        np.testing.assert_array_equal(got["counts"][a:b], want["counts"][c:d])
        assert got["path_length"][i] == want["path_length"][i]
        assert got["num_paths"][i] == want["num_paths"][i]
    assert (np.diff(got["offsets"])[cut] == 0).all()


def test_noalloc_rejects_graphs_beyond_the_scratch(sb):
    """A graph with more nodes than one sampler slot of the fixed scratch
    holds is refused before anything is launched, with the limit named."""
    n = 1_489_409  # one node beyond the limit
    g = sb.Graph.from_pairs(np.array([[0, 1], [1, n - 1]], np.uint32), directed=False)
    assert g.n == n
    lib = sb.load()
    z = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.silvan_replay_samples_noalloc(g.h, 1, 0, 10, 2.3, 0, z, z, z, z, z, 0, z, None)
    assert rc == sb.E_CAPACITY
    assert b"1489408" in lib.silvan_last_error()
    small = sb.Graph.from_pairs(np.array([[0, 1], [1, n - 2]], np.uint32), directed=False)
    got = noalloc_replay(sb, small, 3, 0, 64, 2.3, cap=1 << 12)
    want = small.replay(3, 0, 64, 2.3)
    for f in ("path_length", "num_paths", "vis_edges", "status"):
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)
