"""Conditions the reference does not survive are reported as status codes,
sample by sample and for the whole run (include/silvan.h):
  * a 64-bit path count that wraps to 0: the reference takes get_max(0) and
    dies of SIGFPE (silvan/src/Sp_sampler.cpp:172-178); here the sample's
    status is SILVAN_E_OVERFLOW and a run stops with it;
  * more than np_cap paths for one sample (alpha * W, Sp_sampler.cpp:165-170):
    the reference loops for hours; here SILVAN_E_NP_CAP.
Every other sample of the same replay stays exactly the oracle's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ladder(layers):
    """Layer 0 is one node, every later layer two; consecutive layers are
    fully connected, so a pair d layers apart has 2^(d-1) shortest paths."""
    pairs = []
    prev = [0]
    nxt = 1
    for _ in range(layers):
        cur = [nxt, nxt + 1]
        nxt += 2
        pairs += [(a, b) for a in prev for b in cur]
        prev = cur
    return np.array(pairs, np.uint32)


def test_wrapped_path_count_is_reported(sb, port):
    hg = sb.HostGraph.from_pairs(ladder(150), False)
    csr = hg.csr()
    g = sb.Graph.from_host(hg)
    count = 200
    got = g.replay(11, 0, count, -1.0)
    pg = port.graph(csr.n, False, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj, csr.cc)
    overflow = 0
    for i in range(count):
        o = pg.replay(11, i, 1, -1.0)
        if o.zero_modulus:
            overflow += 1
            assert got["status"][i] == sb.E_OVERFLOW, i
        else:
            assert got["status"][i] == 0, i
            assert got["path_length"][i] == o.path_length[0]
            assert got["num_paths"][i] == o.num_paths[0]
            assert got["vis_edges"][i] == o.vis_edges[0]
    assert overflow > 10  # most pairs 65+ layers apart
    with pytest.raises(sb.SilvanError) as e:
        sb.Probabilistic(g, 0.05, 0.1, alpha=-1.0, alpha_given=True, seed=11).run()
    assert e.value.code == sb.E_OVERFLOW


def test_path_cap_is_reported(sb, port, small_graphs):
    hg, csr, _ = small_graphs["ba2k"]
    g = sb.Graph.from_host(hg)
    cap, count = 4, 400
    got = g.replay(3, 0, count, 2.3, np_cap=cap)
    o = port.graph(csr.n, False, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj,
                   csr.cc).replay(3, 0, count, 2.3)
    over = o.num_paths > cap
    assert over.any() and (~over).any()
    np.testing.assert_array_equal(got["status"][over], sb.E_NP_CAP)
    np.testing.assert_array_equal(got["status"][~over], 0)
    np.testing.assert_array_equal(got["num_paths"][~over], o.num_paths[~over])
    with pytest.raises(sb.SilvanError) as e:
        sb.Probabilistic(g, 0.05, 0.1, np_cap=cap, seed=3).run()
    assert e.value.code == sb.E_NP_CAP


def test_lattice_at_default_alpha_stops_with_the_cap(sb):
    """A 48 x 48 lattice at the reference's default alpha 2.3: path counts
    explode (the reference does not finish); the run ends with NP_CAP."""
    hg = sb.HostGraph.from_pairs(sb.grid(48, 0.0, 0.0, 1), False)
    with pytest.raises(sb.SilvanError) as e:
        sb.Probabilistic(sb.Graph.from_host(hg), 0.05, 0.1, seed=1).run()
    assert e.value.code == sb.E_NP_CAP
