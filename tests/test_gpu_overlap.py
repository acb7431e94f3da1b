"""Stopping-rule checks overlapped with the next commit round.

In absolute mode the engine commits the samples up to the next schedule
point while the host evaluates a check (silvan/src/Probabilistic.cpp:
1060-1087), with a journal of what that round changes; the round is kept
when the check lets the run go on with the same next point, and undone when
the check stops the run or moves the point (the m_hat bound lowering omega
below it).  Either way the run must be the one that evaluates every check
before committing further: the same counters bit for bit, the same scalars,
the same status lines, and the oracle's results."""
import tempfile

import numpy as np
import pytest

from conftest import port_graph

pytestmark = pytest.mark.gpu

SCALARS = ["num_samples", "vis_edges", "iteration_index", "num_partitions", "omega",
           "first_stopping_samples", "last_stopping_samples", "alpha_sp_sampling",
           "first_pass_samples", "stop_reason", "void_samples", "backtracked_paths",
           "checks", "eps_stop", "sup_bcest", "sup_emp_wimpy_var", "max_num_samples"]


def run(sb, g, eps, delta, **kw):
    job = sb.Probabilistic(g, eps, delta, **kw)
    return job, job.run()


def lines_without_times(text):
    return [ln for ln in text.splitlines() if "time" not in ln and "seconds" not in ln]


def same_run(a, b):
    (ja, ra), (jb, rb) = a, b
    for f in SCALARS:
        assert ra[f] == rb[f], (f, ra[f], rb[f])
    ca, cb = ja.counters(), jb.counters()
    for f in ("approx", "wimpy", "mcrade", "partition_index"):
        np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)


@pytest.mark.parametrize("name,eps,kw", [
    ("rmat11d", 0.02, {}),
    ("ba2k", 0.02, {}),
    ("er3k", 0.03, {"m_hat": False}),
    ("grid40", 0.03, {"alpha": 0.0, "alpha_given": True}),
])
def test_overlapped_checks_match_serial_and_oracle(sb, port, small_graphs, name, eps, kw):
    hg, csr, _ = small_graphs[name]
    g = sb.Graph.from_host(hg)
    ov = run(sb, g, eps, 0.1, seed=21, **kw)
    se = run(sb, g, eps, 0.1, seed=21, serial_checks=True, **kw)
    same_run(ov, se)
    assert se[1]["overlapped_checks"] == 0
    if ov[1]["checks"] > 1:
        assert ov[1]["overlapped_checks"] > 0
    okw = dict(kw)
    if "m_hat" in okw:
        okw["mhat"] = okw.pop("m_hat")
    o = port_graph(port, csr).run(csr.diameter, eps, 0.1, seed=21, **okw)
    for f in ("num_samples", "iteration_index", "omega", "last_stopping_samples",
              "stop_reason"):
        assert ov[1][f] == o[f], (f, ov[1][f], o[f])
    np.testing.assert_array_equal(ov[0].counters()["mcrade"], o["mcrade"])


@pytest.mark.parametrize("seed", [3, 4, 5])
def test_overlap_with_moving_omega(sb, seed):
    """A directed R-MAT graph where the m_hat bound lowers omega at every
    check, so that the last kept point moves and the journaled round after
    it is undone; the status lines must match too."""
    pairs = sb.rmat(15, 16, 7, True)
    g = sb.Graph.from_host(sb.HostGraph.from_pairs(pairs, True))
    logs, runs = [], []
    for serial in (False, True):
        job = sb.Probabilistic(g, 0.01, 0.05, seed=seed, serial_checks=serial)
        with tempfile.TemporaryFile("w+") as f:
            res = job.run(log=f)
            f.seek(0)
            logs.append(lines_without_times(f.read()))
        runs.append((job, res))
    same_run(runs[0], runs[1])
    assert logs[0] == logs[1]
    assert runs[1][1]["overlapped_checks"] == 0
