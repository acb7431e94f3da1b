"""The reference's own CLI wrapper, scripts/run_silvan.py, unmodified, in
front of the drop-in binary (scripts/run_silvan.py:18,50-99): it maps its
flags to the binary's, runs `../silvan/silvan ... > output.txt`, scrapes
fifteen stdout patterns and appends one `;`-separated row to
results_silvan.csv (results_silvan_topk.csv in top-k mode).

The wrapper is read from the reference checkout (it never enters this
repository) and the drop-in binary needs a GPU, so the drop-in's side comes
from fixtures (tests/golden/make_cli_golden.py): the binary arguments the
wrapper builds for each case, and the drop-in's standard output for exactly
those arguments, recorded on a B200 (tests/test_gpu_cli.py keeps the
fixture tied to the live binary).  Here the unmodified wrapper runs over
that output and over the reference binary itself (oracle/_ref/silvan, one
thread), and the two results rows must agree: the same columns filled, the
same diameter bound and, in absolute mode, the same first-pass size (tau,
which does not depend on the random stream)."""
import json
import os
import sys
import tempfile

import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_cli_golden as mk  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "silvan")
HEADER = ("graph_name;epsilon;delta;k;type;m_hat_enabled;emp_peel_enabled;emp_peel_a;alpha;m;"
          "time;diameter;first_samples;first_time;eps_mcera;iter_index_mcera;top1_est;top1_ub;"
          "avg_spl_est;avg_spl_ub;samples_bound;time_bfs;time_critical;eps_final_topk")
COLS = HEADER.split(";")

pytestmark = pytest.mark.skipif(mk.reference_wrapper() is None,
                                reason="the reference's scripts/run_silvan.py is not present")

with open(mk.CASES) as _f:
    CASES = json.load(_f)


def results(scripts, k):
    path = os.path.join(scripts, "results_silvan_topk.csv" if k else "results_silvan.csv")
    lines = open(path).read().splitlines()
    assert lines[0] == HEADER
    assert len(lines) == 2
    row = lines[1].split(";")
    assert len(row) == len(COLS)
    return dict(zip(COLS, row))


def wrapper_row(name, binary=None):
    c = CASES[name]
    k = int(c["wrapper_flags"][c["wrapper_flags"].index("-k") + 1]) \
        if "-k" in c["wrapper_flags"] else 0
    with tempfile.TemporaryDirectory() as tmp:
        text = None
        if binary is None:
            text = open(os.path.join(mk.CLI_DIR, f"{name}.stdout.txt")).read()
        scripts, bindir = mk.wrapper_sandbox(tmp, binary=binary, stdout_text=text)
        graph = os.path.join(tmp, "graph.txt")
        with open(os.path.join(mk.HERE, c["graph"])) as src, open(graph, "w") as dst:
            dst.write(src.read())
        r = mk.run_wrapper(scripts, graph, c["wrapper_flags"], env={"OMP_NUM_THREADS": "1"})
        assert r.returncode == 0, r.stderr
        assert "terminated with errors" not in r.stdout
        if binary is None:
            # the wrapper still builds the argument list the fixture was made for
            argv = open(os.path.join(bindir, "argv.txt")).read().splitlines()
            assert [mk.GRAPH_TOKEN if a == graph else a for a in argv] == c["binary_argv"]
        return results(scripts, k), k


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference binary not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_wrapper_rows_agree(name):
    got, k = wrapper_row(name)
    want, _ = wrapper_row(name, binary=REF_BIN)
    for col in COLS[1:9]:  # the wrapper's own arguments
        assert got[col] == want[col], col
    # every column the reference fills is filled, and only those; the
    # MCRADE columns depend on which stopping condition fired, which depends
    # on the random stream (the reference binary keeps its own LCG)
    for col in COLS[9:]:
        if col in ("eps_mcera", "iter_index_mcera"):
            continue
        assert bool(got[col]) == bool(want[col]), (col, got[col], want[col])
    assert got["diameter"] == want["diameter"]
    if k == 0:
        assert got["first_samples"] == want["first_samples"]  # tau
    for col in COLS[9:]:
        if got[col]:
            float(got[col])
