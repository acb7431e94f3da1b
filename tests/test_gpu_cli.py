"""The drop-in binary end to end: scripts/run_silvan.py runs `silvan` with the
reference's flags, scrapes fixed stdout patterns into its `;`-separated
results row (scripts/run_silvan.py:79-100) and reads the -o file.  The binary
here must print those lines with the oracle's values, write the -o file in
the reference's format (Probabilistic.cpp:1116-1136: `id,value` with six
significant digits; every node in absolute mode, the ranked nodes in top-k
mode), and print the same set of scraped lines as the reference binary.
The unmodified wrapper itself runs in tests/test_cli_wrapper.py over the
drop-in output recorded in tests/golden/cli/; the last test here keeps that
recording equal to what the live binary prints."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, port_graph

pytestmark = pytest.mark.gpu

# the patterns of scripts/run_silvan.py:79, in its order
PATTERNS = ["Finished after ", "Total time: ", "estimated diameter of the graph: ",
            "First pass finished after ", "time for first pass ", "MCRADE STOPS WITH eps ",
            "MCRADE STOPS at iteration ", "top-1 bc first pass: ", "    top1bc_upperbound: ",
            "avg_diam_firstpass: ", "avg_diam_upperbound: ", "max_num_samples: ",
            "Time bfs: ", "Time critical: ", "eps_final_topk "]

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "silvan")


def scrape(stdout):
    """run_silvan.py's get_result over every pattern: the text after the
    pattern on the last line that contains it ('' when none does)."""
    out = []
    for pat in PATTERNS:
        val = ""
        for line in stdout.splitlines():
            if pat in line:
                val = line[len(pat):]
        val = val.replace(" iterations.", "").replace(" iteration", "")
        out.append(val)
    return out


def write_graph(path, csr):
    with open(path, "w") as f:
        for u in range(csr.n):
            for v in csr.out_adj[csr.out_off[u]:csr.out_off[u + 1]]:
                if csr.directed or u <= v:
                    f.write(f"{u} {v}\n")


def run_bin(binary, args, env=None):
    return subprocess.run([binary, *args], capture_output=True, text=True, timeout=600, env=env)


@pytest.mark.parametrize("name,flags", [("ba2k", []), ("rmat11d", ["-d"]),
                                        ("rmat11u", ["-k", "5"])])
def test_cli_output_and_file(sb, port, small_graphs, tmp_path, name, flags):
    hg, csr, directed = small_graphs[name]
    gpath = str(tmp_path / "g.txt")
    write_graph(gpath, csr)
    out = str(tmp_path / "out.txt")
    eps, delta = (0.1, 0.1) if "-k" in flags else (0.03, 0.1)
    r = run_bin(sb.CLI_PATH, [*flags, "--seed", "7", "-o", out, str(eps), str(delta), gpath])
    assert r.returncode == 0, r.stderr
    row = scrape(r.stdout)
    k = int(flags[flags.index("-k") + 1]) if "-k" in flags else 0
    o = port_graph(port, csr).run(csr.diameter, eps, delta, k=k, seed=7)
    assert row[0] == str(o["num_samples"])
    assert row[2] == str(csr.diameter)
    assert row[3] == str(o["first_pass_samples"])
    float(row[1]), float(row[12]), float(row[13])
    if k == 0:
        assert float(row[11]) > 0  # the m_hat bound after pass 1
    lines = open(out).read().splitlines()
    if k == 0:
        assert len(lines) == csr.n
        want = o["approx"] / o["num_samples"]
        ids = np.array([int(ln.split(",")[0]) for ln in lines])
        vals = np.array([float(ln.split(",")[1]) for ln in lines])
        np.testing.assert_array_equal(ids, np.arange(csr.n))
        np.testing.assert_allclose(vals, want, rtol=5e-6, atol=0)
        assert lines[0] == f"0,{want[0]:.6g}"
    else:
        cnt = o["numresults_topk"]
        assert len(lines) == cnt
        ids = [int(ln.split(",")[0]) for ln in lines]
        assert ids == list(o["ranking_elements"][:cnt])
    if os.path.exists(REF_BIN):
        env = dict(os.environ, OMP_NUM_THREADS="1")
        rr = run_bin(REF_BIN, [*flags, "-o", str(tmp_path / "ref.txt"), str(eps), str(delta),
                               gpath], env=env)
        assert rr.returncode == 0, rr.stderr
        ref_row = scrape(rr.stdout)
        # the MCRADE lines depend on which stopping condition fired, which
        # depends on the random stream (the reference binary keeps its LCG)
        stable = [i for i, p in enumerate(PATTERNS) if not p.startswith("MCRADE")]
        assert [bool(row[i]) for i in stable] == [bool(ref_row[i]) for i in stable]
        assert row[2] == ref_row[2]
        if k == 0:
            assert row[3] == ref_row[3]  # tau-sized first pass


def test_cli_assist_items_gives_the_same_output(sb, small_graphs, tmp_path):
    """--assist-items only changes how wide levels are expanded (by several
    sampler CTAs), never the estimates: the -o files and the sample counts
    of a run that posts every level, one that posts none and the default
    agree."""
    hg, csr, directed = small_graphs["rmat11d"]
    gpath = str(tmp_path / "g.txt")
    write_graph(gpath, csr)
    outs = []
    for items in (None, "1", "4294967295"):
        out = str(tmp_path / f"out_{items}.txt")
        extra = [] if items is None else ["--assist-items", items]
        r = run_bin(sb.CLI_PATH, ["-d", "--seed", "3", *extra, "-o", out, "0.03", "0.1", gpath])
        assert r.returncode == 0, r.stderr
        row = scrape(r.stdout)
        outs.append((row[0], row[3], open(out).read()))
    assert outs[0] == outs[1] == outs[2]


# Lines of the drop-in's output that do not depend on wall time, by pattern.
STABLE_LINES = ["Finished after ", "estimated diameter of the graph: ",
                "First pass finished after ", "MCRADE STOPS WITH eps ",
                "MCRADE STOPS at iteration ", "max_num_samples: ", "eps_final_topk "]


def _cli_cases():
    import json
    path = os.path.join(ROOT, "tests", "golden", "cli", "cases.json")
    with open(path) as f:
        return json.load(f)


@pytest.mark.parametrize("name", sorted(_cli_cases()))
def test_cli_fixture_matches_live_binary(sb, name):
    """The drop-in output that tests/test_cli_wrapper.py feeds to the
    reference's unmodified run_silvan.py (tests/golden/cli/) is what the live
    binary prints for the arguments that wrapper builds: every line of the
    patterns it scrapes that does not depend on wall time is identical."""
    c = _cli_cases()[name]
    gdir = os.path.join(ROOT, "tests", "golden")
    argv = [os.path.join(gdir, c["graph"]) if a == "@GRAPH@" else a for a in c["binary_argv"]]
    r = run_bin(sb.CLI_PATH, argv)
    assert r.returncode == 0, r.stderr
    want = open(os.path.join(gdir, "cli", f"{name}.stdout.txt")).read()

    def stable(text):
        return [ln for ln in text.splitlines() if any(p in ln for p in STABLE_LINES)]

    assert stable(r.stdout) == stable(want)
    assert stable(r.stdout)
