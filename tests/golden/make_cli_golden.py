"""Fixtures of the end-to-end test of the reference's CLI wrapper
(scripts/run_silvan.py) in front of the drop-in binary.

The wrapper is the reference's own Python script.  It stays where it lies
(it is read from the reference checkout, never copied into this
repository), so it can run only on a machine that has the reference, and the
drop-in binary can run only on a machine with a GPU.  The fixtures connect
the two:

  argv    (needs the reference; no GPU) runs the unmodified wrapper for
          every case below in a scratch directory whose ../silvan/silvan is a
          stub that records its argument list, and writes
          tests/golden/cli/cases.json: the wrapper's flags and the binary
          arguments it produced (the graph path as a placeholder);
  stdout  (needs a GPU; no reference) runs the drop-in binary with each
          recorded argument list on the committed graph file and writes its
          standard output to <out_dir>/<case>.stdout.txt, which is then
          committed as tests/golden/cli/<case>.stdout.txt.

tests/test_cli_wrapper.py runs the unmodified wrapper over the recorded
output and over the reference binary itself and compares the results rows;
tests/test_gpu_cli.py checks that the live binary still prints what the
fixture holds.

Usage: python tests/golden/make_cli_golden.py argv
       python tests/golden/make_cli_golden.py stdout <out_dir>
"""
import json
import os
import shutil
import stat
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CLI_DIR = os.path.join(HERE, "cli")
CASES = os.path.join(CLI_DIR, "cases.json")
GRAPH_TOKEN = "@GRAPH@"

# name -> (committed graph file, wrapper flags after -db)
CASE_FLAGS = {
    "abs_undirected": ("ba600.txt", ["-e", "0.03", "-d", "0.1"]),
    "abs_directed": ("rmat9d.txt", ["-t", "1", "-e", "0.03", "-d", "0.1"]),
    "topk": ("ba600.txt", ["-k", "5", "-e", "0.2", "-d", "0.1"]),
    "options": ("er500.txt", ["-e", "0.04", "-d", "0.1", "-s", "3.0", "-a", "3", "-mh", "0"]),
    "no_peeling": ("er500.txt", ["-e", "0.04", "-d", "0.1", "-eempp", "0"]),
}

STUB = """#!/bin/sh
# stands in for ../silvan/silvan: records the argument list, prints the
# output it is given (if any)
d=$(dirname "$0")
printf '%s\\n' "$@" > "$d/argv.txt"
if [ -f "$d/stdout.txt" ]; then cat "$d/stdout.txt"; fi
"""


def reference_wrapper():
    """Path of the reference's scripts/run_silvan.py, or None."""
    src = os.environ.get("SILVAN_REFERENCE_SRC", "/root/reference/silvan")
    p = os.path.join(os.path.dirname(src.rstrip("/")), "scripts", "run_silvan.py")
    return p if os.path.exists(p) else None


def wrapper_sandbox(tmp, binary=None, stdout_text=None):
    """tmp/scripts/run_silvan.py (the reference's file, unmodified) and
    tmp/silvan/silvan: the given binary, or the recording stub."""
    scripts = os.path.join(tmp, "scripts")
    bindir = os.path.join(tmp, "silvan")
    os.makedirs(scripts, exist_ok=True)
    os.makedirs(bindir, exist_ok=True)
    shutil.copyfile(reference_wrapper(), os.path.join(scripts, "run_silvan.py"))
    exe = os.path.join(bindir, "silvan")
    if binary:
        os.symlink(os.path.abspath(binary), exe)
    else:
        with open(exe, "w") as f:
            f.write(STUB)
        os.chmod(exe, os.stat(exe).st_mode | stat.S_IXUSR | stat.S_IXGRP | stat.S_IXOTH)
        if stdout_text is not None:
            with open(os.path.join(bindir, "stdout.txt"), "w") as f:
                f.write(stdout_text)
    return scripts, bindir


def run_wrapper(scripts, graph, flags, env=None):
    return subprocess.run([sys.executable, "run_silvan.py", "-db", graph, *flags], cwd=scripts,
                          capture_output=True, text=True, timeout=600,
                          env=dict(os.environ, **(env or {})))


def record_argv():
    if reference_wrapper() is None:
        sys.exit("the reference's scripts/run_silvan.py is not available")
    cases = {}
    for name, (gfile, flags) in CASE_FLAGS.items():
        with tempfile.TemporaryDirectory() as tmp:
            scripts, bindir = wrapper_sandbox(tmp)
            graph = os.path.join(tmp, "graph.txt")
            shutil.copyfile(os.path.join(HERE, gfile), graph)
            r = run_wrapper(scripts, graph, flags)
            if r.returncode != 0:
                sys.exit(r.stderr)
            argv = open(os.path.join(bindir, "argv.txt")).read().splitlines()
        cases[name] = {"graph": gfile, "wrapper_flags": flags,
                       "binary_argv": [GRAPH_TOKEN if a == graph else a for a in argv]}
    os.makedirs(CLI_DIR, exist_ok=True)
    with open(CASES, "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"wrote {CASES}")


def record_stdout(out_dir):
    sys.path.insert(0, ROOT)
    import silvan_b200 as sb
    os.makedirs(out_dir, exist_ok=True)
    with open(CASES) as f:
        cases = json.load(f)
    for name, c in sorted(cases.items()):
        argv = [os.path.join(HERE, c["graph"]) if a == GRAPH_TOKEN else a
                for a in c["binary_argv"]]
        r = subprocess.run([sb.CLI_PATH, *argv], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            sys.exit(f"{name}: {r.stderr}")
        with open(os.path.join(out_dir, f"{name}.stdout.txt"), "w") as f:
            f.write(r.stdout)
        print(f"{name}: {len(r.stdout.splitlines())} lines")


if __name__ == "__main__":
    if len(sys.argv) >= 2 and sys.argv[1] == "argv":
        record_argv()
    elif len(sys.argv) >= 3 and sys.argv[1] == "stdout":
        record_stdout(sys.argv[2])
    else:
        sys.exit(__doc__)
