"""The C-ABI library loads without a GPU and exports every function that
include/silvan.h declares; the CLI rejects bad arguments the way the
reference binary does (silvan/main.cpp:74-153) before touching a device."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "silvan.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(silvan_[a-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_header_declarations_exported(sb):
    lib = sb.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(sb.EXPORTS) == names


def test_library_is_in_tree(sb):
    assert os.path.dirname(sb.LIB_PATH) == os.path.join(ROOT, "silvan_b200")
    assert os.path.exists(sb.CLI_PATH)


def run_cli(sb, *args):
    return subprocess.run([sb.CLI_PATH, *args], capture_output=True, text=True, timeout=60)


def test_cli_help(sb):
    r = run_cli(sb, "-h")
    assert r.returncode == 0
    assert "USAGE:" in r.stderr


@pytest.mark.parametrize("args,msg", [
    ((), "Wrong number of arguments"),
    (("0.5", "0.1"), "Wrong number of arguments"),
    (("1.5", "0.1", "x"), "The error err should be greater than 0"),
    (("0.1", "0", "x"), "Delta should be greater than 0"),
    (("-k", "-3", "0.1", "0.1", "x"), "The value k should be between"),
    (("-v", "-1", "0.1", "0.1", "x"), "The verbosity should be"),
])
def test_cli_argument_errors(sb, args, msg):
    r = run_cli(sb, *args)
    assert r.returncode == 1
    assert msg in r.stderr
    assert "USAGE:" in r.stderr


def test_cli_missing_graph(sb, tmp_path):
    r = run_cli(sb, "0.1", "0.1", str(tmp_path / "none.txt"))
    assert r.returncode == 1
    assert "Problems with input graph file" in r.stderr
