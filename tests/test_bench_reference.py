"""The reference arm of bench.py (`--impl reference`): the reference's own
OpenMP build of the estimator, timed on the host cores on the benchmark's
workload, printed as one JSON line with the same metric as the GPU arm.
Under torchrun only rank 0 runs it; the other ranks exit 0 without output."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libsilvan_refbench.so")


def run_bench(args, env=None):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                          capture_output=True, text=True, timeout=300, env=e, cwd=ROOT)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
def test_reference_arm_line():
    r = run_bench(["--impl", "reference", "--config", "ba10k", "--steps", "1", "--warmup", "0"])
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "paths/sec" and d["unit"] == "paths/s" and d["higher_is_better"]
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "ba_n10000_m5_seed1"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "paths/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run_bench(["--impl", "reference", "--config", "ba10k", "--steps", "1", "--warmup", "0"],
                  env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build not present")
def test_reference_arm_loads_no_product_code():
    """The reference arm generates its graph inside the reference harness
    (oracle/_ref/libsilvan_refbench.so), so its process maps no library of
    this project and imports no part of the package; the graph is the GPU
    arm's graph (same CSR checksum)."""
    code = (
        "import sys, json, types; sys.argv = ['bench.py', '--impl', 'reference', '--config', "
        "'ba10k', '--steps', '1', '--warmup', '0']; import bench; bench.main(); "
        "maps = open('/proc/self/maps').read(); "
        "print(json.dumps({'mods': [m for m in sys.modules if m.startswith('silvan_b200')], "
        "'lib': 'libsilvan_b200' in maps, 'ref': 'libsilvan_refbench' in maps}))")
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env=e, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert probe == {"mods": [], "lib": False, "ref": True}
    import bench
    import silvan_b200 as sb
    csr = bench.make_graph(bench.CONFIGS["ba10k"]).csr()
    assert line["config"]["csr_sha1_16"] == bench.csr_checksum(csr)
