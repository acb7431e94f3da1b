"""Builds the in-tree native artefacts of silvan_b200.

* ``silvan_b200/libsilvan_b200.so`` -- CUDA kernels for sm_100a, the host
  engine and the C-ABI of ``include/silvan.h``.
* ``silvan_b200/bin/silvan`` -- the drop-in command-line binary.

Run ``python -m silvan_b200.build`` (or call ``build()``).  Compilation is
incremental on source timestamps; nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libsilvan_b200.so")
BIN = os.path.join(PKG, "bin", "silvan")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["graph_host.cpp", "gen.cpp", "graph_dev.cu", "sampler.cu", "counters.cu", "engine.cu",
           "server.cu", "noalloc.cu", "ingest.cu", "components.cu", "brandes.cu", "capi.cu"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _headers():
    hs = [os.path.join(INC, "silvan.h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False) -> str:
    nvcc, cxx = _nvcc(), _host_cxx()
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    hdrs = _headers()
    common = ["-std=c++17", "-O3", "-lineinfo", "-ccbin", cxx, "-Xcompiler", "-fPIC",
              "-I" + INC, "-I" + CSRC] + ARCH
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            cmd = [nvcc] + common + (["-x", "cu"] if s.endswith(".cu") else []) + \
                ["-c", src, "-o", obj]
            jobs.append(cmd)
    log = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            log.append(out)
    if jobs or _stale(LIB, objs):
        log.append(_run([nvcc, "-shared", "-ccbin", cxx] + ARCH + objs + ["-o", LIB]))
    cli = os.path.join(CSRC, "silvan_cli.cpp")
    if _stale(BIN, [cli, LIB, os.path.join(INC, "silvan.h")]):
        log.append(_run([cxx, "-std=c++17", "-O2", "-I" + INC, cli, "-o", BIN,
                         "-L" + PKG, "-lsilvan_b200", "-Wl,-rpath,$ORIGIN/.."]))
    text = "".join(log)
    if verbose and text:
        print(text)
    return text


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
    print(BIN)
