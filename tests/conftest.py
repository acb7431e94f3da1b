"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device; everything else
runs on the CPU (oracle, host ingest, C-ABI exports, CLI argument errors)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def sb():
    import silvan_b200
    silvan_b200.load()
    return silvan_b200


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port
    return Port()


# Small graphs used across the parity tests: (name, generator kwargs, directed).
SMALL_GRAPHS = {
    "ba2k": ("ba", dict(n=2000, m=4, seed=11), False),
    "er3k": ("er", dict(n=3000, mean_degree=5.0, seed=12), False),
    "rmat11d": ("rmat", dict(scale=11, edge_factor=8, seed=13, directed=True), True),
    "rmat11u": ("rmat", dict(scale=11, edge_factor=6, seed=14, directed=False), False),
    "grid40": ("grid", dict(side=40, delete_frac=0.05, shortcut_frac=0.001, seed=15), False),
}


def make_pairs(sb, kind, kw):
    if kind == "ba":
        return sb.barabasi_albert(kw["n"], kw["m"], kw["seed"])
    if kind == "er":
        return sb.erdos_renyi(kw["n"], kw["mean_degree"], kw["seed"])
    if kind == "rmat":
        return sb.rmat(kw["scale"], kw["edge_factor"], kw["seed"], kw["directed"])
    if kind == "grid":
        return sb.grid(kw["side"], kw["delete_frac"], kw["shortcut_frac"], kw["seed"])
    raise ValueError(kind)


@pytest.fixture(scope="session")
def small_graphs(sb):
    """name -> (HostGraph, CSR, directed)"""
    out = {}
    for name, (kind, kw, directed) in SMALL_GRAPHS.items():
        pairs = make_pairs(sb, kind, kw)
        hg = sb.HostGraph.from_pairs(pairs, directed)
        out[name] = (hg, hg.csr(), directed)
    return out


def port_graph(port, csr):
    return port.graph(csr.n, csr.directed, csr.out_off, csr.out_adj, csr.in_off, csr.in_adj,
                      csr.cc)
