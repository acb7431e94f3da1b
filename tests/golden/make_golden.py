"""Generates the committed golden fixtures of tests/golden/.

The fixtures are outputs of the REFERENCE'S OWN SOURCES (silvan/src/*.cpp,
unmodified) compiled with the Philox stream into oracle/_ref/libsilvan_ref.so
by oracle/Makefile; they pin the CPU oracle and the device path on machines
where the reference is not available.

For every graph below (written by this library's seeded generators and
committed as small edge-list files):
  * per-sample replay of samples [0, 600) for alpha 2.3 and -1 (path length,
    number of paths, edges visited, path map);
  * a full estimator run (Probabilistic::run with one thread): the final
    approx / emp_wimpy_vars / mcrade / partition counters, the schedule
    scalars and the ranking list.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built with the
reference sources present).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Ref  # noqa: E402

# name -> (generator, kwargs, directed, run kwargs)
GRAPHS = {
    "ba600": ("ba", dict(n=600, m=3, seed=21), False, dict(eps=0.03, delta=0.1)),
    "rmat9d": ("rmat", dict(scale=9, edge_factor=8, seed=22, directed=True), True,
               dict(eps=0.03, delta=0.1)),
    "er500": ("er", dict(n=500, mean_degree=4.0, seed=23), False, dict(eps=0.04, delta=0.1)),
    "grid20": ("grid", dict(side=20, delete_frac=0.05, shortcut_frac=0.002, seed=24), False,
               dict(eps=0.05, delta=0.1, alpha=0.0, alpha_given=True)),
    "ba600_top5": ("ba", dict(n=600, m=3, seed=21), False, dict(eps=0.2, delta=0.1, k=5)),
}
SEED = 1234
REPLAY = 600


def pairs_for(kind, kw):
    import silvan_b200 as sb
    if kind == "ba":
        return sb.barabasi_albert(kw["n"], kw["m"], kw["seed"])
    if kind == "er":
        return sb.erdos_renyi(kw["n"], kw["mean_degree"], kw["seed"])
    if kind == "rmat":
        return sb.rmat(kw["scale"], kw["edge_factor"], kw["seed"], kw["directed"])
    return sb.grid(kw["side"], kw["delete_frac"], kw["shortcut_frac"], kw["seed"])


def main():
    import silvan_b200 as sb
    ref = Ref()
    manifest = {}
    for name, (kind, kw, directed, runkw) in GRAPHS.items():
        gname = name.split("_")[0]
        path = os.path.join(HERE, gname + ".txt")
        if not os.path.exists(path):
            sb.write_edge_list(path, pairs_for(kind, kw))
        rg = ref.graph(path, directed)
        D, cc, nc = rg.diameter()
        oo, oa, io, ia = rg.csr()
        out = dict(n=np.array(rg.n), diameter=np.array(D), n_components=np.array(nc), cc=cc,
                   out_off=oo, out_adj=oa, in_off=io, in_adj=ia)
        if name == gname:
            for alpha, tag in ((2.3, "a23"), (-1.0, "am1")):
                r = rg.replay(SEED, 0, REPLAY, alpha)
                out.update({f"{tag}_path_length": r.path_length, f"{tag}_num_paths": r.num_paths,
                            f"{tag}_vis_edges": r.vis_edges, f"{tag}_offsets": r.offsets,
                            f"{tag}_nodes": r.nodes, f"{tag}_counts": r.counts})
        res = ref.run(path, directed, seed=SEED, **runkw)
        for f in ("approx", "wimpy", "mcrade", "partition_index", "ranking_elements",
                  "ranking_values", "sp_lengths", "epsilon_partition", "partition_ids"):
            out["run_" + f] = res[f]
        scal = {f: res[f] for f in ("num_samples", "vis_edges", "iteration_index",
                                    "num_partitions", "omega", "first_stopping_samples",
                                    "last_stopping_samples", "alpha_sp_sampling", "sup_bcest",
                                    "sup_emp_wimpy_var", "union_sample")}
        if runkw.get("k", 0) > 0:
            scal["numresults_topk"] = res["numresults_topk"]
            scal["eps_final_topk"] = res["eps_final_topk"]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = dict(graph=gname + ".txt", directed=directed, generator=kind,
                              generator_args=kw, run=runkw, seed=SEED, replay=REPLAY,
                              scalars=scal)
        print(name, "n", rg.n, "D", D, "samples", res["num_samples"])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
