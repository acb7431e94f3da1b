"""The first sampler rounds of one estimation job on a generated benchmark
graph, with a chosen slot count and CTA size: a bounded workload (one
persistent sampler launch of about a thousand samples) for profiler captures
of sampler_kernel and the commit kernels.

    python -m silvan_b200.profile_round --graph grid2048 --slots 16 --block 512

A complete estimation of these graphs runs many launches over seconds; this
runs `--rounds` rounds of the job's own schedule and stops.
"""
import argparse
import time

import silvan_b200 as sb

GRAPHS = {
    # name: (generator, job parameters)
    "rmat20": (lambda: sb.HostGraph.from_pairs(sb.rmat(20, 16, 2, True), True),
               dict(eps=0.005, delta=0.05)),
    # the same generator at 2^18 and 2^17 nodes: every resident slot fits in
    # a few GB, so a capture can run the sampler at full occupancy
    "rmat18": (lambda: sb.HostGraph.from_pairs(sb.rmat(18, 16, 2, True), True),
               dict(eps=0.005, delta=0.05)),
    "rmat17": (lambda: sb.HostGraph.from_pairs(sb.rmat(17, 16, 2, True), True),
               dict(eps=0.005, delta=0.05)),
    "grid2048": (lambda: sb.HostGraph.from_pairs(sb.grid(2048, 0.05, 0.001, 3), False),
                 dict(eps=0.1, delta=0.05, k=10, alpha=0.0, alpha_given=True)),
    "ba10k": (lambda: sb.HostGraph.from_pairs(sb.barabasi_albert(10000, 5, 1), False),
              dict(eps=0.01, delta=0.05)),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--graph", default="rmat20", choices=sorted(GRAPHS))
    ap.add_argument("--slots", type=int, default=32)
    ap.add_argument("--block", type=int, default=512, choices=[128, 256, 512, 1024])
    ap.add_argument("--rounds", type=int, default=1)
    args = ap.parse_args()
    make, kw = GRAPHS[args.graph]
    g = sb.Graph.from_host(make())
    job = sb.Probabilistic(g, kw.pop("eps"), kw.pop("delta"), slots=args.slots, block=args.block,
                           **kw)
    t0 = time.perf_counter()
    st = job.step(args.rounds)
    print(f"{args.graph}: {args.rounds} round(s) in {time.perf_counter() - t0:.3f} s, "
          f"pass {st['pass_']}, samples {st['samples']}, done {st['done']}")


if __name__ == "__main__":
    main()
