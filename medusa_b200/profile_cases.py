"""One measured case per invocation, for profilers (ncu launch lists and
single-kernel captures) and quick timings:

    python -m medusa_b200.profile_cases CASE [--reps N] [--hostloop]

CASE: c2-bfs, c2-sssp (R-MAT 2^20 / 2^24, source 0), c2-msssp (the same
graph, SSSP from sources 0..31 in one batched traversal; NAME-msssp on any
graph below), c4a-msssp (R-MAT
2^22 / 2^26, sources 0..31), c1-pr (uniform
2^18 / 2^22, 10 supersteps), c5-bfs, c5-sssp (R-MAT 2^24 / 2^28,
(0.57,0.19,0.19,0.05)), c5-pr (20 supersteps), c3-bfs, c3-sssp (1448^2
grid), c5s-bfs, c5s-sssp, c5s-pr (the C5 generator at 2^21 / 2^25: a case
small enough for full ncu captures), unif-bfs, unif-sssp (uniform random
2^20 / 2^24, weights 1..1000), path-bfs, path-sssp (a directed path
of 200 vertices, persistent tail off: every superstep is one select kernel
and one push over a one-vertex frontier -- the fixed cost of a superstep).
--pr-order fixed|reference picks PageRank's summation order (default: the
library's, the reference's).  Prints one line per repetition with
the library's device time.  --hostloop runs the host-driven loop (kernels in
conditional-node graphs are invisible to ncu); --trace prints each superstep
of the last repetition (BFS 8 B per frontier out-edge + 20 B per frontier
vertex, SSSP 12 + 20, as algorithmic bytes).  --set NAME=VALUE sets a
tunable (medusa_b200.api.TUNABLES) before the runs; repeatable.
--sssp-delta W sets the single-source near-far width."""
import argparse
import sys

import numpy as np

from . import api

SEED = 1


def params(case):
    if case.startswith("c2"):
        return api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=SEED, wmin=1, wmax=1000)
    if case.startswith("c4a"):
        return api.rmat_params(22, 1 << 26, 0.45, 0.15, 0.15, seed=SEED, wmin=1, wmax=1000)
    if case.startswith("c1"):
        return api.uniform_params(1 << 18, 1 << 22, seed=SEED)
    if case.startswith("unif"):
        return api.uniform_params(1 << 20, 1 << 24, seed=SEED, wmin=1, wmax=1000)
    if case.startswith("c5s"):
        return api.rmat_params(21, 1 << 25, 0.57, 0.19, 0.19, seed=SEED, wmin=1, wmax=1000)
    if case.startswith("c5"):
        return api.rmat_params(24, 1 << 28, 0.57, 0.19, 0.19, seed=SEED, wmin=1, wmax=1000)
    if case.startswith("c3"):
        return api.grid_params(1448, 1448, 0.1, 0.005, seed=SEED, wmin=1, wmax=100)
    raise SystemExit("unknown case " + case)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--hostloop", action="store_true")
    ap.add_argument("--trace", action="store_true",
                    help="print every superstep (branch, frontier, CUDA-event ms) of the last rep")
    ap.add_argument("--pr-order", choices=["fixed", "reference"], default=None)
    ap.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                    help="a tunable for the runs (e.g. sssp_async=1)")
    ap.add_argument("--sssp-delta", type=float, default=None,
                    help="single-source SSSP near-far width (0: none; -1: the per-graph default)")
    args = ap.parse_args(argv)
    ctx = api.Context(0)
    if args.hostloop:
        ctx.set_graph_capture(False)
    for kv in args.set:
        name, value = kv.split("=", 1)
        ctx.set_tunable(name, int(value))
    if args.sssp_delta is not None:
        ctx.set_sssp_delta(args.sssp_delta)
    if args.pr_order:
        ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED if args.pr_order == "fixed"
                               else api.MB_PR_ORDER_REFERENCE)
    if args.case.startswith("path"):
        n = 200
        src = np.arange(n - 1, dtype=np.int32)
        g = ctx.graph_from_edges(n, src, src + 1, np.ones(n - 1, np.float32))
        ctx.set_persistent_tail(False)
    else:
        g = ctx.generate(params(args.case))
    kind = args.case.split("-")[1]
    for i in range(args.reps):
        if args.trace and i == args.reps - 1:
            ctx.set_tracing(True)
        if kind == "bfs":
            _, st = g.bfs([0])
        elif kind == "sssp":
            _, st = g.sssp([0])
        elif kind == "msssp":
            _, st = g.sssp(list(range(32)))
        elif kind == "pr":
            _, st = g.pagerank(20 if args.case.startswith("c5") else 10, 1.0 / g.V)
        else:
            raise SystemExit("unknown case " + args.case)
        print("%s rep %d: %.4f ms, %d supersteps, %d launches" %
              (args.case, i, st["device_ms"], st["supersteps"], st["kernel_launches"]), flush=True)
    if args.trace:
        per_edge = 8 if kind == "bfs" else 12
        print("step branch sched frontier_vertices frontier_edges ms algorithmic_bytes")
        for r in ctx.get_trace():
            b = per_edge * int(r["frontier_edges"]) + 20 * int(r["frontier_vertices"])
            print("%d %d %d %d %d %.4f %d" % (r["step"], r["branch"], r["sched"],
                                             r["frontier_vertices"], r["frontier_edges"], r["ms"], b))
        ctx.set_tracing(False)
    g.close()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
