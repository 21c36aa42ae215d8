"""Autotuner for the library's launch and routing parameters (MB_TUNE_*).

The tunables change only how fast a run goes, never its result (the tests
check every path against the oracle), so the tuner simply times candidate
settings on the caller's own graph with the library's device clock and keeps
the fastest.  Search: coordinate descent -- one tunable at a time over its
candidate values, the others held at their best so far -- for `passes`
rounds.  Every candidate is timed `reps` times after one untimed run (the
first run after a change rebuilds the loop's CUDA graph); the median counts.

    from medusa_b200 import api, autotune
    best, table = autotune.tune_sssp(ctx, graph, source=0)   # leaves best set
"""
import numpy as np


# threshold steps of the asynchronous SSSP tried (-1: the per-graph default,
# 8 x mean weight / mean out-degree; 0: no threshold)
ASYNC_DELTAS = [-1, 0, 50, 200, 800, 3200]


def _median_ms(fn, reps):
    fn()
    return float(np.median([fn()["device_ms"] for _ in range(reps)]))


def _get(ctx, name):
    return ctx.sssp_delta if name == "sssp_delta" else ctx.get_tunable(name)


def _set(ctx, name, value):
    if name == "sssp_delta":  # the near-far bucket width (0: off, -1: per-graph default)
        ctx.set_sssp_delta(value)
    else:
        ctx.set_tunable(name, value)


def tune(ctx, run, space, reps=3, passes=1):
    """Coordinate descent over `space` ({tunable name: [values]}); `run()`
    performs one run and returns its stats.  Leaves the best values set and
    returns (best {name: value}, [(setting, ms), ...])."""
    best = {k: _get(ctx, k) for k in space}
    table = []
    best_ms = _median_ms(run, reps)
    table.append((dict(best), best_ms))
    for _ in range(passes):
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                _set(ctx, name, v)
                ms = _median_ms(run, reps)
                trial = dict(best)
                trial[name] = v
                table.append((trial, ms))
                if ms < best_ms:
                    best_ms, best[name] = ms, v
            _set(ctx, name, best[name])
    return best, table


def tune_joint(ctx, run, names, candidates, reps=3):
    """Try each tuple of `candidates` for the tunables `names` together (for
    settings that only matter jointly, such as a kernel switch and its
    parameter); leaves the fastest set.  Returns (best {name: value}, table)."""
    best = tuple(_get(ctx, n) for n in names)
    best_ms = _median_ms(run, reps)
    table = [(dict(zip(names, best)), best_ms)]
    for cand in candidates:
        if tuple(cand) == best:
            continue
        for n, v in zip(names, cand):
            _set(ctx, n, v)
        ms = _median_ms(run, reps)
        table.append((dict(zip(names, cand)), ms))
        if ms < best_ms:
            best_ms, best = ms, tuple(cand)
    for n, v in zip(names, best):
        _set(ctx, n, v)
    return dict(zip(names, best)), table


# (MB_TUNE_SSSP_ASYNC, MB_TUNE_ASYNC_DELTA) and (MB_TUNE_BFS_ASYNC,
# MB_TUNE_BFS_ASYNC_DELTA) pairs tried together
SSSP_ASYNC_PAIRS = [(-1, -1), (0, -1)] + [(1, d) for d in ASYNC_DELTAS]
# (MB_TUNE_SSSP_ASYNC, MB_TUNE_ASYNC_DELTA, MB_TUNE_ASYNC_BELOW): the
# defaults, the BSP loop alone, the kernel from the first superstep with each
# step, and the BSP supersteps while the frontier is large, then the kernel
SSSP_ASYNC_TRIPLES = [(-1, -1, -1), (0, -1, -1)] + [(1, d, 0) for d in ASYNC_DELTAS] + \
    [(1, 0, 1 << b) for b in (18, 20, 22)]
BFS_ASYNC_PAIRS = [(-1, -1), (1, -1), (1, 2), (1, 4), (1, 8)]


def tune_sssp(ctx, g, source=0, reps=3):
    """Asynchronous kernel on or off and its threshold step and grid, then
    the bitmap-output push threshold and push grid for SSSP on graph g."""
    E = max(int(g.E), 1)
    run = lambda: g.sssp([source])[1]
    best, table = tune_joint(ctx, run, ("sssp_async", "async_delta", "async_below"), SSSP_ASYNC_TRIPLES, reps)
    space = {"async_blocks_per_sm": [-1, 2, 3],
             "sssp_bm_push_min": sorted({-1, 0, 1 << 16, 1 << 18, 1 << 20, 1 << 22, E // 8, E // 32}),
             "push_blocks_per_sm": [-1, 4, 6, 12, 16],
             "bulk_stage": [-1, 1]}
    b2, t2 = tune(ctx, run, space, reps)
    best.update(b2)
    return best, table + t2


def tune_bfs(ctx, g, source=0, reps=3):
    """Asynchronous BFS on or off and its threshold step, the persistent-tail
    size and the push / per-vertex grids for BFS on g."""
    run = lambda: g.bfs([source])[1]
    best, table = tune_joint(ctx, run, ("bfs_async", "bfs_async_delta"), BFS_ASYNC_PAIRS, reps)
    space = {"tail_edges": [-1, 0, 2048, 4096, 6144],
             "push_blocks_per_sm": [-1, 4, 6, 12, 16],
             "vertex_blocks_per_sm": [-1, 4, 12, 16],
             "bfs_alpha": [-1, 0, 4, 60],
             "bfs_beta": [-1, 5, 80],
             "bfs_gamma": [-1, 0, 64]}
    b2, t2 = tune(ctx, run, space, reps)
    best.update(b2)
    return best, table + t2


# near-far widths of the batched SSSP tried (-1: the per-graph default;
# 0: no buckets)
MSS_DELTAS = [-1, 0, 50, 100, 150, 200, 400, 800, 2000]


def tune_batched_sssp(ctx, g, sources, reps=3):
    """The near-far width of the batched SSSP (2..32 sources per traversal)
    over `sources` on graph g; leaves the fastest set."""
    run = lambda: g.sssp(list(sources))[1]
    return tune(ctx, run, {"mss_delta": MSS_DELTAS}, reps)


def tune_traversals(ctx, g, source=0, reps=3):
    """Every BFS/SSSP tunable at once, timing one BFS plus one SSSP (the
    tunables are per context and the two apps share the push grid)."""
    E = max(int(g.E), 1)

    def run():
        sb = g.bfs([source])[1]
        ss = g.sssp([source])[1]
        return {"device_ms": sb["device_ms"] + ss["device_ms"]}

    best, table = tune_joint(ctx, run, ("sssp_async", "async_delta", "async_below"), SSSP_ASYNC_TRIPLES, reps)
    b2, t2 = tune_joint(ctx, run, ("bfs_async", "bfs_async_delta"), BFS_ASYNC_PAIRS, reps)
    best.update(b2)
    table += t2
    space = {"async_blocks_per_sm": [-1, 2, 3],
             "sssp_bm_push_min": sorted({-1, 0, 1 << 18, 1 << 20, 1 << 22, E // 8, E // 32}),
             "sssp_delta": [0.0, -1.0, 100.0, 1000.0, 10000.0],
             "tail_edges": [-1, 0, 2048, 4096],
             "push_blocks_per_sm": [-1, 4, 6, 12, 16],
             "vertex_blocks_per_sm": [-1, 4, 12, 16],
             "bfs_alpha": [-1, 0, 4, 60],
             "bfs_beta": [-1, 5, 80],
             "bfs_gamma": [-1, 0, 64],
             "bulk_stage": [-1, 1]}
    b3, t3 = tune(ctx, run, space, reps)
    best.update(b3)
    return best, table + t3


def tune_pagerank(ctx, g, iters=10, reps=3, out=None):
    """Light vertices per lane of the fused pull, and, in the reference's
    order, the in-degree above which a vertex is summed by one CTA's integer
    scan (else short heavy blocks per warp of the fixed order), timing
    `iters` PageRank supersteps on g (out: a rank buffer to reuse, e.g. a
    device tensor)."""
    from medusa_b200 import api
    space = {"pr_light_vpl": [-1, 1, 2, 4]}
    if getattr(ctx, "pr_order", api.MB_PR_ORDER_REFERENCE) == api.MB_PR_ORDER_REFERENCE:
        space["pr_hub_min"] = [-1, 256, 512, 1024, 4096]
        space["pr_hub_ctas"] = [-1, 148, 592]
    else:
        space["pr_short_pair"] = [-1, 1, 2]
    return tune(ctx, lambda: g.pagerank(iters, 1.0 / g.V, out=out)[1], space, reps)


def tune_batch(ctx, batch, pr_iters=20, reps=3, ranks=None, levels=None):
    """CTA size and edges per CTA (team size) of the many-graph kernel.
    ranks/levels: output buffers to reuse (device tensors avoid the copies)."""
    if ranks is None:
        ranks = np.empty(batch.total_V, np.float32)
    if levels is None:
        levels = np.empty(batch.total_V, np.int32)
    space = {"batch_threads": [-1, 128, 512],
             "batch_edges_per_cta": [-1, 1 << 14, 1 << 15, 1 << 17, 1 << 18]}
    return tune(ctx, lambda: batch.run(pr_iters, None, ranks, levels)[2], space, reps, passes=2)
