"""Near-far buckets of the single-source SSSP (medusa_b200/csrc/sssp.cu
work_far_split, engine.cuh choose_next), restated on the CPU superstep by
superstep, on random graphs with random widths and weights up to past 2^24.

A push relaxes the near queue's out-edges: a neighbour whose new distance is
below the threshold T joins the next queue (once per superstep), one at or
above it joins the far pile unless its pile bit is set already.  When the
queue runs dry the threshold rises to max(T + width, kept + width), kept
being the least distance the last split left in the pile (one float step
further where a sum rounds back), and a split drops the pile's vertices
below the previous threshold (they were expanded at that distance through
the near queue), queues those below the new one and keeps the rest,
recording the least distance kept.  Checked here: the distances equal
Bellman-Ford's, and the supersteps stay within the loop's cap of 4 V + 16.
"""
import numpy as np
import pytest

INF = np.float32(np.inf)


def bellman_ford(V, src, dst, w, s):
    d = np.full(V, INF, np.float32)
    d[s] = 0.0
    for _ in range(V + 1):
        nd = (d[src] + w).astype(np.float32)
        upd = nd < d[dst]
        if not upd.any():
            break
        np.minimum.at(d, dst[upd], nd[upd])
    return d


def next_up(x):
    return np.nextafter(np.float32(x), np.float32(np.inf))


def near_far(V, src, dst, w, s, width):
    order = np.argsort(src, kind="stable")
    src, dst, w = src[order], dst[order], w[order]
    row = np.searchsorted(src, np.arange(V + 1))
    dist = np.full(V, INF, np.float32)
    dist[s] = 0.0
    width = np.float32(width)
    T, T_prev, kept = width, np.float32(0.0), INF
    queue = [s] if row[s + 1] > row[s] else []
    pile, inpile = [], np.zeros(V, bool)
    steps = 0
    while True:
        if not queue:
            if not pile:
                return dist, steps
            # raise: skip empty buckets; one float step where a sum rounds back
            t = np.float32(T + width)
            if kept < INF:
                t = max(t, np.float32(kept + width))
            if not t > T:
                t = next_up(T)
            if kept < INF and not t > kept:
                t = next_up(kept)
            T_prev, T, kept = T, t, INF
            # split
            rest = []
            for v in pile:
                if dist[v] < T:
                    inpile[v] = False
                    if dist[v] >= T_prev and row[v + 1] > row[v]:
                        queue.append(v)
                else:
                    rest.append(v)
                    kept = min(kept, dist[v])
            pile = rest
            steps += 1
            continue
        nxt, seen = [], set()
        for u in queue:
            for e in range(row[u], row[u + 1]):
                v = dst[e]
                nd = np.float32(dist[u] + w[e])
                if nd < dist[v]:
                    dist[v] = nd
                    if nd < T:
                        if v not in seen and row[v + 1] > row[v]:
                            seen.add(v)
                            nxt.append(v)
                    elif not inpile[v]:
                        inpile[v] = True
                        pile.append(v)
        queue = nxt
        steps += 1


@pytest.mark.parametrize("seed", range(60))
def test_near_far_reaches_bellman_ford_within_the_cap(seed):
    rng = np.random.default_rng(seed)
    V = int(rng.integers(2, 50))
    E = int(rng.integers(0, 4 * V))
    src = rng.integers(0, V, E).astype(np.int32)
    dst = rng.integers(0, V, E).astype(np.int32)
    wmax = float(rng.choice([3.0, 1000.0, 3.0e7]))  # 3e7: distances past 2^24
    w = np.floor(rng.uniform(0, wmax, E)).astype(np.float32)
    width = float(rng.choice([0.5, 1.0, 7.0, 999.0, 1e9]))
    s = int(rng.integers(0, V))
    dist, steps = near_far(V, src, dst, w, s, width)
    np.testing.assert_array_equal(dist, bellman_ford(V, src, dst, w, s),
                                  err_msg="width %g, weights < %g" % (width, wmax))
    assert steps <= 4 * V + 16, (steps, V)


def test_distances_far_apart_in_units_of_the_width():
    """A path of weight-1000 edges at width 1: without the skip, 7000 empty
    buckets; with it, a few supersteps per vertex."""
    n = 8
    src = np.arange(n - 1, dtype=np.int32)
    w = np.full(n - 1, 1000.0, np.float32)
    dist, steps = near_far(n, src, src + 1, w, 0, 1.0)
    np.testing.assert_array_equal(dist, np.arange(n, dtype=np.float32) * 1000)
    assert steps <= 4 * n + 16
