"""Near-far buckets of the batched SSSP (medusa_b200/csrc/mssssp.cu), restated
on the CPU superstep by superstep, on random graphs with random widths.

A superstep relaxes every queued (vertex, source) pair's out-edges; an
improved pair is marked near (new distance below the threshold T) or far
in its head's two masks, and near wins for a pair improved both ways.  The
commit queues the near pairs and parks the far ones in far[v], appending v
to the live far list only when far[v] was empty.  When the queue runs dry a
far pass raises T to fmin + width, where fmin is the least distance recorded
for a parked pair since the last pass (at parking time, or the exact rest
after a pass), requeues the parked pairs now below T and moves the rest to
the other far list.  Checked here, on every step of every run:

  * a far list never holds a vertex twice, and holds exactly the vertices
    with a nonzero far mask;
  * at each far pass fmin >= T (it was recorded under the current
    threshold), so T only rises;
  * progress: fmin was set by a pair whose distance is at most fmin, so the
    pass requeues that pair -- unless that pair was also improved below T in
    the same superstep (near wins, it is not parked).  Then the pass may
    requeue nothing, but it leaves fmin exact (the least parked distance),
    so the next pass, which follows at once, requeues at least one pair;
  * the run ends, and every source's distances are the Bellman-Ford fixpoint.

A parked pair's distance can drop later through a near improvement without
touching fmin: such a pair lies below T and is simply requeued (once more)
by the next pass, so fmin need not bound every parked pair from below.
"""
import numpy as np
import pytest

INF = np.float32(np.inf)


def bellman_ford(V, src, dst, w, s):
    d = np.full(V, INF, np.float32)
    d[s] = 0.0
    for _ in range(V + 1):
        nd = d[src] + w
        upd = nd < d[dst]
        if not upd.any():
            break
        np.minimum.at(d, dst[upd], nd[upd])
    return d


def batched_near_far(V, src, dst, w, sources, width):
    order = np.argsort(src, kind="stable")
    src, dst, w = src[order], dst[order], w[order]
    row = np.searchsorted(src, np.arange(V + 1))
    deg = np.diff(row)
    S = len(sources)
    dist = np.full((V, S), INF, np.float32)
    front = np.zeros(V, np.int64)
    queue = []
    for i, s in enumerate(sources):
        if front[s] == 0 and deg[s] > 0:
            queue.append(s)
        front[s] |= 1 << i
        dist[s, i] = 0.0
    T = np.float32(width)
    fmin = INF
    far = np.zeros(V, np.int64)
    lists = [[], []]
    fl = 0
    steps = 0
    must_requeue = False  # the last far pass requeued nothing
    while True:
        # the far-list invariant
        live = lists[fl]
        assert len(live) == len(set(live))
        assert set(live) == set(np.nonzero(far)[0].tolist())
        if not queue:
            if not lists[fl]:
                return dist, steps
            # advance
            assert fmin >= T
            T = np.float32(fmin + np.float32(width))
            fmin = INF
            scan, fl = lists[fl], fl ^ 1
            lists[fl] = []
            for v in scan:
                m = int(far[v])
                near = 0
                for i in range(S):
                    if (m >> i) & 1 and dist[v, i] < T:
                        near |= 1 << i
                rem = m & ~near
                far[v] = rem
                if rem:
                    lists[fl].append(v)
                    fmin = min(fmin, min(dist[v, i] for i in range(S) if (rem >> i) & 1))
                if near:
                    front[v] = near
                    queue.append(v)
            if not queue:
                assert not must_requeue, "two far passes in a row requeued nothing"
                must_requeue = True
                steps += 1  # the GPU loop runs an empty superstep here
                continue
            must_requeue = False
        # push
        nxt_near = {}
        nxt_far = {}
        for u in queue:
            fm = int(front[u])
            for e in range(row[u], row[u + 1]):
                v = dst[e]
                for i in range(S):
                    if not (fm >> i) & 1:
                        continue
                    nd = np.float32(dist[u, i] + w[e])
                    if nd < dist[v, i]:
                        dist[v, i] = nd
                        if nd < T:
                            nxt_near[v] = nxt_near.get(v, 0) | (1 << i)
                        else:
                            nxt_far[v] = nxt_far.get(v, 0) | (1 << i)
                            fmin = min(fmin, nd)
        # commit
        queue = []
        for v in sorted(set(nxt_near) | set(nxt_far)):
            near = nxt_near.get(v, 0)
            fm = nxt_far.get(v, 0) & ~near
            if deg[v] > 0 and fm:
                if far[v] == 0:
                    lists[fl].append(v)
                far[v] |= fm
            if deg[v] > 0 and near:
                front[v] = near
                queue.append(v)
        steps += 1
        assert steps < 100 * (V + 2), "the run did not end"


@pytest.mark.parametrize("seed", range(40))
def test_buckets_reach_the_bellman_ford_fixpoint(seed):
    rng = np.random.default_rng(seed)
    V = int(rng.integers(2, 60))
    E = int(rng.integers(0, 5 * V))
    src = rng.integers(0, V, E).astype(np.int32)
    dst = rng.integers(0, V, E).astype(np.int32)
    w = rng.integers(0, int(rng.choice([3, 20, 1000])), E).astype(np.float32)  # zeros included
    S = int(rng.integers(1, 9))
    sources = rng.integers(0, V, S)
    if S > 1:
        sources[-1] = sources[0]  # a repeated source
    width = int(rng.choice([1, 2, 7, 50, 400, 100000]))
    dist, _ = batched_near_far(V, src, dst, w, list(sources), width)
    for i, s in enumerate(sources):
        np.testing.assert_array_equal(dist[:, i], bellman_ford(V, src, dst, w, s),
                                      err_msg="source %d, width %d" % (s, width))


def test_a_narrow_width_takes_more_supersteps_than_a_wide_one():
    rng = np.random.default_rng(99)
    V, E = 200, 1200
    src = rng.integers(0, V, E).astype(np.int32)
    dst = rng.integers(0, V, E).astype(np.int32)
    w = rng.integers(1, 100, E).astype(np.float32)
    d1, narrow = batched_near_far(V, src, dst, w, [0, 1, 2, 3], 1)
    d2, wide = batched_near_far(V, src, dst, w, [0, 1, 2, 3], 10 ** 6)
    np.testing.assert_array_equal(d1, d2)
    assert narrow > wide
