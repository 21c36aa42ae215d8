"""Batched SSSP (up to 32 sources per traversal) with near-far buckets over
(vertex, source) pairs: zero weights and a zero-weight cycle, non-integer
weights, one source repeated 32 times, and the superstep cap.  Every
distance is the oracle's (or, for non-integer weights, the plain frontier
Bellman-Ford's: both reach the least fixpoint of
d[v] = min over in-edges of fl(d[u] + w), which does not depend on the
order of relaxations because fl(a + w) is monotone in a)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

WIDTHS = (-1, 0, 1, 3, 100)


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


@pytest.fixture
def bctx(gpu_ctx):
    gpu_ctx.set_batching(True)
    yield gpu_ctx
    gpu_ctx.set_tunable("mss_delta", -1)
    gpu_ctx.set_tunable("step_cap", -1)


def _random_graph(seed, V, E, weights):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, V, E).astype(np.int32)
    dst = rng.integers(0, V, E).astype(np.int32)
    return rng, src, dst, weights(rng, E)


def test_zero_weights_and_a_zero_cycle(bctx):
    """A fifth of the weights are 0, plus a zero-weight cycle through a
    source: a pair only re-enters the frontier when its distance drops, so
    the run ends; every source's distances are the oracle's at every width."""
    V = 3000
    _, src, dst, w = _random_graph(31, V, 20000, lambda r, n: r.integers(0, 5, n).astype(np.float32))
    cyc = np.arange(10, dtype=np.int32)
    src = np.concatenate([src, cyc])
    dst = np.concatenate([dst, (cyc + 1) % 10])
    w = np.concatenate([w, np.zeros(10, np.float32)])
    g = bctx.graph_from_edges(V, src, dst, w)
    try:
        srcs = [0, 5, 9] + list(range(100, 3000, 100))
        want = [O.sssp(V, src, dst, w, s)[0] for s in srcs]
        for delta in WIDTHS:
            bctx.set_tunable("mss_delta", delta)
            got, _ = g.sssp(srcs)
            for i, s in enumerate(srcs):
                np.testing.assert_array_equal(got[i].view(np.uint32), want[i].view(np.uint32),
                                              err_msg="width %d, source %d" % (delta, s))
    finally:
        g.close()


def test_fractional_weights_equal_the_plain_batched_loop(bctx):
    V = 20000
    _, src, dst, w = _random_graph(32, V, 160000,
                                   lambda r, n: r.uniform(0.001, 3.0, n).astype(np.float32))
    g = bctx.graph_from_edges(V, src, dst, w)
    try:
        srcs = list(range(0, 32 * 611, 611))
        bctx.set_tunable("mss_delta", 0)
        ref, _ = g.sssp(srcs)
        for delta in (1, 2, 5):
            bctx.set_tunable("mss_delta", delta)
            got, _ = g.sssp(srcs)
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32),
                                          err_msg="width %d" % delta)
    finally:
        g.close()


def test_one_source_in_every_lane(bctx, api):
    """The same source 32 times: every lane's pairs move between the buckets
    together; all 32 rows equal the single-source run."""
    p = api.rmat_params(14, 1 << 18, 0.45, 0.15, 0.15, seed=33, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    g = bctx.generate(p)
    try:
        want, _ = O.sssp(V, s, d, w, 7)
        for delta in (-1, 50):
            bctx.set_tunable("mss_delta", delta)
            got, _ = g.sssp([7] * 32)
            for i in range(32):
                np.testing.assert_array_equal(got[i].view(np.uint32), want.view(np.uint32))
    finally:
        g.close()


def test_buckets_with_every_pair_at_its_own_distance(bctx, api):
    """A 20-vertex path whose edge weights make every (vertex, source)
    distance distinct, 20 sources, width 1: a bucket may advance a single
    pair, 190 buckets in all -- more than 4 V + 16 supersteps, within the
    cap of the bucketed loop (which scales with the sources)."""
    n = 20
    src = np.arange(n - 1, dtype=np.int32)
    dst = src + 1
    w = (1000 + 37 * np.arange(n - 1) ** 2).astype(np.float32)
    g = bctx.graph_from_edges(n, src, dst, w)
    try:
        bctx.set_tunable("mss_delta", 1)
        srcs = list(range(n))
        got, st = g.sssp(srcs)
        for i, s0 in enumerate(srcs):
            np.testing.assert_array_equal(got[i], O.sssp(n, src, dst, w, s0)[0])
        assert st["supersteps"] > 4 * n + 16
    finally:
        g.close()


def test_superstep_cap_with_buckets(bctx, api):
    """A superstep cap of 1 stops the bucketed loop with MB_ERR_TIMEOUT; the
    same context then runs it to the oracle's distances."""
    p = api.rmat_params(14, 1 << 18, 0.45, 0.15, 0.15, seed=34, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    g = bctx.generate(p)
    try:
        bctx.set_tunable("mss_delta", 100)
        bctx.set_tunable("step_cap", 1)
        with pytest.raises(api.MedusaError) as e:
            g.sssp(list(range(32)))
        assert e.value.code == api.MB_ERR_TIMEOUT and "cap" in str(e.value)
        bctx.set_tunable("step_cap", -1)
        got, _ = g.sssp(list(range(32)))
        for i in (0, 13, 31):
            want, _ = O.sssp(V, s, d, w, i)
            np.testing.assert_array_equal(got[i].view(np.uint32), want.view(np.uint32))
    finally:
        g.close()
