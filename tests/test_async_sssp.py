"""The asynchronous SSSP kernel (MB_TUNE_SSSP_ASYNC): the rest of a traversal
in one cooperative launch, with no superstep barriers.

Shortest-path distances over integer weights stored as float are exact and
unique, so any order of relaxations reaches the reference's distances bit for
bit: every golden graph (fixtures made by the reference's own CPU superstep),
every threshold step, both loop modes, graphs whose hubs are split into
chunks, and the full-size configurations against the BSP supersteps."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


@pytest.fixture(params=[False, True], ids=["hostloop", "graph"])
def actx(request, gpu_ctx, api):
    gpu_ctx.set_graph_capture(request.param)
    gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    gpu_ctx.set_tunable("sssp_async", 1)
    gpu_ctx.set_tunable("async_below", 0)  # the kernel from the first superstep
    yield gpu_ctx
    for k in ("sssp_async", "async_delta", "async_blocks_per_sm", "async_below"):
        gpu_ctx.set_tunable(k, -1)
    gpu_ctx.set_graph_capture(True)


@pytest.mark.parametrize("name", golden_names())
def test_async_sssp_matches_reference(actx, name):
    c = load_golden(name)
    g = actx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        # -1: the per-graph step; 0: no threshold; 1: one weight unit; huge
        for delta in (-1, 0, 1, 1 << 30):
            actx.set_tunable("async_delta", delta)
            for i, s in enumerate(c["sources"]):
                d, st = g.sssp([int(s)])
                np.testing.assert_array_equal(d[0].view(np.uint32), c["sssp_dist"][i].view(np.uint32),
                                              err_msg="delta %d source %d" % (delta, s))
    finally:
        g.close()


@pytest.mark.parametrize("seed", [9, 10])
def test_async_sssp_hub_chunks(actx, api, seed):
    """Skewed R-MAT (0.57, 0.19, 0.19) with hubs of several thousand
    out-edges: a hub's edges are relaxed as 128-edge chunks by many warps."""
    p = api.rmat_params(14, 1 << 20, 0.57, 0.19, 0.19, seed=seed, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    assert np.bincount(s, minlength=V).max() > 4 * 1024
    want, _ = O.sssp(V, s, d, w, 0)
    g = actx.generate(p)
    try:
        for delta in (-1, 0, 50):
            actx.set_tunable("async_delta", delta)
            for bps in (-1, 1):
                actx.set_tunable("async_blocks_per_sm", bps)
                got, st = g.sssp([0])
                np.testing.assert_array_equal(got[0].view(np.uint32), want.view(np.uint32),
                                              err_msg="delta %d blocks %d" % (delta, bps))
                # every reached vertex's out-edges relaxed at least once
                assert st["edges_scanned"] >= st["edges_traversed"]
    finally:
        g.close()


def test_async_sssp_star_hub_and_isolated_source(actx, api):
    """One vertex with 5000 out-edges (40 chunks), a chain behind it, and a
    source with no out-edges (nothing to relax)."""
    rng = np.random.default_rng(3)
    V = 7000
    src = np.concatenate([np.zeros(5000, np.int32), np.arange(5000, 6998, dtype=np.int32)])
    dst = np.concatenate([np.arange(1, 5001, dtype=np.int32), np.arange(5001, 6999, dtype=np.int32)])
    w = rng.integers(1, 100, len(src)).astype(np.float32)
    g = actx.graph_from_edges(V, src, dst, w)
    try:
        for s0 in (0, 6999):
            want, _ = O.sssp(V, src, dst, w, s0)
            got, _ = g.sssp([s0])
            np.testing.assert_array_equal(got[0].view(np.uint32), want.view(np.uint32))
    finally:
        g.close()


def test_async_sssp_negative_weight_takes_the_bsp_loop(gpu_ctx, api):
    """A graph with a negative weight runs the BSP loop even when the
    asynchronous kernel is asked for (the loop's superstep cap is what bounds
    such a run); without a negative cycle it gets the oracle's distances."""
    V = 4
    src = np.array([0, 1, 0, 2], np.int32)
    dst = np.array([1, 2, 2, 3], np.int32)
    w = np.array([5, -2, 4, 1], np.float32)
    g = gpu_ctx.graph_from_edges(V, src, dst, w)
    try:
        gpu_ctx.set_tunable("sssp_async", 1)
        got, st = g.sssp([0])
        want, _ = O.sssp(V, src, dst, w, 0)
        np.testing.assert_array_equal(got[0], want)
    finally:
        gpu_ctx.set_tunable("sssp_async", -1)
        g.close()


@pytest.mark.parametrize("which", ["c2_rmat", "c3_grid"])
def test_async_sssp_full_size_equals_bsp(gpu_ctx, api, which):
    """C2 (R-MAT 2^20 / 2^24) and C3 (1448^2 grid): the asynchronous kernel
    and the BSP supersteps give the same distances bit for bit; with a
    threshold step of 100 the asynchronous one relaxes fewer edges."""
    if which == "c2_rmat":
        p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=1, wmin=1, wmax=1000)
    else:
        p = api.grid_params(1448, 1448, 0.1, 0.005, seed=1, wmin=1, wmax=100)
    g = gpu_ctx.generate(p)
    try:
        gpu_ctx.set_tunable("sssp_async", 0)
        ref, st0 = g.sssp([0])
        gpu_ctx.set_tunable("sssp_async", 1)
        gpu_ctx.set_tunable("async_below", 0)  # the kernel from the first superstep
        for delta in (-1, 100):
            gpu_ctx.set_tunable("async_delta", delta)
            got, st1 = g.sssp([0])
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
            assert st1["edges_traversed"] == st0["edges_traversed"]
        assert st1["edges_scanned"] < st0["edges_scanned"]
    finally:
        for k in ("sssp_async", "async_delta", "async_below"):
            gpu_ctx.set_tunable(k, -1)
        g.close()


@pytest.mark.parametrize("name", golden_names())
def test_async_bfs_matches_reference(gpu_ctx, api, name):
    """MB_TUNE_BFS_ASYNC: BFS as the asynchronous kernel with every weight 1
    (levels are hop distances, exact in float): the reference's levels for
    every threshold step, both loop modes."""
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        gpu_ctx.set_tunable("bfs_async", 1)
        for capture in (True, False):
            gpu_ctx.set_graph_capture(capture)
            for delta in (-1, 2, 1 << 20):
                gpu_ctx.set_tunable("bfs_async_delta", delta)
                for i, s in enumerate(c["sources"]):
                    lv, st = g.bfs([int(s)])
                    np.testing.assert_array_equal(lv[0], c["bfs_level"][i],
                                                  err_msg="delta %d source %d" % (delta, s))
    finally:
        for k in ("bfs_async", "bfs_async_delta"):
            gpu_ctx.set_tunable(k, -1)
        gpu_ctx.set_graph_capture(True)
        g.close()


@pytest.mark.parametrize("which", ["c2_rmat", "c3_grid"])
def test_async_bfs_full_size_equals_bsp(gpu_ctx, api, which):
    if which == "c2_rmat":
        p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=1, wmin=1, wmax=1000)
    else:
        p = api.grid_params(1448, 1448, 0.1, 0.005, seed=1, wmin=1, wmax=100)
    g = gpu_ctx.generate(p)
    try:
        ref, st0 = g.bfs([0])
        gpu_ctx.set_tunable("bfs_async", 1)
        got, st1 = g.bfs([0])
        np.testing.assert_array_equal(got, ref)
        assert st1["edges_traversed"] == st0["edges_traversed"]
        assert st1["vertices_reached"] == st0["vertices_reached"]
    finally:
        gpu_ctx.set_tunable("bfs_async", -1)
        g.close()


@pytest.mark.parametrize("name", golden_names())
def test_hybrid_route_matches_reference(actx, name):
    """MB_TUNE_ASYNC_BELOW: BSP supersteps while the frontier is large, then
    the asynchronous kernel for the rest (a threshold of 1 edge: the kernel
    takes over right after the first frontier with out-edges)."""
    c = load_golden(name)
    g = actx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for below, delta in ((1, 0), (64, -1), (1 << 30, 0)):
            actx.set_tunable("async_below", below)
            actx.set_tunable("async_delta", delta)
            for i, s in enumerate(c["sources"]):
                d, _ = g.sssp([int(s)])
                np.testing.assert_array_equal(d[0].view(np.uint32), c["sssp_dist"][i].view(np.uint32),
                                              err_msg="below %d source %d" % (below, s))
    finally:
        actx.set_tunable("async_below", -1)
        g.close()


def test_hybrid_route_full_size_c2(gpu_ctx, api):
    """C2 at full size: BSP supersteps until the frontier drops below 2^18 /
    2^20 out-edges after its peak, then the asynchronous kernel: the BSP
    loop's distances bit for bit."""
    p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=1, wmin=1, wmax=1000)
    g = gpu_ctx.generate(p)
    try:
        gpu_ctx.set_tunable("sssp_async", 0)
        ref, st0 = g.sssp([0])
        gpu_ctx.set_tunable("sssp_async", 1)
        gpu_ctx.set_tunable("async_delta", 0)
        for below in (1 << 18, 1 << 20):
            gpu_ctx.set_tunable("async_below", below)
            got, st = g.sssp([0])
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
            assert st["edges_traversed"] == st0["edges_traversed"]
            assert 1 < st["supersteps"] < st0["supersteps"] + 8
    finally:
        for k in ("sssp_async", "async_delta", "async_below"):
            gpu_ctx.set_tunable(k, -1)
        g.close()


def test_learned_policy_takes_the_asynchronous_route(gpu_ctx, api):
    """Under the learned policy schedule 0 may run as the asynchronous kernel
    too (on a hub-free graph, its default), with the fixed rule's distances;
    under the replay policy it never does (every superstep is named)."""
    p = api.uniform_params(1 << 14, 1 << 17, seed=5, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    want, _ = O.sssp(V, s, d, w, 0)
    g = gpu_ctx.generate(p)
    try:
        w0 = np.zeros(api.lib.mb_scheduler_num_params(), np.float32)
        gpu_ctx.scheduler_set_weights(w0, api.MB_MODEL_SSSP)  # ties: the fixed rule's choice
        for policy in (api.MB_POLICY_LEARNED, api.MB_POLICY_ORACLE_BEST):
            if policy == api.MB_POLICY_ORACLE_BEST:
                gpu_ctx.set_replay([0] * 8)
            else:
                gpu_ctx.set_policy(policy)
            got, st = g.sssp([0])
            np.testing.assert_array_equal(got[0].view(np.uint32), want.view(np.uint32))
            if policy == api.MB_POLICY_ORACLE_BEST:
                assert st["schedule_count"][0] > 3  # one superstep per BSP step
            else:
                assert st["schedule_count"][0] == 1  # the whole traversal in one launch
    finally:
        gpu_ctx.set_policy(api.MB_POLICY_FIXED)
        g.close()


def test_async_sssp_zero_weights_and_a_zero_cycle(actx, api):
    """Zero weights, including a zero-weight cycle: a relaxation only counts
    when it lowers a distance, so the kernel ends; the distances are the
    oracle's."""
    rng = np.random.default_rng(21)
    V = 3000
    src = rng.integers(0, V, 20000).astype(np.int32)
    dst = rng.integers(0, V, 20000).astype(np.int32)
    w = rng.integers(0, 5, 20000).astype(np.float32)  # a fifth of the weights are 0
    cyc = np.arange(10, dtype=np.int32)
    src = np.concatenate([src, cyc])
    dst = np.concatenate([dst, (cyc + 1) % 10])
    w = np.concatenate([w, np.zeros(10, np.float32)])
    g = actx.graph_from_edges(V, src, dst, w)
    try:
        for s0 in (0, 5):
            want, _ = O.sssp(V, src, dst, w, s0)
            for delta in (-1, 0, 1):
                actx.set_tunable("async_delta", delta)
                got, _ = g.sssp([s0])
                np.testing.assert_array_equal(got[0].view(np.uint32), want.view(np.uint32))
    finally:
        g.close()


def test_async_sssp_threshold_past_2_24(actx, api):
    """Distances past 2^24 with a threshold step of 1, where T + 1 rounds
    back to T: the step goes one float past the least distance above T, so
    the run ends with the oracle's distances."""
    n = 8
    src = np.concatenate([np.arange(n - 1), [0]]).astype(np.int32)
    dst = np.concatenate([np.arange(1, n), [5]]).astype(np.int32)
    w = np.full(n, 3.0e7, np.float32)
    w[-1] = 1.35e8
    g = actx.graph_from_edges(n, src, dst, w)
    try:
        want, _ = O.sssp(n, src, dst, w, 0)
        for delta in (1, 2, 100):
            actx.set_tunable("async_delta", delta)
            got, st = g.sssp([0])
            np.testing.assert_array_equal(got[0], want, err_msg="delta %d" % delta)
    finally:
        actx.set_tunable("async_delta", -1)
        g.close()


def test_async_sssp_fractional_weights_equal_the_bsp_loop(gpu_ctx, api):
    """Non-integer weights: the distances are the least fixpoint of
    d[v] = min over in-edges of fl(d[u] + w), which every order of
    relaxations reaches (fl(a + w) is monotone in a), so the asynchronous
    kernel gives the BSP loop's floats bit for bit."""
    rng = np.random.default_rng(22)
    V = 20000
    src = rng.integers(0, V, 160000).astype(np.int32)
    dst = rng.integers(0, V, 160000).astype(np.int32)
    w = rng.uniform(0.001, 3.0, 160000).astype(np.float32)
    g = gpu_ctx.graph_from_edges(V, src, dst, w)
    try:
        gpu_ctx.set_tunable("sssp_async", 0)
        ref, _ = g.sssp([0])
        gpu_ctx.set_tunable("sssp_async", 1)
        gpu_ctx.set_tunable("async_below", 0)
        for delta in (-1, 0, 1):
            gpu_ctx.set_tunable("async_delta", delta)
            got, _ = g.sssp([0])
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
    finally:
        for k in ("sssp_async", "async_delta", "async_below"):
            gpu_ctx.set_tunable(k, -1)
        g.close()


@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "rmat_skew_s12"])
def test_near_far_width_turns_the_kernel_off(actx, name):
    """The asynchronous kernel starts from the queue frontier only, so with
    near-far buckets on (vertices parked in the far pile) it must not run,
    whatever the tunable says: distances stay the reference's for every
    width, with the kernel asked for from the first superstep and as a tail."""
    c = load_golden(name)
    g = actx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for below in (0, 1, 64):
            actx.set_tunable("async_below", below)
            for width in (1.0, 37.0, 500.0, -1.0):
                actx.set_sssp_delta(width)
                for i, s in enumerate(c["sources"]):
                    d, _ = g.sssp([int(s)])
                    np.testing.assert_array_equal(d[0].view(np.uint32), c["sssp_dist"][i].view(np.uint32),
                                                  err_msg="width %g below %d" % (width, below))
    finally:
        actx.set_sssp_delta(0.0)
        g.close()
