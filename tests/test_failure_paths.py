"""The error paths of the bounded device waits and of the superstep cap.

Every wait on the device is bounded: the grid barrier of the persistent BSP
kernels, the team barrier of the many-graph kernel, the wait for a bulk copy
into shared memory and the start barrier and idle polls of the asynchronous
SSSP kernel give up after a number of polls, record an error
flag and return, and the run fails with MB_ERR_TIMEOUT; a loop that passes
its superstep cap does the same.  MB_TUNE_WAIT_POLLS = 0 makes every such
wait give up at once and MB_TUNE_STEP_CAP = 1 stops a loop after one
superstep, so each path runs here on purpose, without a hang or a fault.
After each failure the same context runs the traversal again with the
defaults and gets the oracle's result: the context is still usable."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


@pytest.fixture(scope="module")
def graph(api):
    ctx = api.Context(0)
    p = api.rmat_params(14, 1 << 18, 0.45, 0.15, 0.15, seed=11, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    g = ctx.generate(p)
    want_l, _ = O.bfs(V, s, d, [0])
    want_d, _ = O.sssp(V, s, d, w, 0)
    yield ctx, g, want_l, want_d
    g.close()
    ctx.close()


def _reset(ctx, api):
    for k in api.TUNABLES:
        ctx.set_tunable(k, -1)
    ctx.set_persistent_grid(False)
    ctx.set_persistent_tail(True)
    ctx.set_graph_capture(True)


def _still_works(ctx, api, g, want_l, want_d):
    _reset(ctx, api)
    lv, _ = g.bfs([0])
    np.testing.assert_array_equal(lv[0], want_l)
    d, _ = g.sssp([0])
    np.testing.assert_array_equal(d[0].view(np.uint32), want_d.view(np.uint32))


@pytest.mark.parametrize("capture", [True, False], ids=["graph", "hostloop"])
def test_superstep_cap_stops_the_loop(api, graph, capture):
    ctx, g, want_l, want_d = graph
    try:
        ctx.set_graph_capture(capture)
        ctx.set_tunable("step_cap", 1)
        for run in (g.bfs, g.sssp):
            with pytest.raises(api.MedusaError) as e:
                run([0])
            assert e.value.code == api.MB_ERR_TIMEOUT
            assert "cap" in str(e.value)
    finally:
        _still_works(ctx, api, g, want_l, want_d)


def test_grid_barrier_gives_up(api, graph):
    """The persistent cooperative grid with a zero poll budget: every block
    but the last to arrive gives up at the first barrier."""
    ctx, g, want_l, want_d = graph
    try:
        ctx.set_persistent_tail(False)
        ctx.set_persistent_grid(True)
        ctx.set_tunable("wait_polls", 0)
        for run in (g.bfs, g.sssp):
            with pytest.raises(api.MedusaError) as e:
                run([0])
            assert e.value.code == api.MB_ERR_TIMEOUT
            assert "barrier" in str(e.value)
    finally:
        _still_works(ctx, api, g, want_l, want_d)


def test_bulk_copy_wait_gives_up(api, graph):
    """The staged SSSP push (bulk copies of each tile's queue entries into
    shared memory, completed on an mbarrier) with a zero poll budget: the
    first wait gives up, the copy is still waited for, the run reports it."""
    ctx, g, want_l, want_d = graph
    try:
        ctx.set_persistent_tail(False)
        ctx.set_tunable("sssp_async", 0)  # the staged push is a BSP superstep
        ctx.set_tunable("bulk_stage", 1)
        ctx.set_tunable("wait_polls", 0)
        with pytest.raises(api.MedusaError) as e:
            g.sssp([0])
        assert e.value.code == api.MB_ERR_TIMEOUT
        assert "bulk copy" in str(e.value)
    finally:
        _still_works(ctx, api, g, want_l, want_d)


@pytest.mark.parametrize("capture", [True, False], ids=["graph", "hostloop"])
def test_async_sssp_wait_gives_up(api, graph, capture):
    """The asynchronous SSSP kernel with a zero poll budget: every CTA but the
    last to arrive gives up at the start barrier, every warp leaves, and the
    run reports the wait."""
    ctx, g, want_l, want_d = graph
    try:
        ctx.set_graph_capture(capture)
        ctx.set_tunable("sssp_async", 1)
        ctx.set_tunable("async_below", 0)  # the kernel from the first superstep
        ctx.set_tunable("wait_polls", 0)
        with pytest.raises(api.MedusaError) as e:
            g.sssp([0])
        assert e.value.code == api.MB_ERR_TIMEOUT
        assert "asynchronous" in str(e.value)
    finally:
        _still_works(ctx, api, g, want_l, want_d)


def test_team_barrier_gives_up(api, graph):
    """The many-graph kernel with teams of several CTAs per graph and a zero
    poll budget; afterwards the same batch runs to the single-graph results."""
    ctx, g, want_l, want_d = graph
    ps = [api.rmat_params(12, 1 << 16, 0.45, 0.15, 0.15, seed=40 + i) for i in range(3)]
    b = ctx.batch_generate(ps)
    try:
        ctx.set_tunable("batch_edges_per_cta", 4096)  # several CTAs per graph
        ctx.set_tunable("wait_polls", 0)
        with pytest.raises(api.MedusaError) as e:
            b.run(5)
        assert e.value.code == api.MB_ERR_TIMEOUT
        assert "team barrier" in str(e.value)
        ctx.set_tunable("wait_polls", -1)
        ranks, levels, _ = b.run(5)
        for i, p in enumerate(ps):
            V, s, d, _ = api.generate_edges_host(p)
            want, _ = O.bfs(V, s, d, [0])
            np.testing.assert_array_equal(levels[b.vbase[i]:b.vbase[i + 1]], want)
    finally:
        b.close()
        _still_works(ctx, api, g, want_l, want_d)
