"""GPU parity: the CUDA path through the C ABI against the reference's own
outputs (golden fixtures) and the CPU oracle, for every schedule, in both
loop modes (CUDA graph with device-side convergence, and host-driven)."""
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
def ctx(request, gpu_ctx, api):
    gpu_ctx.set_graph_capture(request.param)
    gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    yield gpu_ctx
    gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    gpu_ctx.set_graph_capture(True)


@pytest.mark.parametrize("name", golden_names())
def test_layout_matches_reference_aa(gpu_ctx, name):
    """CSR order, msg_index and msgDstID equal the reference's buildAA."""
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"], reference_order=True)
    lay = g.export()
    aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    np.testing.assert_array_equal(lay["row"], aa.edge_index)
    np.testing.assert_array_equal(lay["col"], aa.e_dst[:aa.E])
    np.testing.assert_array_equal(lay["w"], aa.e_w[:aa.E])
    np.testing.assert_array_equal(lay["rrow"], aa.msg_index)
    np.testing.assert_array_equal(lay["mslot"], aa.msg_dst[:aa.E])
    rcol = np.empty(aa.E, np.int32)
    rcol[aa.msg_dst[:aa.E]] = aa.e_src[:aa.E]
    np.testing.assert_array_equal(lay["rcol"], rcol)
    g.close()


@pytest.mark.parametrize("name", golden_names())
def test_bfs_matches_reference(ctx, name):
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    for i, s in enumerate(c["sources"]):
        lv, st = g.bfs([s])
        np.testing.assert_array_equal(lv[0], c["bfs_level"][i])
        reached = c["bfs_level"][i] >= 0
        outdeg = np.bincount(c["src"], minlength=c["V"])
        assert st["vertices_reached"] == int(reached.sum())
        assert st["edges_traversed"] == int(outdeg[reached].sum())
    g.close()


@pytest.mark.parametrize("name", golden_names())
def test_sssp_matches_reference(ctx, name):
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    for i, s in enumerate(c["sources"]):
        d, st = g.sssp([s])
        np.testing.assert_array_equal(d[0].view(np.uint32), c["sssp_dist"][i].view(np.uint32))
    g.close()


@pytest.mark.parametrize("name", golden_names())
def test_sssp_bulk_staged_push_matches_reference(ctx, api, name):
    """The edge-balanced pushes with each tile's queue entries brought into
    shared memory by TMA bulk copies (queue and bitmap output, the latter
    forced by a threshold of one edge): distances equal the reference's."""
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    ctx.set_tunable("bulk_stage", 1)
    ctx.set_tunable("sssp_async", 0)  # the BSP supersteps
    try:
        for bm_min in (-1, 1):
            ctx.set_tunable("sssp_bm_push_min", bm_min)
            ctx.set_tunable("tail_edges", 0)  # every superstep on the multi-CTA pushes
            for i, s in enumerate(c["sources"]):
                d, st = g.sssp([s])
                np.testing.assert_array_equal(d[0].view(np.uint32), c["sssp_dist"][i].view(np.uint32),
                                              err_msg="bm_push_min %d" % bm_min)
    finally:
        for k in ("bulk_stage", "sssp_bm_push_min", "tail_edges", "sssp_async"):
            ctx.set_tunable(k, -1)
        g.close()


@pytest.mark.parametrize("name", golden_names())
def test_pagerank_matches_reference(ctx, api, name):
    """The default order is the reference's: its FP32 ranks bit for bit (the
    1e-5 rule with 0 error), and the oracle's MEG-order fold equally.  The
    fixed parallel order equals the oracle run in that order bit for bit and
    stays within the FP32 summation bound of the FP64 ranks."""
    from test_oracle import check_pagerank
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        r, st = g.pagerank(c["pr_iters"], 1.0 / c["V"])
        np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32))
        assert check_pagerank(r, c["pr_rank"]) == 0.0
        aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
        ro = O.pagerank(c["V"], aa, None, c["pr_iters"], 1.0 / c["V"])
        np.testing.assert_array_equal(r.view(np.uint32), ro.view(np.uint32))
        ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
        rf, _ = g.pagerank(c["pr_iters"], 1.0 / c["V"])
        rd = O.pagerank(c["V"], aa, None, c["pr_iters"], 1.0 / c["V"], order="device")
        np.testing.assert_array_equal(rf.view(np.uint32), rd.view(np.uint32))
        r64 = O.pagerank(c["V"], aa, None, c["pr_iters"], 1.0 / c["V"], fp64=True)
        bound = (float(np.diff(aa.msg_index).max(initial=0)) + 8) * 2.0 ** -24 * 4
        assert (np.abs(rf - r64) / r64).max(initial=0) <= bound
    finally:
        ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
        g.close()


def test_pagerank_launch_shapes_keep_every_bit(ctx, api):
    """Every light-vertices-per-lane and short-blocks-per-warp setting, for
    both PageRank schedules, on a skewed R-MAT whose in-degrees cover light
    vertices, short and long heavy blocks and multi-block hubs: ranks equal
    the oracle run in the kernels' summation order, bit for bit."""
    p = api.rmat_params(14, 1 << 19, 0.57, 0.19, 0.19, seed=7)
    V, src, dst, _ = api.generate_edges_host(p)
    indeg = np.bincount(dst, minlength=V)
    assert indeg.max() > 4096 and ((indeg > 512) & (indeg <= 4096)).any()
    assert ((indeg > 64) & (indeg <= 512)).any()
    aa = O.AAGraph(V, src, dst, None)
    ro = O.pagerank(V, aa, None, 5, 1.0 / V, order="device")
    g = ctx.graph_from_edges(V, src, dst, None)
    ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
    try:
        for vpl in (1, 2, 4):
            for pair in (1, 2, 4):
                ctx.set_tunable("pr_light_vpl", vpl)
                ctx.set_tunable("pr_short_pair", pair)
                for sched in (0, 6):
                    ctx.set_policy(api.MB_POLICY_FORCED, sched)
                    r, _ = g.pagerank(5, 1.0 / V)
                    np.testing.assert_array_equal(r.view(np.uint32), ro.view(np.uint32),
                                                  err_msg="vpl %d pair %d schedule %d" % (vpl, pair, sched))
    finally:
        ctx.set_policy(api.MB_POLICY_FIXED)
        ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
        ctx.set_tunable("pr_light_vpl", -1)
        ctx.set_tunable("pr_short_pair", -1)
        g.close()


@pytest.mark.parametrize("name", golden_names())
def test_pagerank_reference_order_is_the_reference_bit_for_bit(ctx, api, name):
    """MB_PR_ORDER_REFERENCE replays GraphIR::sortByDegree + buildMEG: the
    ranks equal the reference's own FP32 output (the golden fixture made by
    its CPU path over the MEG layout), hubs included, for both PageRank
    schedules."""
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
    try:
        for sched in (0, 6):
            ctx.set_policy(api.MB_POLICY_FORCED, sched)
            r, _ = g.pagerank(c["pr_iters"], 1.0 / c["V"])
            np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32),
                                          err_msg="schedule %d" % sched)
    finally:
        ctx.set_policy(api.MB_POLICY_FIXED)
        g.close()


@pytest.mark.parametrize("name", ["tiny", "rmat_s10", "grid_24", "hub", "uniform_2k"])
def test_every_schedule_bit_identical(gpu_ctx, api, name):
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    s = int(c["sources"][0])
    try:
        for sched in range(api.NUM_SCHEDULES):
            gpu_ctx.set_policy(api.MB_POLICY_FORCED, sched)
            lv, st = g.bfs([s])
            np.testing.assert_array_equal(lv[0], c["bfs_level"][0], err_msg="bfs sched %d" % sched)
            d, st = g.sssp([s])
            np.testing.assert_array_equal(d[0], c["sssp_dist"][0], err_msg="sssp sched %d" % sched)
        r = {}
        for sched in (0, 6):
            gpu_ctx.set_policy(api.MB_POLICY_FORCED, sched)
            r[sched] = g.pagerank(c["pr_iters"], 1.0 / c["V"])[0]
        np.testing.assert_array_equal(r[0].view(np.uint32), r[6].view(np.uint32))
    finally:
        gpu_ctx.set_policy(api.MB_POLICY_FIXED)
        g.close()


@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "uniform_2k"])
def test_persistent_tail_and_grid_on_off_identical(gpu_ctx, api, name):
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for tail, grid in ((False, False), (True, False), (False, True), (True, True)):
            gpu_ctx.set_persistent_tail(tail)
            gpu_ctx.set_persistent_grid(grid)
            for i, s in enumerate(c["sources"]):
                lv, _ = g.bfs([s])
                np.testing.assert_array_equal(lv[0], c["bfs_level"][i])
                d, _ = g.sssp([s])
                np.testing.assert_array_equal(d[0], c["sssp_dist"][i])
    finally:
        gpu_ctx.set_persistent_tail(True)
        gpu_ctx.set_persistent_grid(False)
        g.close()


@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "rmat_skew_s12", "tiny"])
def test_sssp_every_delta_identical(gpu_ctx, api, name):
    """Near-far bucket widths (and plain Bellman-Ford) give the same distances."""
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for delta in (0.0, 1.0, 37.0, 500.0, 5000.0, -1.0):
            gpu_ctx.set_sssp_delta(delta)
            for i, s in enumerate(c["sources"]):
                d, _ = g.sssp([s])
                np.testing.assert_array_equal(d[0], c["sssp_dist"][i], err_msg="delta %g" % delta)
    finally:
        gpu_ctx.set_sssp_delta(0.0)
        g.close()


def test_sssp_near_far_skips_empty_buckets(gpu_ctx, api):
    """Distances far apart in units of the width: a directed 8-vertex path of
    weight-1000 edges (plus a shortcut) spans 7000 buckets of width 1, far
    more than the superstep cap (4 V + 16 = 48); the raise skips to the
    least parked distance, so every width ends with the oracle's distances.
    Weights of 3e7 put distances past 2^24, where T + 1 rounds back to T:
    the threshold then steps one float past the least parked distance."""
    n = 8
    src = np.concatenate([np.arange(n - 1), [0]]).astype(np.int32)
    dst = np.concatenate([np.arange(1, n), [5]]).astype(np.int32)
    for wv in (1000.0, 3.0e7):
        w = np.full(n, wv, np.float32)
        w[-1] = 4.5 * wv  # the shortcut 0 -> 5
        g = gpu_ctx.graph_from_edges(n, src, dst, w)
        want, _ = O.sssp(n, src, dst, w, 0)
        try:
            for delta in (1.0, 0.5, 3.0, 999.0):
                gpu_ctx.set_sssp_delta(delta)
                d, st = g.sssp([0])
                np.testing.assert_array_equal(d[0], want, err_msg="weights %g, delta %g" % (wv, delta))
                assert st["supersteps"] <= 4 * n + 16
            # batched, with near-far buckets over the (vertex, source) pairs
            gpu_ctx.set_sssp_delta(0.0)
            gpu_ctx.set_tunable("mss_delta", 1)
            db, _ = g.sssp([0, 1, 0])
            np.testing.assert_array_equal(db[0], want)
            np.testing.assert_array_equal(db[1], O.sssp(n, src, dst, w, 1)[0])
        finally:
            gpu_ctx.set_sssp_delta(0.0)
            gpu_ctx.set_tunable("mss_delta", -1)
            g.close()


def test_oracle_replay_policy(gpu_ctx, api):
    """A per-superstep schedule list (alternating push/pull) gives the same levels."""
    c = load_golden("rmat_s10")
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for seq in ([0, 4, 0, 4, 0, 4, 0, 4], [4, 5, 2, 3, 1, 6, 7, 0], [6] * 20):
            gpu_ctx.set_replay(seq)
            lv, st = g.bfs([0])
            np.testing.assert_array_equal(lv[0], c["bfs_level"][0])
            d, _ = g.sssp([0])
            np.testing.assert_array_equal(d[0], c["sssp_dist"][0])
            n = st["supersteps"]
            want = np.bincount(np.array(seq + [seq[-1]] * 64)[:n], minlength=8)
            assert list(want) == st["schedule_count"]
    finally:
        gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    g.close()


def test_device_generator_equals_host_generator(gpu_ctx, api):
    for p in (api.rmat_params(12, 50000, 0.45, 0.15, 0.15, seed=4, wmin=1, wmax=1000),
              api.uniform_params(3000, 20000, seed=8, wmin=1, wmax=1000),
              api.grid_params(30, 17, seed=5)):
        V, s, d, w = api.generate_edges_host(p)
        g1 = gpu_ctx.generate(p)
        g2 = gpu_ctx.graph_from_edges(V, s, d, w)
        a, b = g1.export(), g2.export()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        g1.close()
        g2.close()


def test_multi_source_equals_single(gpu_ctx):
    c = load_golden("rmat_s10")
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    srcs = [0, 17, 5, 1000]
    lv, st = g.bfs(srcs)
    d, _ = g.sssp(srcs)
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(lv[i], O.bfs(c["V"], c["src"], c["dst"], [s])[0])
        np.testing.assert_array_equal(d[i], O.sssp(c["V"], c["src"], c["dst"], c["w"], s)[0])
    g.close()


def test_bad_arguments_fail_loudly(gpu_ctx, api):
    c = load_golden("tiny")
    with pytest.raises(api.MedusaError) as e:
        gpu_ctx.graph_from_edges(4, c["src"], c["dst"], c["w"])
    assert e.value.code == api.MB_ERR_INVALID
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    with pytest.raises(api.MedusaError):
        g.bfs([c["V"]])
    with pytest.raises(api.MedusaError):
        gpu_ctx.set_policy(api.MB_POLICY_FORCED, 99)
    g.close()


# ---- full-size property checks (R-MAT 2^20 / 2^24, 1448^2 grid) ---------------

def bfs_certificate(V, src, dst, lv, s):
    """Levels are BFS levels iff: lv[s]=0; every edge from a reached vertex
    reaches a vertex at most one level deeper; every reached vertex other than
    s has an in-edge from the level above; edges from unreached vertices are
    irrelevant."""
    assert lv[s] == 0
    lu, lvv = lv[src], lv[dst]
    reached_u = lu >= 0
    assert (lvv[reached_u] >= 0).all()
    assert (lvv[reached_u] <= lu[reached_u] + 1).all()
    parent_ok = np.zeros(V, bool)
    tight = reached_u & (lvv == lu + 1)
    parent_ok[dst[tight]] = True
    need = lv > 0
    assert parent_ok[need].all()


def sssp_certificate(V, src, dst, w, d, s):
    assert d[s] == 0
    du, dv = d[src], d[dst]
    reached_u = du < 1e9
    assert (dv[reached_u] <= du[reached_u] + w[reached_u]).all()
    tight = reached_u & (dv == du + w)
    ok = np.zeros(V, bool)
    ok[dst[tight]] = True
    need = (d < 1e9) & (np.arange(V) != s)
    assert ok[need].all()
    assert (d[~(d < 1e9)] == np.float32(1e9)).all()


@pytest.mark.parametrize("which", ["c2_rmat", "c3_grid"])
def test_full_size_bfs_sssp_certificates(gpu_ctx, api, which):
    if which == "c2_rmat":
        p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=1, wmin=1, wmax=1000)
    else:
        p = api.grid_params(1448, 1448, 0.1, 0.005, seed=1, wmin=1, wmax=100)
    V, s_, d_, w_ = api.generate_edges_host(p)
    g = gpu_ctx.generate(p)
    lv, st = g.bfs([0])
    bfs_certificate(V, s_, d_, lv[0], 0)
    dist, st2 = g.sssp([0])
    sssp_certificate(V, s_, d_, w_, dist[0], 0)
    # every schedule policy path agrees at full size
    gpu_ctx.set_policy(api.MB_POLICY_FORCED, api.SCHEDULE_NAMES.index("push_edge_queue"))
    lv2, _ = g.bfs([0])
    d2, _ = g.sssp([0])
    gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    np.testing.assert_array_equal(lv2, lv)
    np.testing.assert_array_equal(d2, dist)
    g.close()


def test_full_size_pagerank_c1_against_oracle(gpu_ctx, api):
    """C1: uniform 2^18 vertices / 2^22 edges, 10 supersteps from 1/N."""
    p = api.uniform_params(1 << 18, 1 << 22, seed=1)
    V, s_, d_, _ = api.generate_edges_host(p)
    g = gpu_ctx.generate(p)
    r, st = g.pagerank(10, 1.0 / V)
    aa = O.AAGraph(V, s_, d_)
    ro = O.pagerank(V, aa, None, 10, 1.0 / V)
    # the reference's MEG-order fold, bit for bit
    np.testing.assert_array_equal(r.view(np.uint32), ro.view(np.uint32))
    # the fixed order: in-degrees are all <= 64, so it is the sequential
    # fold in AA slot order
    assert np.diff(aa.msg_index).max() <= 64
    gpu_ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
    try:
        rf, _ = g.pagerank(10, 1.0 / V)
    finally:
        gpu_ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
    ra = O.pagerank(V, aa, None, 10, 1.0 / V, order="aa")
    np.testing.assert_array_equal(rf.view(np.uint32), ra.view(np.uint32))
    g.close()


@pytest.mark.parametrize("name", golden_names())
def test_sssp_bitmap_output_push(ctx, api, name):
    """Every schedule-0 superstep through the bitmap-output push (threshold
    1, persistent tail off): distances equal the reference's."""
    c = load_golden(name)
    if c["w"] is None:
        pytest.skip("unweighted")
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    ctx.set_tunable("sssp_bm_push_min", 1)
    ctx.set_tunable("tail_edges", 0)
    ctx.set_tunable("sssp_async", 0)  # the BSP supersteps
    try:
        for i, s in enumerate(c["sources"]):
            d, st = g.sssp([int(s)])
            np.testing.assert_array_equal(d[0], c["sssp_dist"][i])
        # the bitmap push followed by every other schedule (replayed list
        # 0, s, 0, s, ...): each must see the frontier the push left
        s0 = int(c["sources"][0])
        for other in range(1, 8):
            ctx.set_replay([0, other] * 64)
            ctx.set_policy(api.MB_POLICY_ORACLE_BEST)
            d, st = g.sssp([s0])
            ctx.set_policy(api.MB_POLICY_FIXED)
            np.testing.assert_array_equal(d[0], c["sssp_dist"][0], err_msg="0,%d" % other)
    finally:
        ctx.set_policy(api.MB_POLICY_FIXED)
        ctx.set_tunable("sssp_bm_push_min", -1)
        ctx.set_tunable("tail_edges", -1)
        ctx.set_tunable("sssp_async", -1)
        g.close()


@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "rmat_skew_s12", "uniform_2k"])
def test_random_schedule_sequences(ctx, api, name):
    """Seeded random schedule sequences (replayed), with the bitmap-output
    push and the persistent tail on and off: every mix of schedules gives
    the reference's levels and distances (the learned policy can produce
    any mix)."""
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    rng = np.random.default_rng(11)
    s0 = int(c["sources"][0])
    try:
        for trial in range(6):
            ctx.set_tunable("sssp_bm_push_min", 1 if trial % 2 == 0 else -1)
            ctx.set_tunable("tail_edges", 0 if (trial // 2) % 2 == 0 else -1)
            ctx.set_replay(list(rng.integers(0, 8, 512)))
            ctx.set_policy(api.MB_POLICY_ORACLE_BEST)
            lv, _ = g.bfs([s0])
            d, _ = g.sssp([s0])
            ctx.set_policy(api.MB_POLICY_FIXED)
            np.testing.assert_array_equal(lv[0], c["bfs_level"][0], err_msg="bfs trial %d" % trial)
            np.testing.assert_array_equal(d[0], c["sssp_dist"][0], err_msg="sssp trial %d" % trial)
    finally:
        ctx.set_policy(api.MB_POLICY_FIXED)
        ctx.set_tunable("sssp_bm_push_min", -1)
        ctx.set_tunable("tail_edges", -1)
        g.close()


def test_tunables_validate_and_reset(gpu_ctx, api):
    assert gpu_ctx.get_tunable("push_blocks_per_sm") == -1
    gpu_ctx.set_tunable("push_blocks_per_sm", 4)
    assert gpu_ctx.get_tunable("push_blocks_per_sm") == 4
    with pytest.raises(api.MedusaError):
        gpu_ctx.set_tunable("push_blocks_per_sm", 0)
    with pytest.raises(api.MedusaError):
        gpu_ctx.set_tunable(99, 1)
    for bad in (0, 3, 8):
        with pytest.raises(api.MedusaError):
            gpu_ctx.set_tunable("pr_light_vpl", bad)
        with pytest.raises(api.MedusaError):
            gpu_ctx.set_tunable("pr_short_pair", bad)
    gpu_ctx.set_tunable("push_blocks_per_sm", -1)
    assert gpu_ctx.get_tunable("push_blocks_per_sm") == -1


@pytest.mark.parametrize("direction", [None, 0, 4], ids=["fixed", "push", "pull"])
@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "rmat_skew_s12", "tiny", "empty"])
def test_batched_bfs_equals_single_source_runs(ctx, api, name, direction):
    """64-bit-mask batched BFS (fixed rule, all-push, all-pull; CUDA graph
    and host loop): levels of every source equal the oracle's."""
    gpu_ctx = ctx
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    rng = np.random.default_rng(3)
    srcs = list(rng.integers(0, c["V"], size=min(70, 3 * c["V"])))
    srcs[:len(c["sources"])] = list(c["sources"])
    if len(srcs) > 2:
        srcs[2] = srcs[1]  # a repeated source
    if direction is not None:
        gpu_ctx.set_policy(api.MB_POLICY_FORCED, direction)
    lv, st = g.bfs(srcs)
    gpu_ctx.set_policy(api.MB_POLICY_FIXED)
    if direction == 0:
        assert st["schedule_count"][4] == 0
    elif direction == 4:
        assert st["schedule_count"][0] == 0
    aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    outdeg = aa.out_degree()
    er = 0
    for i, s in enumerate(srcs):
        want, _ = O.bfs(c["V"], aa, None, [s])
        np.testing.assert_array_equal(lv[i], want, err_msg="source %d (#%d)" % (s, i))
        er += int(outdeg[want >= 0].sum())
    assert st["edges_traversed"] == er
    gpu_ctx.set_batching(False)
    lv2, _ = g.bfs(srcs)
    gpu_ctx.set_batching(True)
    np.testing.assert_array_equal(lv, lv2)
    g.close()


def test_batched_bfs_c4_size_certificates(gpu_ctx, api):
    """64 sources on a 2^20-vertex R-MAT: each source's levels pass the BFS certificate."""
    p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=2)
    V, s_, d_, _ = api.generate_edges_host(p)
    g = gpu_ctx.generate(p)
    srcs = list(range(64))
    lv, st = g.bfs(srcs)
    for i in (0, 1, 17, 63):
        bfs_certificate(V, s_, d_, lv[i], srcs[i])
    single, _ = g.bfs([17])
    gpu_ctx.set_batching(True)
    np.testing.assert_array_equal(lv[17], single[0])
    g.close()


@pytest.mark.parametrize("delta", [-1, 0, 1, 7, 100, 5000], ids=lambda d: "delta%d" % d)
@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "rmat_skew_s12", "tiny", "empty"])
def test_batched_sssp_equals_single_source_runs(gpu_ctx, api, name, delta):
    """32-source batched SSSP: distances of every source equal the oracle's,
    with plain frontier Bellman-Ford (delta 0), the default near-far width
    and widths from 1 (one bucket per distance) to past the largest
    distance (a single bucket)."""
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    rng = np.random.default_rng(5)
    srcs = list(rng.integers(0, c["V"], size=min(40, 3 * c["V"])))
    srcs[:len(c["sources"])] = list(c["sources"])
    if len(srcs) > 2:
        srcs[2] = srcs[1]
    gpu_ctx.set_tunable("mss_delta", delta)
    try:
        d, st = g.sssp(srcs)
    finally:
        gpu_ctx.set_tunable("mss_delta", -1)
    aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    for i, s in enumerate(srcs):
        want, _ = O.sssp(c["V"], aa, None, None, s)
        np.testing.assert_array_equal(d[i], want, err_msg="source %d (#%d)" % (s, i))
    g.close()


def test_batched_sssp_near_far_full_size(gpu_ctx, api):
    """32 sources on the 2^20 / 2^24 R-MAT: near-far buckets at the default
    width and at 100 give the same distances as plain frontier Bellman-Ford;
    source 5 also equals its single-source run."""
    p = api.rmat_params(20, 1 << 24, 0.45, 0.15, 0.15, seed=1, wmin=1, wmax=1000)
    g = gpu_ctx.generate(p)
    srcs = list(range(32))
    try:
        gpu_ctx.set_tunable("mss_delta", 0)
        d0, st0 = g.sssp(srcs)
        for delta in (-1, 100):
            gpu_ctx.set_tunable("mss_delta", delta)
            d1, st1 = g.sssp(srcs)
            np.testing.assert_array_equal(d1, d0, err_msg="delta %d" % delta)
            assert st1["edges_traversed"] == st0["edges_traversed"]
    finally:
        gpu_ctx.set_tunable("mss_delta", -1)
    gpu_ctx.set_batching(False)
    one, _ = g.sssp([5])
    gpu_ctx.set_batching(True)
    np.testing.assert_array_equal(d0[5], one[0])
    g.close()
