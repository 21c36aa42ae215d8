"""Many independent graphs in one persistent launch (mb_batch_*): every
graph's PageRank equals mb_pagerank on that graph bit for bit, and its BFS
levels equal the oracle's, for several team shapes."""
import numpy as np
import pytest

from oracle import oracle as O


def small_batch_params(api):
    rng = np.random.default_rng(4)
    ps = []
    for i in range(12):
        scale = int(rng.integers(6, 13))
        deg = float(rng.uniform(2, 24))
        ps.append(api.rmat_params(scale, int(deg * (1 << scale)), 0.57, 0.19, 0.19, seed=50 + i))
    ps.append(api.uniform_params(3000, 40000, seed=7))
    ps.append(api.grid_params(30, 40, 0.1, 0.01, seed=8))
    # a star-heavy graph: in-degrees above the 4096-edge block
    ps.append(api.rmat_params(12, 60000, 0.9, 0.03, 0.03, seed=9))
    return ps


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(-1, -1), (64, 256), (512, 4096), (128, 1 << 30)],
                         ids=["default", "t64_small_teams", "t512", "one_cta_per_graph"])
def test_batch_matches_single_graph_runs(gpu_ctx, api, shape):
    threads, epc = shape
    gpu_ctx.set_tunable("batch_threads", threads)
    gpu_ctx.set_tunable("batch_edges_per_cta", epc)
    ps = small_batch_params(api)
    b = gpu_ctx.batch_generate(ps)
    rng = np.random.default_rng(1)
    srcs = [int(rng.integers(0, api.num_vertices_of(p))) for p in ps]
    try:
        ranks, levels, st = b.run(20, srcs)
        ranks2, levels2, _ = b.run(20, srcs)  # a second run reuses the batch
        np.testing.assert_array_equal(ranks, ranks2)
        np.testing.assert_array_equal(levels, levels2)
        er = 0
        for i, p in enumerate(ps):
            V, s, d, _ = api.generate_edges_host(p)
            g = gpu_ctx.generate(p)
            gpu_ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)  # the many-graph kernel's order
            try:
                r, _ = g.pagerank(20, 1.0 / V)
            finally:
                gpu_ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
            g.close()
            got_r = ranks[b.vbase[i]:b.vbase[i + 1]]
            np.testing.assert_array_equal(got_r.view(np.uint32), r.view(np.uint32),
                                          err_msg="graph %d ranks" % i)
            want_l, _ = O.bfs(V, s, d, [srcs[i]])
            np.testing.assert_array_equal(levels[b.vbase[i]:b.vbase[i + 1]], want_l,
                                          err_msg="graph %d levels" % i)
            outdeg = np.bincount(s, minlength=V)
            er += int(outdeg[want_l >= 0].sum())
        assert st["edges_traversed"] == 20 * b.total_E + er
        assert st["kernel_launches"] == 1
    finally:
        b.close()
        gpu_ctx.set_tunable("batch_threads", -1)
        gpu_ctx.set_tunable("batch_edges_per_cta", -1)


@pytest.mark.gpu
def test_batch_zero_iterations_and_bad_source(gpu_ctx, api):
    ps = small_batch_params(api)[:3]
    b = gpu_ctx.batch_generate(ps)
    try:
        ranks, levels, _ = b.run(0)
        for i in range(b.n):
            V = b.vbase[i + 1] - b.vbase[i]
            assert (ranks[b.vbase[i]:b.vbase[i + 1]] == np.float32(1.0 / V)).all()
        with pytest.raises(api.MedusaError):
            b.run(1, [0, 0, 1 << 20])
    finally:
        b.close()


def test_c4b_workload_shape(api):
    ps = api.c4b_params(256, seed=1)
    Vs = np.array([api.num_vertices_of(p) for p in ps])
    degs = np.array([p.num_edges for p in ps]) / Vs
    assert Vs.min() >= 1 << 10 and Vs.max() <= 1 << 18
    assert degs.min() >= 4 and degs.max() <= 32
