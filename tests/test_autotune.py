"""The autotuner: it leaves a valid setting behind, and tuned runs return
the same results as default ones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_traversals_keeps_results(gpu_ctx):
    from medusa_b200 import api, autotune
    g = gpu_ctx.generate(api.rmat_params(14, 1 << 18, 0.45, 0.15, 0.15, seed=3, wmin=1, wmax=1000))
    try:
        lv0, _ = g.bfs([0])
        d0, _ = g.sssp([0])
        best, table = autotune.tune_traversals(gpu_ctx, g, 0, reps=1)
        assert len(table) > 5
        for k, v in best.items():
            assert autotune._get(gpu_ctx, k) == v
        lv1, _ = g.bfs([0])
        d1, _ = g.sssp([0])
        np.testing.assert_array_equal(lv0, lv1)
        np.testing.assert_array_equal(d0.view(np.uint32), d1.view(np.uint32))
    finally:
        g.close()
        for k in api.TUNABLES:
            gpu_ctx.set_tunable(k, -1)
        gpu_ctx.set_sssp_delta(0.0)


def test_tune_batched_sssp_keeps_results(gpu_ctx):
    """The batched SSSP's near-far width: every candidate tried, the best
    left set, the distances unchanged."""
    from medusa_b200 import api, autotune
    g = gpu_ctx.generate(api.grid_params(96, 96, seed=4))
    try:
        srcs = list(range(0, 9216, 300))[:32]
        d0, _ = g.sssp(srcs)
        best, table = autotune.tune_batched_sssp(gpu_ctx, g, srcs, reps=1)
        assert set(best) == {"mss_delta"} and len(table) == len(autotune.MSS_DELTAS)
        assert gpu_ctx.get_tunable("mss_delta") == best["mss_delta"]
        d1, _ = g.sssp(srcs)
        np.testing.assert_array_equal(d0.view(np.uint32), d1.view(np.uint32))
    finally:
        g.close()
        gpu_ctx.set_tunable("mss_delta", -1)


def test_tune_batch(gpu_ctx):
    from medusa_b200 import api, autotune
    b = gpu_ctx.batch_generate([api.rmat_params(s, 8 << s, 0.45, 0.15, 0.15, seed=s)
                                for s in range(8, 14)])
    try:
        r0, l0, _ = b.run(5)
        best, table = autotune.tune_batch(gpu_ctx, b, 5, reps=1)
        assert set(best) == {"batch_threads", "batch_edges_per_cta"}
        r1, l1, _ = b.run(5)
        np.testing.assert_array_equal(r0.view(np.uint32), r1.view(np.uint32))
        np.testing.assert_array_equal(l0, l1)
    finally:
        b.close()
        gpu_ctx.set_tunable("batch_threads", -1)
        gpu_ctx.set_tunable("batch_edges_per_cta", -1)


def test_tune_pagerank_keeps_results(gpu_ctx):
    """Both summation orders: the tuned launch shapes (hub threshold in the
    reference's order, short-block pairing in the fixed order) change no bit."""
    from medusa_b200 import api, autotune
    g = gpu_ctx.generate(api.rmat_params(14, 1 << 18, 0.57, 0.19, 0.19, seed=3))
    try:
        for order, keys in ((api.MB_PR_ORDER_REFERENCE, {"pr_light_vpl", "pr_hub_min", "pr_hub_ctas"}),
                            (api.MB_PR_ORDER_FIXED, {"pr_light_vpl", "pr_short_pair"})):
            gpu_ctx.set_pagerank_order(order)
            r0, _ = g.pagerank(5, 1.0 / g.V)
            best, table = autotune.tune_pagerank(gpu_ctx, g, 5, reps=1)
            assert set(best) == keys and len(table) >= 5
            r1, _ = g.pagerank(5, 1.0 / g.V)
            np.testing.assert_array_equal(r0.view(np.uint32), r1.view(np.uint32))
            for k in keys:
                gpu_ctx.set_tunable(k, -1)
    finally:
        gpu_ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
        g.close()
        for k in ("pr_light_vpl", "pr_short_pair", "pr_hub_min", "pr_hub_ctas"):
            gpu_ctx.set_tunable(k, -1)
