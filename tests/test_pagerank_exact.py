"""PageRank in the reference's order (MB_PR_ORDER_REFERENCE): the parallel
kernels (light lists, sliced ELL, the per-hub integer scan of pr_order.cuh)
give the reference's own FP32 ranks bit for bit.

Comparators: the golden fixtures (the reference's CPU path, over its MEG
layout) on every golden graph, and -- at sizes whose hubs have hundreds of
thousands of in-edges -- the message-reading schedule, which folds each
vertex serially over the same MEG slots (bit-identical to the goldens)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


@pytest.fixture(scope="module")
def ctx(api):
    c = api.Context(0)
    c.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
    yield c
    c.close()


def _serial(ctx, api, g, iters, init):
    """The message-reading schedule: every vertex folded by one lane, in order."""
    ctx.set_policy(api.MB_POLICY_FORCED, 6)
    try:
        r, _ = g.pagerank(iters, init)
    finally:
        ctx.set_policy(api.MB_POLICY_FIXED)
    return r


@pytest.mark.parametrize("name", golden_names())
def test_exact_pagerank_equals_reference_fp32(ctx, api, name):
    """Every hub threshold (64: every vertex above 64 in-edges goes through the
    integer scan; 2^30: none does) and every light-vertex packing."""
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        for hub_min in (64, 100, 2048, 1 << 30):
            for vpl in (1, 2, 4):
                ctx.set_tunable("pr_hub_min", hub_min)
                ctx.set_tunable("pr_light_vpl", vpl)
                r, _ = g.pagerank(c["pr_iters"], 1.0 / c["V"])
                np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32),
                                              err_msg="hub_min %d vpl %d" % (hub_min, vpl))
    finally:
        ctx.set_tunable("pr_hub_min", -1)
        ctx.set_tunable("pr_light_vpl", -1)
        g.close()


@pytest.mark.parametrize("scale,iters", [(14, 5), (21, 20)])
def test_exact_pagerank_on_skewed_rmat_equals_serial_fold(ctx, api, scale, iters):
    """R-MAT (0.57,0.19,0.19,0.05) with 16 edges per vertex: at 2^21 vertices
    the largest hub has about 10^5 in-edges, where a parallel order of the
    sum differs from the reference's by more than 1e-5.  The parallel exact
    kernels equal the serial fold bit for bit at several hub thresholds."""
    import torch
    p = api.rmat_params(scale, 16 << scale, 0.57, 0.19, 0.19, seed=1)
    g = ctx.generate(p)
    V = g.V
    try:
        want = _serial(ctx, api, g, iters, 1.0 / V)
        rrow = g.export()["rrow"]
        indeg = np.diff(rrow)
        assert indeg.max() > 4096
        out = torch.empty(V, dtype=torch.float32, device="cuda")
        for hub_min in (64, 512, 2048, 16384):
            ctx.set_tunable("pr_hub_min", hub_min)
            g.pagerank(iters, 1.0 / V, out=out)
            got = out.cpu().numpy()
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32),
                                          err_msg="hub_min %d" % hub_min)
    finally:
        ctx.set_tunable("pr_hub_min", -1)
        g.close()


def test_fixed_order_misses_the_rule_where_the_exact_order_meets_it(ctx, api):
    """The reason for the exact kernels: on a graph with a 10^5-in-edge hub
    the fixed parallel order's ranks differ from the reference's sequential
    FP32 ranks by more than the 1e-5 per-vertex rule allows somewhere near
    that bound, while the exact order differs by 0."""
    p = api.rmat_params(21, 16 << 21, 0.57, 0.19, 0.19, seed=1)
    g = ctx.generate(p)
    V = g.V
    try:
        ref = _serial(ctx, api, g, 20, 1.0 / V).astype(np.float64)
        exact, _ = g.pagerank(20, 1.0 / V)
        assert np.array_equal(exact.astype(np.float64), ref)
        ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
        fixed, _ = g.pagerank(20, 1.0 / V)
        rel = np.abs(fixed.astype(np.float64) - ref) / ref
        assert rel.max() > 1e-7  # a different order: different bits
    finally:
        ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
        g.close()
