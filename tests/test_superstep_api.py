"""mb_superstep: the BSP loop driven from the host one superstep at a time,
as the reference's main.cu files drive Medusa_Exec (ResetToExecute;
Medusa_Exec; exe = RetriveToExecute; super_step++).  The stepped runs give
the whole-run results (the reference's, from the golden fixtures) bit for
bit, under the policy's schedules and under random forced ones."""
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
    yield c
    c.close()


def stepped(g, app, source, schedules=None, steps=None):
    step, cont = 0, True
    while cont:
        sched = -1 if schedules is None else int(schedules[step % len(schedules)])
        cont = g.superstep(app, step, source, sched)
        step += 1
        if steps is not None and step >= steps:
            break
    out, st = g.superstep_result(app)
    return out, st, step


@pytest.mark.parametrize("name", golden_names())
def test_stepped_bfs_sssp_pagerank_equal_the_reference(ctx, api, name):
    c = load_golden(name)
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    s0 = int(c["sources"][0])
    rng = np.random.default_rng(len(name))
    try:
        lv, st, n = stepped(g, api.MB_APP_BFS, s0)
        np.testing.assert_array_equal(lv, c["bfs_level"][0])
        # one superstep per call (a source with no out-edges needs none)
        assert st["supersteps"] == n or (n == 1 and st["supersteps"] == 0)
        lv, _, _ = stepped(g, api.MB_APP_BFS, s0, rng.integers(0, 8, 64))
        np.testing.assert_array_equal(lv, c["bfs_level"][0])
        d, _, _ = stepped(g, api.MB_APP_SSSP, s0)
        np.testing.assert_array_equal(d.view(np.uint32), c["sssp_dist"][0].view(np.uint32))
        d, _, _ = stepped(g, api.MB_APP_SSSP, s0, rng.integers(0, 8, 64))
        np.testing.assert_array_equal(d.view(np.uint32), c["sssp_dist"][0].view(np.uint32))
        iters = int(c["pr_iters"])
        r, _, _ = stepped(g, api.MB_APP_PAGERANK, 0, steps=iters)
        np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32))
        r, _, _ = stepped(g, api.MB_APP_PAGERANK, 0, schedules=[0, 6], steps=iters)
        np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32))
    finally:
        g.close()


def test_stepped_run_ends_with_a_whole_run_and_rejects_misuse(ctx, api):
    c = load_golden("rmat_s10")
    g = ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        assert g.superstep(api.MB_APP_BFS, 0, 0)
        g.bfs([0])  # a whole run on the same graph ends the stepped one
        with pytest.raises(api.MedusaError):
            g.superstep(api.MB_APP_BFS, 1, 0)
        with pytest.raises(api.MedusaError):
            g.superstep_result(api.MB_APP_BFS)
        with pytest.raises(api.MedusaError):
            g.superstep(api.MB_APP_SSSP, 0, c["V"])  # source out of range
        with pytest.raises(api.MedusaError):
            g.superstep(7, 0, 0)
    finally:
        g.close()
