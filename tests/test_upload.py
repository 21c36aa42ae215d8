"""Graphs from the caller's own arrays: a CSR (mb_graph_upload) and a batch of
edge lists (mb_graph_upload_batch).  An uploaded CSR rebuilds exactly the
graph it was exported from (every device array, so every traversal), a bad
row_ptr or column id is rejected with MB_ERR_INVALID and leaves the context
usable, and a batch of uploaded edge lists runs exactly as the same graphs
generated on the device."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import api as a
    return a


def _export(g):
    return g.export()


@pytest.mark.parametrize("reference_order", [True, False], ids=["reference_order", "input_order"])
@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "tiny", "empty"])
def test_upload_rebuilds_the_exported_graph(gpu_ctx, api, name, reference_order):
    c = load_golden(name)
    g1 = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"], reference_order=reference_order)
    d1 = _export(g1)
    g2 = gpu_ctx.graph_upload(c["V"], d1["row"], d1["col"], d1["w"])
    try:
        d2 = _export(g2)
        for k in d1:
            np.testing.assert_array_equal(d1[k], d2[k], err_msg=k)
        s = int(c["sources"][0]) if len(c["sources"]) else 0
        for g in (g1, g2):
            lv, _ = g.bfs([s])
            dist, _ = g.sssp([s])
            np.testing.assert_array_equal(lv[0], O.bfs(c["V"], c["src"], c["dst"], [s])[0])
            np.testing.assert_array_equal(dist[0], O.sssp(c["V"], c["src"], c["dst"], c["w"], s)[0])
    finally:
        g1.close()
        g2.close()


def test_upload_from_device_tensors(gpu_ctx, api):
    import torch
    c = load_golden("rmat_s10")
    g1 = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    d1 = _export(g1)
    g2 = gpu_ctx.graph_upload(c["V"], torch.from_numpy(d1["row"]).cuda(),
                              torch.from_numpy(d1["col"]).cuda(), torch.from_numpy(d1["w"]).cuda())
    try:
        d2 = _export(g2)
        for k in d1:
            np.testing.assert_array_equal(d1[k], d2[k], err_msg=k)
    finally:
        g1.close()
        g2.close()


def test_upload_without_weights(gpu_ctx, api):
    row = np.array([0, 2, 2, 3], np.int32)  # vertex 1 has no out-edges
    col = np.array([1, 2, 0], np.int32)
    g = gpu_ctx.graph_upload(3, row, col)
    try:
        d = _export(g)
        np.testing.assert_array_equal(d["row"], row)
        np.testing.assert_array_equal(d["col"], col)
        lv, _ = g.bfs([0])
        np.testing.assert_array_equal(lv[0], [0, 1, 1])
    finally:
        g.close()


@pytest.mark.parametrize("case", ["row0", "decreasing", "last_row", "column", "no_vertices"])
def test_upload_rejects_a_bad_csr(gpu_ctx, api, case):
    row = np.array([0, 2, 3, 4], np.int32)
    col = np.array([1, 2, 0, 1], np.int32)
    V = 3
    if case == "row0":
        row = np.array([1, 2, 3, 4], np.int32)
    elif case == "decreasing":
        row = np.array([0, 3, 2, 4], np.int32)
    elif case == "last_row":
        row = np.array([0, 2, 3, 3], np.int32)
    elif case == "column":
        col = np.array([1, 2, 3, 1], np.int32)
    elif case == "no_vertices":
        V = 0
    with pytest.raises(api.MedusaError) as e:
        gpu_ctx.graph_upload(V, row if V else row[:1], col)
    assert e.value.code == api.MB_ERR_INVALID
    # the context still works
    g = gpu_ctx.graph_upload(3, np.array([0, 2, 3, 4], np.int32), np.array([1, 2, 0, 1], np.int32))
    lv, _ = g.bfs([0])
    np.testing.assert_array_equal(lv[0], [0, 1, 1])
    g.close()


def test_upload_batch_runs_as_the_generated_batch(gpu_ctx, api):
    rng = np.random.default_rng(12)
    ps = [api.rmat_params(int(rng.integers(6, 11)), int(rng.integers(200, 8000)), 0.57, 0.19, 0.19,
                          seed=70 + i) for i in range(6)]
    ps.append(api.grid_params(20, 30, 0.1, 0.01, seed=71))
    ps.append(api.uniform_params(50, 0, seed=72))  # a graph without edges
    host = [api.generate_edges_host(p) for p in ps]
    b1 = gpu_ctx.batch_generate(ps)
    b2 = gpu_ctx.batch_upload([(V, s, d) for V, s, d, _ in host])
    try:
        assert (b1.n, b1.total_V, b1.total_E) == (b2.n, b2.total_V, b2.total_E)
        np.testing.assert_array_equal(b1.vbase, b2.vbase)
        srcs = [int(rng.integers(0, V)) for V, _, _, _ in host]
        r1, l1, _ = b1.run(10, srcs)
        r2, l2, _ = b2.run(10, srcs)
        np.testing.assert_array_equal(r1.view(np.uint32), r2.view(np.uint32))
        np.testing.assert_array_equal(l1, l2)
        for i, (V, s, d, _) in enumerate(host):
            want, _ = O.bfs(V, s, d, [srcs[i]])
            np.testing.assert_array_equal(l2[b2.vbase[i]:b2.vbase[i + 1]], want, err_msg="graph %d" % i)
    finally:
        b1.close()
        b2.close()


def test_upload_batch_rejects_bad_input(gpu_ctx, api):
    with pytest.raises(api.MedusaError) as e:
        gpu_ctx.batch_upload([(3, [0, 1], [1, 3])])  # vertex id 3 of a 3-vertex graph
    assert e.value.code == api.MB_ERR_INVALID
    with pytest.raises(api.MedusaError) as e:
        gpu_ctx.batch_upload([(0, [], [])])
    assert e.value.code == api.MB_ERR_INVALID
