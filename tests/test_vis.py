"""Visualisation coordinates (DrawNodes / DrawEdges of the reference's
MedusaRT/GraphRenderingAPI.cu) into a headless buffer, against a numpy
restatement of the quad and endpoint arithmetic."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_node_quads(gpu_ctx):
    rng = np.random.default_rng(2)
    V = 100003
    pos = rng.uniform(-500, 500, (V, 2)).astype(np.float32)
    r = rng.integers(1, 20, V).astype(np.int32)
    q = gpu_ctx.vis_node_quads(pos, r)
    x, y, rf = pos[:, 0], pos[:, 1], r.astype(np.float32)
    want = np.stack([np.stack([x - rf, y + rf - 1], 1), np.stack([x + rf - 1, y + rf - 1], 1),
                     np.stack([x + rf - 1, y - rf], 1), np.stack([x - rf, y - rf], 1)], 1)
    np.testing.assert_array_equal(q, want.astype(np.float32))


@pytest.mark.parametrize("name", ["rmat_s10", "tiny"])
def test_edge_lines_follow_the_edge_array(gpu_ctx, name):
    c = load_golden(name)
    g = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], c["w"])
    try:
        pos = np.random.default_rng(3).uniform(0, 1000, (c["V"], 2)).astype(np.float32)
        lines = g.vis_edge_lines(pos)
        ex = g.export()
        src = np.repeat(np.arange(c["V"]), np.diff(ex["row"]))
        np.testing.assert_array_equal(lines[:, 0], pos[src])
        np.testing.assert_array_equal(lines[:, 1], pos[ex["col"]])
    finally:
        g.close()
