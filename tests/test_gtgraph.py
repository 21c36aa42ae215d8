"""GTgraph text ingest on the GPU (mb_graph_from_gtgraph) against the same
edges given as arrays, and against the format rules of the reference's reader
(MultipleGPU/PartitionManager.cu:153-213)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gt_text(V, src, dst, w, junk=True):
    rng = np.random.default_rng(1)
    lines = ["c generated for a test", "c another comment"]
    if junk:
        lines.append("a 1 1 5")  # before the p line: skipped, as the reference does
    lines.append("p sp %d %d" % (V, len(src)))
    for k, (u, v, x) in enumerate(zip(src, dst, w)):
        sep = " \t"[rng.integers(0, 2)] if junk else " "
        wtxt = ("%d" % int(x)) if (x == int(x) and k % 3) else repr(float(x))
        lines.append("a%s%d%s%d %s" % (sep, u + 1, sep, v + 1, wtxt))
        if junk and k % 97 == 0:
            lines.append("c mid-file comment")
    eol = "\r\n" if junk else "\n"
    return (eol.join(lines) + eol).encode()


@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "uniform_2k", "tiny"])
def test_gtgraph_equals_edge_arrays(gpu_ctx, name):
    from conftest import load_golden
    c = load_golden(name)
    w = c["w"].astype(np.float32)
    w[::5] += np.float32(0.5)  # some non-integer weights
    g1 = gpu_ctx.graph_from_edges(c["V"], c["src"], c["dst"], w)
    g2 = gpu_ctx.graph_from_gtgraph(gt_text(c["V"], c["src"], c["dst"], w))
    try:
        assert (g2.V, g2.E) == (g1.V, g1.E)
        a, b = g1.export(), g2.export()
        for k in ("row", "col", "rrow", "rcol", "mslot"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        np.testing.assert_array_equal(a["w"].view(np.uint32), b["w"].view(np.uint32))
        s0 = int(c["sources"][0])
        np.testing.assert_array_equal(g2.bfs([s0])[0][0], c["bfs_level"][0])
    finally:
        g1.close()
        g2.close()


def test_gtgraph_from_file_and_device_buffer(gpu_ctx, tmp_path):
    import torch
    from medusa_b200 import api
    p = api.rmat_params(12, 30000, 0.45, 0.15, 0.15, seed=3, wmin=1, wmax=100)
    V, s, d, w = api.generate_edges_host(p)
    text = gt_text(V, s, d, w, junk=False)
    path = tmp_path / "g.gr"
    path.write_bytes(text)
    g1 = gpu_ctx.graph_from_gtgraph(str(path))
    dev = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    g2 = gpu_ctx.graph_from_gtgraph(dev)
    try:
        want, _ = O.bfs(V, s, d, [0])
        for g in (g1, g2):
            np.testing.assert_array_equal(g.bfs([0])[0][0], want)
            dist, _ = g.sssp([0])
            np.testing.assert_array_equal(dist[0], O.sssp(V, s, d, w, 0)[0])
    finally:
        g1.close()
        g2.close()


@pytest.mark.parametrize("text", [b"c no p line\na 1 2 3\n", b"p sp 3 1\na 1 4 1\n",
                                  b"p sp 3 1\na 1 x 1\n", b"p sp 3 1\na 0 1 1\n"],
                         ids=["no_p", "id_above_V", "not_a_number", "id_zero"])
def test_gtgraph_rejects_bad_text(gpu_ctx, text):
    from medusa_b200 import api
    with pytest.raises(api.MedusaError):
        gpu_ctx.graph_from_gtgraph(text)
