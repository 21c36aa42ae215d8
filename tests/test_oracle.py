"""The CPU oracle (oracle/medusa_oracle.c) against the golden fixtures made by
the reference's own CPU code, and (when oracle/_ref is built) against the
reference directly on random graphs."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from oracle import oracle as O


@pytest.mark.parametrize("name", golden_names())
def test_oracle_bfs_sssp_match_reference_bit_exact(name):
    c = load_golden(name)
    g = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    for i, s in enumerate(c["sources"]):
        lv, _ = O.bfs(c["V"], g, None, [s])
        np.testing.assert_array_equal(lv, c["bfs_level"][i])
        d, _ = O.sssp(c["V"], g, None, None, s)
        np.testing.assert_array_equal(d.view(np.uint32), c["sssp_dist"][i].view(np.uint32))


@pytest.mark.parametrize("name", golden_names())
def test_oracle_pagerank_within_tolerance(name):
    c = load_golden(name)
    g = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    r = O.pagerank(c["V"], g, None, c["pr_iters"], 1.0 / c["V"])
    r64 = O.pagerank(c["V"], g, None, c["pr_iters"], 1.0 / c["V"], fp64=True)
    check_pagerank(r, c["pr_rank"], r64, np.diff(g.msg_index))


def check_pagerank(got, ref, r64, indeg, tol=1e-5, hub=2048):
    """The PageRank parity rule.  The reference sums each vertex's messages in
    FP32 in its MEG slot order; another order rounds differently.  A graph
    whose in-degrees are all <= `hub`: every vertex within `tol` relative of
    the reference.  A graph with larger in-degrees: a hub's FP32 sum can
    differ by up to (n-1)*2^-24 relative between two orders, and that error
    flows to the hub's out-neighbours, so both results are held to that
    summation bound (x4 for the supersteps' carry) against the FP64 oracle."""
    got = got.astype(np.float64)
    ref = ref.astype(np.float64)
    if indeg.max(initial=0) <= hub:
        rel = np.abs(got - ref) / np.abs(ref)
        assert rel.max(initial=0) <= tol, rel.max()
        return
    bound = (float(indeg.max()) + 8) * 2.0 ** -24 * 4
    assert (np.abs(got - r64) / r64).max() <= bound
    assert (np.abs(ref - r64) / r64).max() <= bound


def test_oracle_layout_matches_reference_builders():
    # msg_index is the prefix of in-degrees; msg_dst hands out slots per
    # destination in AA edge order (SSSP/EdgeDataType.cu:181-182)
    src = np.array([0, 0, 1, 2, 2, 1], np.int32)
    dst = np.array([1, 2, 2, 0, 1, 2], np.int32)
    g = O.AAGraph(3, src, dst)
    # AA order: per source, reverse insertion order
    np.testing.assert_array_equal(g.e_src, [0, 0, 1, 1, 2, 2])
    np.testing.assert_array_equal(g.e_dst, [2, 1, 2, 2, 1, 0])
    np.testing.assert_array_equal(g.edge_index, [0, 2, 4, 6])
    np.testing.assert_array_equal(g.msg_index, [0, 1, 3, 6])
    np.testing.assert_array_equal(g.msg_dst, [3, 1, 4, 5, 2, 0])


def test_oracle_rejects_bad_ids():
    with pytest.raises(ValueError):
        O.AAGraph(3, np.array([0, 3], np.int32), np.array([1, 1], np.int32))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_equals_reference_random(seed):
    rng = np.random.default_rng(seed)
    V = int(rng.integers(2, 3000))
    E = int(rng.integers(0, 20000))
    src = rng.integers(0, V, E).astype(np.int32)
    dst = rng.integers(0, V, E).astype(np.int32)
    w = rng.integers(1, 1001, E).astype(np.float32)
    s = int(rng.integers(0, V))
    lv, _ = O.bfs(V, src, dst, [s])
    rb = O.RefGraph("bfs", V, src, dst)
    np.testing.assert_array_equal(lv, rb.bfs(s)[0])
    d, _ = O.sssp(V, src, dst, w, s)
    rs = O.RefGraph("sssp", V, src, dst, w)
    np.testing.assert_array_equal(d, rs.sssp(s)[0])
    r = O.pagerank(V, src, dst, 10, 1.0 / V)
    rp = O.RefGraph("pr", V, src, dst)
    ref = rp.pagerank(10, 1.0 / V)[0]
    assert (np.abs(r - ref) / ref).max() <= 1e-5
