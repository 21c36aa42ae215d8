"""The header-only operator API (include/medusa/medusa.h): the reference's
BFS, SSSP and PageRank written as Medusa functors (medusa_b200/apps) run
through the generic FunctorHolder kernels and give the reference's results.
The apps read GTgraph files through the GPU parser."""
import os
import subprocess

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "medusa_b200", "apps", "medusa_apps")


def write_gt(path, V, src, dst, w):
    with open(path, "w") as f:
        f.write("c test graph\np sp %d %d\n" % (V, len(src)))
        for u, v, x in zip(src, dst, w):
            f.write("a %d %d %d\n" % (u + 1, v + 1, int(x)))


def run_app(app, gt, arg, out, dtype):
    r = subprocess.run([APPS, app, str(gt), str(arg), str(out)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    return np.fromfile(out, dtype=dtype)


def test_apps_binary_is_built_and_checks_arguments():
    assert os.access(APPS, os.X_OK)
    r = subprocess.run([APPS], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["rmat_s10", "grid_24", "hub", "uniform_2k", "tiny"])
def test_operator_api_apps_match_reference(name, tmp_path):
    c = load_golden(name)
    gt = tmp_path / "g.gr"
    write_gt(gt, c["V"], c["src"], c["dst"], c["w"])
    s0 = int(c["sources"][0])
    lv = run_app("bfs", gt, s0, tmp_path / "lv", np.int32)
    np.testing.assert_array_equal(lv, c["bfs_level"][0])
    d = run_app("sssp", gt, s0, tmp_path / "d", np.float32)
    np.testing.assert_array_equal(d, c["sssp_dist"][0])
    r = run_app("pr", gt, 10, tmp_path / "r", np.float32)
    # the generic combiner folds each vertex's slots in order: the reference's
    # CPU fold over the AA layout, bit for bit
    aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    want = O.pagerank(c["V"], aa, None, 10, 1.0 / c["V"], order="aa")
    np.testing.assert_array_equal(r.view(np.uint32), want.view(np.uint32))


def _damped_message_pagerank(c, iters):
    """numpy restatement of msg_app (medusa_b200/apps/msg_ops.cuh): messages
    rank/outdeg, each scaled by 0.85 (float * double -> float), folded per
    vertex in AA slot order in float, rank = 0.15 + sum (double -> float)."""
    V = c["V"]
    aa = O.AAGraph(V, c["src"], c["dst"], c["w"])
    outdeg = aa.out_degree()
    rank = np.full(V, np.float32(1.0 / V), np.float32)
    slot_src = np.empty(aa.E, np.int64)
    slot_src[aa.msg_dst[:aa.E]] = aa.e_src[:aa.E]
    for _ in range(iters):
        m = (rank[slot_src] / outdeg[slot_src].astype(np.float32)).astype(np.float32)
        m = (m.astype(np.float64) * 0.85).astype(np.float32)
        new = np.empty(V, np.float32)
        for v in range(V):
            acc = np.float32(0)
            for x in m[aa.msg_index[v]:aa.msg_index[v + 1]]:
                acc = np.float32(acc + x)
            new[v] = np.float32(0.15 + np.float64(acc))
        rank = new
    return rank


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "rmat_s10", "uniform_2k"])
def test_edge_ht_and_message_functors(name, tmp_path):
    """FunctorHolder<EDGE_HT> sends and FunctorHolder<MESSAGE> rewrites every
    message before the combiner: the ranks equal the numpy restatement."""
    c = load_golden(name)
    gt = tmp_path / "g.gr"
    write_gt(gt, c["V"], c["src"], c["dst"], c["w"])
    r = run_app("prmsg", gt, 3, tmp_path / "r", np.float32)
    want = _damped_message_pagerank(c, 3)
    np.testing.assert_array_equal(r.view(np.uint32), want.view(np.uint32))
    # and the message functor really ran: without it the ranks differ
    plain = run_app("pr", gt, 3, tmp_path / "p", np.float32)
    assert not np.array_equal(r, plain) or c["V"] <= 8
