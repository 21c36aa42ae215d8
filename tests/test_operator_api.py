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
    want = O.pagerank(c["V"], aa, None, 10, 1.0 / c["V"])
    np.testing.assert_array_equal(r.view(np.uint32), want.view(np.uint32))
