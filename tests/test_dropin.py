"""The reference's three apps in their own shape (medusa_b200/apps/dropin):
vertex attributes from a field list with the generated accessors
(get_distance / set_updated / get_level ...), the functors and the BSP loop
of the reference's main.cu files, and one line that routes each app's send
functor to the library's kernels.

Each app runs twice: routed (mb_bfs / mb_sssp / mb_pagerank_from ran, and no
generic functor kernel launched) and with the routing off (the generic
FunctorHolder kernels).  Both give the reference's results."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden
from oracle import oracle as O
from test_operator_api import write_gt

DROPIN = os.path.join(ROOT, "medusa_b200", "apps", "dropin")
NAMES = ["tiny", "rmat_s10", "grid_24", "hub", "uniform_2k", "rmat_skew_s12"]
BUILTIN_BFS, BUILTIN_SSSP, BUILTIN_PAGERANK = 1, 2, 3


def run(app, gt, arg, out, dtype, generic=False):
    cmd = [os.path.join(DROPIN, "medusa_dropin_" + app), str(gt), str(arg), str(out)]
    if generic:
        cmd.append("generic")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = [x for x in r.stdout.splitlines() if x.startswith("path=")][-1]
    rep = dict(kv.split("=") for kv in line.split())
    rep = {k: (list(map(int, v.split(","))) if k == "schedules" else int(v)) for k, v in rep.items()}
    return np.fromfile(out, dtype=dtype), rep


def test_dropin_binaries_are_built_and_check_arguments():
    for app in ("bfs", "sssp", "pagerank"):
        exe = os.path.join(DROPIN, "medusa_dropin_" + app)
        assert os.access(exe, os.X_OK), exe
        r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
        assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_dropin_apps_routed_and_generic_match_reference(name, tmp_path):
    c = load_golden(name)
    gt = tmp_path / "g.gr"
    write_gt(gt, c["V"], c["src"], c["dst"], c["w"])
    s0 = int(c["sources"][0])
    # BFS
    lv, rep = run("bfs", gt, s0, tmp_path / "lv", np.int32)
    np.testing.assert_array_equal(lv, c["bfs_level"][0])
    assert rep["path"] == BUILTIN_BFS and rep["generic_launches"] == 0
    assert rep["kernel_launches"] > 0 and sum(rep["schedules"]) > 0
    lv, rep = run("bfs", gt, s0, tmp_path / "lv", np.int32, generic=True)
    np.testing.assert_array_equal(lv, c["bfs_level"][0])
    assert rep["path"] == 0 and rep["generic_launches"] > 0
    # SSSP
    d, rep = run("sssp", gt, s0, tmp_path / "d", np.float32)
    np.testing.assert_array_equal(d.view(np.uint32), c["sssp_dist"][0].view(np.uint32))
    assert rep["path"] == BUILTIN_SSSP and rep["generic_launches"] == 0
    assert rep["kernel_launches"] > 0
    d, rep = run("sssp", gt, s0, tmp_path / "d", np.float32, generic=True)
    np.testing.assert_array_equal(d.view(np.uint32), c["sssp_dist"][0].view(np.uint32))
    assert rep["path"] == 0
    # PageRank: routed, the reference's own FP32 ranks; generic, the combiner
    # folds each vertex's slots in AA order
    iters = int(c["pr_iters"])
    r, rep = run("pagerank", gt, iters, tmp_path / "r", np.float32)
    np.testing.assert_array_equal(r.view(np.uint32), c["pr_rank"].view(np.uint32))
    assert rep["path"] == BUILTIN_PAGERANK and rep["generic_launches"] == 0
    r, rep = run("pagerank", gt, iters, tmp_path / "r", np.float32, generic=True)
    aa = O.AAGraph(c["V"], c["src"], c["dst"], c["w"])
    want = O.pagerank(c["V"], aa, None, iters, 1.0 / c["V"], order="aa")
    np.testing.assert_array_equal(r.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_dropin_bfs_and_sssp_on_a_larger_rmat_take_the_fast_schedules(tmp_path):
    """On an R-MAT with 2^16 vertices the routed BFS uses the direction-
    optimising schedules (push and pull supersteps) and the routed SSSP the
    edge-balanced push: the library's kernels, not the functor kernels."""
    from medusa_b200 import api
    p = api.rmat_params(16, 1 << 20, 0.45, 0.15, 0.15, seed=5, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    gt = tmp_path / "g.gr"
    write_gt(gt, V, s, d, w)
    lv, rep = run("bfs", gt, 0, tmp_path / "lv", np.int32)
    want, _ = O.bfs(V, s, d, [0])
    np.testing.assert_array_equal(lv, want)
    sched = rep["schedules"]
    assert sched[0] + sched[1] > 0 and sched[4] + sched[5] > 0  # push and pull supersteps
    assert rep["generic_launches"] == 0
    dist, rep = run("sssp", gt, 0, tmp_path / "d", np.float32)
    want_d, _ = O.sssp(V, s, d, w, 0)
    np.testing.assert_array_equal(dist.view(np.uint32), want_d.view(np.uint32))
    assert rep["schedules"][0] > 0 and rep["generic_launches"] == 0
