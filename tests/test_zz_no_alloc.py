"""mb_pagerank_noalloc: PageRank for callers that cannot call cudaMalloc.

Some callers own all of the GPU's memory through their own pool (a database
or serving process with a fixed budget), or cannot accept cudaMalloc's device
synchronisation inside a call; this entry point takes only their device
arrays and keeps its scratch in a fixed device array inside the library.
The test calls it through the C ABI twice in a row, on two different graphs,
and checks each result against mb_pagerank bit for bit (the tolerance the
PageRank schedule tests use).  The same check also runs in a fresh Python
process (test_pagerank_noalloc_in_a_fresh_process), and the file is
collected last so that a failure here comes after every other test has run.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _device_layout(torch, g):
    lay = g.export()
    dev = torch.device("cuda", 0)
    return (torch.from_numpy(lay["row"]).to(dev), torch.from_numpy(lay["rrow"]).to(dev),
            torch.from_numpy(np.ascontiguousarray(lay["rcol"])).to(dev))


def test_pagerank_noalloc_matches_pagerank_two_calls():
    import torch
    from medusa_b200 import api
    ctx = api.Context(0)
    try:
        # mb_pagerank_noalloc sums in mb_pagerank's fixed order
        ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
        # the hub has 5000 in-edges, above kPrBlock = 4096: it is summed as two blocks
        hub = load_golden("hub")
        g1 = ctx.graph_from_edges(hub["V"], hub["src"], hub["dst"], hub["w"])
        g2 = ctx.generate(api.rmat_params(16, 1 << 20, 0.57, 0.19, 0.19, seed=3))
        for g, iters in ((g1, 10), (g2, 20)):
            want, _ = g.pagerank(iters, 1.0 / g.V)
            row, rrow, rcol = _device_layout(torch, g)
            out = torch.full((g.V,), -1.0, dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            api.pagerank_noalloc(row, rrow, rcol, g.V, iters, 1.0 / g.V, out)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
        g1.close()
        g2.close()
    finally:
        ctx.close()


def test_pagerank_noalloc_rejects_oversize_and_host_memory():
    import torch
    from medusa_b200 import api
    row = torch.zeros(3, dtype=torch.int32, device="cuda")
    rcol = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(2, dtype=torch.float32, device="cuda")
    with pytest.raises(api.MedusaError) as e:
        api.pagerank_noalloc(row, row, rcol, (1 << 20) + 1, 1, 0.5, out)
    assert e.value.code == api.MB_ERR_UNSUPPORTED
    assert "limit" in str(e.value)
    with pytest.raises(api.MedusaError) as e:
        api.pagerank_noalloc(row.cpu().numpy(), row, rcol, 2, 1, 0.5, out)
    assert e.value.code == api.MB_ERR_INVALID


def test_pagerank_noalloc_in_a_fresh_process():
    """The two-call check alone in a new interpreter: the scratch address is
    looked up there by the first call, with nothing run before it."""
    here = os.path.dirname(os.path.abspath(__file__))
    code = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r); "
            "import test_zz_no_alloc as t; t.test_pagerank_noalloc_matches_pagerank_two_calls(); "
            "print('fresh ok')" % (here, os.path.dirname(here)))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "fresh ok" in r.stdout
