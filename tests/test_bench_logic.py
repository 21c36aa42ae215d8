"""bench.py's roofline bookkeeping on the host (no GPU): the dominant kernel
is the loop branch with the most traced time, its achieved bandwidth comes
from the per-superstep algorithmic bytes, and its DRAM traffic from the
committed ncu ratio."""
import bench


class FakeGraph:
    def bfs(self, sources):
        return None, {}

    def sssp(self, sources):
        return None, {}


class FakeCtx:
    def __init__(self, trace):
        self.trace = trace
        self.tracing = False

    def set_tracing(self, on):
        self.tracing = on

    def get_trace(self):
        assert self.tracing
        return self.trace


def rec(app, branch, n, m, ms):
    return {"app": app, "branch": branch, "frontier_vertices": n, "frontier_edges": m, "ms": ms}


def test_measured_ratio_is_read_from_the_committed_summary():
    r = bench.measured_traffic_ratio("k_push_edge_bm + k_nbm2q")
    assert r is not None and 0.5 < r < 2.0
    assert bench.measured_traffic_ratio("no such kernel") is None


def test_dominant_branch_and_its_roofline():
    trace = [rec(0, 17, 1, 100, 0.01),          # BFS tail
             rec(0, 4, 1000, 10 ** 6, 0.02),    # BFS pull
             rec(1, 19, 2000, 2 * 10 ** 6, 0.05),  # SSSP bitmap-output push, twice
             rec(1, 19, 1000, 10 ** 6, 0.03),
             rec(1, 0, 10, 1000, 0.01)]
    ctx = FakeCtx(trace)
    r = bench.kernel_roofline(ctx, FakeGraph(), 1 << 20, 6000.0, "measured")
    assert not ctx.tracing
    assert r["kernel"] == "k_push_edge_bm + k_nbm2q (SSSP, branch 19)"
    assert r["launches"] == 2
    byts = 12 * 3 * 10 ** 6 + 20 * 3000
    assert r["algorithmic_bytes_per_launch"] == round(byts / 2)
    assert abs(r["achieved"] - byts / 0.08e-3 / 1e9) < 0.1
    assert abs(r["frac"] - r["achieved"] / 6000.0) < 1e-4
    ratio = bench.measured_traffic_ratio("k_push_edge_bm + k_nbm2q")
    assert r["traffic"] == round(ratio * byts / 2)
    assert abs(r["share_of_traced_time"] - 0.08 / 0.12) < 1e-3


def test_verify_against_bsp_compares_and_restores_the_tuned_settings():
    """The bench checks its tuned outputs against one default BSP run and
    puts every tuned setting back afterwards."""
    import torch
    from medusa_b200 import api

    class Ctx:
        def __init__(self):
            self.t = {k: -1 for k in api.TUNABLES}
            self.sssp_delta = 0.0
            self.seen = None

        def get_tunable(self, k):
            return self.t[k]

        def set_tunable(self, k, v):
            self.t[k] = v

        def set_sssp_delta(self, d):
            self.sssp_delta = d

    ctx = Ctx()

    class G:
        def bfs(self, src, out):
            ctx.seen = dict(ctx.t)
            out.copy_(torch.arange(4, dtype=torch.int32))
            return out, {}

        def sssp(self, src, out):
            out.copy_(torch.tensor([0.0, 1.0, 2.0, 3.0]))
            return out, {}

    ctx.t["sssp_async"] = 1
    ctx.t["async_below"] = 1 << 20
    ctx.sssp_delta = 100.0
    lv = torch.arange(4, dtype=torch.int32)
    r = bench.verify_against_bsp(ctx, api, G(), lv, torch.tensor([0.0, 1.0, 2.0, 3.0]))
    assert r == {"bfs_levels": True, "sssp_distances": True}
    # the reference run: defaults, the asynchronous kernels off
    assert ctx.seen["sssp_async"] == 0 and ctx.seen["bfs_async"] == 0 and ctx.seen["async_below"] == -1
    assert ctx.t["sssp_async"] == 1 and ctx.t["async_below"] == 1 << 20 and ctx.sssp_delta == 100.0
    r = bench.verify_against_bsp(ctx, api, G(), lv, torch.tensor([0.0, 1.0, 2.0, 4.0]))
    assert r == {"bfs_levels": True, "sssp_distances": False}
