"""The autotuner's search on the host (no GPU): coordinate descent over a
fake context whose run time is a known function of the settings."""
from medusa_b200 import autotune


class FakeCtx:
    def __init__(self):
        self.t = {"a": -1, "b": -1}
        self.sssp_delta = 0.0

    def get_tunable(self, name):
        return self.t[name]

    def set_tunable(self, name, value):
        self.t[name] = value

    def set_sssp_delta(self, value):
        self.sssp_delta = value


def cost(ctx):
    # best at a = 4, b = 16, delta = 100, separable
    a = 8 if ctx.t["a"] == -1 else ctx.t["a"]
    b = 32 if ctx.t["b"] == -1 else ctx.t["b"]
    return {"device_ms": abs(a - 4) + abs(b - 16) / 4 + abs(ctx.sssp_delta - 100) / 100 + 1.0}


def test_coordinate_descent_finds_the_separable_optimum_and_leaves_it_set():
    ctx = FakeCtx()
    space = {"a": [-1, 2, 4, 6], "b": [-1, 8, 16], "sssp_delta": [0.0, 100.0, 1000.0]}
    best, table = autotune.tune(ctx, lambda: cost(ctx), space, reps=1)
    assert best == {"a": 4, "b": 16, "sssp_delta": 100.0}
    assert ctx.t == {"a": 4, "b": 16} and ctx.sssp_delta == 100.0
    # the default setting, then every other candidate of every tunable once
    assert len(table) == 1 + 3 + 2 + 2
    assert min(ms for _, ms in table) == cost(ctx)["device_ms"]


def test_a_worse_candidate_is_never_kept():
    ctx = FakeCtx()
    ctx.t["a"] = 4
    best, _ = autotune.tune(ctx, lambda: cost(ctx), {"a": [-1, 0, 100]}, reps=3)
    assert best["a"] == 4 and ctx.t["a"] == 4


def test_joint_search_tries_a_switch_with_each_of_its_parameters():
    """A kernel switch that only pays with the right parameter: coordinate
    descent one tunable at a time would keep the switch off (off beats on at
    the default parameter); the joint search finds (on, 200)."""
    ctx = FakeCtx()

    def run():
        on, d = ctx.t["a"], ctx.t["b"]
        if on != 1:
            return {"device_ms": 5.0}
        return {"device_ms": 7.0 if d == -1 else 1.0 + abs(d - 200) / 100}

    best, table = autotune.tune_joint(ctx, run, ("a", "b"), [(-1, -1), (1, -1), (1, 50), (1, 200), (1, 800)],
                                      reps=1)
    assert best == {"a": 1, "b": 200} and ctx.t == {"a": 1, "b": 200}
    assert len(table) == 5  # the current setting, then the four others


def test_batched_sssp_width_search_keeps_the_fastest_width():
    """tune_batched_sssp times every candidate width over the given sources
    and leaves the fastest set."""
    from medusa_b200 import autotune

    class Ctx:
        def __init__(self):
            self.t = {"mss_delta": -1}

        def get_tunable(self, name):
            return self.t[name]

        def set_tunable(self, name, value):
            self.t[name] = value

    ctx = Ctx()
    seen = []

    class Graph:
        def sssp(self, sources):
            seen.append(list(sources))
            d = ctx.t["mss_delta"]
            return None, {"device_ms": 5.0 if d <= 0 else abs(d - 150) / 50 + 1.0}

    best, table = autotune.tune_batched_sssp(ctx, Graph(), range(32), reps=1)
    assert best == {"mss_delta": 150} and ctx.t["mss_delta"] == 150
    assert sorted(t["mss_delta"] for t, _ in table) == sorted(autotune.MSS_DELTAS)
    assert all(s == list(range(32)) for s in seen)
