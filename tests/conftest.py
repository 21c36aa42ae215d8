"""Shared fixtures: golden cases and the GPU marker.

Tests marked ``gpu`` need a B200 and the built libmedusa_b200.so; everything
else runs on a CPU-only machine.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def golden_names():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return sorted(json.load(f))


def edges_sha(src, dst, w):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(src, np.int32).tobytes())
    h.update(np.ascontiguousarray(dst, np.int32).tobytes())
    if w is not None:
        h.update(np.ascontiguousarray(w, np.float32).tobytes())
    return h.hexdigest()


def gen_params(d):
    from medusa_b200 import api
    d = dict(d)
    kind = d.pop("kind")
    if kind == "rmat":
        return api.rmat_params(d["scale"], d["num_edges"], d["a"], d["b"], d["c"],
                               seed=d["seed"], wmin=d["wmin"], wmax=d["wmax"])
    if kind == "uniform":
        return api.uniform_params(d["num_vertices"], d["num_edges"], seed=d["seed"],
                                  wmin=d["wmin"], wmax=d["wmax"])
    return api.grid_params(d["rows"], d["cols"], d["drop_frac"], d["shortcut_frac"],
                           seed=d["seed"], wmin=d["wmin"], wmax=d["wmax"])


def load_golden(name):
    """Return dict(V, src, dst, w, sources, bfs_level, sssp_dist, pr_rank, pr_iters)."""
    with open(os.path.join(GOLDEN, "index.json")) as f:
        meta = json.load(f)[name]
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {k: z[k] for k in z.files}
    out["V"] = int(out["V"])
    out["pr_iters"] = int(out["pr_iters"])
    if meta["kind"] == "generated":
        from medusa_b200 import api
        V, src, dst, w = api.generate_edges_host(gen_params(meta["params"]))
        assert edges_sha(src, dst, w) == meta["edges_sha256"], "generator output changed"
        out.update(src=src, dst=dst, w=w)
    out["name"] = name
    return out


@pytest.fixture(scope="session")
def gpu_ctx():
    from medusa_b200 import api
    ctx = api.Context(0)
    yield ctx
    ctx.close()
