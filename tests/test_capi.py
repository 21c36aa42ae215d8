"""CPU-only checks of the C ABI library: it loads without a GPU, exports every
symbol include/medusa_b200.h declares, its host generator is deterministic
and shaped as specified, and calls fail with status codes (no crash) when no
device is present or arguments are bad."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "medusa_b200.h")


@pytest.fixture(scope="module")
def api():
    from medusa_b200 import build
    build.build()
    from medusa_b200 import api as a
    return a


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(api):
    syms = declared_symbols()
    assert len(syms) >= 15
    lib = ctypes.CDLL(api.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_tunable_ids_match_the_header(api):
    """api.TUNABLES names every MB_TUNE_* of include/medusa_b200.h with the
    same id, and nothing else."""
    text = open(os.path.join(ROOT, "include", "medusa_b200.h")).read()
    ids = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"#define MB_TUNE_(\w+) (\d+)", text)}
    count = int(re.search(r"#define MB_NUM_TUNABLES (\d+)", text).group(1))
    assert ids == api.TUNABLES
    assert sorted(ids.values()) == list(range(count))


def test_schedule_ids_match_the_header(api):
    """The Python MB_SCHED_* ids and SCHEDULE_NAMES follow the header's."""
    text = open(os.path.join(ROOT, "include", "medusa_b200.h")).read()
    ids = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (MB_SCHED_\w+) (\d+)", text)}
    count = int(re.search(r"#define MB_NUM_SCHEDULES (\d+)", text).group(1))
    assert count == api.NUM_SCHEDULES == len(api.SCHEDULE_NAMES)
    assert ids and all(getattr(api, k) == v for k, v in ids.items())
    for k, v in ids.items():
        assert api.SCHEDULE_NAMES[v] == k[len("MB_SCHED_"):].lower()


def test_version(api):
    assert "sm_100a" in api.version()


def test_create_without_gpu_returns_error(api):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.MedusaError) as e:
        api.Context(0)
    assert e.value.code in (api.MB_ERR_CUDA, api.MB_ERR_INVALID)


def test_rmat_generator_deterministic_and_skewed(api):
    p = api.rmat_params(14, 200000, 0.57, 0.19, 0.19, seed=42, wmin=1, wmax=1000)
    V, s1, d1, w1 = api.generate_edges_host(p)
    _, s2, d2, w2 = api.generate_edges_host(p)
    assert V == 1 << 14 and len(s1) == 200000
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(w1, w2)
    assert s1.min() >= 0 and s1.max() < V and d1.min() >= 0 and d1.max() < V
    assert w1.min() >= 1 and w1.max() <= 1000 and (w1 == np.round(w1)).all()
    # quadrant (0,0) carries probability a at the top level
    top_s, top_d = s1 >> 13, d1 >> 13
    frac = np.mean((top_s == 0) & (top_d == 0))
    assert abs(frac - 0.57) < 0.01
    assert abs(np.mean(top_s == 1) - 0.24) < 0.01   # c + d
    deg = np.bincount(s1, minlength=V)
    assert deg.max() > 50 * deg.mean()              # heavy skew
    p2 = api.rmat_params(14, 200000, 0.57, 0.19, 0.19, seed=43)
    _, s3, _, w3 = api.generate_edges_host(p2)
    assert w3 is None and not np.array_equal(s1, s3)


def test_uniform_generator(api):
    p = api.uniform_params(1000, 100000, seed=3, wmin=1, wmax=1000)
    V, s, d, w = api.generate_edges_host(p)
    assert V == 1000
    assert abs(np.bincount(s, minlength=V).mean() - 100) < 1e-9
    assert np.bincount(s, minlength=V).std() < 20
    assert (s == d).sum() > 0  # self-loops kept


def test_grid_generator_shape(api):
    R, C = 50, 40
    p = api.grid_params(R, C, drop_frac=0.1, shortcut_frac=0.005, seed=9)
    V, s, d, w = api.generate_edges_host(p)
    assert V == R * C
    und = R * (C - 1) + (R - 1) * C
    shortcuts = round(0.005 * V)
    kept = (len(s) - 2 * shortcuts) // 2
    assert abs(kept / und - 0.9) < 0.03
    # bidirectional with one shared weight per undirected edge
    np.testing.assert_array_equal(s[0::2], d[1::2])
    np.testing.assert_array_equal(d[0::2], s[1::2])
    np.testing.assert_array_equal(w[0::2], w[1::2])
    assert w.min() >= 1 and w.max() <= 100
    grid = len(s) - 2 * shortcuts
    ds = np.abs(s[:grid].astype(np.int64) - d[:grid])
    assert set(np.unique(ds)) <= {1, C}


def test_generator_rejects_bad_params(api):
    bad = [api.rmat_params(40, 10, 0.5, 0.2, 0.2),
           api.rmat_params(10, 10, 0.6, 0.3, 0.3),
           api.uniform_params(0, 10),
           api.grid_params(0, 5)]
    for p in bad:
        with pytest.raises(api.MedusaError):
            api.generate_edges_host(p)


def test_pagerank_noalloc_rejects_bad_sizes_without_touching_memory(api):
    """Size and null checks come before any CUDA call: an oversize graph is
    MB_ERR_UNSUPPORTED with the limit in the message, a null array or a
    negative count MB_ERR_INVALID (no GPU needed)."""
    lib = api.lib
    rc = lib.mb_pagerank_noalloc(None, None, None, (1 << 20) + 1, 10, 1, 0.5, None, None)
    assert rc == api.MB_ERR_UNSUPPORTED
    assert b"limit" in lib.mb_last_error(None)
    assert lib.mb_pagerank_noalloc(None, None, None, 4, 10, 1, 0.5, None, None) == api.MB_ERR_INVALID
    assert lib.mb_pagerank_noalloc(None, None, None, 0, 10, 1, 0.5, None, None) == api.MB_ERR_INVALID
    assert lib.mb_pagerank_noalloc(None, None, None, 4, -1, 1, 0.5, None, None) == api.MB_ERR_INVALID
    assert lib.mb_pagerank_noalloc(None, None, None, 4, 10, -1, 0.5, None, None) == api.MB_ERR_INVALID
