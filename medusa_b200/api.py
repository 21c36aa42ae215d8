"""ctypes binding of libmedusa_b200.so (the C ABI in include/medusa_b200.h).

This is plumbing for Python callers, tests and the benchmark: every call goes
straight to the CUDA library, and there is no CPU fallback -- if the shared
library is missing or cannot load, importing the binding raises.

Arrays may be numpy arrays (host memory; results are copied back) or CUDA
torch tensors (device memory, used in place).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmedusa_b200.so")

MB_OK = 0
MB_ERR_INVALID, MB_ERR_CUDA, MB_ERR_OOM, MB_ERR_TIMEOUT, MB_ERR_UNSUPPORTED = 1, 2, 3, 4, 5
MB_ORDER_INPUT, MB_ORDER_REFERENCE = 0, 1
MB_POLICY_FIXED, MB_POLICY_LEARNED, MB_POLICY_FORCED, MB_POLICY_ORACLE_BEST = 0, 1, 2, 3
MB_GEN_RMAT, MB_GEN_UNIFORM, MB_GEN_GRID = 0, 1, 2
MB_MODEL_BFS, MB_MODEL_BATCHED, MB_MODEL_SSSP = 0, 1, 2
MB_PR_ORDER_FIXED, MB_PR_ORDER_REFERENCE = 0, 1
MB_TUNE_SSSP_BM_PUSH_MIN, MB_TUNE_PUSH_BLOCKS_PER_SM, MB_TUNE_VERTEX_BLOCKS_PER_SM, \
    MB_TUNE_TAIL_EDGES, MB_TUNE_BATCH_THREADS, MB_TUNE_BATCH_EDGES_PER_CTA, \
    MB_TUNE_PR_LIGHT_VPL, MB_TUNE_PR_SHORT_PAIR, MB_TUNE_BFS_ALPHA, MB_TUNE_BFS_BETA, \
    MB_TUNE_BULK_STAGE, MB_TUNE_BFS_GAMMA, MB_TUNE_PR_HUB_MIN, MB_TUNE_WAIT_POLLS, \
    MB_TUNE_STEP_CAP, MB_TUNE_SMALL_PUSH_EDGES, MB_TUNE_PR_HUB_CTAS, MB_TUNE_SSSP_ASYNC, \
    MB_TUNE_ASYNC_DELTA, MB_TUNE_ASYNC_BLOCKS_PER_SM, MB_TUNE_BFS_ASYNC, MB_TUNE_BFS_ASYNC_DELTA, \
    MB_TUNE_ASYNC_BELOW, MB_TUNE_MSS_DELTA = \
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23
TUNABLES = {"sssp_bm_push_min": 0, "push_blocks_per_sm": 1, "vertex_blocks_per_sm": 2,
            "tail_edges": 3, "batch_threads": 4, "batch_edges_per_cta": 5,
            "pr_light_vpl": 6, "pr_short_pair": 7, "bfs_alpha": 8, "bfs_beta": 9,
            "bulk_stage": 10, "bfs_gamma": 11, "pr_hub_min": 12, "wait_polls": 13,
            "step_cap": 14, "small_push_edges": 15, "pr_hub_ctas": 16, "sssp_async": 17,
            "async_delta": 18, "async_blocks_per_sm": 19, "bfs_async": 20, "bfs_async_delta": 21,
            "async_below": 22, "mss_delta": 23}
NUM_SCHEDULES = 8
# schedule ids (MB_SCHED_* in include/medusa_b200.h)
MB_SCHED_PUSH_EDGE_QUEUE, MB_SCHED_PUSH_WARP_QUEUE, MB_SCHED_PUSH_EDGE_BITMAP, \
    MB_SCHED_PUSH_WARP_BITMAP, MB_SCHED_PULL_THREAD, MB_SCHED_PULL_WARP, MB_SCHED_PUSH_UNFUSED, \
    MB_SCHED_PULL_UNFUSED = range(8)
SCHEDULE_NAMES = ["push_edge_queue", "push_warp_queue", "push_edge_bitmap", "push_warp_bitmap",
                  "pull_thread", "pull_warp", "push_unfused", "pull_unfused"]
MEDUSA_MAX = np.float32(1e9)


class MedusaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("medusa_b200 error %d: %s" % (code, msg))
        self.code = code


class GenParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("scale", ctypes.c_int32),
                ("num_vertices", ctypes.c_int64), ("num_edges", ctypes.c_int64),
                ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double),
                ("rows", ctypes.c_int32), ("cols", ctypes.c_int32),
                ("drop_frac", ctypes.c_double), ("shortcut_frac", ctypes.c_double),
                ("wmin", ctypes.c_int32), ("wmax", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [("supersteps", ctypes.c_int32), ("status_flags", ctypes.c_int32),
                ("edges_traversed", ctypes.c_int64), ("vertices_reached", ctypes.c_int64),
                ("device_ms", ctypes.c_double),
                ("schedule_count", ctypes.c_int32 * NUM_SCHEDULES),
                ("kernel_launches", ctypes.c_int64), ("edges_scanned", ctypes.c_int64)]

    def as_dict(self):
        return {"supersteps": self.supersteps, "status_flags": self.status_flags,
                "edges_traversed": self.edges_traversed,
                "vertices_reached": self.vertices_reached, "device_ms": self.device_ms,
                "schedule_count": list(self.schedule_count),
                "kernel_launches": self.kernel_launches,
                "edges_scanned": self.edges_scanned}


def _load():
    # MEDUSA_B200_LIB: another build of the library (a variant for comparisons)
    path = os.environ.get("MEDUSA_B200_LIB", LIB_PATH)
    if not os.path.exists(path):
        raise ImportError("libmedusa_b200.so is not built: run `python -m medusa_b200.build`")
    lib = ctypes.CDLL(path)
    P, I32, I64, U32, F32 = (ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                             ctypes.c_float)
    sigs = {
        "mb_version": (ctypes.c_char_p, []),
        "mb_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(P)]),
        "mb_destroy": (ctypes.c_int, [P]),
        "mb_last_error": (ctypes.c_char_p, [P]),
        "mb_set_schedule_policy": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int]),
        "mb_set_graph_capture": (ctypes.c_int, [P, ctypes.c_int]),
        "mb_set_schedule_replay": (ctypes.c_int, [P, P, I32]),
        "mb_set_sssp_delta": (ctypes.c_int, [P, F32]),
        "mb_set_persistent_tail": (ctypes.c_int, [P, ctypes.c_int]),
        "mb_set_persistent_grid": (ctypes.c_int, [P, ctypes.c_int]),
        "mb_set_batching": (ctypes.c_int, [P, ctypes.c_int]),
        "mb_graph_from_edges": (ctypes.c_int, [P, I32, I64, P, P, P, U32, ctypes.POINTER(P)]),
        "mb_graph_upload": (ctypes.c_int, [P, I32, I64, P, P, P, ctypes.POINTER(P)]),
        "mb_graph_generate": (ctypes.c_int, [P, ctypes.POINTER(GenParams), U32,
                                             ctypes.POINTER(P)]),
        "mb_generate_edges_host": (ctypes.c_int, [ctypes.POINTER(GenParams), P, P, P,
                                                  ctypes.POINTER(I64)]),
        "mb_graph_info": (ctypes.c_int, [P, ctypes.POINTER(I32), ctypes.POINTER(I64)]),
        "mb_graph_export": (ctypes.c_int, [P, P, P, P, P, P, P, P]),
        "mb_graph_destroy": (ctypes.c_int, [P]),
        "mb_bfs": (ctypes.c_int, [P, P, P, I32, P, ctypes.POINTER(Stats)]),
        "mb_sssp": (ctypes.c_int, [P, P, P, I32, P, ctypes.POINTER(Stats)]),
        "mb_pagerank": (ctypes.c_int, [P, P, I32, F32, P, ctypes.POINTER(Stats)]),
        "mb_pagerank_noalloc": (ctypes.c_int, [P, P, P, I32, I64, I32, F32, P, P]),
        "mb_pagerank_from": (ctypes.c_int, [P, P, I32, P, P, ctypes.POINTER(Stats)]),
        "mb_superstep": (ctypes.c_int, [P, P, I32, I32, I32, I32, ctypes.POINTER(I32)]),
        "mb_superstep_result": (ctypes.c_int, [P, P, I32, P, ctypes.POINTER(Stats)]),
        "mb_scheduler_collect": (ctypes.c_int, [P, P, I32, I32, P, P, P, I32, ctypes.POINTER(I32)]),
        "mb_scheduler_train": (ctypes.c_int, [P, I32, P, P, I32, I32, F32, ctypes.c_uint64,
                                              ctypes.POINTER(F32)]),
        "mb_scheduler_num_params": (I32, []),
        "mb_set_tunable": (ctypes.c_int, [P, I32, ctypes.c_int64]),
        "mb_set_pagerank_order": (ctypes.c_int, [P, I32]),
        "mb_set_tracing": (ctypes.c_int, [P, ctypes.c_int]),
        "mb_get_trace": (ctypes.c_int, [P, P, I32, ctypes.POINTER(I32)]),
        "mb_vis_node_quads": (ctypes.c_int, [P, I32, P, P, P]),
        "mb_vis_edge_lines": (ctypes.c_int, [P, P, P, P]),
        "mb_batch_generate": (ctypes.c_int, [P, I32, P, ctypes.POINTER(P)]),
        "mb_graph_upload_batch": (ctypes.c_int, [P, I32, P, P, P, P, ctypes.POINTER(P)]),
        "mb_batch_info": (ctypes.c_int, [P, ctypes.POINTER(I32), ctypes.POINTER(I64),
                                         ctypes.POINTER(I64)]),
        "mb_batch_vertex_offsets": (ctypes.c_int, [P, P]),
        "mb_batch_run": (ctypes.c_int, [P, P, I32, P, P, P, P]),
        "mb_batch_destroy": (ctypes.c_int, [P]),
        "mb_graph_from_gtgraph": (ctypes.c_int, [P, P, I64, U32, ctypes.POINTER(P)]),
        "mb_get_tunable": (ctypes.c_int, [P, I32, ctypes.POINTER(ctypes.c_int64)]),
        "mb_scheduler_get_weights": (ctypes.c_int, [P, I32, P]),
        "mb_scheduler_set_weights": (ctypes.c_int, [P, I32, P]),
        "mb_scheduler_grad": (ctypes.c_int, [P, P, P, P, I32, P, ctypes.POINTER(F32)]),
        "mb_scheduler_pick": (ctypes.c_int, [P, I32, P, P, I32, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def version():
    return lib.mb_version().decode()


def _ptr(x):
    """Address of a numpy array or torch tensor (host or device)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return x.data_ptr()
    raise TypeError("expected a numpy array or a torch tensor, got %r" % type(x))


def _check(rc, ctx=None):
    if rc != MB_OK:
        msg = lib.mb_last_error(ctx).decode(errors="replace")
        raise MedusaError(rc, msg)


def gen_params(kind, seed=1, scale=0, num_vertices=0, num_edges=0, a=0.57, b=0.19, c=0.19,
               rows=0, cols=0, drop_frac=0.0, shortcut_frac=0.0, wmin=0, wmax=0):
    return GenParams(kind, scale, num_vertices, num_edges, a, b, c, rows, cols, drop_frac,
                     shortcut_frac, wmin, wmax, seed)


def rmat_params(scale, num_edges, a, b, c, seed=1, wmin=0, wmax=0):
    return gen_params(MB_GEN_RMAT, seed=seed, scale=scale, num_edges=num_edges, a=a, b=b, c=c,
                      wmin=wmin, wmax=wmax)


def uniform_params(num_vertices, num_edges, seed=1, wmin=0, wmax=0):
    return gen_params(MB_GEN_UNIFORM, seed=seed, num_vertices=num_vertices, num_edges=num_edges,
                      wmin=wmin, wmax=wmax)


def grid_params(rows, cols, drop_frac=0.1, shortcut_frac=0.005, seed=1, wmin=1, wmax=100):
    return gen_params(MB_GEN_GRID, seed=seed, rows=rows, cols=cols, drop_frac=drop_frac,
                      shortcut_frac=shortcut_frac, wmin=wmin, wmax=wmax)


def num_vertices_of(p):
    if p.kind == MB_GEN_RMAT:
        return 1 << p.scale
    if p.kind == MB_GEN_UNIFORM:
        return int(p.num_vertices)
    return int(p.rows) * int(p.cols)


def generate_edges_host(p, weighted=None):
    """The seeded generator run on the host: (V, src, dst, w or None)."""
    E = ctypes.c_int64(0)
    _check(lib.mb_generate_edges_host(ctypes.byref(p), None, None, None, ctypes.byref(E)))
    n = E.value
    src = np.empty(max(n, 1), np.int32)
    dst = np.empty(max(n, 1), np.int32)
    if weighted is None:
        weighted = p.wmax > 0
    w = np.empty(max(n, 1), np.float32) if weighted else None
    _check(lib.mb_generate_edges_host(ctypes.byref(p), src.ctypes.data, dst.ctypes.data,
                                      None if w is None else w.ctypes.data, ctypes.byref(E)))
    return num_vertices_of(p), src[:n], dst[:n], (None if w is None else w[:n])


def pagerank_noalloc(row, rrow, rcol, num_vertices, iters, init, rank_out, stream=None):
    """mb_pagerank_noalloc on caller-owned CUDA tensors (no allocation inside).
    Asynchronous on `stream` (a raw cudaStream_t value, or None for the
    default stream)."""
    _check(lib.mb_pagerank_noalloc(_ptr(row), _ptr(rrow), _ptr(rcol), int(num_vertices),
                                   int(rcol.shape[0]), int(iters), float(init), _ptr(rank_out),
                                   stream))


class Graph:
    """A device-resident graph (CSR + reverse CSR + message slots)."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = ctypes.c_void_p(handle)
        V = ctypes.c_int32(0)
        E = ctypes.c_int64(0)
        _check(lib.mb_graph_info(self.h, ctypes.byref(V), ctypes.byref(E)))
        self.V, self.E = V.value, E.value

    def close(self):
        if self.h:
            lib.mb_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        """Device layout as numpy arrays: row, col, w, rrow, rcol, mslot."""
        V, E = self.V, self.E
        row = np.empty(V + 1, np.int32)
        rrow = np.empty(V + 1, np.int32)
        col = np.empty(max(E, 1), np.int32)
        w = np.empty(max(E, 1), np.float32)
        rcol = np.empty(max(E, 1), np.int32)
        mslot = np.empty(max(E, 1), np.int32)
        _check(lib.mb_graph_export(self.ctx.h, self.h, row.ctypes.data, col.ctypes.data,
                                   w.ctypes.data, rrow.ctypes.data, rcol.ctypes.data,
                                   mslot.ctypes.data), self.ctx.h)
        return {"row": row, "col": col[:E], "w": w[:E], "rrow": rrow, "rcol": rcol[:E],
                "mslot": mslot[:E]}

    def bfs(self, sources, out=None):
        src = np.ascontiguousarray(np.atleast_1d(sources), dtype=np.int32)
        if out is None:
            out = np.empty((len(src), self.V), np.int32)
        st = Stats()
        _check(lib.mb_bfs(self.ctx.h, self.h, src.ctypes.data, len(src), _ptr(out),
                          ctypes.byref(st)), self.ctx.h)
        return out, st.as_dict()

    def sssp(self, sources, out=None):
        src = np.ascontiguousarray(np.atleast_1d(sources), dtype=np.int32)
        if out is None:
            out = np.empty((len(src), self.V), np.float32)
        st = Stats()
        _check(lib.mb_sssp(self.ctx.h, self.h, src.ctypes.data, len(src), _ptr(out),
                           ctypes.byref(st)), self.ctx.h)
        return out, st.as_dict()

    def vis_edge_lines(self, pos):
        """Endpoints of every edge (DrawEdges) in edge order: pos [V,2] -> [E,2,2]."""
        pos = np.ascontiguousarray(pos, np.float32)
        out = np.empty((self.E, 2, 2), np.float32)
        _check(lib.mb_vis_edge_lines(self.ctx.h, self.h, pos.ctypes.data, out.ctypes.data), self.ctx.h)
        return out

    def pagerank(self, iters, init=None, out=None):
        if init is None:
            init = 1.0 / self.V
        if out is None:
            out = np.empty(self.V, np.float32)
        st = Stats()
        _check(lib.mb_pagerank(self.ctx.h, self.h, int(iters), float(init), _ptr(out),
                               ctypes.byref(st)), self.ctx.h)
        return out, st.as_dict()


def _pagerank_from(self, iters, init_ranks, out=None):
    """`iters` supersteps from a rank per vertex (mb_pagerank_from)."""
    if not hasattr(init_ranks, "data_ptr"):
        init_ranks = np.ascontiguousarray(init_ranks, np.float32)
    if out is None:
        out = np.empty(self.V, np.float32)
    st = Stats()
    _check(lib.mb_pagerank_from(self.ctx.h, self.h, int(iters), _ptr(init_ranks), _ptr(out),
                                ctypes.byref(st)), self.ctx.h)
    return out, st.as_dict()


Graph.pagerank_from = _pagerank_from

MB_APP_BFS, MB_APP_SSSP, MB_APP_PAGERANK = 0, 1, 2


def _superstep(self, app, step, source=0, schedule=-1):
    """One superstep of a stepped run (mb_superstep): True while another is needed."""
    cont = ctypes.c_int32(0)
    _check(lib.mb_superstep(self.ctx.h, self.h, int(app), int(step), int(source), int(schedule),
                            ctypes.byref(cont)), self.ctx.h)
    return bool(cont.value)


def _superstep_result(self, app, out=None):
    """The stepped run's levels / distances / ranks and statistics; ends the run."""
    if out is None:
        out = np.empty(self.V, np.int32 if app == MB_APP_BFS else np.float32)
    st = Stats()
    _check(lib.mb_superstep_result(self.ctx.h, self.h, int(app), _ptr(out), ctypes.byref(st)),
           self.ctx.h)
    return out, st.as_dict()


Graph.superstep = _superstep
Graph.superstep_result = _superstep_result


class Batch:
    """Many independent graphs run together (mb_batch_*)."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = ctypes.c_void_p(handle)
        n = ctypes.c_int32(0)
        V = ctypes.c_int64(0)
        E = ctypes.c_int64(0)
        _check(lib.mb_batch_info(self.h, ctypes.byref(n), ctypes.byref(V), ctypes.byref(E)))
        self.n, self.total_V, self.total_E = n.value, V.value, E.value
        self.vbase = np.zeros(self.n + 1, np.int64)
        _check(lib.mb_batch_vertex_offsets(self.h, self.vbase.ctypes.data))

    def close(self):
        if self.h:
            lib.mb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, pr_iters=20, sources=None, ranks=None, levels=None):
        """PageRank then one BFS on every graph, one launch: (ranks, levels, stats),
        concatenated by vbase."""
        src = None
        if sources is not None:
            src = np.ascontiguousarray(sources, np.int32)
            assert len(src) == self.n
        if ranks is None:
            ranks = np.empty(self.total_V, np.float32)
        if levels is None:
            levels = np.empty(self.total_V, np.int32)
        st = Stats()
        _check(lib.mb_batch_run(self.ctx.h, self.h, int(pr_iters), _ptr(src), _ptr(ranks),
                                _ptr(levels), ctypes.byref(st)), self.ctx.h)
        return ranks, levels, st.as_dict()

    def split(self, arr):
        return [arr[self.vbase[i]:self.vbase[i + 1]] for i in range(self.n)]


def c4b_params(n=256, seed=1):
    """The many-graph workload: n R-MAT graphs, (a,b,c) = (0.45,0.15,0.15),
    vertices 2^10..2^18 log-uniform (2^s with s uniform in [10, 18], rounded to
    a whole scale), average degree uniform in [4, 32]; seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        scale = int(rng.integers(10, 19))
        deg = float(rng.uniform(4, 32))
        out.append(rmat_params(scale, int(round(deg * (1 << scale))), 0.45, 0.15, 0.15,
                               seed=seed * 100003 + i))
    return out


class Context:
    """One CUDA device, one stream, and the device scratch of every run."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(lib.mb_create(int(device), ctypes.byref(h)))
        self.h = h
        self.policy = (MB_POLICY_FIXED, 0)
        self.sssp_delta = 0.0
        self.pr_order = MB_PR_ORDER_REFERENCE

    def close(self):
        if self.h:
            lib.mb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_policy(self, policy, schedule=0):
        _check(lib.mb_set_schedule_policy(self.h, int(policy), int(schedule)), self.h)
        self.policy = (int(policy), int(schedule))

    def set_replay(self, schedules):
        arr = np.ascontiguousarray(schedules, dtype=np.int8)
        _check(lib.mb_set_schedule_replay(self.h, arr.ctypes.data, len(arr)), self.h)

    def set_sssp_delta(self, delta):
        """SSSP near-far bucket width (> 0), 0 for plain Bellman-Ford, < 0 per-graph default."""
        _check(lib.mb_set_sssp_delta(self.h, float(delta)), self.h)
        self.sssp_delta = float(delta)

    def set_persistent_tail(self, enable):
        _check(lib.mb_set_persistent_tail(self.h, 1 if enable else 0), self.h)

    def set_persistent_grid(self, enable):
        _check(lib.mb_set_persistent_grid(self.h, 1 if enable else 0), self.h)

    # ---- learned scheduler ----
    def scheduler_collect(self, g, app, source, max_samples=4096):
        """Timing traces of one run (app 0 BFS, 1 SSSP, 2 batched BFS from
        `source` and the 63 vertices after it): features [n,6],
        per-schedule superstep times [n,8] (ms, -1 unmeasured) and the
        schedule the fixed rule chose at each superstep [n]."""
        X = np.zeros((max_samples, 6), np.float32)
        T = np.zeros((max_samples, 8), np.float32)
        S = np.zeros(max_samples, np.int32)
        n = ctypes.c_int32(0)
        _check(lib.mb_scheduler_collect(self.h, g.h, int(app), int(source), X.ctypes.data,
                                        T.ctypes.data, S.ctypes.data, max_samples,
                                        ctypes.byref(n)), self.h)
        k = n.value
        return X[:k].copy(), T[:k].copy(), S[:k].copy()

    def scheduler_train(self, X, T, epochs=1500, lr=3e-3, seed=1, model=MB_MODEL_BFS):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = ctypes.c_float(0)
        _check(lib.mb_scheduler_train(self.h, int(model), X.ctypes.data, T.ctypes.data, len(X),
                                      int(epochs), float(lr), int(seed), ctypes.byref(loss)),
               self.h)
        return loss.value

    def scheduler_weights(self, model=MB_MODEL_BFS):
        w = np.zeros(lib.mb_scheduler_num_params(), np.float32)
        _check(lib.mb_scheduler_get_weights(self.h, int(model), w.ctypes.data), self.h)
        return w

    def scheduler_set_weights(self, w, model=MB_MODEL_BFS):
        w = np.ascontiguousarray(w, np.float32)
        assert len(w) == lib.mb_scheduler_num_params()
        _check(lib.mb_scheduler_set_weights(self.h, int(model), w.ctypes.data), self.h)

    def scheduler_grad(self, w, X, T):
        w = np.ascontiguousarray(w, np.float32)
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        g = np.zeros(lib.mb_scheduler_num_params(), np.float32)
        loss = ctypes.c_float(0)
        _check(lib.mb_scheduler_grad(self.h, w.ctypes.data, X.ctypes.data, T.ctypes.data, len(X),
                                     g.ctypes.data, ctypes.byref(loss)), self.h)
        return g, loss.value

    def scheduler_pick(self, X, model=MB_MODEL_BFS, fallback=None):
        """The model's choice per feature row; with `fallback` (the fixed
        rule's choices), the in-run rule that overrides them only by a margin."""
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros(len(X), np.int32)
        fb = None
        if fallback is not None:
            fb = np.ascontiguousarray(fallback, np.int32)
            assert len(fb) == len(X)
        _check(lib.mb_scheduler_pick(self.h, int(model), X.ctypes.data,
                                     fb.ctypes.data if fb is not None else None, len(X),
                                     out.ctypes.data), self.h)
        return out

    def set_tunable(self, which, value):
        """Launch/routing parameter (name from TUNABLES or MB_TUNE_* id); -1: default."""
        w = TUNABLES[which] if isinstance(which, str) else int(which)
        _check(lib.mb_set_tunable(self.h, w, int(value)), self.h)

    def get_tunable(self, which):
        w = TUNABLES[which] if isinstance(which, str) else int(which)
        v = ctypes.c_int64(0)
        _check(lib.mb_get_tunable(self.h, w, ctypes.byref(v)), self.h)
        return v.value

    def vis_node_quads(self, pos, radius):
        """Quad corners of every vertex (DrawNodes): pos [V,2] float32, radius
        [V] int32 -> [V,4,2] float32."""
        pos = np.ascontiguousarray(pos, np.float32)
        radius = np.ascontiguousarray(radius, np.int32)
        out = np.empty((len(radius), 4, 2), np.float32)
        _check(lib.mb_vis_node_quads(self.h, len(radius), pos.ctypes.data, radius.ctypes.data,
                                     out.ctypes.data), self.h)
        return out

    TRACE_DTYPE = np.dtype([("app", np.int32), ("step", np.int32), ("sched", np.int32),
                            ("branch", np.int32), ("frontier_vertices", np.uint32),
                            ("frontier_edges", np.uint64), ("ms", np.float32)], align=True)

    def set_tracing(self, enable):
        """Host-driven loops with every superstep timed alone (CUDA events)."""
        _check(lib.mb_set_tracing(self.h, 1 if enable else 0), self.h)

    def get_trace(self, max_records=1 << 16):
        out = np.zeros(max_records, self.TRACE_DTYPE)
        n = ctypes.c_int32(0)
        _check(lib.mb_get_trace(self.h, out.ctypes.data, max_records, ctypes.byref(n)), self.h)
        return out[:n.value].copy()

    def set_pagerank_order(self, order):
        """MB_PR_ORDER_REFERENCE (default: the reference's MEG order, its FP32
        result bit for bit) or MB_PR_ORDER_FIXED (a fixed parallel order)."""
        _check(lib.mb_set_pagerank_order(self.h, int(order)), self.h)
        self.pr_order = int(order)

    def set_batching(self, enable):
        _check(lib.mb_set_batching(self.h, 1 if enable else 0), self.h)

    def set_graph_capture(self, enable):
        _check(lib.mb_set_graph_capture(self.h, 1 if enable else 0), self.h)

    def graph_from_edges(self, V, src, dst, w=None, reference_order=True):
        src = src if hasattr(src, "data_ptr") else np.ascontiguousarray(src, dtype=np.int32)
        dst = dst if hasattr(dst, "data_ptr") else np.ascontiguousarray(dst, dtype=np.int32)
        if w is not None and not hasattr(w, "data_ptr"):
            w = np.ascontiguousarray(w, dtype=np.float32)
        E = int(src.shape[0])
        g = ctypes.c_void_p()
        flags = MB_ORDER_REFERENCE if reference_order else MB_ORDER_INPUT
        _check(lib.mb_graph_from_edges(self.h, int(V), E, _ptr(src) if E else None,
                                       _ptr(dst) if E else None, _ptr(w) if E else None,
                                       flags, ctypes.byref(g)), self.h)
        return Graph(self, g.value)

    def graph_upload(self, V, row, col, w=None):
        """Graph from a CSR (mb_graph_upload): row[V+1], col[E], optional w[E];
        each row keeps its order."""
        row = row if hasattr(row, "data_ptr") else np.ascontiguousarray(row, dtype=np.int32)
        col = col if hasattr(col, "data_ptr") else np.ascontiguousarray(col, dtype=np.int32)
        if w is not None and not hasattr(w, "data_ptr"):
            w = np.ascontiguousarray(w, dtype=np.float32)
        E = int(col.shape[0])
        g = ctypes.c_void_p()
        _check(lib.mb_graph_upload(self.h, int(V), E, _ptr(row), _ptr(col) if E else None,
                                   _ptr(w) if (E and w is not None) else None, ctypes.byref(g)), self.h)
        return Graph(self, g.value)

    def graph_from_gtgraph(self, text, reference_order=True):
        """Graph from GTgraph text: bytes, a str path, or a device uint8 tensor
        (parsed on the GPU)."""
        if isinstance(text, str):
            with open(text, "rb") as f:
                text = f.read()
        if isinstance(text, (bytes, bytearray)):
            buf = np.frombuffer(bytes(text), np.uint8)
            ptr, n = (buf.ctypes.data if len(buf) else None), len(buf)
        else:
            ptr, n = _ptr(text), int(text.numel())
        g = ctypes.c_void_p()
        flags = MB_ORDER_REFERENCE if reference_order else MB_ORDER_INPUT
        _check(lib.mb_graph_from_gtgraph(self.h, ptr, n, flags, ctypes.byref(g)), self.h)
        return Graph(self, g.value)

    def batch_generate(self, params_list):
        arr = (GenParams * len(params_list))(*params_list)
        h = ctypes.c_void_p()
        _check(lib.mb_batch_generate(self.h, len(params_list), ctypes.cast(arr, ctypes.c_void_p),
                                     ctypes.byref(h)), self.h)
        return Batch(self, h.value)

    def batch_upload(self, graphs):
        """A batch from the caller's graphs (mb_graph_upload_batch): a list of
        (V, src, dst) with ids local to each graph."""
        nv = np.ascontiguousarray([int(V) for V, _, _ in graphs], dtype=np.int32)
        ne = np.ascontiguousarray([len(s) for _, s, _ in graphs], dtype=np.int64)
        src = np.ascontiguousarray(np.concatenate([np.asarray(s, np.int32) for _, s, _ in graphs]))
        dst = np.ascontiguousarray(np.concatenate([np.asarray(d, np.int32) for _, _, d in graphs]))
        h = ctypes.c_void_p()
        _check(lib.mb_graph_upload_batch(self.h, len(graphs), nv.ctypes.data, ne.ctypes.data,
                                         src.ctypes.data if len(src) else None,
                                         dst.ctypes.data if len(dst) else None, ctypes.byref(h)), self.h)
        return Batch(self, h.value)

    def generate(self, params, reference_order=True):
        g = ctypes.c_void_p()
        flags = MB_ORDER_REFERENCE if reference_order else MB_ORDER_INPUT
        _check(lib.mb_graph_generate(self.h, ctypes.byref(params), flags, ctypes.byref(g)),
               self.h)
        return Graph(self, g.value)
