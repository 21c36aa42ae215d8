"""ctypes front end of the CPU oracle and of the reference's own CPU path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg, as the checker.  The product (medusa_b200) never
imports this module.

Two back ends:
  * ``liboracle.so`` -- medusa_oracle.c, the C restatement of the reference's
    superstep, and meg_order.cpp, the reference's MEG message order (C++ for
    std::sort), built by :func:`build_oracle`;
  * ``_ref/libref_{bfs,sssp,pr}.so`` -- the reference's unmodified CPU code
    (Algorithm|SSSP|MPG/CPUFunctorHoster.cpp and its host builders) plus
    ref/ref_harness.cpp, built by ref/build_ref.py when the reference tree is
    present; the files travel prebuilt otherwise.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

MEDUSA_MAX = np.float32(1e9)

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build_oracle(force=False):
    """Compile medusa_oracle.c (gcc) and meg_order.cpp (g++) into liboracle.so
    (no GPU needed)."""
    srcs = [os.path.join(HERE, "medusa_oracle.c"), os.path.join(HERE, "meg_order.cpp"),
            os.path.join(HERE, "gen.c")]
    if (not force and os.path.exists(ORACLE_SO)
            and all(os.path.getmtime(ORACLE_SO) >= os.path.getmtime(x) for x in srcs)):
        return ORACLE_SO
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        o1, o2, o3 = (os.path.join(tmp, x) for x in ("orc.o", "meg.o", "gen.o"))
        subprocess.check_call(["gcc", "-O2", "-std=c99", "-fopenmp", "-fPIC", "-c", srcs[0], "-o", o1])
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-c", srcs[1], "-o", o2])
        subprocess.check_call(["gcc", "-O2", "-std=c99", "-fopenmp", "-fPIC", "-c", srcs[2], "-o", o3])
        out = ORACLE_SO + ".tmp"
        subprocess.check_call(["g++", "-shared", "-fopenmp", o1, o2, o3, "-o", out, "-lm"])
        os.replace(out, ORACLE_SO)
    return ORACLE_SO


_lib = None


def _oracle():
    global _lib
    if _lib is None:
        build_oracle()  # rebuilds when the source is newer than the library
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_build_aa.restype = ctypes.c_int
        lib.orc_build_aa.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p,
                                     ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p,
                                     _f32p, _i32p, ctypes.c_void_p]
        lib.orc_bfs.restype = ctypes.c_int
        lib.orc_bfs.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p]
        lib.orc_sssp.restype = ctypes.c_int
        lib.orc_sssp.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _f32p, _i32p,
                                 _i32p, _f32p]
        lib.orc_pagerank_f32.restype = ctypes.c_int
        lib.orc_pagerank_f32.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p,
                                         _i32p, _i32p, ctypes.c_int, _f32p, ctypes.c_int]
        lib.orc_meg_slots.restype = ctypes.c_int
        lib.orc_meg_slots.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, _i32p]
        lib.gen_rmat.restype = None
        lib.gen_rmat.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                 _i32p, _i32p, ctypes.c_void_p]
        lib.gen_uniform.restype = None
        lib.gen_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                    ctypes.c_int32, _i32p, _i32p, ctypes.c_void_p]
        lib.gen_grid.restype = ctypes.c_int64
        lib.gen_grid.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p]
        lib.orc_pagerank_f64.restype = ctypes.c_int
        lib.orc_pagerank_f64.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p,
                                         _i32p, _i32p, ctypes.c_int, _f64p]
        _lib = lib
    return _lib


def generate(kind, seed=1, scale=0, num_vertices=0, num_edges=0, a=0.57, b=0.19, c=0.19,
             rows=0, cols=0, drop_frac=0.0, shortcut_frac=0.0, wmin=0, wmax=0):
    """The seeded generators (gen.c): (V, src, dst, w or None) for kind
    "rmat", "uniform" or "grid" -- the same edge lists the product's
    generator makes from the same parameters."""
    lib = _oracle()
    weighted = wmax > 0
    if kind == "grid":
        E = lib.gen_grid(seed, rows, cols, drop_frac, shortcut_frac, wmin, wmax, None, None, None)
        V = rows * cols
    else:
        E = int(num_edges)
        V = (1 << scale) if kind == "rmat" else int(num_vertices)
    src = np.empty(max(E, 1), np.int32)
    dst = np.empty(max(E, 1), np.int32)
    w = np.empty(max(E, 1), np.float32) if weighted else None
    wp = None if w is None else w.ctypes.data
    if kind == "rmat":
        lib.gen_rmat(seed, scale, E, a, b, c, wmin, wmax, src, dst, wp)
    elif kind == "uniform":
        lib.gen_uniform(seed, V, E, wmin, wmax, src, dst, wp)
    elif kind == "grid":
        lib.gen_grid(seed, rows, cols, drop_frac, shortcut_frac, wmin, wmax, src.ctypes.data,
                     dst.ctypes.data, wp)
    else:
        raise ValueError(kind)
    return V, src[:E], dst[:E], (None if w is None else w[:E])


class AAGraph:
    """The reference's AA layout of an edge list (orc_build_aa)."""

    def __init__(self, V, src, dst, w=None):
        lib = _oracle()
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        E = int(src.shape[0])
        self.V, self.E = int(V), E
        self.edge_index = np.zeros(V + 1, np.int32)
        self.msg_index = np.zeros(V + 1, np.int32)
        self.e_src = np.zeros(max(E, 1), np.int32)
        self.e_dst = np.zeros(max(E, 1), np.int32)
        self.e_w = np.zeros(max(E, 1), np.float32)
        self.msg_dst = np.zeros(max(E, 1), np.int32)
        self.perm = np.zeros(max(E, 1), np.int64)
        wp = None
        if w is not None:
            self._w = np.ascontiguousarray(w, dtype=np.float32)
            wp = self._w.ctypes.data
        rc = lib.orc_build_aa(V, E, src if E else np.zeros(1, np.int32),
                              dst if E else np.zeros(1, np.int32), wp,
                              self.edge_index, self.msg_index, self.e_src, self.e_dst,
                              self.e_w, self.msg_dst, self.perm.ctypes.data)
        if rc != 0:
            raise ValueError("orc_build_aa failed (bad vertex id?)")

    def out_degree(self):
        return np.diff(self.edge_index)

    @property
    def meg_slot(self):
        """Message slot of each AA edge in the reference's MEG order
        (GraphIR::sortByDegree + EdgeArray::buildMEG; meg_order.cpp)."""
        if getattr(self, "_meg_slot", None) is None:
            ms = np.zeros(max(self.E, 1), np.int32)
            if _oracle().orc_meg_slots(self.V, self.E, self.edge_index, self.e_dst,
                                       self.msg_index, ms) != 0:
                raise MemoryError("orc_meg_slots")
            self._meg_slot = ms
        return self._meg_slot


def bfs(V, src, dst, sources):
    """Levels (int32, -1 unreached) and supersteps of the reference's BFS."""
    g = src if isinstance(src, AAGraph) else AAGraph(V, src, dst)
    level = np.full(g.V, -1, np.int32)
    level[np.asarray(sources, dtype=np.int64)] = 0
    steps = _oracle().orc_bfs(g.V, g.E, g.e_src, g.e_dst, level)
    return level, steps


def sssp(V, src, dst, w, source):
    """Distances (float32, 1e9 unreached) and supersteps of the reference's SSSP."""
    g = src if isinstance(src, AAGraph) else AAGraph(V, src, dst, w)
    dist = np.full(g.V, MEDUSA_MAX, np.float32)
    dist[source] = 0.0
    steps = _oracle().orc_sssp(g.V, g.E, g.e_src, g.e_w, g.msg_dst, g.msg_index, dist)
    if steps < 0:
        raise MemoryError("orc_sssp")
    return dist, steps


def pagerank(V, src, dst, iters, init, fp64=False, order="reference"):
    """Ranks after `iters` supersteps of the reference's PageRank.  order
    "reference": each vertex folds its messages sequentially in the
    reference's MEG slot order -- the reference's FP32 result
    (MPG/CPUFunctorHoster.cpp:21-26 over the layout of MPG/EdgeDataType.cu
    :45-131); "aa": the same fold over the AA slot order
    (SSSP/EdgeDataType.cu:181-182); "device": the fixed order of the
    MB_PR_ORDER_FIXED kernels (sequential up to 64 in-edges, else 4096-edge
    blocks of 32-lane strided folds reduced by an xor butterfly, folded in
    order).  fp64: the same formula in double (order-free up to rounding)."""
    g = src if isinstance(src, AAGraph) else AAGraph(V, src, dst)
    if fp64:
        rank = np.full(g.V, float(init), np.float64)
        rc = _oracle().orc_pagerank_f64(g.V, g.E, g.e_src, g.msg_dst, g.msg_index,
                                        g.edge_index, iters, rank)
    else:
        slots = g.meg_slot if order == "reference" else g.msg_dst
        rank = np.full(g.V, np.float32(init), np.float32)
        rc = _oracle().orc_pagerank_f32(g.V, g.E, g.e_src, slots, g.msg_index,
                                        g.edge_index, iters, rank,
                                        {"reference": 0, "aa": 0, "device": 1}[order])
    if rc < 0:
        raise MemoryError("orc_pagerank")
    return rank


# ---------------------------------------------------------------------------
# The reference's own CPU path (oracle/_ref), when built.

def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % t))
               for t in ("bfs", "sssp", "pr"))


_ref_libs = {}


def _ref(tag):
    if tag not in _ref_libs:
        path = os.path.join(REF_DIR, "libref_%s.so" % tag)
        lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        lib.ref_prepare.restype = ctypes.c_void_p
        lib.ref_prepare.argtypes = [ctypes.c_int, ctypes.c_longlong, _i32p, _i32p,
                                    ctypes.c_void_p]
        lib.ref_release.restype = None
        lib.ref_release.argtypes = [ctypes.c_void_p]
        lib.ref_max_threads.restype = ctypes.c_int
        dbl = ctypes.POINTER(ctypes.c_double)
        if tag == "bfs":
            lib.ref_bfs_run.restype = ctypes.c_int
            lib.ref_bfs_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        _i32p, dbl]
        elif tag == "sssp":
            lib.ref_sssp_run.restype = ctypes.c_int
            lib.ref_sssp_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         _f32p, dbl]
        else:
            lib.ref_pagerank_run.restype = ctypes.c_int
            lib.ref_pagerank_run.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_float, ctypes.c_int, _f32p, dbl]
        _ref_libs[tag] = lib
    return _ref_libs[tag]


class RefGraph:
    """A graph prepared inside the reference's CPU path (GraphIR + layout)."""

    def __init__(self, tag, V, src, dst, w=None):
        self.tag, self.V = tag, int(V)
        self.lib = _ref(tag)
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        E = int(src.shape[0])
        wp = None
        if w is not None:
            self._w = np.ascontiguousarray(w, dtype=np.float32)
            wp = self._w.ctypes.data
        self.h = self.lib.ref_prepare(V, E, src if E else np.zeros(1, np.int32),
                                      dst if E else np.zeros(1, np.int32), wp)
        if not self.h:
            raise ValueError("ref_prepare failed")

    def close(self):
        if self.h:
            self.lib.ref_release(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def max_threads(self):
        return int(self.lib.ref_max_threads())

    def bfs(self, source, nthreads=0):
        out = np.zeros(self.V, np.int32)
        ms = ctypes.c_double(0)
        if self.lib.ref_bfs_run(self.h, int(source), nthreads, out, ctypes.byref(ms)):
            raise RuntimeError("ref_bfs_run failed")
        return out, ms.value

    def sssp(self, source, nthreads=0):
        out = np.zeros(self.V, np.float32)
        ms = ctypes.c_double(0)
        if self.lib.ref_sssp_run(self.h, int(source), nthreads, out, ctypes.byref(ms)):
            raise RuntimeError("ref_sssp_run failed")
        return out, ms.value

    def pagerank(self, iters, init, nthreads=0):
        out = np.zeros(self.V, np.float32)
        ms = ctypes.c_double(0)
        if self.lib.ref_pagerank_run(self.h, int(iters), float(init), nthreads, out,
                                     ctypes.byref(ms)):
            raise RuntimeError("ref_pagerank_run failed")
        return out, ms.value
