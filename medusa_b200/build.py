"""Build libmedusa_b200.so in-tree from medusa_b200/csrc/*.cu for sm_100a.

    python -m medusa_b200.build [--force] [--jobs N]

nvcc compiles each .cu file to an object (in parallel) with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and links them into
``medusa_b200/libmedusa_b200.so`` (static cudart, OpenMP for the host-side
generators).  No GPU is needed to build.
"""
import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmedusa_b200.so")
APPS_DIR = os.path.join(HERE, "apps")
APPS_BIN = os.path.join(APPS_DIR, "medusa_apps")
ROOT = os.path.dirname(HERE)
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-fopenmp,-O3", "-I", os.path.join(ROOT, "include")] + ARCH


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "medusa", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, jobs=None, verbose=False, defines=(), out_dir=None):
    """Compile (when stale) and return the path of the shared library.
    defines/out_dir: a variant build (e.g. ["MB_TILE_EDGES=2048"]) into its own
    directory, for comparisons; the default build is the product."""
    global OBJ, LIB
    if out_dir:
        OBJ = os.path.join(out_dir, "_build")
        LIB = os.path.join(out_dir, "libmedusa_b200.so")
    extra = [f for d in defines for f in ("-D", d)]
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    hdrs = _headers()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            todo.append((s, o))

    def cc(job):
        s, o = job
        cmd = [NVCC] + NVFLAGS + extra + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s" % (s, r.stderr[-6000:]))
        return r.stderr

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for err in ex.map(cc, todo):
                if verbose and err.strip():
                    print(err)
    if force or todo or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s" % r.stderr[-6000:])
    if not out_dir:
        build_apps(force)
    return LIB


def build_apps(force=False):
    """The operator-API apps (medusa_b200/apps) -> medusa_b200/apps/medusa_apps,
    linked against the in-tree library (rpath $ORIGIN/..)."""
    srcs = glob.glob(os.path.join(APPS_DIR, "*.cu")) + glob.glob(os.path.join(APPS_DIR, "*.cuh"))
    deps = srcs + [LIB] + glob.glob(os.path.join(ROOT, "include", "medusa", "*.h"))
    if not force and not _stale(APPS_BIN, deps):
        return APPS_BIN
    cmd = ([NVCC, "-std=c++17", "-O3", "-lineinfo"] + ARCH +
           ["-I", os.path.join(ROOT, "include"), "-I", APPS_DIR,
            os.path.join(APPS_DIR, "apps_main.cu"), "-o", APPS_BIN,
            "-L", HERE, "-lmedusa_b200", "-Xlinker", "-rpath,$ORIGIN/.."])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("apps build failed:\n%s" % r.stderr[-6000:])
    build_dropin(force)
    return APPS_BIN


DROPIN_DIR = os.path.join(APPS_DIR, "dropin")
DROPIN_APPS = ("bfs", "sssp", "pagerank")


def dropin_bin(app):
    return os.path.join(DROPIN_DIR, "medusa_dropin_" + app)


def build_dropin(force=False):
    """The reference's apps in their own shape (medusa_b200/apps/dropin), one
    binary each (each app generates its own vertex field list)."""
    common = glob.glob(os.path.join(DROPIN_DIR, "*.h")) + [LIB] + \
        glob.glob(os.path.join(ROOT, "include", "medusa", "*.h"))
    jobs = []
    for app in DROPIN_APPS:
        src = os.path.join(DROPIN_DIR, "dropin_%s.cu" % app)
        if force or _stale(dropin_bin(app), [src] + common):
            jobs.append([NVCC, "-std=c++17", "-O3", "-lineinfo"] + ARCH +
                        ["-I", os.path.join(ROOT, "include"), "-I", DROPIN_DIR, src,
                         "-o", dropin_bin(app), "-L", HERE, "-lmedusa_b200",
                         "-Xlinker", "-rpath,$ORIGIN/../.."])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("drop-in app build failed:\n%s" % r.stderr[-6000:])

    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            list(ex.map(run, jobs))


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--force", action="store_true")
    p.add_argument("--jobs", type=int, default=None)
    p.add_argument("-v", "--verbose", action="store_true")
    a = p.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
