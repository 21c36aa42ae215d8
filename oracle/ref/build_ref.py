#!/usr/bin/env python3
"""Compile the reference's own CPU superstep path into oracle/_ref/.

TEST INFRASTRUCTURE ONLY (the CPU checker and the timed CPU baseline).

The reference selects an app at build time by placing it at ``Algorithm/``
(reference ``HowToBuild:9-10``); its headers include ``../Algorithm/*.h``.
For each app this script therefore makes ``oracle/_ref/farm_<app>/`` whose
``Algorithm/``, ``MedusaRT/``, ``MultipleGPU/`` and ``Compatibility/`` are real
directories of per-file symlinks into the reference tree (nothing is copied),
with ``Algorithm/`` pointing at the app's own files.  It then compiles, from
those unmodified sources, the host-only files the CPU path needs:

  <app>/CPUFunctorHoster.cpp, <app>/{Edge,Vertex,Message}DataType.cu,
  MedusaRT/GraphConverter.cu, MedusaRT/Utilities.cu, MedusaRT/GraphStorage.cu

with g++ -O3 -fopenmp (as ``-x c++``; none of them holds device code) against
the small stand-in headers in ``oracle/ref/shim/`` for the CUDA-SDK and CUDPP
headers that are not installed, plus ``oracle/ref/ref_harness.cpp``, into
``oracle/_ref/libref_<bfs|sssp|pr>.so``, linked with ``--wrap`` on the
reference's CPUMalloc (see ref_harness.cpp).  Output goes only to
``oracle/_ref/``.

Usage: python oracle/ref/build_ref.py [--reference PATH] [--force]
Exits 0 without doing anything when the reference tree is absent and the
libraries already exist (the GPU box only uses prebuilt files).
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
SHIM = os.path.join(HERE, "shim")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

# app name in the reference tree -> (library tag, harness define)
APPS = {
    "Algorithm": ("bfs", "REF_APP_BFS"),   # the tree's Algorithm/ is the MBFS app
    "SSSP": ("sssp", "REF_APP_SSSP"),
    "MPG": ("pr", "REF_APP_PR"),
}
SUBDIRS = ("MedusaRT", "MultipleGPU", "Compatibility")
APP_SOURCES = ("CPUFunctorHoster.cpp", "EdgeDataType.cu", "VertexDataType.cu",
               "MessageDataType.cu")
RT_SOURCES = ("GraphConverter.cu", "Utilities.cu", "GraphStorage.cu")


def lib_path(tag):
    return os.path.join(OUT, "libref_%s.so" % tag)


def make_farm(ref, app):
    farm = os.path.join(OUT, "farm_" + app)
    if os.path.isdir(farm):
        shutil.rmtree(farm)
    for sub, srcdir in [("Algorithm", app)] + [(s, s) for s in SUBDIRS]:
        d = os.path.join(farm, sub)
        os.makedirs(d)
        full = os.path.join(ref, srcdir)
        for name in sorted(os.listdir(full)):
            os.symlink(os.path.join(full, name), os.path.join(d, name))
    return farm


def compile_one(args):
    cmd, src = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed for %s:\n%s" % (src, r.stderr[-4000:]))


def build_app(ref, app, tag, define):
    farm = make_farm(ref, app)
    objdir = os.path.join(OUT, "obj_" + tag)
    os.makedirs(objdir, exist_ok=True)
    common = ["g++", "-O3", "-fPIC", "-fopenmp", "-w", "-I", SHIM,
              "-I", os.path.join(CUDA, "include"),
              "-include", os.path.join(SHIM, "ref_shim.h")]
    jobs, objs = [], []
    for name in APP_SOURCES:
        src = os.path.join(farm, "Algorithm", name)
        obj = os.path.join(objdir, name + ".o")
        jobs.append((common + ["-x", "c++", "-c", src, "-o", obj], src))
        objs.append(obj)
    for name in RT_SOURCES:
        src = os.path.join(farm, "MedusaRT", name)
        obj = os.path.join(objdir, "rt_" + name + ".o")
        jobs.append((common + ["-x", "c++", "-c", src, "-o", obj], src))
        objs.append(obj)
    harness = os.path.join(HERE, "ref_harness.cpp")
    hobj = os.path.join(objdir, "ref_harness.o")
    jobs.append((common + ["-D" + define, "-I", farm, "-x", "c++", "-c", harness,
                           "-o", hobj], harness))
    objs.append(hobj)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(compile_one, jobs))
    cudalib = os.path.join(CUDA, "lib64")
    # --wrap: see ref_harness.cpp (64 spare bytes on the reference's host blocks)
    link = ["g++", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-Wl,--wrap=_Z9CPUMallocPPvi",
            "-o", lib_path(tag)] + objs + [
        "-L", cudalib, "-lcudart", "-Wl,-rpath," + cudalib]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed for %s:\n%s" % (tag, r.stderr[-4000:]))
    shutil.rmtree(objdir, ignore_errors=True)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--reference", default="/root/reference")
    p.add_argument("--force", action="store_true")
    a = p.parse_args(argv)
    have = all(os.path.exists(lib_path(t)) for t, _ in APPS.values())
    if not os.path.isdir(a.reference):
        if have:
            return 0
        print("reference tree not found at %s; oracle/_ref not built" % a.reference,
              file=sys.stderr)
        return 1
    if have and not a.force:
        newest_input = max(os.path.getmtime(os.path.join(HERE, f))
                           for f in ("ref_harness.cpp", "build_ref.py"))
        if all(os.path.getmtime(lib_path(t)) >= newest_input for t, _ in APPS.values()):
            return 0
    os.makedirs(OUT, exist_ok=True)
    for app, (tag, define) in APPS.items():
        build_app(a.reference, app, tag, define)
    return 0


if __name__ == "__main__":
    sys.exit(main())
