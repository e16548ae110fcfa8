"""Compile generated pipelines into in-tree shared libraries.

The reference writes the generated C++ and runs
``g++ -O3 -march=native -fopenmp -fPIC -shared`` on it
(sandbox/apps/python/cpp_compiler.py:4-43, sandbox/tuner.py:238-254).  Here
the CUDA translation unit is compiled by nvcc for sm_100a only and the host
C++ that tabulates const functions by g++ with the reference's optimization
flags; both link into ``libpm_<name>_<hash>.so`` under
``polymage_b200/_gen`` (inside the package, so a built library travels with
the source tree).  Libraries are cached by the hash of their sources and
flags.
"""

import hashlib
import os
import subprocess
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN_DIR = os.environ.get("PM_GEN_DIR") or os.path.join(HERE, "_gen")

NVCC = os.environ.get("PM_NVCC", "nvcc")
CXX = os.environ.get("PM_CXX", "g++")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Device code at -O3; the host side of a pipeline library (validation,
# descriptors, launches) is compiled at -O1, which halves its compile time
# (it dominates tuning wall-clock) without measurable cost per call.
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O1", "-Xptxas", "-O3"]
# Host code for const tables: the reference's optimization flags.  The
# instruction set is pinned (not -march=native) because a library built on
# one machine may be loaded on another.
HOST_MARCH = os.environ.get("PM_HOST_MARCH", "x86-64-v3")
CXX_FLAGS = ["-O3", "-march=" + HOST_MARCH, "-ftree-vectorize", "-fPIC"]


class BuildError(Exception):
    pass


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       universal_newlines=True)
    if r.returncode != 0:
        raise BuildError("command failed (%d): %s\n%s" % (
            r.returncode, " ".join(cmd), r.stdout[-8000:]))
    return r.stdout


def _runtime_hash():
    h = hashlib.sha1()
    for fn in sorted(os.listdir(CSRC)):
        if fn.endswith((".cuh", ".h")):
            with open(os.path.join(CSRC, fn), "rb") as f:
                h.update(f.read())
    return h.hexdigest()


def library_path(module, out_dir=None):
    out_dir = out_dir or GEN_DIR
    h = hashlib.sha1()
    h.update(module.source.encode())
    h.update((module.host_source or "").encode())
    h.update(_runtime_hash().encode())
    h.update(" ".join(ARCH_FLAGS + NVCC_FLAGS + CXX_FLAGS).encode())
    tag = h.hexdigest()[:16]
    return os.path.join(out_dir, "libpm_%s_%s.so" % (module.name, tag)), tag


_locks = {}
_locks_guard = threading.Lock()


def _lock_for(path):
    with _locks_guard:
        return _locks.setdefault(path, threading.Lock())


def compile_module(module, out_dir=None, verbose=False, force=False):
    """Compile a CudaModule; returns the path of the shared library.  Safe
    to call concurrently (identical modules compile once; temporaries have
    per-process, per-thread names)."""
    out_dir = out_dir or GEN_DIR
    os.makedirs(out_dir, exist_ok=True)
    so, tag = library_path(module, out_dir)
    with _lock_for(so):
        if os.path.exists(so) and not force:
            return so
        base = os.path.join(out_dir, "pm_%s_%s" % (module.name, tag))
        uniq = "%s.%d.%d" % (base, os.getpid(), threading.get_ident())
        with open(base + ".cu", "w") as f:
            f.write(module.source)
        with open(base + ".h", "w") as f:
            f.write(module.header)
        objs = []
        _run([NVCC] + ARCH_FLAGS + NVCC_FLAGS +
             ["-I", CSRC, "-c", base + ".cu", "-o", uniq + ".o"], verbose)
        objs.append(uniq + ".o")
        if module.host_source:
            with open(base + "_host.cpp", "w") as f:
                f.write(module.host_source)
            _run([CXX] + CXX_FLAGS + ["-c", base + "_host.cpp", "-o",
                                      uniq + "_host.o"], verbose)
            objs.append(uniq + "_host.o")
        tmp = uniq + ".so.tmp"
        _run([NVCC] + ARCH_FLAGS + ["-shared", "-o", tmp] + objs, verbose)
        os.replace(tmp, so)
        for o in objs:
            try:
                os.remove(o)
            except OSError:
                pass
        return so


def compile_source(name, path, out_dir=None, verbose=False):
    """Compile a standalone CUDA source of this package (e.g. the cost
    model's kernels) into ``libpm_<name>_<hash>.so``."""
    out_dir = out_dir or GEN_DIR
    os.makedirs(out_dir, exist_ok=True)
    with open(path, "rb") as f:
        src = f.read()
    h = hashlib.sha1(src)
    h.update(_runtime_hash().encode())
    h.update(" ".join(ARCH_FLAGS + NVCC_FLAGS).encode())
    so = os.path.join(out_dir, "libpm_%s_%s.so" % (name, h.hexdigest()[:16]))
    if os.path.exists(so):
        return so
    tmp = so + ".tmp%d" % os.getpid()
    _run([NVCC] + ARCH_FLAGS + NVCC_FLAGS + ["-I", CSRC, "-shared", path,
                                             "-o", tmp], verbose)
    os.replace(tmp, so)
    return so


def build_pipeline(pipeline, out_dir=None, verbose=False):
    from .runtime import CompiledPipeline
    module = pipeline.generate_code()
    so = compile_module(module, out_dir=out_dir, verbose=verbose)
    return CompiledPipeline(pipeline, so, module)
