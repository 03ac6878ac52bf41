"""Build the CUDA library ``mbx_b200/libmbx_b200.so`` for sm_100a.

Steps: regenerate the per-evaluator CUDA sources from the specs and PIP
tables (``codegen/gen_kernels.py``), compile every translation unit with nvcc
(``-gencode arch=compute_100a,code=sm_100a``) in parallel, link one shared
library.  Incremental: a unit is rebuilt when its source or any header it can
see is newer than its object.  A file lock keeps concurrent builds (two
processes importing the package on a fresh checkout) from racing.

The straight-line kernels of the four trie-compiled evaluators are the long
units (about 1-2 minutes each in ptxas); everything else is table-driven and
compiles in seconds, so a clean build takes a few minutes on 8 cores.

Usage: ``python -m mbx_b200.build [-j N] [--verbose]``
"""
import argparse
import concurrent.futures as cf
import contextlib
import fcntl
import os
import subprocess
import sys
import time

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
GEN = os.path.join(CSRC, "gen")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmbx_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
HAND = ("mbx_capi.cu", "nmer_build.cu", "peaks.cu", "noalloc.cu", "table_kernels.cu", "onebody.cu")
HEADERS = ("holder_common.cuh", "holder_kernel.cuh", "term_table.cuh", "launch_cache.cuh", "device_state.h",
           "qf_kernel.cuh")


def deps(src):
    common = [os.path.join(CSRC, h) for h in HEADERS]
    base = os.path.basename(src)
    if base == "terms_blob.cpp":
        return [src, os.path.join(GEN, "terms.bin")]
    if os.path.dirname(src) == GEN:
        name, v = base[:-3].rsplit("_", 1)
        common.append(os.path.join(GEN, name + ".cuh"))
        for variant in {"g": ("pip",), "e": ("pip_e",), "s": ("pip_s32", "qf")}.get(v, ()):
            common.append(os.path.join(GEN, "%s_%s.cuh" % (name, variant)))
    else:
        common += [os.path.join(CSRC, "nmer_build.h"), os.path.join(ROOT, "include", "mbx_b200.h"),
                   os.path.join(GEN, "registry.inc"), os.path.join(GEN, "terms_index.inc"),
                   os.path.join(GEN, "ps1b.inc")]
    return [src] + [d for d in common if os.path.exists(d)]


def obj_of(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "__")
    return os.path.join(OBJ, rel.rsplit(".", 1)[0] + ".o")


def compile_one(src, verbose):
    obj = obj_of(src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps(src)):
        return obj, None, 0.0
    t0 = time.time()
    if src.endswith(".cpp"):
        cmd = ["g++", "-O2", "-fPIC", "-c", src, "-o", obj + ".tmp"]
    else:
        cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr[-6000:], time.time() - t0
    os.replace(obj + ".tmp", obj)
    if verbose and r.stderr:
        with open(obj + ".ptxas.txt", "w") as f:
            f.write(r.stderr)
    return obj, None, time.time() - t0


@contextlib.contextmanager
def build_lock():
    os.makedirs(OBJ, exist_ok=True)
    with open(os.path.join(OBJ, ".lock"), "w") as f:
        fcntl.flock(f, fcntl.LOCK_EX)
        try:
            yield
        finally:
            fcntl.flock(f, fcntl.LOCK_UN)


def build(jobs=None, verbose=False, quiet=False):
    t_start = time.time()
    sys.path.insert(0, ROOT)
    with build_lock():
        from mbx_b200.codegen import gen_kernels
        gen = gen_kernels.main([], quiet=True)
        srcs = [os.path.join(CSRC, f) for f in HAND] + gen
        # the long units first, so that they overlap the rest
        srcs.sort(key=lambda s: -sum(os.path.getsize(d) for d in deps(s)))
        errors = []
        objs = []
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for obj, err, dt in ex.map(lambda s: compile_one(s, verbose), srcs):
                objs.append(obj)
                if err:
                    errors.append((obj, err))
                elif dt and not quiet:
                    print("  compiled %s (%.0fs)" % (os.path.basename(obj), dt), flush=True)
        if errors:
            for obj, err in errors:
                sys.stderr.write("FAILED %s\n%s\n" % (obj, err))
            raise RuntimeError("mbx_b200 build failed")
        newest = max(os.path.getmtime(o) for o in objs)
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
            cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("link failed:\n" + r.stderr[-4000:])
            os.replace(LIB + ".tmp", LIB)
    if not quiet:
        print("built %s (%.0f s)" % (LIB, time.time() - t_start))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(a.j, a.verbose)


if __name__ == "__main__":
    main()
