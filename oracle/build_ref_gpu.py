#!/usr/bin/env python3
"""Build recipe for ``oracle/_ref/libmbx_ref_gpu.so``: the reference's
``bblock::System`` with ``Get2B`` / ``Get3B`` forwarded to ``libmbx_b200.so``.

Test infrastructure: the C++ caller of the drop-in boundary.  It takes the
reference's objects built by ``oracle/build_ref.py`` and replaces
``bblock/system.cpp`` with a copy (written under ``oracle/_ref/obj/gpu``,
never committed) that differs in two inserted lines per term:

* ``bblock/system.h``: the declaration of ``double GpuTerm(int nbody, bool
  do_grads, bool use_ghost);`` after the ``Get3B`` declaration (system.h:1279),
  under ``#ifdef MBX_GPU_2B3B``;
* ``bblock/system.cpp``: ``return GpuTerm(2, do_grads, use_ghost);`` as the
  first statement of ``System::Get2B`` (system.cpp:2425), and the same with 3
  in ``System::Get3B`` (system.cpp:2769), under ``#ifdef MBX_GPU_2B3B``;

then compiles it with ``-DMBX_GPU_2B3B`` beside ``oracle/ref_gpu_glue.cpp``
(``GpuTerm`` over the C ABI) and ``oracle/ref_harness.cpp``, and links the
result against ``mbx_b200/libmbx_b200.so`` (rpath relative to the library, so
the pair travels together).  The class layout of ``System`` is unchanged (one
non-virtual member function added), so the rest of the reference's objects
are reused as built.

Usage: ``python oracle/build_ref_gpu.py [--ref DIR]`` (after build_ref.py and
``python -m mbx_b200.build``); the reference root is ``--ref``, else the
``MBX_REFERENCE`` environment variable.
"""
import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
WORK = os.path.join(OBJ, "gpu")
LIB = os.path.join(OUT, "libmbx_ref_gpu.so")
CUDA_LIB = os.path.join(ROOT, "mbx_b200", "libmbx_b200.so")

HEADER_ANCHOR = "double Get3B(bool do_grads, bool use_ghost = 0);"
HEADER_INSERT = ("\n#ifdef MBX_GPU_2B3B\n"
                 "    // the 2b/3b terms computed by libmbx_b200 (oracle/ref_gpu_glue.cpp)\n"
                 "    double GpuTerm(int nbody, bool do_grads, bool use_ghost);\n"
                 "#endif\n")
BODY_ANCHORS = {2: "double System::Get2B(bool do_grads, bool use_ghost) {",
                3: "double System::Get3B(bool do_grads, bool use_ghost) {"}
BODY_INSERT = "\n#ifdef MBX_GPU_2B3B\n    return GpuTerm(%d, do_grads, use_ghost);\n#endif\n"


def insert_after(text, anchor, insert, what):
    if text.count(anchor) != 1:
        raise RuntimeError("%s: anchor %r found %d times" % (what, anchor, text.count(anchor)))
    i = text.index(anchor) + len(anchor)
    return text[:i] + insert + text[i:]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"))
    ap.add_argument("--cxx", default="/usr/bin/g++")
    args = ap.parse_args(argv)
    if not args.ref:
        print("no reference root (--ref or MBX_REFERENCE); %s not built" % LIB)
        return 0
    src = os.path.join(args.ref, "src")
    objs = sorted(glob.glob(os.path.join(OBJ, "*.o")))
    if not objs or not os.path.exists(CUDA_LIB):
        print("build oracle/_ref (build_ref.py) and mbx_b200/libmbx_b200.so first")
        return 1
    os.makedirs(os.path.join(WORK, "bblock"), exist_ok=True)
    h = open(os.path.join(src, "bblock", "system.h")).read()
    h = insert_after(h, HEADER_ANCHOR, HEADER_INSERT, "system.h")
    c = open(os.path.join(src, "bblock", "system.cpp")).read()
    for nb, anchor in BODY_ANCHORS.items():
        c = insert_after(c, anchor, BODY_INSERT % nb, "system.cpp")
    for name, text in (("system.h", h), ("system.cpp", c)):
        path = os.path.join(WORK, "bblock", name)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
    shim = os.path.join(HERE, "ref_shim")
    base = [args.cxx, "-std=c++17", "-fPIC", "-fopenmp", "-w", "-O2", "-DHAVE_FFTWD=1", "-DMBX_GPU_2B3B",
            "-I" + WORK, "-I" + src, "-I" + os.path.join(src, "bblock"), "-I" + shim,
            "-I" + os.path.join(ROOT, "include")]
    units = [(os.path.join(WORK, "bblock", "system.cpp"), os.path.join(WORK, "system.o")),
             (os.path.join(HERE, "ref_gpu_glue.cpp"), os.path.join(WORK, "glue.o")),
             (os.path.join(HERE, "ref_harness.cpp"), os.path.join(WORK, "harness.o"))]
    for s, o in units:
        deps = [s, os.path.join(WORK, "bblock", "system.h")]
        if os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(d) for d in deps):
            continue
        r = subprocess.run(base + ["-c", s, "-o", o], capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr[-4000:])
            return 1
    keep = [o for o in objs if os.path.basename(o) not in ("bblock__system.o", "ref_harness.o")]
    link = [args.cxx, "-shared", "-fopenmp", "-o", LIB + ".tmp"] + keep + [u[1] for u in units] + \
           ["-L" + os.path.dirname(CUDA_LIB), "-lmbx_b200",
            "-Wl,-rpath,$ORIGIN/../../mbx_b200"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-4000:])
        return 1
    os.replace(LIB + ".tmp", LIB)
    print("built %s" % LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())
