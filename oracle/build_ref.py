#!/usr/bin/env python3
"""Build recipe for the reference oracle library ``oracle/_ref/libmbx_ref.so``.

Test infrastructure only.  It compiles the reference's own C++ sources in place
(nothing is copied into this repository) with g++, using the source lists of
the reference's ``src/Makefile.am`` (``tools_src`` ... ``lj_sources`` and the
N2O5 mini-library), and links them with:

* ``ref_shim/fftw3.h`` + ``ref_shim/fftw_shim.c``: the double-precision FFTW
  names the PME header binds with ``-DHAVE_FFTWD=1``; planners and executors
  abort if called (PME is never reached by the 2-body/3-body path);
* ``ref_shim/mbx_version.h``: the configure-generated version header;
* ``ref_shim/ch4ch4_grad_stub.cpp``: the CH4-CH4 2-body gradient polynomial,
  whose source file is missing from the reference (``.MISSING_LARGE_BLOBS``);
  it differentiates the present energy-only polynomial exactly;
* ``ref_harness.cpp``: ``extern "C"`` entry points over ``bblock::System``.

Optimisation follows the reference's defaults (``-O2``, no ``-march``,
``configure.ac:187,222``) for every file the timed water path executes
(``System::TwoBodyEnergy/ThreeBodyEnergy`` on MB-pol water: the n-mer
search, the MB-pol 2b/3b holders and polynomials, the dispatch); the rest of
the library (other monomer types, 1-body, 4-body, dispersion, ...) is
compiled at ``-O0`` only so that it links quickly, as the reference itself
does for its N2O5 files (``src/Makefile.am:21-25``).  On x86-64 without
``-march`` and ``-ffast-math`` the optimisation level does not change a
double-precision result (SSE2 arithmetic, no FMA contraction, no
reassociation), so the -O0 files give the same numbers as the reference's
own build; they are only slower, and they are not timed.

Usage: ``python oracle/build_ref.py [--ref DIR] [-j N]``; the reference root
is ``--ref``, else the ``MBX_REFERENCE`` environment variable.
Incremental: an object is rebuilt only when its source is newer.
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libmbx_ref.so")

LISTS = [
    "tools_src", "iotools_src", "bblock_src", "liba1b2c4_la_SOURCES", "oneb_sources",
    "twob_sources", "threeb_sources", "fourb_sources", "elec_sources", "disp_sources",
    "buck_sources", "ff_sources", "lj_sources",
]

# Files the timed water path executes: compiled like the reference (-O2).
HOT = {
    "potential/2b/energy2b.cpp", "potential/2b/x2b-v9x.cpp", "potential/2b/poly-2b-v6x.cpp",
    "potential/2b/poly-2b-v6x-nogrd.cpp",
    "potential/3b/energy3b.cpp", "potential/3b/x3b-v2x.cpp", "potential/3b/poly-3b-v2x.cpp",
    "potential/3b/poly-3b-v2x-nogrd.cpp",
    "potential/electrostatics/electrostatics.cpp", "potential/electrostatics/fields.cpp",
}
HOT_DIRS = ("tools/", "io_tools/", "bblock/")
MISSING_GRAD = "potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1x.cpp"


def sources(ref):
    txt = open(os.path.join(ref, "src", "Makefile.am")).read()
    out = []
    for name in LISTS:
        m = re.search(r"^" + name + r"\s*=\s*(.*)$", txt, re.M)
        if not m:
            raise RuntimeError("list %s not found in src/Makefile.am" % name)
        out += [s for s in m.group(1).split() if not s.startswith("$(")]
    return out


def compile_one(cmd, src, obj):
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
        return obj, None, 0.0
    t0 = time.time()
    r = subprocess.run(cmd + ["-c", src, "-o", obj + ".tmp"], capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr[-4000:], time.time() - t0
    os.replace(obj + ".tmp", obj)
    return obj, None, time.time() - t0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"))
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--cxx", default="/usr/bin/g++")
    args = ap.parse_args(argv)
    t_start = time.time()
    if not args.ref:
        print("no reference root (--ref or MBX_REFERENCE); oracle/_ref not built")
        return 0
    src_root = os.path.join(args.ref, "src")
    if not os.path.isdir(src_root):
        print("reference sources not found at %s; oracle/_ref not built" % src_root)
        return 0
    os.makedirs(OBJ, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    base = [args.cxx, "-std=c++17", "-fPIC", "-fopenmp", "-w", "-DHAVE_FFTWD=1", "-I" + src_root, "-I" + shim]
    jobs = []
    for rel in sources(args.ref):
        if rel == MISSING_GRAD:
            src = os.path.join(shim, "ch4ch4_grad_stub.cpp")
            opt = "-O2"
        else:
            src = os.path.join(src_root, rel)
            opt = "-O2" if (rel in HOT or rel.startswith(HOT_DIRS)) else "-O0"
        obj = os.path.join(OBJ, rel.replace("/", "__").replace(".cpp", ".o"))
        jobs.append((base + [opt], src, obj))
    jobs.append((base + ["-O2"], os.path.join(HERE, "ref_harness.cpp"), os.path.join(OBJ, "ref_harness.o")))
    jobs.append(([args.cxx.replace("g++", "gcc"), "-fPIC", "-O2", "-I" + shim],
                 os.path.join(shim, "fftw_shim.c"), os.path.join(OBJ, "fftw_shim.o")))
    # largest files first so the long compiles overlap
    jobs.sort(key=lambda j: -os.path.getsize(j[1]))
    errors = []
    with cf.ThreadPoolExecutor(max_workers=args.j) as ex:
        for obj, err, dt in ex.map(lambda j: compile_one(*j), jobs):
            if err:
                errors.append((obj, err))
            elif dt > 20:
                print("  compiled %s (%.0f s)" % (os.path.basename(obj), dt), flush=True)
    if errors:
        for obj, err in errors:
            sys.stderr.write("FAILED %s\n%s\n" % (obj, err))
        return 1
    objs = [j[2] for j in jobs]
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        r = subprocess.run([args.cxx, "-shared", "-fopenmp", "-o", LIB] + objs, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr[-4000:])
            return 1
    print("built %s (%.0f s)" % (LIB, time.time() - t_start))
    return 0


if __name__ == "__main__":
    sys.exit(main())
