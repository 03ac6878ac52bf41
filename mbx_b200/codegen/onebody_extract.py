#!/usr/bin/env python3
"""Extract the water 1-body model data (Partridge-Schwenke surface) from the
reference's sources into ``mbx_b200/data/ps1b.json``.

The 1-body energy of MB-pol water is the Partridge-Schwenke potential energy
surface as the reference evaluates it in ``ps::pot_nasa``
(potential/1b/ps.cpp:346-640): Morse O-H terms, an exponential H-H term and
a 245-term polynomial in the two O-H stretches and the bend, damped by a
Gaussian in the stretches.  Its constants are model data and must equal the
reference's, so they are read from the source, not retyped:

* the index tables ``idx1``, ``idx2``, ``idx3`` (ps.cpp:61-87) and the four
  coefficient sets ``c5zA``, ``cbasis``, ``ccore``, ``crest`` combined as
  ``c5z = f5z c5zA + fbasis cbasis + fcore ccore + frest crest``
  (ps.cpp:428-430, same operation order);
* the scalar constants of the anonymous namespace (ps.cpp:45-58) and the
  literals of ``pot_nasa`` (equilibrium cosine, energy offset);
* ``constants::cm1_kcalmol`` (tools/constants.h:61), evaluated by compiling
  a three-line program against the reference's header.

Usage: ``python -m mbx_b200.codegen.onebody_extract [--ref DIR]`` (or
MBX_REFERENCE).
"""
import argparse
import json
import math
import os
import re
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "data")
OUT = os.path.join(DATA, "ps1b.json")

SCALARS = ("reoh", "thetae", "b1", "roh", "alphaoh", "deohA", "phh1A", "phh2", "f5z", "fbasis", "fcore", "frest")
ARRAYS = ("idx1", "idx2", "idx3", "c5zA", "cbasis", "ccore", "crest")


def _array(text, name):
    m = re.search(r"const\s+(?:size_t|double)\s+%s\[(\d+)\]\s*=\s*\{" % name, text)
    if not m:
        raise ValueError("array %s not found" % name)
    end = text.index("}", m.end())
    vals = [v for v in text[m.end():end].replace("\n", " ").split(",") if v.strip()]
    if len(vals) != int(m.group(1)):
        raise ValueError("%s: %d values, declared %s" % (name, len(vals), m.group(1)))
    return [float(v) if name.startswith("c") else int(v) for v in vals]


def _scalar(text, name):
    m = re.search(r"const\s+double\s+%s\s*=\s*([-+0-9.eE]+)\s*;" % name, text)
    if not m:
        raise ValueError("constant %s not found" % name)
    return float(m.group(1))


def cm1_kcalmol(ref):
    src = ('#include <cstdio>\n#include "tools/constants.h"\n'
           'int main() { std::printf("%.17g\\n", constants::cm1_kcalmol); return 0; }\n')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "k.cpp")
        exe = os.path.join(d, "k")
        open(c, "w").write(src)
        subprocess.check_call(["g++", "-std=c++17", "-I" + os.path.join(ref, "src"), c, "-o", exe])
        return float(subprocess.check_output([exe]).decode())


def extract(ref):
    path = os.path.join(ref, "src", "potential", "1b", "ps.cpp")
    text = open(path).read()
    d = {name: _scalar(text, name) for name in SCALARS}
    arr = {name: _array(text, name) for name in ARRAYS}
    body = text[text.index("std::vector<double> pot_nasa("):]
    costhe = float(re.search(r"const double costhe\s*=\s*([-+0-9.eE]+)\s*;", body).group(1))
    offset = float(re.search(r"e1\[nv\]\s*\+=\s*([-+0-9.eE]+)\s*;", body).group(1))
    c5z = [((d["f5z"] * a + d["fbasis"] * b) + d["fcore"] * c) + d["frest"] * r
           for a, b, c, r in zip(arr["c5zA"], arr["cbasis"], arr["ccore"], arr["crest"])]
    out = {
        "source": "potential/1b/ps.cpp (ps::pot_nasa)",
        "reoh": d["reoh"], "b1": d["b1"], "roh": d["roh"], "alphaoh": d["alphaoh"], "phh2": d["phh2"],
        "deoh": d["f5z"] * d["deohA"], "phh1": d["f5z"] * d["phh1A"] * math.exp(d["phh2"]),
        "costhe": costhe, "offset": offset, "cm1_kcalmol": cm1_kcalmol(ref),
        "idx1": arr["idx1"], "idx2": arr["idx2"], "idx3": arr["idx3"], "c5z": c5z,
    }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"), required=not os.environ.get("MBX_REFERENCE"))
    args = ap.parse_args(argv)
    d = extract(args.ref)
    with open(OUT, "w") as f:
        json.dump(d, f, indent=1)
    print("wrote %s (%d polynomial terms)" % (OUT, len(d["c5z"])))


if __name__ == "__main__":
    main()
