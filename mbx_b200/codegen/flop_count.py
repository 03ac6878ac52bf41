#!/usr/bin/env python3
"""Algorithmic FLOPs per evaluated n-mer, counted from the reference's programs.

The roofline of the evaluation kernels uses the reference's own gradient
programs as the definition of the work (so a cheaper schedule in this
library shows up as a higher achieved rate, not as less work).  For each
program this tool counts the binary multiplications and additions/subtractions
executed for ONE configuration:

* mbpol2b: poly_2b_v6x::eval(nd, a, x, t, g), potential/2b/poly-2b-v6x.cpp
  (functions f0..f99, each an 8-lane loop; counted per lane);
* mbpol3b: poly_3b_v2x::eval(a, x, t, g), potential/3b/poly-3b-v2x.cpp
  (f0..f54, 8-lane loops, per lane);
* ch4h2o2b: poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x::eval(a, x, g),
  potential/2b/poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp;
* ch4h2o3b: poly_A1B4_C1D2_C1D2_deg3_v1::eval(x, a, g),
  potential/3b/poly_3b_A1B4_C1D2_C1D2_deg3_grad_v1.cpp;
* ch4ch42b: the gradient program is absent from the reference; by convention
  twice the energy-only program poly_2b_A1B4_A1B4_deg4_exp0_v1.cpp.

An FMA in the reference's source is written as a multiply and an add, so
flops = muls + adds.  The variable, switch and chain-rule code of the
evaluators is not counted (it is < 3% of the polynomial).  Output:
``mbx_b200/data/flops.json``.
"""
import argparse
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "data", "flops.json")

PROGRAMS = {
    "mbpol2b": ("potential/2b/poly-2b-v6x.cpp", "lanes"),
    "mbpol3b": ("potential/3b/poly-3b-v2x.cpp", "lanes"),
    "ch4h2o2b": ("potential/2b/poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp", "scalar"),
    "ch4h2o3b": ("potential/3b/poly_3b_A1B4_C1D2_C1D2_deg3_grad_v1.cpp", "scalar"),
    "ch4ch42b": ("potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1.cpp", "scalar_x2"),
}


def strip(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return re.sub(r"#[^\n]*", "", text)


def count_ops(expr):
    # remove array subscripts (index arithmetic is not floating point)
    prev = None
    while prev != expr:
        prev = expr
        expr = re.sub(r"\[[^\[\]]*\]", "", expr)
    mul = expr.count("*")
    # binary + / - : an operator preceded by an operand (name, number or ')')
    add = len(re.findall(r"(?<=[\w)\s])\s*[-+](?=\s*[\w(.])", expr))
    # exponents in numeric literals (1e-5) are not operations
    add -= len(re.findall(r"\d[eE][-+]\d", expr))
    return mul, add


def count_program(ref, rel, mode):
    text = strip(open(os.path.join(ref, "src", rel)).read())
    mul = add = 0
    if mode == "lanes":
        # bodies of the 8-lane loops inside f0..fN
        for m in re.finditer(r"void f\d+\([^)]*\)\s*\{\s*for\s*\((?:int|size_t) i = 0; i < 8; i\+\+\)\s*\{(.*?)\n\s*\}\s*\n\}",
                             text, re.S):
            for stmt in m.group(1).split(";"):
                if "=" in stmt:
                    rhs = stmt.split("=", 1)[1]
                    a, b = count_ops(rhs)
                    mul += a
                    add += b
    else:
        for stmt in text.split(";"):
            if re.search(r"\bt\d+\b\s*=|t\[\d+\]\s*=|\bg\[\d+\]\s*=|return\s", stmt):
                rhs = stmt.split("=", 1)[1] if "=" in stmt else stmt.split("return", 1)[1]
                a, b = count_ops(rhs)
                mul += a
                add += b
        if mode == "scalar_x2":
            mul, add = 2 * mul, 2 * add
    return mul, add


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"), required=not os.environ.get("MBX_REFERENCE"))
    a = ap.parse_args(argv)
    out = {}
    for name, (rel, mode) in PROGRAMS.items():
        mul, add = count_program(a.ref, rel, mode)
        out[name] = {"mul": mul, "add": add, "flops": mul + add, "source": rel,
                     "convention": "2x energy-only program" if mode == "scalar_x2" else "gradient program"}
        print("%-9s mul %7d add %7d flops %7d" % (name, mul, add, mul + add))
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
