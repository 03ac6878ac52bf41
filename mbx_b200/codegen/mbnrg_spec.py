#!/usr/bin/env python3
"""Evaluator specs of the reference's template-generated MB-nrg holders.

The reference writes its newer 2-body and 3-body evaluators
(``potential/2b/mbnrg_2b_*_v1.cpp``, ``potential/3b/mbnrg_3b_*_v1.cpp``) from
one code template: a constructor block per monomer tuple that sets the
coefficients, the non-linear constants ``m_k_*`` / ``m_d_*`` and the switch
radii ``m_ri`` / ``m_ro``; an ``eval`` with gradients that names every site
``coords_<X>_<i>_<m>`` (real atoms copied from the n-mer, lone pairs built by
``monomer::setup`` with the MB-pol gammas), one line per polynomial variable
(``xs[i] = vs[i].v_exp(...)`` and its ``v_exp0`` / ``v_coul`` / ``v_coul0``
siblings, tools/variable.cpp:49-130), the switch product and the skip test.
This tool reads those parts of one evaluator and writes the description
``mbx_b200/specs.py`` needs (``<name>.spec.json`` in ``mbx_b200/data``): the
same fields as a hand-written ``Spec``.  It refuses anything outside the
template (another variable kind, other lone-pair constants, another switch
or skip form) rather than guess.

The extracted specs are checked against the reference's own golden vectors
and against whole systems evaluated by the compiled reference
(tests/test_oracle_goldens.py); ``tests/test_mbnrg_specs.py`` also re-extracts
the template evaluators whose specs are written by hand in specs.py and
compares the two.

Usage: ``python -m mbx_b200.codegen.mbnrg_spec [--ref DIR] (or MBX_REFERENCE) [names...]``
"""
import argparse
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "data")

LP_GAMMA_IN = -9.721486914088159e-02
LP_GAMMA_OUT = 9.859272078406150e-02

# evaluator name -> (source, monomer ids of the constructor block, PIP table,
# polynomial header, reference line of the gradient eval)
SOURCES = {
    "h2h22b": ("potential/2b/mbnrg_2b_A2_A2_deg6_v1.cpp", ("h2", "h2"), "h2h22b",
               "potential/2b/poly_2b_A2_A2_deg6_v1.h"),
    "h2oh22b": ("potential/2b/mbnrg_2b_A1B2Z2_C2_deg5_v1.cpp", ("h2o", "h2"), "h2oh22b",
                "potential/2b/poly_2b_A1B2Z2_C2_deg5_v1.h"),
    "csh22b": ("potential/2b/mbnrg_2b_A1_B2_deg7_v1.cpp", ("cs+", "h2"), "csh22b",
               "potential/2b/poly_2b_A1_B2_deg7_v1.h"),
    "nh3nh32b": ("potential/2b/mbnrg_2b_A1B3_A1B3_deg4_v1.cpp", ("nh3", "nh3"), "nh3nh32b",
                 "potential/2b/poly_2b_A1B3_A1B3_deg4_v1.h"),
    "nh3pbe2b": ("potential/2b/mbnrg_2b_A1B3_A1B3_deg4_v1.cpp", ("nh3pbe0d3bj", "nh3pbe0d3bj"), "nh3nh32b",
                 "potential/2b/poly_2b_A1B3_A1B3_deg4_v1.h"),
    "ch4co22b": ("potential/2b/mbnrg_2b_A1B4_C1D2_deg4_v1.cpp", ("ch4", "co2"), "ch4co22b",
                 "potential/2b/poly_2b_A1B4_C1D2_deg4_v1.h"),
    "mbpbe2b": ("potential/2b/mbnrg_2b_A1B2Z2_A1B2Z2_deg4_vmbpbe.cpp", ("mbpbe", "mbpbe"), "mbpbe2b",
                "potential/2b/poly_2b_A1B2Z2_A1B2Z2_deg4_vmbpbe.h"),
    "co23b": ("potential/3b/mbnrg_3b_A1B2_A1B2_A1B2_deg4_v1.cpp", ("co2", "co2", "co2"), "co23b",
              "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_v1.h"),
    "mbpbe3b": ("potential/3b/mbnrg_3b_A1B2_A1B2_A1B2_deg4_vmbpbe.cpp", ("mbpbe", "mbpbe", "mbpbe"), "mbpbe3b",
                "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_vmbpbe.h"),
    # switches with 1 - cos^2((s12 + s13 + s23 - 1) pi / 2) (the "cos2" form)
    "n2o5h2o3b": ("potential/3b/mbnrg_3b_A1B2C4_D1E2_D1E2_deg3_v1.cpp", ("n2o5", "h2o", "h2o"), "n2o5h2o3b",
                  "potential/3b/poly_3b_A1B2C4_D1E2_D1E2_deg3_v1.h"),
}

# the energy-only program of each table (pip_extract)
PROGRAMS = {
    "h2h22b": "potential/2b/poly_2b_A2_A2_deg6_nograd_v1.cpp",
    "h2oh22b": "potential/2b/poly_2b_A1B2Z2_C2_deg5_nograd_v1.cpp",
    "csh22b": "potential/2b/poly_2b_A1_B2_deg7_nograd_v1.cpp",
    "nh3nh32b": "potential/2b/poly_2b_A1B3_A1B3_deg4_nograd_v1.cpp",
    "ch4co22b": "potential/2b/poly_2b_A1B4_C1D2_deg4_nograd_v1.cpp",
    "mbpbe2b": "potential/2b/poly_2b_A1B2Z2_A1B2Z2_deg4_nograd_vmbpbe.cpp",
    "co23b": "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_nograd_v1.cpp",
    "mbpbe3b": "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_nograd_vmbpbe.cpp",
    "n2o5h2o3b": "potential/3b/poly_3b_A1B2C4_D1E2_D1E2_deg3_nograd_v1.cpp",
}


def poly_size(ref, header):
    """(nvars, ncoef, degree) of a generated polynomial from its header."""
    htext = open(os.path.join(ref, "src", header)).read()
    return (int(re.search(r"n_vars\s*=\s*(\d+)", htext).group(1)), int(re.search(r"size\s*=\s*(\d+)", htext).group(1)),
            int(re.search(r"degree\s*=\s*(\d+)", htext).group(1)))


def fit_pattern(mons):
    """Regex of the coefficient vector of a monomer tuple's constructor block."""
    cond = r"\s+and\s+".join(r'mon%d\s*==\s*"%s"' % (i + 1, re.escape(m)) for i, m in enumerate(mons))
    return r"if\s*\(\s*" + cond + r"\s*\)\s*\{\s*coefficients\s*=\s*std::vector<double>\s*\{"

# template evaluators whose specs are hand-written in specs.py (cross-check)
HANDWRITTEN = {
    "fh2o2b": ("potential/2b/mbnrg_2b_A1_B1C2X2_deg6_v1.cpp", ("f-", "h2o"), "halh2o2b",
               "potential/2b/poly_2b_A1_B1C2X2_deg6_v1.h"),
    "ih2o3b": ("potential/3b/mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp", ("i-", "h2o", "h2o"), "halh2o3b",
               "potential/3b/poly_3b_A1_B1C2X2_B1C2X2_deg4_v1.h"),
    "nacl2b": ("potential/2b/mbnrg_2b_A1_B1_deg9_v1.cpp", ("na+", "cl-"), "a1b12b",
               "potential/2b/poly_2b_A1_B1_deg9_v1.h"),
    "clcl2b": ("potential/2b/mbnrg_2b_A1_A1_deg9_v1.cpp", ("cl-", "cl-"), "a1a12b",
               "potential/2b/poly_2b_A1_A1_deg9_v1.h"),
    "arh2o2b": ("potential/2b/mbnrg_2b_A1_B1C2X2_deg5_v1.cpp", ("ar", "h2o"), "arh2o2b",
                "potential/2b/poly_2b_A1_B1C2X2_deg5_v1.h"),
}

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _braced(text, start):
    """The text between the '{' at or after start and its matching '}'."""
    i = text.index("{", start)
    depth, j = 1, i + 1
    while depth:
        depth += (text[j] == "{") - (text[j] == "}")
        j += 1
    return text[i + 1:j - 1], j


def _ws(s):
    return re.sub(r"\s+", "", s)


def extract(ref, name, source, mons, table, header):
    path = os.path.join(ref, "src", source)
    text = _strip_comments(open(path).read())
    nb = len(mons)
    # constructor block of the monomer tuple
    cond = r"\s+and\s+".join(r'mon%d\s*==\s*"%s"' % (i + 1, re.escape(m)) for i, m in enumerate(mons))
    m = re.search(r"if\s*\(\s*" + cond + r"\s*\)", text)
    if not m:
        raise ValueError("%s: no constructor block for %s" % (source, mons))
    block, _ = _braced(text, m.end())
    consts = {k: float(v) for k, v in re.findall(r"\b(m_\w+)\s*=\s*(%s)\s*;" % NUM, block)}
    for key in ("m_ri", "m_ro"):
        if key not in consts:
            raise ValueError("%s: %s not set for %s" % (source, key, mons))
    # the eval with gradients
    sig = r"::eval\s*\(\s*const double\s*\*\s*xyz1\s*,[^)]*double\s*\*\s*grad1"
    m = re.search(sig, text)
    if not m:
        raise ValueError("%s: no gradient eval" % source)
    body, _ = _braced(text, m.end())
    # f_switch: the cosine switch between m_ri and m_ro
    fs = re.search(r"::f_switch\s*\([^)]*\)", text)
    fbody, _ = _braced(text, fs.end())
    if "M_PI/(m_ro-m_ri)" not in _ws(fbody) or "(1.0+std::cos(x))/2.0" not in _ws(fbody):
        raise ValueError("%s: f_switch is not the cosine switch" % source)
    # real sites in holder order: coords_<X>_<i>_<m> = xyz.data() + offset
    real = re.findall(r"const double\s*\*\s*coords_(\w+)\s*=\s*xyz\.data\(\)\s*\+\s*(\d+)\s*;", body)
    real = sorted(((int(off), nm) for nm, off in real))
    if [off for off, _ in real] != list(range(0, 3 * len(real), 3)):
        raise ValueError("%s: real sites are not contiguous" % source)
    sites = [nm for _, nm in real]
    letters = "abc"[:nb]
    nat = tuple(sum(1 for s in sites if s.endswith("_" + l)) for l in letters)
    if [s[-1] for s in sites] != sorted(s[-1] for s in sites):
        raise ValueError("%s: real sites are not grouped by monomer" % source)
    # lone pairs: mK.setup(coords_O, w12, wcross, coords_Xp, coords_Xm)
    w12 = re.search(r"double\s+w12\s*=\s*(%s)" % NUM, body)
    wcr = re.search(r"double\s+wcross\s*=\s*(%s)" % NUM, body)
    lp = []
    for o, xp, xm in re.findall(r"\w+\.setup\(\s*coords_(\w+)\s*,\s*w12\s*,\s*wcross\s*,\s*coords_(\w+)\s*,"
                                r"\s*coords_(\w+)\s*\)", body):
        if float(w12.group(1)) != LP_GAMMA_IN or float(wcr.group(1)) != LP_GAMMA_OUT:
            raise ValueError("%s: lone-pair constants differ from MB-pol's" % source)
        for v in (xp, xm):
            if v not in sites:
                sites.append(v)
        lp.append((letters.index(o[-1]), sites.index(o), sites.index(xp), sites.index(xm)))
    # variables
    variables = []
    for idx, kind, args in re.findall(r"xs\[(\d+)\]\s*=\s*vs\[\d+\]\.(v_\w+)\(([^)]*)\)\s*;", body):
        a = [x.strip() for x in args.split(",")]
        if kind in ("v_exp0", "v_coul0"):
            d0, k, p, q = consts[a[0]], consts[a[1]], a[2], a[3]
        elif kind in ("v_exp", "v_coul"):
            d0, k, p, q = 0.0, consts[a[0]], a[1], a[2]
        else:
            raise ValueError("%s: variable kind %s is not supported" % (source, kind))
        if int(idx) != len(variables):
            raise ValueError("%s: variables out of order" % source)
        p, q = p.replace("coords_", ""), q.replace("coords_", "")
        variables.append(("exp" if kind.startswith("v_exp") else "coul", sites.index(p), sites.index(q), k, d0))
    # switch and skip
    forms = {"sw12": "pair", "sw12*sw13+sw12*sw23+sw13*sw23": "triple",
             "sw12*sw13+sw12*sw23+sw13*sw23-2*sw12*sw23*sw13": "triple2"}
    cos2 = ("if((sw12+sw13+sw23)<1.0){sw=0.0;}elseif((sw12+sw13+sw23)>2.0){sw=1.0;}"
            "else{sw=std::cos((sw12+sw13+sw23-1.0)*M_PI/2.0);sw=1.0-sw*sw;}")
    cos2_grad = ("if((sw12+sw13+sw23)>1.0&&(sw12+sw13+sw23)<2.0){"
                 "gsw12*=-(M_PI/2.0)*sin(M_PI*(sw12+sw13+sw23))*energies[j]/d12r;")
    if cos2 in _ws(body):
        if cos2_grad not in _ws(body):
            raise ValueError("%s: cos2 switch without its gradient" % source)
        sw = "cos2"
        forms[sw] = "cos2"
    else:
        sw = _ws(re.search(r"\bsw\s*=\s*(sw[^;]*);", body).group(1))
    if sw not in forms:
        raise ValueError("%s: switch %s is not supported" % (source, sw))
    skip_expr = _ws(re.search(r"if\s*\(\s*true\s*&&\s*([^{]*)\)\s*\{\s*continue\s*;", body).group(1))
    skips = {"d12r>m_ro": "pair_gt", "d12r>m_ro&&d13r>m_ro&&d23r>m_ro": "all_three_gt"}
    if skip_expr not in skips:
        raise ValueError("%s: skip rule %s is not supported" % (source, skip_expr))
    # polynomial size
    htext = open(os.path.join(ref, "src", header)).read()
    degree = int(re.search(r"degree\s*=\s*(\d+)", htext).group(1))
    nvars = int(re.search(r"n_vars\s*=\s*(\d+)", htext).group(1))
    ncoef = int(re.search(r"size\s*=\s*(\d+)", htext).group(1))
    if nvars != len(variables):
        raise ValueError("%s: %d variables, polynomial has %d" % (source, len(variables), nvars))
    return {"name": name, "monomers": list(mons), "nat": list(nat), "sites": sites, "lp": lp,
            "variables": variables, "switch": forms[sw], "ri": consts["m_ri"], "rf": consts["m_ro"],
            "skip": skips[skip_expr], "nvars": nvars, "ncoef": ncoef, "degree": degree,
            "ref": "%s:%d" % (source, _eval_line(path)), "table": table}


def _eval_line(path):
    """Line of the gradient eval in the original file."""
    for i, l in enumerate(open(path), 1):
        if re.search(r"::eval\s*\(\s*const double\s*\*\s*xyz1", l) and "grad1" in l:
            return i
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"), required=not os.environ.get("MBX_REFERENCE"))
    ap.add_argument("names", nargs="*", default=list(SOURCES))
    args = ap.parse_args(argv)
    os.makedirs(DATA, exist_ok=True)
    for name in args.names:
        spec = extract(args.ref, name, *SOURCES[name])
        with open(os.path.join(DATA, name + ".spec.json"), "w") as f:
            json.dump(spec, f, indent=1)
            f.write("\n")
        print("%-10s %s: %d sites, %d vars, %s switch, skip %s" % (name, spec["ref"], len(spec["sites"]),
                                                                 spec["nvars"], spec["switch"], spec["skip"]))


if __name__ == "__main__":
    main()
