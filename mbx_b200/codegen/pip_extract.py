#!/usr/bin/env python3
"""Recover the monomial basis of the reference's generated PIP programs.

The reference ships each permutationally-invariant polynomial (PIP) only as a
machine-generated straight-line program (``const double tN = ...;`` or
``t[N] = ...;`` assignments over ``a[k]`` and ``x[j]``) that is linear in the
coefficients ``a``.  This tool parses such a program, expands it symbolically
and writes the polynomial in the explicit form

    P(a, x) = sum_k a[k] * sum_m  c_{k,m} * prod_{j in m} x[j]

as a term table (one line per (k, m) pair).  The build's own CUDA generator
(``gen_kernels.py``) and the oracle restatement (``oracle/mbx_oracle.c``)
both work from these tables; neither contains any of the reference programs.
Every table is checked against the compiled reference polynomial (value
and gradient at random variables) in ``tests/test_oracle_goldens.py``
(``test_table_vs_reference_program``).

Programs parsed (file:line of the energy-only evaluator in the reference):

======== ================================================================ ==== ====
name     source                                                           vars coef
======== ================================================================ ==== ====
mbpol2b  potential/2b/poly-2b-v6x-nogrd.cpp:41 (eval(nd, a, x))          31   1153
mbpol3b  potential/3b/poly-3b-v2x-nogrd.cpp:38 (eval(a, x))              36   1163
ch4h2o2b potential/2b/poly_2b_A1B2Z2_C1D4_deg3_exp0_v1.cpp:38             38   603
ch4ch42b potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1.cpp:44982 (+fmg1-15) 45   1345
ch4h2o3b potential/3b/poly_3b_A1B4_C1D2_C1D2_deg3_nograd_v1.cpp:39        55   1254
h2oion2b potential/2b/poly-2b-A1B2Z2_C-v1.cpp:38 (eval(nd, a, x))        8    429
h2oion3b potential/3b/poly-3b-h2o-ion-v1x_deg4_filtered.cpp:39 (*)       21   1016
halh2o2b potential/2b/poly_2b_A1_B1C2X2_deg6_nograd_v1.cpp:50             8    906
halh2o3b potential/3b/poly_3b_A1_B1C2X2_B1C2X2_deg4_nograd_v1.cpp:50      41   3173
co2co22btab potential/2b/poly_2b_A1B2_A1B2_v1.cpp:39 (**)               15   2269
h2oco22b potential/2b/poly_2b_A1B2Z2_C1D2_v1.cpp:39                      21   1653
hehe2b   potential/2b/poly_2b_A1_A1_deg23_v1.cpp:5                        1    23
h2ohe2b  potential/2b/poly_2b_A1B2Z2_C1_deg5_v1.cpp:5                     8    496
n2o5h2o2b potential/2b/poly_2b_A1B2C4_D1E2_deg3_v1.cpp:5                 45   983
a1a12b   potential/2b/poly_2b_A1_A1_deg9_nograd_v1.cpp:50                 1    9
a1b12b   potential/2b/poly_2b_A1_B1_deg9_nograd_v1.cpp:50                 1    9
arh2o2b  potential/2b/poly_2b_A1_B1C2X2_deg5_nograd_v1.cpp:50             8    496
======== ================================================================ ==== ====

(*) the only program of this polynomial computes value and gradient; the
value is its ``double e = tN;``, and only the assignments tN depends on are
expanded.  (**) the value is the expression assigned to ``double e`` before
``return e;``.

It also extracts the fitted linear coefficients (the model parameters) from
the evaluator classes:

* mbpol2b: ``thefit`` in potential/2b/x2b-v9x.cpp:164-1318
* mbpol3b: ``thefit`` in potential/3b/x3b-v2x.cpp:80-1244
* ch4h2o2b: ``coefficients`` in potential/2b/x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:175
* ch4ch42b: ``coefficients`` in potential/2b/x2b_A1B4_A1B4_deg4_exp0_v1x.cpp
* ch4h2o3b: ``coefficients`` in potential/3b/mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp
* h2oli2b, h2ona2b, h2ok2b, h2orb2b, h2ocs2b (table h2oion2b): ``twobodyfit``
  of the ion's constructor block in potential/2b/x2b-A1B2Z2_C-v1x.cpp:181
  (li+), :628 (na+), :1075 (k+), :1522 (rb+), :1969 (cs+)
* h2oli3b, h2ona3b, h2ok3b, h2orb3b, h2ocs3b (table h2oion3b): ``the_poly`` of
  the ion's constructor block in
  potential/3b/x3b-h2o-ion-v1x-deg4-filtered.cpp:485 (li+), :1522 (na+),
  :2561 (k+), :3602 (rb+), :4639 (cs+)
* fh2o2b, clh2o2b, brh2o2b, ih2o2b (table halh2o2b): ``coefficients`` of the
  halide's constructor block in potential/2b/mbnrg_2b_A1_B1C2X2_deg6_v1.cpp:12
  (f-), :929 (cl-), :1846 (br-), :2763 (i-)
* fh2o3b, clh2o3b, brh2o3b, ih2o3b (table halh2o3b): ``coefficients`` of the
  halide's constructor block in
  potential/3b/mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp:13 (f-), :3204 (cl-),
  :6395 (br-), :9586 (i-)
* nana2b, clcl2b, arar2b (table a1a12b), nacl2b, csar2b (table a1b12b):
  ``coefficients`` of the pair's block in potential/2b/mbnrg_2b_A1_A1_deg9_v1.cpp
  :11 (na+ na+), :27 (cl- cl-), :43 (ar ar) and mbnrg_2b_A1_B1_deg9_v1.cpp :11
  (na+ cl-), :27 (cs+ ar); arh2o2b: mbnrg_2b_A1_B1C2X2_deg5_v1.cpp:11
* co2a2b, co2co22b (table co2co22btab): ``coefficients`` of the model's block
  in potential/2b/x2b_A1B2_A1B2_v1x.cpp :88 (co2_archive), :2373 (co2)

Output (``mbx_b200/data/``): ``<table>.pip.gz`` (term table, gzip) and
``<evaluator>.fit`` (coefficients, one per line, printed with ``repr`` so they
round-trip bit-exactly); an evaluator's table is named after it unless
several evaluators share one polynomial.

Usage: ``python -m mbx_b200.codegen.pip_extract [--ref DIR] (or MBX_REFERENCE)``
"""
import argparse
import gzip
import os
import re
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "data")

PROGRAMS = {
    "mbpol2b": ("potential/2b/poly-2b-v6x-nogrd.cpp", 31, 1153, 4),
    "mbpol3b": ("potential/3b/poly-3b-v2x-nogrd.cpp", 36, 1163, 4),
    "ch4h2o2b": ("potential/2b/poly_2b_A1B2Z2_C1D4_deg3_exp0_v1.cpp", 38, 603, 3),
    "ch4ch42b": ("potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1.cpp", 45, 1345, 4),
    "ch4h2o3b": ("potential/3b/poly_3b_A1B4_C1D2_C1D2_deg3_nograd_v1.cpp", 55, 1254, 3),
    "h2oion2b": ("potential/2b/poly-2b-A1B2Z2_C-v1.cpp", 8, 429, 5),
    "h2oion3b": ("potential/3b/poly-3b-h2o-ion-v1x_deg4_filtered.cpp", 21, 1016, 4),
    "halh2o2b": ("potential/2b/poly_2b_A1_B1C2X2_deg6_nograd_v1.cpp", 8, 906, 6),
    "halh2o3b": ("potential/3b/poly_3b_A1_B1C2X2_B1C2X2_deg4_nograd_v1.cpp", 41, 3173, 4),
    "a1a12b": ("potential/2b/poly_2b_A1_A1_deg9_nograd_v1.cpp", 1, 9, 9),
    "a1b12b": ("potential/2b/poly_2b_A1_B1_deg9_nograd_v1.cpp", 1, 9, 9),
    "arh2o2b": ("potential/2b/poly_2b_A1_B1C2X2_deg5_nograd_v1.cpp", 8, 496, 5),
    "co2co22btab": ("potential/2b/poly_2b_A1B2_A1B2_v1.cpp", 15, 2269, 5),
    "h2oco22b": ("potential/2b/poly_2b_A1B2Z2_C1D2_v1.cpp", 21, 1653, 4),
    "hehe2b": ("potential/2b/poly_2b_A1_A1_deg23_v1.cpp", 1, 23, 23),
    "h2ohe2b": ("potential/2b/poly_2b_A1B2Z2_C1_deg5_v1.cpp", 8, 496, 5),
    "n2o5h2o2b": ("potential/2b/poly_2b_A1B2C4_D1E2_deg3_v1.cpp", 45, 983, 3),
    # 1-body: CH4 (x1b_A1B4_deg5_exp0::x1b_A1B4_v1x, potential/1b/x1b_A1B4_deg5_exp0_v1x.cpp:309-419)
    "ch41b": ("potential/1b/poly_1b_A1B4_deg5_exp0_v1.cpp", 10, 207, 5),
}
# programs whose value is assigned to ``double e`` and then returned
E_ASSIGN = {"co2co22btab", "ch41b"}
# programs whose value is a named temporary (value + gradient programs)
RESULT_VAR = {"h2oion3b": r"double e = (t\d+)\s*;"}

FITS = {
    "mbpol2b": ("potential/2b/x2b-v9x.cpp", r"const double thefit\[\]\s*=\s*\{"),
    "mbpol3b": ("potential/3b/x3b-v2x.cpp", r"thefit\[[^\]]*\]\s*=\s*\{"),
    "ch4h2o2b": ("potential/2b/x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp", r"coefficients\s*=\s*std::vector<double>\s*\{"),
    "ch4ch42b": ("potential/2b/x2b_A1B4_A1B4_deg4_exp0_v1x.cpp", r"coefficients\s*=\s*std::vector<double>\s*\{"),
    "ch4h2o3b": ("potential/3b/mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp", r"coefficients\s*=\s*std::vector<double>\s*\{"),
}
_ION2B = "potential/2b/x2b-A1B2Z2_C-v1x.cpp"
for _ion, _name in (("li", "h2oli2b"), ("na", "h2ona2b"), ("k", "h2ok2b"), ("rb", "h2orb2b"), ("cs", "h2ocs2b")):
    FITS[_name] = (_ION2B, r'if \(mon1 == "h2o" && mon2 == "%s\+"\) \{\s*twobodyfit\s*=\s*std::vector<double>\s*\{' % _ion)

# the template-generated MB-nrg evaluators whose specs codegen/mbnrg_spec.py
# extracts: their energy-only programs and constructor blocks
def _mbnrg_programs():
    from mbx_b200.codegen import mbnrg_spec as ms
    progs, fits, tables = {}, {}, {}
    for name, (source, mons, table, header) in ms.SOURCES.items():
        progs[table] = (ms.PROGRAMS[table], header)
        fits[name] = (source, ms.fit_pattern(mons))
        tables[name] = table
    return progs, fits, tables


MBNRG_PROGRAMS, _fits, _tables = _mbnrg_programs()
FITS.update(_fits)

# evaluator -> the program (table) its coefficients belong to
TABLE_OF = {name: name for name in PROGRAMS if name in FITS}
TABLE_OF.update(_tables)
TABLE_OF.update({n: "h2oion2b" for n in ("h2oli2b", "h2ona2b", "h2ok2b", "h2orb2b", "h2ocs2b")})
_ION3B = "potential/3b/x3b-h2o-ion-v1x-deg4-filtered.cpp"
for _ion in ("li", "na", "k", "rb", "cs"):
    FITS["h2o%s3b" % _ion] = (_ION3B, r'\(m3 == "%s\+"\) \{\s*const double the_poly\[\]\s*=\s*\{' % _ion)
    TABLE_OF["h2o%s3b" % _ion] = "h2oion3b"
for _hal in ("f", "cl", "br", "i"):
    FITS["%sh2o2b" % _hal] = ("potential/2b/mbnrg_2b_A1_B1C2X2_deg6_v1.cpp",
                              r'if \(mon1 == "%s-" and mon2 == "h2o"\) \{\s*coefficients\s*=\s*std::vector<double>\s*\{'
                              % _hal)
    FITS["%sh2o3b" % _hal] = ("potential/3b/mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp",
                              r'if \(mon1 == "%s-" and mon2 == "h2o" and mon3 == "h2o"\) \{\s*coefficients\s*=\s*'
                              r'std::vector<double>\s*\{' % _hal)
    TABLE_OF["%sh2o2b" % _hal] = "halh2o2b"
    TABLE_OF["%sh2o3b" % _hal] = "halh2o3b"
for _m1, _m2, _name, _table, _file in (
        ("na\\+", "na\\+", "nana2b", "a1a12b", "mbnrg_2b_A1_A1_deg9_v1.cpp"),
        ("cl-", "cl-", "clcl2b", "a1a12b", "mbnrg_2b_A1_A1_deg9_v1.cpp"),
        ("ar", "ar", "arar2b", "a1a12b", "mbnrg_2b_A1_A1_deg9_v1.cpp"),
        ("na\\+", "cl-", "nacl2b", "a1b12b", "mbnrg_2b_A1_B1_deg9_v1.cpp"),
        ("cs\\+", "ar", "csar2b", "a1b12b", "mbnrg_2b_A1_B1_deg9_v1.cpp"),
        ("ar", "h2o", "arh2o2b", "arh2o2b", "mbnrg_2b_A1_B1C2X2_deg5_v1.cpp")):
    FITS[_name] = ("potential/2b/" + _file, r'if \(mon1 == "%s" and mon2 == "%s"\) \{\s*coefficients\s*=\s*'
                   r'std::vector<double>\s*\{' % (_m1, _m2))
    TABLE_OF[_name] = _table
for _m, _name in (("co2_archive", "co2a2b"), ("co2", "co2co22b"), ("co2cm5100", "cm5100co22b"),
                  ("co2cm595", "cm595co22b"), ("co2cm590", "cm590co22b"), ("co2cm585", "cm585co22b"),
                  ("co2cm5875", "cm5875co22b"), ("co2cm580", "cm580co22b")):
    FITS[_name] = ("potential/2b/x2b_A1B2_A1B2_v1x.cpp", r'if \(mon1 == "%s" && mon2 == "%s"\) \{\s*coefficients\s*=\s*'
                   r'std::vector<double>\s*\{' % (_m, _m))
    TABLE_OF[_name] = "co2co22btab"
FITS["h2oco22b"] = ("potential/2b/x2b_A1B2Z2_C1D2_v1x.cpp",
                    r'if \(mon1 == "h2o" && mon2 == "co2"\) \{\s*coefficients\s*=\s*std::vector<double>\s*\{')
TABLE_OF["h2oco22b"] = "h2oco22b"
FITS["h2oco2a2b"] = ("potential/2b/x2b_A1B2Z2_C1D2_v1x.cpp",
                     r'if \(mon1 == "h2o" && mon2 == "co2_archive"\) \{\s*coefficients\s*=\s*std::vector<double>\s*\{')
TABLE_OF["h2oco2a2b"] = "h2oco22b"
FITS["ch41b"] = ("potential/1b/x1b_A1B4_deg5_exp0_v1x.cpp",
                 r'if \(mon == "ch4"\) \{\s*coefficients\s*=\s*std::vector<double>\s*\{')
TABLE_OF["ch41b"] = "ch41b"
FITS["n2o5h2o2b"] = ("potential/2b/x2b_A1B2C4_D1E2_deg3_v1x.cpp",
                     r'if \(mon1 == "h2o" && mon2 == "n2o5"\) \{\s*coefficients\s*=\s*std::vector<double>\s*\{')
TABLE_OF["n2o5h2o2b"] = "n2o5h2o2b"
FITS["hehe2b"] = ("potential/2b/x2b_A1_A1_deg23_v1x.cpp",
                  r'if \( mon1 == "he" && mon2 == "he" \) \{\s*coefficients\s*=\s*std::vector<double>\s*\{')
FITS["h2ohe2b"] = ("potential/2b/x2b_A1B2Z2_C1_deg5_v1x.cpp",
                   r'if \(mon1 == "h2o" && mon2  == "he"\) \{[^{}]*?coefficients\s*=\s*std::vector<double>\s*\{')
TABLE_OF["hehe2b"] = "hehe2b"
TABLE_OF["h2ohe2b"] = "h2ohe2b"

TOKEN = re.compile(
    r"\s*(?:(?P<num>\d+\.\d*(?:[eE][-+]?\d+)?|\d+(?:[eE][-+]?\d+)?)"
    r"|(?P<t>t\[\d+\]|t\d+)"
    r"|(?P<a>a\[\d+\])"
    r"|(?P<x>x\[[^\]]*\])"
    r"|(?P<op>[-+*/()]))"
)


# ---------------------------------------------------------------------------
# Sparse polynomials linear in a: dict {(k, mono): coef}; k = -1 means "no a",
# mono = sorted tuple of variable indices (with repetition).
# ---------------------------------------------------------------------------

def padd(p, q, sign=1.0):
    r = dict(p)
    for key, c in q.items():
        v = r.get(key, 0.0) + sign * c
        if v == 0.0:
            r.pop(key, None)
        else:
            r[key] = v
    return r


def pmul(p, q):
    if len(p) > len(q):
        p, q = q, p
    r = {}
    for (k1, m1), c1 in p.items():
        for (k2, m2), c2 in q.items():
            if k1 >= 0 and k2 >= 0:
                raise ValueError("program is not linear in the coefficients")
            key = (k1 if k1 >= 0 else k2, tuple(sorted(m1 + m2)))
            v = r.get(key, 0.0) + c1 * c2
            if v == 0.0:
                r.pop(key, None)
            else:
                r[key] = v
    return r


class Parser:
    def __init__(self, env, xindex):
        self.env = env
        self.xindex = xindex

    def parse(self, text):
        self.toks = []
        pos = 0
        text = text.strip()
        while pos < len(text):
            m = TOKEN.match(text, pos)
            if not m or m.end() == pos:
                raise ValueError("cannot tokenise: %r" % text[pos:pos + 40])
            self.toks.append((m.lastgroup, m.group(m.lastgroup)))
            pos = m.end()
            while pos < len(text) and text[pos].isspace():
                pos += 1
        self.i = 0
        v = self.expr()
        if self.i != len(self.toks):
            raise ValueError("trailing tokens in %r" % text[:80])
        return v

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else (None, None)

    def expr(self):
        v = self.term()
        while True:
            kind, tok = self.peek()
            if kind == "op" and tok in "+-":
                self.i += 1
                v = padd(v, self.term(), 1.0 if tok == "+" else -1.0)
            else:
                return v

    def term(self):
        v = self.factor()
        while True:
            kind, tok = self.peek()
            if kind == "op" and tok == "*":
                self.i += 1
                v = pmul(v, self.factor())
            elif kind == "op" and tok == "/":
                self.i += 1
                d = self.factor()
                if len(d) != 1 or next(iter(d)) != (-1, ()):
                    raise ValueError("division by a non-constant")
                c = next(iter(d.values()))
                v = {key: val / c for key, val in v.items()}
            else:
                return v

    def factor(self):
        kind, tok = self.peek()
        self.i += 1
        if kind == "op" and tok == "-":
            return {key: -c for key, c in self.factor().items()}
        if kind == "op" and tok == "+":
            return self.factor()
        if kind == "op" and tok == "(":
            v = self.expr()
            k2, t2 = self.peek()
            if t2 != ")":
                raise ValueError("missing )")
            self.i += 1
            return v
        if kind == "num":
            return {(-1, ()): float(tok)}
        if kind == "t":
            return self.env[tok.replace("[", "").replace("]", "")]
        if kind == "a":
            return {(int(tok[2:-1]), ()): 1.0}
        if kind == "x":
            return {(-1, (self.xindex(tok),)): 1.0}
        raise ValueError("unexpected token %r" % (tok,))


def xindex_factory(src):
    def xi(tok):
        inner = tok[2:-1].replace(" ", "")
        m = re.fullmatch(r"(\d+)", inner)
        if m:
            return int(m.group(1))
        m = re.fullmatch(r"nv\+nd\*(\d+)", inner)
        if m:
            return int(m.group(1))
        raise ValueError("unknown x index form %r in %s" % (tok, src))
    return xi


ASSIGN = re.compile(r"(?:const\s+double\s+)?(t\d+|t\[\d+\])\s*=\s*([^;]*);", re.S)


def statements(body):
    """Yield (target, expr) for assignments and ('<result>', expr) for the result."""
    for stmt in body.split(";"):
        s = " ".join(stmt.split()).replace(" [", "[")
        if not s:
            continue
        m = re.fullmatch(r"(?:const double )?(t\d+|t\[\d+\]) = (.*)", s)
        if m:
            yield m.group(1).replace("[", "").replace("]", ""), m.group(2)
            continue
        m = re.fullmatch(r"(?:return ?\(?|energy\[nv\] = )(.*)", s)
        if m and ("t" in m.group(1)):
            expr = m.group(1)
            if re.match(r"return ?\(", s) and expr.endswith(")") and expr.count("(") < expr.count(")"):
                expr = expr[:-1]
            yield "<result>", expr


def function_bodies(text, names):
    """Return the bodies of the named functions, in the order given."""
    out = []
    for name in names:
        m = re.search(r"\b" + re.escape(name) + r"\s*\([^)]*\)\s*\{", text)
        if not m:
            raise ValueError("function %s not found" % name)
        depth, i = 1, m.end()
        while depth:
            c = text[i]
            depth += (c == "{") - (c == "}")
            i += 1
        out.append(text[m.end():i - 1])
    return out


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def extract_program(ref, name):
    rel, nvars, ncoef, degree = program(ref, name)
    path = os.path.join(ref, "src", rel)
    text = strip_comments(open(path).read())
    text = re.sub(r"#ifdef DEBUG.*?#endif", "", text, flags=re.S)
    if name in E_ASSIGN:
        text = re.sub(r"\bdouble e\s*=", "return", text).replace("return e;", "")
    if name == "ch4ch42b":
        bodies = function_bodies(text, ["fmg%d" % i for i in range(1, 16)])
        main = re.search(r"::eval\(const double a\[1345\], const double x\[45\]\)\s*\{(.*?)\n\}", text, re.S).group(1)
        bodies.append(main)
    elif name in ("mbpol2b", "h2oion2b"):
        m = re.search(r"for \(size_t nv = 0; nv < nd; nv\+\+\) \{(.*?)\n    \}\n    return energy;", text, re.S)
        bodies = [m.group(1)]
    else:
        m = re.search(r"::eval\([^)]*\)\s*\{(.*)\}\s*\}\s*//\s*namespace", text, re.S)
        if not m:
            m = re.search(r"::eval\([^)]*\)\s*\{(.*)\}", text, re.S)
        bodies = [m.group(1)]
    env = {}
    parser = Parser(env, xindex_factory(rel))
    result = None
    if name in RESULT_VAR:
        return _terms(extract_result_var(bodies[0], RESULT_VAR[name], parser, env), rel, nvars, ncoef, degree)
    for body in bodies:
        for target, expr in statements(body):
            if target in ("fmg%d" % i for i in range(1, 16)):
                continue
            if re.fullmatch(r"fmg\d+\(x, a, t\)", expr or ""):
                continue
            v = parser.parse(expr)
            if target == "<result>":
                result = v
            else:
                env[target] = v
    if result is None:
        raise ValueError("no result expression found in %s" % rel)
    return _terms(result, rel, nvars, ncoef, degree)


def extract_result_var(body, pattern, parser, env):
    """The polynomial a value + gradient program returns as ``double e = tN``:
    the assignments tN depends on (transitively), expanded in program order."""
    exprs = {}
    order = []
    for target, expr in statements(body):
        if target != "<result>":
            exprs[target] = expr
            order.append(target)
    root = re.search(pattern, body).group(1)
    need, stack = set(), [root]
    while stack:
        t = stack.pop()
        if t in need:
            continue
        need.add(t)
        stack += [d.replace("[", "").replace("]", "") for d in re.findall(r"\bt\[?\d+\]?", exprs[t])]
    for t in order:
        if t in need:
            env[t] = parser.parse(exprs[t])
    return env[root]


def _terms(result, rel, nvars, ncoef, degree):
    terms = []
    for (k, mono), c in result.items():
        if k < 0:
            raise ValueError("term without a coefficient in %s" % rel)
        if len(mono) > degree or (mono and max(mono) >= nvars) or k >= ncoef:
            raise ValueError("term out of range in %s: %r" % (rel, (k, mono)))
        terms.append((k, mono, c))
    terms.sort(key=lambda t: (t[0], len(t[1]), t[1]))
    return terms


def program(ref, name):
    """(source, nvars, ncoef, degree) of a table's energy-only program."""
    if name in PROGRAMS:
        return PROGRAMS[name]
    from mbx_b200.codegen.mbnrg_spec import poly_size
    rel, header = MBNRG_PROGRAMS[name]
    return (rel,) + poly_size(ref, header)


def extract_fit(ref, name, ncoef):
    rel, pattern = FITS[name]
    text = strip_comments(open(os.path.join(ref, "src", rel)).read())
    m = re.search(pattern, text)
    if not m:
        raise ValueError("coefficients not found in %s" % rel)
    end = text.index("}", m.end())
    vals = [float(v) for v in text[m.end():end].replace(",", " ").split()]
    if len(vals) != ncoef:
        raise ValueError("%s: expected %d coefficients, found %d" % (rel, ncoef, len(vals)))
    return vals


def write_table(name, terms, nvars, ncoef, degree):
    os.makedirs(DATA, exist_ok=True)
    with gzip.GzipFile(os.path.join(DATA, name + ".pip.gz"), "wb", mtime=0) as gz, \
            __import__("io").TextIOWrapper(gz) as f:
        f.write("# PIP term table: k coef nvar v1..vn  (P = sum a[k] * coef * prod x[v])\n")
        f.write("%d %d %d %d\n" % (nvars, ncoef, degree, len(terms)))
        for k, mono, c in terms:
            ci = int(c)
            cs = str(ci) if ci == c else repr(c)
            f.write("%d %s %d %s\n" % (k, cs, len(mono), " ".join(map(str, mono))))


def write_fit(name, fit):
    os.makedirs(DATA, exist_ok=True)
    with open(os.path.join(DATA, name + ".fit"), "w") as f:
        for v in fit:
            f.write(repr(v) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"), required=not os.environ.get("MBX_REFERENCE"))
    ap.add_argument("names", nargs="*", default=list(PROGRAMS) + list(MBNRG_PROGRAMS))
    args = ap.parse_args(argv)
    for name in args.names:
        t0 = time.time()
        rel, nvars, ncoef, degree = program(args.ref, name)
        terms = extract_program(args.ref, name)
        used = sorted({t[0] for t in terms})
        write_table(name, terms, nvars, ncoef, degree)
        fits = [e for e, t in TABLE_OF.items() if t == name]
        for e in fits:
            write_fit(e, extract_fit(args.ref, e, ncoef))
        print("%-9s %6d terms, %4d/%d coefficients used, fits %s, %.1fs" %
              (name, len(terms), len(used), ncoef, ",".join(fits), time.time() - t0))
    return 0


if __name__ == "__main__":
    sys.exit(main())
