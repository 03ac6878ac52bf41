#!/usr/bin/env python3
"""Generate the per-evaluator CUDA device code from the declarative specs.

For each evaluator in ``mbx_b200.specs.SPECS`` this writes
``mbx_b200/csrc/gen/<name>.cuh`` holding:

* ``<name>_vars``: the polynomial variables (straight-line FP64: differences,
  sqrt, exp) and the factor that turns dP/dv into a Cartesian gradient;
* ``<name>_pip``: the polynomial and its reverse-mode gradient, as a
  multivariate Horner trie over the expanded term table;
* ``<name>_pip_e``: the energy-only Horner evaluation;
* ``<name>_pip_mixed``: the same trie with the leaf level (three quarters of
  all terms) in FP32 and the upper levels and every accumulation above the
  leaves in FP64;
* ``<name>_dcoef``: per-coefficient monomial sums dP/da_k (for the adjoint with
  respect to the linear coefficients), recomputed from x.

The trie.  Every term is a monomial x_v1 x_v2 ... (variables sorted in a fixed
order); the monomials form a prefix tree.  With P(n) the product along the path
to node n and V(n) = c_n + sum_children x_var(child) V(child), the polynomial
is V(root) and reverse mode gives dP/dx_var(n) += P(parent(n)) V(n) for every
node.  A depth-first walk keeps only one (P, V) pair per depth live, so the
whole evaluation runs out of registers: nvars values, nvars gradient
accumulators and eight temporaries.  Each leaf costs two FMAs (one into V,
one into its gradient), each inner node one multiply and two FMAs.

Coefficients come from ``coef[k]``, ``coef`` being a template parameter of
the generated functions (a view of a ``__constant__`` array or of a global
pointer).
"""
import argparse
import collections
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
sys.path.insert(0, os.path.dirname(PKG))

from mbx_b200.specs import SPECS, LP_GAMMA_IN, LP_GAMMA_OUT  # noqa: E402
from mbx_b200.tables import load_pip  # noqa: E402

OUT = os.path.join(PKG, "csrc", "gen")

# Larger polynomials (CH4-CH4: 201k terms) use the table-driven warp kernel.
STRAIGHT_LINE_MAX_TERMS = 60000


def lit(v):
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return r


class Trie:
    def __init__(self, table):
        freq = collections.Counter()
        for t in range(table.nterms):
            for v in set(table.var[t, :table.deg[t]].tolist()):
                freq[v] += 1
        order = [v for v, _ in freq.most_common()] + [v for v in range(table.nvars) if v not in freq]
        self.rank = {v: i for i, v in enumerate(order)}
        self.root = {"coef": [], "kids": collections.OrderedDict()}
        for t in range(table.nterms):
            mono = sorted(table.var[t, :table.deg[t]].tolist(), key=lambda v: self.rank[v])
            node = self.root
            for v in mono:
                node = node["kids"].setdefault(v, {"coef": [], "kids": collections.OrderedDict()})
            node["coef"].append((int(table.k[t]), float(table.coef[t])))
        self._sort(self.root)

    def _sort(self, node):
        node["kids"] = collections.OrderedDict(sorted(node["kids"].items(), key=lambda kv: self.rank[kv[0]]))
        for ch in node["kids"].values():
            self._sort(ch)

    def counts(self):
        leaves = inner = 0
        stack = [self.root]
        while stack:
            n = stack.pop()
            for ch in n["kids"].values():
                if ch["kids"]:
                    inner += 1
                    stack.append(ch)
                else:
                    leaves += 1
        return leaves, inner


def coef_expr(coefs, conv=""):
    """Sum of COEF(k)*c for the terms ending exactly at a node."""
    parts = []
    for k, c in coefs:
        if c == 1.0:
            parts.append("%scoef[%d]" % (conv, k))
        else:
            parts.append("%s(coef[%d] * %s)" % (conv, k, lit(c)))
    return " + ".join(parts) if parts else None


def emit_pip(trie, nvars, name, out):
    """FP64 value + gradient: double name(const double* x, double* g)."""
    w = out.append
    w("// %s: polynomial and reverse-mode gradient (multivariate Horner trie)" % name)
    w("template <class Coef>")
    w("__device__ __forceinline__ double %s(const Coef& coef, const double (&x)[%d], double (&g)[%d]) {" %
      (name, nvars, nvars))
    w("    double E = 0.0;")

    def node(n, var, depth, pexpr):
        # pexpr: expression for P(parent), None at the root's children (P = 1)
        P = "P%d" % depth
        V = "V%d" % depth
        if pexpr is None:
            w("    { const double %s = x[%d];" % (P, var))
        else:
            w("    { const double %s = %s * x[%d];" % (P, pexpr, var))
        ce = coef_expr(n["coef"])
        w("      double %s = %s;" % (V, ce if ce else "0.0"))
        for cv, ch in n["kids"].items():
            if ch["kids"]:
                node(ch, cv, depth + 1, P)
            else:
                c = coef_expr(ch["coef"])
                w("      %s = fma(%s, x[%d], %s); g[%d] = fma(%s, %s, g[%d]);" % (V, c, cv, V, cv, c, P, cv))
        if pexpr is None:
            w("      g[%d] += %s; E = fma(x[%d], %s, E); }" % (var, V, var, V))
        else:
            w("      g[%d] = fma(%s, %s, g[%d]); V%d = fma(x[%d], %s, V%d); }" %
              (var, pexpr, V, var, depth - 1, var, V, depth - 1))

    for var, ch in trie.root["kids"].items():
        if ch["kids"]:
            node(ch, var, 1, None)
        else:
            c = coef_expr(ch["coef"])
            w("    E = fma(%s, x[%d], E); g[%d] += %s;" % (c, var, var, c))
    w("    return E;")
    w("}")


def emit_pip_energy(trie, nvars, name, out):
    """FP64 value only: plain Horner over the trie."""
    w = out.append
    w("template <class Coef>")
    w("__device__ __forceinline__ double %s(const Coef& coef, const double (&x)[%d]) {" % (name, nvars))
    w("    double E = 0.0;")

    def node(n, var, depth):
        V = "V%d" % depth
        ce = coef_expr(n["coef"])
        w("    { double %s = %s;" % (V, ce if ce else "0.0"))
        for cv, ch in n["kids"].items():
            if ch["kids"]:
                node(ch, cv, depth + 1)
            else:
                w("      %s = fma(%s, x[%d], %s);" % (V, coef_expr(ch["coef"]), cv, V))
        tgt = "E" if depth == 1 else "V%d" % (depth - 1)
        w("      %s = fma(x[%d], %s, %s); }" % (tgt, var, V, tgt))

    for var, ch in trie.root["kids"].items():
        if ch["kids"]:
            node(ch, var, 1)
        else:
            w("    E = fma(%s, x[%d], E);" % (coef_expr(ch["coef"]), var))
    w("    return E;")
    w("}")


def emit_pip_mixed(trie, nvars, name, out):
    """Mixed precision: products and leaf-level sums in FP32, everything that
    accumulates across leaf groups (inner-node values, the energy) in FP64.

    Leaf gradient contributions go to FP32 accumulators gf[] (each receives one
    product per leaf); inner-node gradient contributions go to FP64 g[].  The
    caller adds gf into g at the end."""
    w = out.append
    w("template <class Coef>")
    w("__device__ __forceinline__ double %s(const Coef& coef, const float (&xf)[%d], const double (&x)[%d], "
      "double (&g)[%d], float (&gf)[%d]) {" % (name, nvars, nvars, nvars, nvars))
    w("    double E = 0.0;")

    def node(n, var, depth, pexpr_f, pexpr_d):
        # FP32 product P and FP64 product PD along the path; inner-node values
        # V in FP64 except the last inner level, whose leaf sums are FP32.
        Pf = "Pf%d" % depth
        Pd = "Pd%d" % depth
        leaf_only = all(not ch["kids"] for ch in n["kids"].values())
        if pexpr_f is None:
            w("    { const float %s = xf[%d]; const double %s = x[%d];" % (Pf, var, Pd, var))
        else:
            w("    { const float %s = %s * xf[%d]; const double %s = %s * x[%d];" %
              (Pf, pexpr_f, var, Pd, pexpr_d, var))
        if leaf_only:
            V = "Vf%d" % depth
            ce = coef_expr(n["coef"], "(float)")
            w("      float %s = %s;" % (V, ce if ce else "0.0f"))
            for cv, ch in n["kids"].items():
                c = coef_expr(ch["coef"], "(float)")
                w("      %s = fmaf(%s, xf[%d], %s); gf[%d] = fmaf(%s, %s, gf[%d]);" % (V, c, cv, V, cv, c, Pf, cv))
            Vd = "(double)%s" % V
        else:
            V = "Vd%d" % depth
            ce = coef_expr(n["coef"])
            w("      double %s = %s;" % (V, ce if ce else "0.0"))
            for cv, ch in n["kids"].items():
                if ch["kids"]:
                    node(ch, cv, depth + 1, Pf, Pd)
                else:
                    c = coef_expr(ch["coef"])
                    w("      %s = fma(%s, x[%d], %s); g[%d] = fma(%s, %s, g[%d]);" % (V, c, cv, V, cv, c, Pd, cv))
            Vd = V
        if pexpr_f is None:
            w("      g[%d] += %s; E = fma(x[%d], %s, E); }" % (var, Vd, var, Vd))
        else:
            w("      g[%d] = fma(%s, %s, g[%d]); Vd%d = fma(x[%d], %s, Vd%d); }" %
              (var, pexpr_d, Vd, var, depth - 1, var, Vd, depth - 1))

    for var, ch in trie.root["kids"].items():
        if ch["kids"]:
            node(ch, var, 1, None, None)
        else:
            c = coef_expr(ch["coef"])
            w("    E = fma(%s, x[%d], E); g[%d] += %s;" % (c, var, var, c))
    w("    return E;")
    w("}")


def emit_dcoef(table, nvars, name, out):
    """dP/da_k = sum of the monomials of coefficient k; calls SINK(k, value)."""
    w = out.append
    w("template <class Sink>")
    w("__device__ __forceinline__ void %s(const double (&x)[%d], Sink&& SINK) {" % (name, nvars))
    by_k = collections.defaultdict(list)
    for t in range(table.nterms):
        by_k[int(table.k[t])].append((float(table.coef[t]), table.var[t, :table.deg[t]].tolist()))
    for k in sorted(by_k):
        terms = []
        for c, mono in by_k[k]:
            prod = " * ".join("x[%d]" % v for v in mono) if mono else "1.0"
            terms.append(prod if c == 1.0 else "%s * %s" % (lit(c), prod))
        w("    SINK(%d, %s);" % (k, " + ".join(terms)))
    w("}")


def emit_vars(spec, out):
    """Sites (incl. lone pairs), variables and their Cartesian derivative factors."""
    w = out.append
    ns = len(spec.sites)
    nv = spec.nvars
    w("// sites, variables and dv/d(p1-p2) factors for %s (%s)" % (spec.name, spec.ref))
    w("__device__ __forceinline__ void %s_sites(const double (&r)[%d][3], double (&s)[%d][3]) {" %
      (spec.name, spec.nreal, ns))
    w("#pragma unroll")
    w("    for (int i = 0; i < %d; ++i) { s[i][0] = r[i][0]; s[i][1] = r[i][1]; s[i][2] = r[i][2]; }" % spec.nreal)
    for (m, o, xp, xm) in spec.lp:
        w("    lp_sites(s[%d], s[%d], s[%d], s[%d], s[%d]);" % (o, o + 1, o + 2, xp, xm))
    w("}")
    w("__device__ __forceinline__ void %s_vars(const double (&s)[%d][3], double (&x)[%d]) {" % (spec.name, ns, nv))
    for v, (kind, a, b, k, d0) in enumerate(spec.variables):
        fn = "var_exp" if kind == "exp" else "var_coul"
        w("    x[%d] = %s(s[%d], s[%d], %s, %s);" % (v, fn, a, b, lit(k), lit(d0)))
    w("}")
    # chain rule: site gradients from dP/dv (g), scaled by sw
    w("__device__ __forceinline__ void %s_chain(const double (&s)[%d][3], const double (&g)[%d], "
      "double (&sg)[%d][3]) {" % (spec.name, ns, nv, ns))
    w("#pragma unroll")
    w("    for (int i = 0; i < %d; ++i) { sg[i][0] = 0.0; sg[i][1] = 0.0; sg[i][2] = 0.0; }" % ns)
    for v, (kind, a, b, k, d0) in enumerate(spec.variables):
        fn = "dvar_exp" if kind == "exp" else "dvar_coul"
        w("    %s(s[%d], s[%d], %s, %s, g[%d], sg[%d], sg[%d]);" % (fn, a, b, lit(k), lit(d0), v, a, b))
    for (m, o, xp, xm) in spec.lp:
        w("    lp_grads(s[%d], s[%d], s[%d], sg[%d], sg[%d], sg[%d], sg[%d], sg[%d]);" %
          (o, o + 1, o + 2, xp, xm, o, o + 1, o + 2))
    w("}")


def emit_traits(spec, table, straight, out):
    """Compile-time description the kernel templates in holder_kernel.cuh use."""
    w = out.append
    n = spec.name
    nat = list(spec.nat) + [0] * (3 - len(spec.nat))
    first = [0, nat[0], nat[0] + nat[1]]
    ns = len(spec.sites)
    w("struct %s_T {" % n)
    w("    static constexpr int NBODY = %d, NVARS = %d, NREAL = %d, NSITES = %d, NCOEF = %d, NTERMS = %d;" %
      (spec.nbody, spec.nvars, spec.nreal, ns, spec.ncoef, table.nterms))
    w("    static constexpr int NAT0 = %d, NAT1 = %d, NAT2 = %d;" % tuple(nat))
    w("    static constexpr int FIRST0 = %d, FIRST1 = %d, FIRST2 = %d;" % tuple(first))
    w("    static constexpr int SWITCH_TRIPLE = %d, SKIP = %d, STRAIGHT = %d, DEGREE = %d;" %
      (1 if spec.switch == "triple" else 0, {"pair_gt": 0, "two_of_three_gt": 1, "all_three_gt": 2}[spec.skip],
       1 if straight else 0, spec.degree))
    w("    static constexpr double RI = %s, RF = %s;" % (lit(spec.ri), lit(spec.rf)))
    w("    __device__ static void sites(const double (&r)[%d][3], double (&s)[%d][3]) { %s_sites(r, s); }" %
      (spec.nreal, ns, n))
    w("    __device__ static void vars(const double (&s)[%d][3], double (&x)[%d]) { %s_vars(s, x); }" %
      (ns, spec.nvars, n))
    w("    __device__ static void chain(const double (&s)[%d][3], const double (&g)[%d], double (&sg)[%d][3]) "
      "{ %s_chain(s, g, sg); }" % (ns, spec.nvars, ns, n))
    if straight:
        w("    template <class C> __device__ static double pip(const C& c, const double (&x)[%d], double (&g)[%d]) "
          "{ return %s_pip(c, x, g); }" % (spec.nvars, spec.nvars, n))
        w("    template <class C> __device__ static double pip_e(const C& c, const double (&x)[%d]) "
          "{ return %s_pip_e(c, x); }" % (spec.nvars, n))
        w("    template <class C> __device__ static double pip_mixed(const C& c, const float (&xf)[%d], "
          "const double (&x)[%d], double (&g)[%d], float (&gf)[%d]) { return %s_pip_mixed(c, xf, x, g, gf); }" %
          (spec.nvars, spec.nvars, spec.nvars, spec.nvars, n))
        w("    template <class S> __device__ static void dcoef(const double (&x)[%d], S&& sink) "
          "{ %s_dcoef(x, sink); }" % (spec.nvars, n))
    w("};")


def generate(name):
    spec = SPECS[name]
    table = load_pip(name)
    trie = Trie(table)
    leaves, inner = trie.counts()
    out = ["// Generated by mbx_b200/codegen/gen_kernels.py from mbx_b200/specs.py and",
           "// mbx_b200/data/%s.pip -- do not edit." % name,
           "// %d terms: %d leaves, %d inner nodes" % (table.nterms, leaves, inner),
           "#pragma once",
           "#define %s_NVARS %d" % (name.upper(), spec.nvars),
           "#define %s_NCOEF %d" % (name.upper(), spec.ncoef),
           "#define %s_NSITES %d" % (name.upper(), len(spec.sites)),
           "#define %s_NREAL %d" % (name.upper(), spec.nreal),
           "#define %s_NTERMS %d" % (name.upper(), table.nterms),
           "#define %s_TRIE_LEAVES %d" % (name.upper(), leaves),
           "#define %s_TRIE_INNER %d" % (name.upper(), inner)]
    emit_vars(spec, out)
    if table.nterms <= STRAIGHT_LINE_MAX_TERMS:
        out.append("#define %s_STRAIGHT_LINE 1" % name.upper())
        emit_pip(trie, spec.nvars, name + "_pip", out)
        emit_pip_energy(trie, spec.nvars, name + "_pip_e", out)
        emit_pip_mixed(trie, spec.nvars, name + "_pip_mixed", out)
        emit_dcoef(table, spec.nvars, name + "_dcoef", out)
    else:
        out.append("#define %s_STRAIGHT_LINE 0" % name.upper())
    emit_traits(spec, table, table.nterms <= STRAIGHT_LINE_MAX_TERMS, out)
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, name + ".cuh")
    text = "\n".join(out) + "\n"
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)
    return path, leaves, inner


KERNELS_CU = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// Kernel instantiations and launchers for the %(name)s evaluator.
#include "../holder_kernel.cuh"
#include "../launch.h"
#include "%(name)s.cuh"

__constant__ double c_%(name)s[%(ncoef)d];
struct %(name)s_CC {
    __device__ __forceinline__ double operator[](int k) const { return c_%(name)s[k]; }
};

int mbx_set_coef_%(name)s(const double* a, int from_device, cudaStream_t s) {
    return (int)cudaMemcpyToSymbolAsync(c_%(name)s, a, sizeof(double) * %(ncoef)d, 0,
                                        from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
}

int mbx_launch_%(name)s(const HolderArgs& A, int mode, int grid, int block, cudaStream_t s) {
%(body)s
    return (int)cudaGetLastError();
}

int mbx_launch_dcoef_%(name)s(const HolderArgs& A, const double* w, double* out, int grid, int block,
                              cudaStream_t s) {
%(dbody)s
    return (int)cudaGetLastError();
}
"""

STRAIGHT_BODY = """    if (A.n <= 0) return 0;
    switch (mode) {
        case HM_ENERGY: holder_kernel<%(name)s_T, %(name)s_CC, HM_ENERGY, false><<<grid, block, 0, s>>>(A); break;
        case HM_GRAD_FP64: holder_kernel<%(name)s_T, %(name)s_CC, HM_GRAD_FP64, false><<<grid, block, 0, s>>>(A); break;
        case HM_GRAD_MIXED: holder_kernel<%(name)s_T, %(name)s_CC, HM_GRAD_MIXED, false><<<grid, block, 0, s>>>(A); break;
        default: return (int)cudaErrorInvalidValue;
    }"""

WARP_BODY = """    if (A.n <= 0) return 0;
    if (mode != HM_ENERGY && mode != HM_GRAD_FP64 && mode != HM_GRAD_MIXED) return (int)cudaErrorInvalidValue;
    holder_warp_kernel<%(name)s_T, 4><<<grid, 128, 0, s>>>(A, mode != HM_ENERGY);"""

STRAIGHT_DBODY = """    if (A.n <= 0) return 0;
    holder_dcoef_kernel<%(name)s_T><<<grid, block, 0, s>>>(A, w, out);"""

WARP_DBODY = """    (void)A; (void)w; (void)out; (void)grid; (void)block; (void)s;
    return (int)cudaErrorNotSupported;"""


def write_kernels_cu(name):
    spec = SPECS[name]
    table = load_pip(name)
    straight = table.nterms <= STRAIGHT_LINE_MAX_TERMS
    d = {"name": name, "ncoef": spec.ncoef}
    d["body"] = (STRAIGHT_BODY if straight else WARP_BODY) % d
    d["dbody"] = (STRAIGHT_DBODY if straight else WARP_DBODY) % d
    text = KERNELS_CU % d
    path = os.path.join(OUT, name + "_kernels.cu")
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)
    return path


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=list(SPECS))
    args = ap.parse_args(argv)
    for n in args.names:
        path, leaves, inner = generate(n)
        write_kernels_cu(n)
        print("%s: %d leaves, %d inner -> %s" % (n, leaves, inner, path))


if __name__ == "__main__":
    main()
