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


# Code-shape options of the generated evaluators: how the trie is cut into
# separately compiled pieces ("top": whole top-level subtrees, "terms":
# contiguous term ranges) and into how many independent FMA chains the leaf sum
# of a node is split (1 = one serial chain per node).
SPLIT = "terms"
ACC_CHAINS = 1


def coef_expr(coefs, fp32=False):
    """Sum of coef[k]*c for the terms ending exactly at a node (FP32: the
    float copy of the coefficients, coef.f(k))."""
    parts = []
    for k, c in coefs:
        ref = ("coef.f(%d)" if fp32 else "coef[%d]") % k
        if c == 1.0:
            parts.append(ref)
        else:
            parts.append("(%s * %s)" % (ref, lit(c) + ("f" if fp32 else "")))
    return " + ".join(parts) if parts else None


def subtree_size(n):
    return 1 + sum(subtree_size(c) for c in n["kids"].values())


def partition(trie, nparts):
    """Top-level subtrees split into nparts groups of similar size (greedy)."""
    kids = sorted(trie.root["kids"].items(), key=lambda kv: -subtree_size(kv[1]))
    nparts = max(1, min(nparts, len(kids)))
    parts = [[] for _ in range(nparts)]
    load = [0] * nparts
    for var, ch in kids:
        i = load.index(min(load))
        parts[i].append((var, ch))
        load[i] += subtree_size(ch)
    return [p for p in parts if p]


def split_terms(trie, nparts):
    """The trie cut into nparts sub-tries of contiguous terms in depth-first
    order, each carrying the path nodes its terms hang from.  A path node's
    own coefficient goes with the range that holds it, so every term is in
    exactly one sub-trie; each sub-trie evaluates to its share of the
    polynomial (the trie value is linear in the terms)."""
    terms = []

    def walk(node, path):
        if node is not trie.root and node["coef"]:
            terms.append((path, node["coef"]))
        for v, ch in node["kids"].items():
            walk(ch, path + (v,))
    walk(trie.root, ())
    per = -(-len(terms) // max(1, nparts))
    roots = []
    for lo in range(0, len(terms), per):
        root = {"coef": [], "kids": collections.OrderedDict()}
        for path, coefs in terms[lo:lo + per]:
            node = root
            for v in path:
                node = node["kids"].setdefault(v, {"coef": [], "kids": collections.OrderedDict()})
            node["coef"].extend(coefs)
        roots.append(root)
    return [list(r["kids"].items()) for r in roots]


def lock_threads(nvars):
    """Threads of a lockstep evaluation block.  Up to 32 variables the
    variables and their gradient accumulators (4 registers per variable) fit
    under 168 registers, so a block of 384 threads (12 warps per SM) is
    resident; wider polynomials need the full 255 registers (256 threads)."""
    return 384 if nvars <= 32 else 256


def parts_for(nterms, nvars=36):
    """Number of separately compiled pieces of a trie.  A single straight-line
    function of 10^4-10^5 FMAs leaves the register allocator live ranges it
    cannot fit (kilobytes of spills), and the code of a piece should stay
    small enough for the instruction cache that the warps of a lockstep block
    share: ~400 terms per piece in 384-thread blocks, ~700 in 256-thread
    blocks (measured on the MB-pol 2b/3b tries)."""
    per = 400 if lock_threads(nvars) == 384 else 700
    return max(1, (nterms + per - 1) // per)


def emit_split(trie, nvars, name, out, nparts, arrays, body, ret="double"):
    """Emits name_partK as __noinline__ functions over pointers to the
    caller's arrays and a __forceinline__ name() that calls them in turn.

    arrays: [(name, ctype, role)] with role "in" (read: copied into a local
    register array on entry) or "acc" (accumulated: zeroed locally, added to
    the caller's array on exit).  body(w, subtrees) writes the evaluation of
    the subtrees into the local arrays and into E."""
    import re
    w = out.append
    pieces = split_terms(trie, nparts) if SPLIT == "terms" else partition(trie, nparts)
    for i, sub in enumerate(pieces):
        text = []
        body(text.append, sub)
        code = "\n".join(text)
        params = ", ".join("%s%s* __restrict__ %sm" % ("const " if role == "in" else "", ct, a)
                           for a, ct, role in arrays)
        w("template <class Coef>")
        w("__device__ __noinline__ %s %s_part%d(const Coef& coef, %s) {" % (ret, name, i, params))
        for a, ct, role in arrays:
            used = sorted({int(v) for v in re.findall(r"\b%s\[(\d+)\]" % a, code)})
            w("    %s %s[%d];" % (ct, a, nvars))
            for v in used:
                w("    %s[%d] = %s;" % (a, v, ("%sm[%d]" % (a, v)) if role == "in" else
                                        ("0.0f" if ct == "float" else "0.0")))
        w("    %s E = 0.0;" % ret)
        w(code)
        for a, ct, role in arrays:
            if role == "acc":
                used = sorted({int(v) for v in re.findall(r"\b%s\[(\d+)\]" % a, code)})
                for v in used:
                    w("    %sm[%d] += %s[%d];" % (a, v, a, v))
        w("    return E;")
        w("}")
    sig = ", ".join("%s%s (&%s)[%d]" % ("const " if role == "in" else "", ct, a, nvars) for a, ct, role in arrays)
    for lock in (False, True):
        # name(): the pieces in turn; name_lock(): the same with a block
        # barrier after every piece, so that all warps of a block run the same
        # piece at the same time and share its instruction fetches
        w("template <class Coef>")
        w("__device__ __forceinline__ %s %s%s(const Coef& coef, %s) {" % (ret, name, "_lock" if lock else "", sig))
        w("    %s E = 0.0;" % ret)
        for i in range(len(pieces)):
            w("    E += %s_part%d(coef, %s);%s" % (name, i, ", ".join(a for a, _, _ in arrays),
                                                 " __syncthreads();" if lock else ""))
        w("    return E;")
        w("}")


def emit_pip(trie, nvars, name, out, nparts=1):
    """FP64 value + gradient (multivariate Horner trie, reverse mode)."""
    out.append("// %s: polynomial and reverse-mode gradient (multivariate Horner trie)" % name)

    def body(w, subtrees):
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
            nleaf = sum(1 for ch in n["kids"].values() if not ch["kids"])
            split = ACC_CHAINS > 1 and nleaf >= 2 * ACC_CHAINS
            if split:
                # leaf sums in ACC_CHAINS independent chains, joined at the end
                for j in range(1, ACC_CHAINS):
                    w("      double %s_%d = 0.0;" % (V, j))
            li = 0
            for cv, ch in n["kids"].items():
                if ch["kids"]:
                    node(ch, cv, depth + 1, P)
                else:
                    c = coef_expr(ch["coef"])
                    acc = V if not split or li % ACC_CHAINS == 0 else "%s_%d" % (V, li % ACC_CHAINS)
                    li += 1
                    w("      %s = fma(%s, x[%d], %s); g[%d] = fma(%s, %s, g[%d]);" % (acc, c, cv, acc, cv, c, P, cv))
            if split:
                w("      %s += %s;" % (V, " + ".join("%s_%d" % (V, j) for j in range(1, ACC_CHAINS))))
            if pexpr is None:
                w("      g[%d] += %s; E = fma(x[%d], %s, E); }" % (var, V, var, V))
            else:
                w("      g[%d] = fma(%s, %s, g[%d]); V%d = fma(x[%d], %s, V%d); }" %
                  (var, pexpr, V, var, depth - 1, var, V, depth - 1))

        for var, ch in subtrees:
            if ch["kids"]:
                node(ch, var, 1, None)
            else:
                c = coef_expr(ch["coef"])
                w("    E = fma(%s, x[%d], E); g[%d] += %s;" % (c, var, var, c))

    emit_split(trie, nvars, name, out, nparts, [("x", "double", "in"), ("g", "double", "acc")], body)


def emit_pip_energy(trie, nvars, name, out, nparts=1):
    """FP64 value only: plain Horner over the trie."""
    def body(w, subtrees):
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

        for var, ch in subtrees:
            if ch["kids"]:
                node(ch, var, 1)
            else:
                w("    E = fma(%s, x[%d], E);" % (coef_expr(ch["coef"]), var))

    emit_split(trie, nvars, name, out, nparts, [("x", "double", "in")], body)


def emit_pip_mixed(trie, nvars, name, out, nparts=1):
    """Mixed precision: products and leaf-level sums in FP32, everything that
    accumulates across leaf groups (inner-node values, the energy) in FP64.

    Leaf gradient contributions go to FP32 accumulators gf[] (each receives one
    product per leaf); inner-node gradient contributions go to FP64 g[].  The
    caller adds gf into g at the end."""
    def body(w, subtrees):
        def node(n, var, depth, pexpr_f, pexpr_d):
            Pf = "Pf%d" % depth
            Pd = "Pd%d" % depth
            leaf_only = all(not ch["kids"] for ch in n["kids"].values())
            if pexpr_f is None:
                w("    { const float %s = xf[%d];" % (Pf, var))
                if not leaf_only:
                    w("      const double %s = x[%d];" % (Pd, var))
            else:
                w("    { const float %s = %s * xf[%d];" % (Pf, pexpr_f, var))
                if not leaf_only:
                    w("      const double %s = %s * x[%d];" % (Pd, pexpr_d, var))
            if leaf_only:
                V = "Vf%d" % depth
                ce = coef_expr(n["coef"], True)
                w("      float %s = %s;" % (V, ce if ce else "0.0f"))
                for cv, ch in n["kids"].items():
                    c = coef_expr(ch["coef"], True)
                    w("      %s = fmaf(%s, xf[%d], %s); gf[%d] = fmaf(%s, %s, gf[%d]);" %
                      (V, c, cv, V, cv, c, Pf, cv))
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
                        w("      %s = fma(%s, x[%d], %s); g[%d] = fma(%s, %s, g[%d]);" %
                          (V, c, cv, V, cv, c, Pd, cv))
                Vd = V
            if pexpr_f is None:
                w("      g[%d] += %s; E = fma(x[%d], %s, E); }" % (var, Vd, var, Vd))
            else:
                w("      g[%d] = fma(%s, %s, g[%d]); Vd%d = fma(x[%d], %s, Vd%d); }" %
                  (var, pexpr_d, Vd, var, depth - 1, var, Vd, depth - 1))

        for var, ch in subtrees:
            if ch["kids"]:
                node(ch, var, 1, None, None)
            else:
                c = coef_expr(ch["coef"])
                w("    E = fma(%s, x[%d], E); g[%d] += %s;" % (c, var, var, c))

    emit_split(trie, nvars, name, out, nparts,
               [("xf", "float", "in"), ("x", "double", "in"), ("g", "double", "acc"), ("gf", "float", "acc")], body)


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
    w("    static constexpr int LOCK_THREADS = %d;  // threads of a lockstep evaluation block" %
      lock_threads(spec.nvars))
    w("    __device__ __forceinline__ static void sites(const double (&r)[%d][3], double (&s)[%d][3]) { %s_sites(r, s); }" %
      (spec.nreal, ns, n))
    w("    __device__ __forceinline__ static void vars(const double (&s)[%d][3], double (&x)[%d]) { %s_vars(s, x); }" %
      (ns, spec.nvars, n))
    w("    __device__ __forceinline__ static void chain(const double (&s)[%d][3], const double (&g)[%d], double (&sg)[%d][3]) "
      "{ %s_chain(s, g, sg); }" % (ns, spec.nvars, ns, n))
    if straight:
        for lk in ("", "_lock"):
            w("    template <class C> __device__ __forceinline__ static double pip%s(const C& c, const double (&x)[%d], "
              "double (&g)[%d]) { return %s_pip%s(c, x, g); }" % (lk, spec.nvars, spec.nvars, n, lk))
            w("    template <class C> __device__ __forceinline__ static double pip_e%s(const C& c, const double (&x)[%d]) "
              "{ return %s_pip_e%s(c, x); }" % (lk, spec.nvars, n, lk))
            w("    template <class C> __device__ __forceinline__ static double pip_mixed%s(const C& c, "
              "const float (&xf)[%d], const double (&x)[%d], double (&g)[%d], float (&gf)[%d]) "
              "{ return %s_pip_mixed%s(c, xf, x, g, gf); }" % (lk, spec.nvars, spec.nvars, spec.nvars, spec.nvars, n, lk))
        w("    template <class S> __device__ __forceinline__ static void dcoef(const double (&x)[%d], S&& sink) "
          "{ %s_dcoef(x, sink); }" % (spec.nvars, n))
    w("};")


def write_if_changed(path, text):
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)


def generate(name):
    """Writes <name>.cuh (sizes, sites, variables, chain rule, traits) and one
    header per polynomial variant, so that a change to one variant rebuilds
    only the units that include it."""
    spec = SPECS[name]
    table = load_pip(name)
    trie = Trie(table)
    leaves, inner = trie.counts()
    straight = table.nterms <= STRAIGHT_LINE_MAX_TERMS
    head = ["// Generated by mbx_b200/codegen/gen_kernels.py from mbx_b200/specs.py and",
            "// mbx_b200/data/%s.pip.gz -- do not edit." % name]
    out = head + ["// %d terms: %d leaves, %d inner nodes" % (table.nterms, leaves, inner),
                  "#pragma once",
                  "#define %s_STRAIGHT_LINE %d" % (name.upper(), 1 if straight else 0)]
    emit_vars(spec, out)
    nv = spec.nvars
    if straight:
        for lk in ("", "_lock"):
            out += ["template <class Coef> __device__ __forceinline__ double %s_pip%s(const Coef&, const double (&)[%d], "
                    "double (&)[%d]);" % (name, lk, nv, nv),
                    "template <class Coef> __device__ __forceinline__ double %s_pip_e%s(const Coef&, "
                    "const double (&)[%d]);" % (name, lk, nv),
                    "template <class Coef> __device__ __forceinline__ double %s_pip_mixed%s(const Coef&, "
                    "const float (&)[%d], const double (&)[%d], double (&)[%d], float (&)[%d]);" %
                    (name, lk, nv, nv, nv, nv)]
        out += ["template <class Sink> __device__ __forceinline__ void %s_dcoef(const double (&)[%d], Sink&&);" %
                (name, nv)]
    emit_traits(spec, table, straight, out)
    os.makedirs(OUT, exist_ok=True)
    write_if_changed(os.path.join(OUT, name + ".cuh"), "\n".join(out) + "\n")
    if straight:
        nparts = parts_for(table.nterms, spec.nvars)
        for suffix, emitter, arg in (("pip", emit_pip, trie), ("pip_e", emit_pip_energy, trie),
                                     ("pip_mixed", emit_pip_mixed, trie), ("dcoef", emit_dcoef, table)):
            body = head + ["#pragma once", '#include "%s.cuh"' % name]
            if emitter is emit_dcoef:
                emitter(arg, nv, "%s_%s" % (name, suffix), body)
            else:
                emitter(arg, nv, "%s_%s" % (name, suffix), body, nparts)
            write_if_changed(os.path.join(OUT, "%s_%s.cuh" % (name, suffix)), "\n".join(body) + "\n")
    return os.path.join(OUT, name + ".cuh"), leaves, inner


TU_HEAD = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// %(what)s for the %(name)s evaluator.
#include <vector>
#include "../holder_kernel.cuh"
#include "%(name)s.cuh"
%(include)s
static __constant__ double c_%(name)s[%(ncoef)d];
static __constant__ float cf_%(name)s[%(ncoef)d];
struct %(name)s_CC {
    __device__ __forceinline__ double operator[](int k) const { return c_%(name)s[k]; }
    __device__ __forceinline__ float f(int k) const { return cf_%(name)s[k]; }
};

int mbx_set_coef_%(name)s_%(v)s(const double* a, int from_device, cudaStream_t s) {
    cudaError_t e = cudaMemcpyToSymbolAsync(c_%(name)s, a, sizeof(double) * %(ncoef)d, 0,
                                            from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return (int)e;
    // FP32 copy for the mixed-precision leaf sums (a warp-uniform FFMA operand)
    std::vector<double> h(%(ncoef)d);
    if (from_device) {
        e = cudaMemcpyAsync(h.data(), a, sizeof(double) * %(ncoef)d, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return (int)e;
    } else {
        for (int k = 0; k < %(ncoef)d; ++k) h[k] = a[k];
    }
    static thread_local std::vector<float> f;
    f.resize(%(ncoef)d);
    for (int k = 0; k < %(ncoef)d; ++k) f[k] = (float)h[k];
    e = cudaMemcpyToSymbolAsync(cf_%(name)s, f.data(), sizeof(float) * %(ncoef)d, 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return (int)e;
}
"""

VARIANTS = {
    # variant: (description, body)
    "g": ("FP64 energy + gradient kernel", """
int mbx_launch_%(name)s_g(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // persistent grid of lockstep blocks: every resident block slot once
    // (blocks claim chunks of LOCK_THREADS n-mers dynamically)
    auto kern = holder_lock_kernel<%(name)s_T, %(name)s_CC, HM_GRAD_FP64, false>;
    block = %(name)s_T::LOCK_THREADS;
    static int bps = 0, sms = 0, bps_block = 0;
    if (!bps || bps_block != block) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, block, 0);
        if (bps < 1) bps = 1;
        bps_block = block;
    }
    const long need = (A.n + block - 1) / block;
    grid = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    if (grid < 1) grid = 1;
    kern<<<grid, block, 0, s>>>(A);
    return (int)cudaGetLastError();
}
"""),
    "e": ("FP64 energy-only kernel", """
int mbx_launch_%(name)s_e(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // persistent grid of lockstep blocks: every resident block slot once
    // (blocks claim chunks of LOCK_THREADS n-mers dynamically)
    auto kern = holder_lock_kernel<%(name)s_T, %(name)s_CC, HM_ENERGY, false>;
    block = %(name)s_T::LOCK_THREADS;
    static int bps = 0, sms = 0, bps_block = 0;
    if (!bps || bps_block != block) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, block, 0);
        if (bps < 1) bps = 1;
        bps_block = block;
    }
    const long need = (A.n + block - 1) / block;
    grid = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    if (grid < 1) grid = 1;
    kern<<<grid, block, 0, s>>>(A);
    return (int)cudaGetLastError();
}
"""),
    "m": ("mixed-precision energy + gradient kernel", """
int mbx_launch_%(name)s_m(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // persistent grid of lockstep blocks: every resident block slot once
    // (blocks claim chunks of LOCK_THREADS n-mers dynamically)
    auto kern = holder_lock_kernel<%(name)s_T, %(name)s_CC, HM_GRAD_MIXED, false>;
    block = %(name)s_T::LOCK_THREADS;
    static int bps = 0, sms = 0, bps_block = 0;
    if (!bps || bps_block != block) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, block, 0);
        if (bps < 1) bps = 1;
        bps_block = block;
    }
    const long need = (A.n + block - 1) / block;
    grid = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    if (grid < 1) grid = 1;
    kern<<<grid, block, 0, s>>>(A);
    return (int)cudaGetLastError();
}
"""),
    "c": ("coefficient-gradient (adjoint) kernel", """
int mbx_launch_%(name)s_c(const HolderArgs& A, const double* w, double* out, int grid, int block, cudaStream_t s) {
    holder_dcoef_kernel<%(name)s_T><<<grid, block, 0, s>>>(A, w, out);
    return (int)cudaGetLastError();
}
"""),
    "p": ("generated-polynomial (SoA) kernel", """
int mbx_launch_%(name)s_p(long nd, const double* x, double* g, double* e, int grid, int block, cudaStream_t s) {
    poly_soa_kernel<%(name)s_T, %(name)s_CC><<<grid, block, 0, s>>>(nd, x, g, e);
    return (int)cudaGetLastError();
}
"""),
    "w": ("table-driven warp kernel (energy, gradient)", """
int mbx_launch_%(name)s_w(const HolderArgs& A, int grads, int grid, cudaStream_t s) {
    holder_warp_kernel<%(name)s_T, 4><<<grid, 128, 0, s>>>(A, grads);
    return (int)cudaGetLastError();
}
"""),
}


def variants_of(name):
    return "gemcp" if load_pip(name).nterms <= STRAIGHT_LINE_MAX_TERMS else "w"


def write_tu(path, text):
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)


def write_kernels_cu(name):
    spec = SPECS[name]
    paths = []
    inc = {"g": "pip", "e": "pip_e", "m": "pip_mixed", "c": "dcoef", "p": "pip", "w": None}
    for v in variants_of(name):
        what, body = VARIANTS[v]
        d = {"name": name, "ncoef": spec.ncoef, "v": v, "what": what,
             "include": ('#include "%s_%s.cuh"\n' % (name, inc[v])) if inc[v] else ""}
        path = os.path.join(OUT, "%s_%s.cu" % (name, v))
        write_tu(path, (TU_HEAD + body) % d)
        paths.append(path)
    return paths


def write_registry():
    """Host tables: evaluator descriptions, default coefficients, term tables."""
    from mbx_b200.tables import load_fit
    lines = ["// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.", "#pragma once",
             '#include "../holder_kernel.cuh"', ""]
    for name in SPECS:
        vs = variants_of(name)
        for v in "gemcpw":
            if v not in vs:
                continue
            if v in "gem":
                lines.append("int mbx_launch_%s_%s(const HolderArgs& A, int grid, int block, cudaStream_t s);" %
                             (name, v))
            elif v == "c":
                lines.append("int mbx_launch_%s_c(const HolderArgs& A, const double* w, double* out, int grid, "
                             "int block, cudaStream_t s);" % name)
            elif v == "p":
                lines.append("int mbx_launch_%s_p(long nd, const double* x, double* g, double* e, int grid, "
                             "int block, cudaStream_t s);" % name)
            else:
                lines.append("int mbx_launch_%s_w(const HolderArgs& A, int grads, int grid, cudaStream_t s);" % name)
            lines.append("int mbx_set_coef_%s_%s(const double* a, int from_device, cudaStream_t s);" % (name, v))
        fit = load_fit(name)
        lines.append("static const double mbx_fit_%s[%d] = {" % (name, len(fit)))
        for i in range(0, len(fit), 4):
            lines.append("    " + ", ".join(repr(float(x)) for x in fit[i:i + 4]) + ",")
        lines.append("};")
    lines.append("")
    lines.append("static const EvaluatorInfo mbx_evaluators[] = {")
    for name, spec in SPECS.items():
        vs = variants_of(name)
        ids = list(spec.monomers) + ["", ""][:3 - len(spec.monomers)]
        skip = {"pair_gt": 0, "two_of_three_gt": 1, "all_three_gt": 2}[spec.skip]

        def fn(v, kind):
            return ("mbx_%s_%s_%s" % (kind, name, v)) if v in vs else "nullptr"
        lines.append('    {"%s", %d, {"%s", "%s", "%s"}, %s, %d, %d, %d, %d, mbx_fit_%s, %s, %s, %s, %s, %s, %s,' %
                     (name, spec.nbody, ids[0], ids[1], ids[2], lit(spec.rf), skip, spec.ncoef, spec.nreal,
                      spec.nvars, name, fn("g", "launch"), fn("e", "launch"), fn("m", "launch"), fn("c", "launch"),
                      fn("p", "launch"), fn("w", "launch")))
        lines.append("     {%s}}," % ", ".join(fn(v, "set_coef") for v in "gemcpw"))
    lines.append("};")
    lines.append("static const int mbx_num_evaluators = %d;" % len(SPECS))
    write_tu(os.path.join(OUT, "registry.inc"), "\n".join(lines) + "\n")


def write_term_tables():
    """Packed term tables for the warp kernel (types without straight-line code)."""
    lines = ["// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.", "#pragma once", ""]
    for name in SPECS:
        if "w" not in variants_of(name):
            continue
        t = load_pip(name)
        lines.append("static const int mbx_terms_%s[%d][4] = {" % (name, t.nterms))
        for q in range(t.nterms):
            packed = 0
            for i in range(4):
                v = int(t.var[q, i]) if i < t.deg[q] else 255
                packed |= (v & 255) << (8 * i)
            if packed >= 1 << 31:
                packed -= 1 << 32
            lines.append("{%d,%d,%d,0}," % (t.k[q], packed, t.deg[q]))
        lines.append("};")
        lines.append("static const double mbx_tcoef_%s[%d] = {%s};" %
                     (name, t.nterms, ",".join(repr(float(c)) for c in t.coef)))
    write_tu(os.path.join(OUT, "terms.inc"), "\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=list(SPECS))
    args = ap.parse_args(argv)
    os.makedirs(OUT, exist_ok=True)
    write_registry()
    write_term_tables()
    for n in args.names:
        path, leaves, inner = generate(n)
        write_kernels_cu(n)
        print("%s: %d leaves, %d inner -> %s" % (n, leaves, inner, path))


if __name__ == "__main__":
    main()
