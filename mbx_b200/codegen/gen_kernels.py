#!/usr/bin/env python3
"""Generate the per-evaluator CUDA device code from the declarative specs.

For each evaluator in ``mbx_b200.specs.SPECS`` this writes
``mbx_b200/csrc/gen/<name>.cuh`` holding:

* ``<name>_vars``: the polynomial variables (straight-line FP64: differences,
  sqrt, exp) and the factor that turns dP/dv into a Cartesian gradient;
* ``<name>_pip``: the polynomial and its reverse-mode gradient, as a
  multivariate Horner trie over the expanded term table;
* ``<name>_pip_e``: the energy-only Horner evaluation;
* ``<name>_pip_s32`` (types in SHIFT_TYPES): the FP32 trie of the type's FP32
  basis (codegen/shift.py), the mixed-precision polynomial.

The tries are generated for STRAIGHT_TYPES only; every evaluator also gets a
table unit ``<name>_t.cu`` (coefficient adjoint and, without a trie, the
evaluation itself) over the term tables that ``write_term_tables`` packs into
one binary embedded in the library.

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

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
sys.path.insert(0, os.path.dirname(PKG))

from mbx_b200.specs import SPECS, ONEBODY_SPECS, LP_GAMMA_IN, LP_GAMMA_OUT  # noqa: E402
from mbx_b200.tables import load_pip  # noqa: E402

OUT = os.path.join(PKG, "csrc", "gen")



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
# of a node is split (1 = one serial chain per node; 2 chains measured slower
# on the MB-pol 3b gradient kernel with the code prefetched: 1.38 vs 1.32 ms
# back to back, 2048-water trimers).
SPLIT = "terms"
ACC_CHAINS = 1

# Mixed precision (paired FP32 trie, the "s" kernels).  "median": the
# polynomial is re-expanded around a symmetric reference point in the middle
# of liquid data (codegen/shift.py); "identity": the original basis in FP32.
# Types not listed run FP64 in the mixed mode.  MB-pol 2b is not listed: in
# FP32 (identity basis, FP32 coefficients and leaf sums) its energy over the
# 2048-water box is off by 1.1e-5 even with the dimers below 4.5 A in FP64
# (the shifted basis does not condition it either).
SHIFT_TYPES = {"mbpol3b": "median"}
# Types of SHIFT_TYPES whose mixed kernel is the quadratic form on the tensor
# cores (codegen/qf.py, csrc/qf_kernel.cuh) instead of the paired FP32 trie:
# MB-pol 3b, 442 products of degree 2 in the basis (data/mbpol3b.qf.json).
QF_TYPES = {"mbpol3b"}
# Optional: n-mers whose first-atom distance is below this radius (A) run the
# FP64 kernel in the mixed mode (a type of SHIFT_TYPES whose short-range
# n-mers cancel too strongly for FP32); the builder puts them in a bucket of
# their own.
MIXED_FP64_RADIUS = {}


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
    if nvars > 56:
        # x and g columns of 256 threads would exceed the 227 KB of shared memory
        return 128
    return 384 if nvars <= 32 else 256


def parts_for(nterms, nvars=36):
    """Number of separately compiled pieces of a trie.  A single straight-line
    function of 10^4-10^5 FMAs leaves the register allocator live ranges it
    cannot fit (kilobytes of spills), and the code of a piece should stay
    small enough for the instruction cache that the warps of a lockstep block
    share: ~400 terms per piece in 384-thread blocks, ~600 in 256-thread
    blocks with shared-memory x/g columns (MB-pol 3b gradient kernel on the
    2048-water trimers: 1.42/1.39/1.35/1.32/1.47 ms at 300/375/450/600/700
    terms per piece, and 2.1 ms at 800-900, past the instruction cache)."""
    per = 400 if lock_threads(nvars) == 384 else 600
    if nvars > 56:
        # a piece loads every variable it uses into registers: fewer terms per
        # piece for the widest polynomials
        per = 200
    return max(1, (nterms + per - 1) // per)


# FP64 kernels whose coefficients are copied to shared memory per block (the
# trie reads them from there instead of the constant bank): measured on the
# 2048-water trimers, MB-pol 3b 1.37 ms (shared, 450-term pieces) vs 1.58 ms
# (constant); MB-pol 2b is faster from the constant bank (0.18 vs 0.25 ms).
SMEM_COEF_TYPES = {"mbpol3b"}

# Types whose tries are generated in the coset form (codegen/coset.py): a
# polynomial R of ~1/24 of the terms, run once per permutation of a
# transversal of the symmetry group, so that its code stays in the
# instruction cache; the kernels' coefficients are scaled on the host.
# COSET_PIECE_TERMS: terms of R per separately compiled piece.
# Measured on the 2048-water trimers (L2 flushed between calls, the code
# prefetch launch in use): MB-pol 3b FP64 1.73 ms in the coset form against
# 1.36 ms for the full trie, paired FP32 0.96 against 0.91 ms -- with the
# prefetch the full trie's code is L2-resident already, and the coset form's
# 10% more arithmetic and per-permutation loads then cost more than its
# smaller code saves.  No type uses it; the form is kept for polynomials
# whose trie does not fit in L2.
COSET_TYPES = set()
COSET_PIECE_TERMS = 400


_COSET = {}


def coset_of(name, shifted_basis=False):
    """(coset form, R table) of an evaluator's polynomial, or of its FP32
    (shifted) basis."""
    key = (name, shifted_basis)
    if key not in _COSET:
        from mbx_b200.codegen.coset import coset_form, CosetTable
        spec = SPECS[name]
        if shifted_basis:
            from mbx_b200.codegen.shift import ShiftedTable
            sp = shifted_pip(name)
            cf = coset_form(spec, ShiftedTable(sp, name), sp.group)
        else:
            cf = coset_form(spec, load_pip(name))
        _COSET[key] = (cf, CosetTable(cf, spec.nvars, name))
    return _COSET[key]


def emit_split(trie, nvars, name, out, nparts, arrays, body, ret="double", perms=None):
    """Emits name_partK as __noinline__ functions over strided pointers to the
    caller's arrays, and the wrappers that call them in turn.

    arrays: [(name, ctype, role)] with role "in" (read: copied into a local
    register array on entry) or "acc" (accumulated: zeroed locally, added to
    the caller's array on exit).  A piece reads element v of an array at
    pointer[v * S], S a template parameter: S = 1 for a thread's own local
    array, S = block size for a shared-memory array laid out [v][thread] (the
    lockstep kernels keep x and g there: shared memory instead of the
    thread's stack for the values every piece loads and stores).  body(w,
    subtrees) writes the evaluation of the subtrees into the local arrays and
    into E.

    perms (coset form, codegen/coset.py): the trie is R and every piece runs
    its subtrees once per permutation p_t, reading variable v of the caller's
    arrays at column p_t[v] and adding its gradient there; the permutations
    sit in a constant-memory table, and a piece's code is reused |T| times in
    a row while it is in the instruction cache."""
    import re
    w = out.append
    zero = {"float": "0.0f", "double": "0.0", "f2_t": "0ull"}
    e0 = "make_double2(0.0, 0.0)" if ret == "double2" else "0.0"
    pieces = split_terms(trie, nparts) if SPLIT == "terms" else partition(trie, nparts)
    params = ", ".join("%s%s* __restrict__ %sm" % ("const " if role == "in" else "", ct, a) for a, ct, role in arrays)
    if perms is not None:
        # the table lives in constant memory and is copied to shared memory
        # by the lock / piece entry points; the pieces read it with a
        # non-removable load at every use, so that the 36 column offsets are
        # not kept in registers across the piece (they would spill)
        w("// coset form: %d permutations of the %d variables (x_local[v] = x[perm[t][v]])" % (len(perms), nvars))
        w("static __constant__ int %s_perm[%d] = {%s};" %
          (name, len(perms) * nvars, ", ".join(str(v) for p in perms for v in p)))
        w("static __shared__ int %s_sperm[%d];" % (name, len(perms) * nvars))
        w("__device__ __forceinline__ void %s_load_perm() {" % name)
        w("    for (int i = threadIdx.x; i < %d; i += blockDim.x) %s_sperm[i] = %s_perm[i];" %
          (len(perms) * nvars, name, name))
        w("    __syncthreads();")
        w("}")
    for i, sub in enumerate(pieces):
        text = []
        body(text.append, sub)
        code = "\n".join(text)
        w("template <class Coef, int S>")
        w("__device__ __noinline__ %s %s_part%d(const Coef& coef, %s) {" % (ret, name, i, params))
        w("    %s E = %s;" % (ret, e0))
        pad = "    "
        if perms is not None:
            w("#pragma unroll 1")
            w("    for (int t = 0; t < %d; ++t) {" % len(perms))
            w("    const int* o = %s_sperm + t * %d;" % (name, nvars))
        for a, ct, role in arrays:
            used = sorted({int(v) for v in re.findall(r"\b%s\[(\d+)\]" % a, code)})
            w("    %s %s[%d];" % (ct, a, nvars))
            for v in used:
                col = ("lds_pinned(o + %d)" % v) if perms is not None else str(v)
                w("    %s[%d] = %s;" % (a, v, ("%sm[%s * S]" % (a, col)) if role == "in" else zero[ct]))
        w(code)
        for a, ct, role in arrays:
            if role == "acc":
                used = sorted({int(v) for v in re.findall(r"\b%s\[(\d+)\]" % a, code)})
                for v in used:
                    col = ("lds_pinned(o + %d)" % v) if perms is not None else str(v)
                    if ct == "f2_t":
                        w("    %sm[%s * S] = f2_add(%sm[%s * S], %s[%d]);" % (a, col, a, col, a, v))
                    else:
                        w("    %sm[%s * S] += %s[%d];" % (a, col, a, v))
        if perms is not None:
            w("    }")
        w("    return E;")
        w("}")

    def calls(lock, targs, args):
        for i in range(len(pieces)):
            call = "%s_part%d<%s>(coef, %s)" % (name, i, targs, args)
            bar = " __syncthreads();" if lock else ""
            if ret == "double2":
                w("    { const double2 e = %s; E.x += e.x; E.y += e.y; }%s" % (call, bar))
            else:
                w("    E += %s;%s" % (call, bar))

    # name(coef, x[], g[]): the pieces in turn over the thread's own arrays
    sig = ", ".join("%s%s (&%s)[%d]" % ("const " if role == "in" else "", ct, a, nvars) for a, ct, role in arrays)
    w("template <class Coef>")
    w("__device__ __forceinline__ %s %s(const Coef& coef, %s) {" % (ret, name, sig))
    w("    %s E = %s;" % (ret, e0))
    calls(False, "Coef, 1", ", ".join(a for a, _, _ in arrays))
    w("    return E;")
    w("}")
    # name_lock<S>(coef, xm, gm): over shared arrays [v][S] (pointers at the
    # thread's column), a block barrier after every piece so that all warps
    # of a block run the same piece at the same time and share its
    # instruction fetches
    w("template <int S, class Coef>")
    w("__device__ __forceinline__ %s %s_lock(const Coef& coef, %s) {" % (ret, name, params))
    if perms is not None:
        w("    %s_load_perm();" % name)
    w("    %s E = %s;" % (ret, e0))
    calls(True, "Coef, S", ", ".join("%sm" % a for a, _, _ in arrays))
    w("    return E;")
    w("}")
    # name_piece<S>(k, coef, xm, gm): piece k alone, the same instantiation
    # as name_lock<S> calls (holder_prime_kernel runs one piece per block to
    # bring the code of all pieces into L2 in parallel)
    w("static constexpr int %s_NPIECES = %d;" % (name, len(pieces)))
    w("template <int S, class Coef>")
    w("__device__ __forceinline__ %s %s_piece(int k, const Coef& coef, %s) {" % (ret, name, params))
    if perms is not None:
        w("    %s_load_perm();" % name)
    w("    switch (k) {")
    args = ", ".join("%sm" % a for a, _, _ in arrays)
    for i in range(len(pieces)):
        w("    case %d: return %s_part%d<Coef, S>(coef, %s);" % (i, name, i, args))
    w("    default: return %s;" % e0)
    w("    }")
    w("}")


def emit_pip(trie, nvars, name, out, nparts=1, perms=None):
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

    emit_split(trie, nvars, name, out, nparts, [("x", "double", "in"), ("g", "double", "acc")], body, perms=perms)


def emit_pip_f32x2(trie, nvars, name, out, nparts=1, perms=None):
    """FP32 value + gradient over the trie for two n-mers at once (the low and
    high halves of every f2_t, paired FP32 instructions): monomials,
    coefficients and leaf sums in FP32; the top-level products are added to
    the two energies in FP64."""
    out.append("// %s: paired FP32 polynomial and reverse-mode gradient (multivariate Horner trie)" % name)

    def cexpr(coefs):
        if not coefs:
            return None
        assert all(c == 1.0 for _, c in coefs)
        parts = ["coef.f2(%d)" % k for k, _ in coefs]
        e = parts[0]
        for p in parts[1:]:
            e = "f2_add(%s, %s)" % (e, p)
        return e

    def body(w, subtrees):
        def node(n, var, depth, pexpr):
            P = "P%d" % depth
            V = "V%d" % depth
            if pexpr is None:
                w("    { const f2_t %s = x[%d];" % (P, var))
            else:
                w("    { const f2_t %s = f2_mul(%s, x[%d]);" % (P, pexpr, var))
            ce = cexpr(n["coef"])
            w("      f2_t %s = %s;" % (V, ce if ce else "0ull"))
            for cv, ch in n["kids"].items():
                if ch["kids"]:
                    node(ch, cv, depth + 1, P)
                else:
                    c = cexpr(ch["coef"])
                    w("      { const f2_t c = %s; %s = f2_fma(c, x[%d], %s); g[%d] = f2_fma(c, %s, g[%d]); }" %
                      (c, V, cv, V, cv, P, cv))
            if pexpr is None:
                w("      g[%d] = f2_add(g[%d], %s);" % (var, var, V))
                w("      E.x = fma((double)f2_lo(x[%d]), (double)f2_lo(%s), E.x); "
                  "E.y = fma((double)f2_hi(x[%d]), (double)f2_hi(%s), E.y); }" % (var, V, var, V))
            else:
                w("      g[%d] = f2_fma(%s, %s, g[%d]); V%d = f2_fma(x[%d], %s, V%d); }" %
                  (var, pexpr, V, var, depth - 1, var, V, depth - 1))

        for var, ch in subtrees:
            if ch["kids"]:
                node(ch, var, 1, None)
            else:
                c = cexpr(ch["coef"])
                w("    { const f2_t c = %s; g[%d] = f2_add(g[%d], c);" % (c, var, var))
                w("      E.x = fma((double)f2_lo(c), (double)f2_lo(x[%d]), E.x); "
                  "E.y = fma((double)f2_hi(c), (double)f2_hi(x[%d]), E.y); }" % (var, var))

    emit_split(trie, nvars, name, out, nparts, [("x", "f2_t", "in"), ("g", "f2_t", "acc")], body, ret="double2",
               perms=perms)


def shifted_pip(name):
    """codegen.shift.ShiftedPip of a type in SHIFT_TYPES (cached)."""
    from mbx_b200.codegen import shift
    if name in _SHIFTED:
        return _SHIFTED[name]
    spec, table = SPECS[name], load_pip(name)
    if SHIFT_TYPES[name] == "median":
        sp = shift.shifted(spec, table)
    else:
        monos = [tuple(sorted(table.var[t, :table.deg[t]].tolist())) for t in range(table.nterms)]
        sp = shift.ShiftedPip(spec.nvars, spec.ncoef, np.zeros(spec.nvars), monos,
                              [int(k) for k in table.k], {}, [{k: 1.0} for k in range(spec.ncoef)], [])
        # the identity basis keeps the term multiplicities of the table
        assert all(c == 1.0 for c in table.coef)
    _SHIFTED[name] = sp
    return sp


_SHIFTED = {}


def emit_pip_energy(trie, nvars, name, out, nparts=1, perms=None):
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

    emit_split(trie, nvars, name, out, nparts, [("x", "double", "in")], body, perms=perms)


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
    # the variables with their radial factors, for a chain rule in another
    # kernel that reads the factors back (NAME_chain_q); q.put(v, factor)
    # stores each as soon as it is known
    w("template <class QW>")
    w("__device__ __forceinline__ void %s_vars_q(const double (&s)[%d][3], double (&x)[%d], QW& q) {" %
      (spec.name, ns, nv))
    for v, (kind, a, b, k, d0) in enumerate(spec.variables):
        fn = "var_exp_q" if kind == "exp" else "var_coul_q"
        w("    { double f; x[%d] = %s(s[%d], s[%d], %s, %s, f); q.put(%d, f); }" % (v, fn, a, b, lit(k), lit(d0), v))
    w("}")
    w("template <class G, class Q>")
    w("__device__ __forceinline__ void %s_chain_q(const double (&s)[%d][3], const G& g, const Q& q, "
      "double (&sg)[%d][3]) {" % (spec.name, ns, ns))
    w("#pragma unroll")
    w("    for (int i = 0; i < %d; ++i) { sg[i][0] = 0.0; sg[i][1] = 0.0; sg[i][2] = 0.0; }" % ns)
    for v, (kind, a, b, k, d0) in enumerate(spec.variables):
        w("    dvar_q(s[%d], s[%d], g[%d], q[%d], sg[%d], sg[%d]);" % (a, b, v, v, a, b))
    for (m, o, xp, xm) in spec.lp:
        w("    lp_grads(s[%d], s[%d], s[%d], sg[%d], sg[%d], sg[%d], sg[%d], sg[%d]);" %
          (o, o + 1, o + 2, xp, xm, o, o + 1, o + 2))
    w("}")
    # chain rule: site gradients from dP/dv (g, an array of NVARS doubles or
    # anything indexable the same way, e.g. a reader of the FP32 gradients in
    # global memory that loads each where it is used), scaled by sw
    w("template <class G>")
    w("__device__ __forceinline__ void %s_chain(const double (&s)[%d][3], const G& g, "
      "double (&sg)[%d][3]) {" % (spec.name, ns, ns))
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
      ({"pair": 0, "triple": 1, "triple2": 2, "cos2": 3, "none": 0}[spec.switch],
       {"pair_gt": 0, "two_of_three_gt": 1, "all_three_gt": 2, "none": 0}[spec.skip],
       1 if straight else 0, spec.degree))
    w("    static constexpr int TPAIRS = %d;  // (variable, exponent) pairs of a term, at most" %
      term_pairs_max(table))
    w("    static constexpr double RI = %s, RF = %s;" % (lit(spec.ri), lit(spec.rf)))
    w("    static constexpr int VIRIAL_RAW = %d;  // virial of the unswitched polynomial gradient" %
      (1 if spec.virial == "raw" else 0))
    w("    static constexpr int LOCK_THREADS = %d;  // threads of a lockstep evaluation block" %
      lock_threads(spec.nvars))
    shifted_type = straight and n in SHIFT_TYPES
    w("    static constexpr int SHIFTED = %d, LOCK_THREADS_S = %d;  // paired FP32 (shifted-basis) kernel" %
      (1 if shifted_type else 0, 256 if shifted_type else lock_threads(spec.nvars)))
    w("    static constexpr int NORB = %d;  // coefficients of the FP32 basis" %
      (shifted_pip(n).norb if shifted_type else 1))
    w("    static constexpr int SMEM_COEF = %d;  // FP64 kernel reads its coefficients from shared memory" %
      (1 if n in SMEM_COEF_TYPES else 0))

    if shifted_type:
        w("    __device__ __forceinline__ static void shift(const double (&x)[%d], float (&xf)[%d]) "
          "{ %s_shift(x, xf); }" % (spec.nvars, spec.nvars, n))
    if shifted_type and n not in QF_TYPES:
        w("    template <int S, class C> __device__ __forceinline__ static double2 pip_s32_lock(const C& c, "
          "const f2_t* __restrict__ x, f2_t* __restrict__ g) { return %s_pip_s32_lock<S>(c, x, g); }" % n)
        w("    template <int S, class C> __device__ __forceinline__ static double2 pip_s32_piece(int k, const C& c, "
          "const f2_t* __restrict__ x, f2_t* __restrict__ g) { return %s_pip_s32_piece<S>(k, c, x, g); }" % n)
    w("    __device__ __forceinline__ static void sites(const double (&r)[%d][3], double (&s)[%d][3]) { %s_sites(r, s); }" %
      (spec.nreal, ns, n))
    w("    __device__ __forceinline__ static void vars(const double (&s)[%d][3], double (&x)[%d]) { %s_vars(s, x); }" %
      (ns, spec.nvars, n))
    w("    template <class G> __device__ __forceinline__ static void chain(const double (&s)[%d][3], const G& g, "
      "double (&sg)[%d][3]) { %s_chain(s, g, sg); }" % (ns, ns, n))
    w("    template <class QW> __device__ __forceinline__ static void vars_q(const double (&s)[%d][3], "
      "double (&x)[%d], QW& q) { %s_vars_q(s, x, q); }" % (ns, spec.nvars, n))
    w("    template <class G, class Q> __device__ __forceinline__ static void chain_q(const double (&s)[%d][3], "
      "const G& g, const Q& q, double (&sg)[%d][3]) { %s_chain_q(s, g, q, sg); }" % (ns, ns, n))
    if straight:
        w("    template <class C> __device__ __forceinline__ static double pip(const C& c, const double (&x)[%d], "
          "double (&g)[%d]) { return %s_pip(c, x, g); }" % (spec.nvars, spec.nvars, n))
        w("    template <class C> __device__ __forceinline__ static double pip_e(const C& c, const double (&x)[%d]) "
          "{ return %s_pip_e(c, x); }" % (spec.nvars, n))
        w("    template <int S, class C> __device__ __forceinline__ static double pip_lock(const C& c, "
          "const double* __restrict__ x, double* __restrict__ g) { return %s_pip_lock<S>(c, x, g); }" % n)
        w("    template <int S, class C> __device__ __forceinline__ static double pip_e_lock(const C& c, "
          "const double* __restrict__ x) { return %s_pip_e_lock<S>(c, x); }" % n)
        w("    template <int S, class C> __device__ __forceinline__ static double pip_piece(int k, const C& c, "
          "const double* __restrict__ x, double* __restrict__ g) { return %s_pip_piece<S>(k, c, x, g); }" % n)
        w("    template <int S, class C> __device__ __forceinline__ static double pip_e_piece(int k, const C& c, "
          "const double* __restrict__ x) { return %s_pip_e_piece<S>(k, c, x); }" % n)

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
    spec = SPECS[name] if name in SPECS else ONEBODY_SPECS[name]
    table = load_pip(name)
    straight = name in STRAIGHT_TYPES
    trie = Trie(table) if straight else None
    leaves, inner = trie.counts() if straight else (table.nterms, 0)
    head = ["// Generated by mbx_b200/codegen/gen_kernels.py from mbx_b200/specs.py and",
            "// mbx_b200/data/%s.pip.gz -- do not edit." % name]
    out = head + ["// %d terms: %d leaves, %d inner nodes" % (table.nterms, leaves, inner),
                  "#pragma once",
                  "#define %s_STRAIGHT_LINE %d" % (name.upper(), 1 if straight else 0)]
    emit_vars(spec, out)
    nv = spec.nvars
    if straight:
        out += ["template <class Coef> __device__ __forceinline__ double %s_pip(const Coef&, const double (&)[%d], "
                "double (&)[%d]);" % (name, nv, nv),
                "template <class Coef> __device__ __forceinline__ double %s_pip_e(const Coef&, "
                "const double (&)[%d]);" % (name, nv),
                "template <int S, class Coef> __device__ __forceinline__ double %s_pip_lock(const Coef&, "
                "const double* __restrict__, double* __restrict__);" % name,
                "template <int S, class Coef> __device__ __forceinline__ double %s_pip_e_lock(const Coef&, "
                "const double* __restrict__);" % name,
                "template <int S, class Coef> __device__ __forceinline__ double %s_pip_piece(int, const Coef&, "
                "const double* __restrict__, double* __restrict__);" % name,
                "template <int S, class Coef> __device__ __forceinline__ double %s_pip_e_piece(int, const Coef&, "
                "const double* __restrict__);" % name]
        if name in SHIFT_TYPES:
            sp = shifted_pip(name)
            if name not in QF_TYPES:
                out.append("template <int S, class Coef> __device__ __forceinline__ double2 %s_pip_s32_lock("
                           "const Coef&, const f2_t* __restrict__, f2_t* __restrict__);" % name)
                out.append("template <int S, class Coef> __device__ __forceinline__ double2 %s_pip_s32_piece(int, "
                           "const Coef&, const f2_t* __restrict__, f2_t* __restrict__);" % name)
            out.append("// dx = x - x0, the reference point of the FP32 basis (%s)" % SHIFT_TYPES[name])
            out.append("__device__ __forceinline__ void %s_shift(const double (&x)[%d], float (&xf)[%d]) {" %
                       (name, nv, nv))
            for v in range(nv):
                if sp.x0[v] == 0.0:
                    out.append("    xf[%d] = (float)x[%d];" % (v, v))
                else:
                    out.append("    xf[%d] = (float)(x[%d] - %s);" % (v, v, lit(float(sp.x0[v]))))
            out.append("}")
    emit_traits(spec, table, straight, out)
    os.makedirs(OUT, exist_ok=True)
    write_if_changed(os.path.join(OUT, name + ".cuh"), "\n".join(out) + "\n")
    if straight:
        nparts = parts_for(table.nterms, spec.nvars)
        perms = None
        if name in COSET_TYPES:
            cf, ctab = coset_of(name)
            trie = Trie(ctab)
            perms = cf.perms
            nparts = max(1, (ctab.nterms + COSET_PIECE_TERMS - 1) // COSET_PIECE_TERMS)
        for suffix, emitter, arg in (("pip", emit_pip, trie), ("pip_e", emit_pip_energy, trie)):
            body = head + ["#pragma once", '#include "%s.cuh"' % name]
            if perms is not None:
                body.append("// coset form: %d terms of R x %d permutations (%d terms in the table)" %
                            (ctab.nterms, len(perms), table.nterms))
            emitter(arg, nv, "%s_%s" % (name, suffix), body, nparts, perms=perms)
            write_if_changed(os.path.join(OUT, "%s_%s.cuh" % (name, suffix)), "\n".join(body) + "\n")
        if name in QF_TYPES:
            from mbx_b200.codegen import qf
            write_if_changed(os.path.join(OUT, "%s_qf.cuh" % name),
                             qf.emit_cuda(qf.QuadForm(name, shifted_pip(name)), name, nv))
        elif name in SHIFT_TYPES:
            from mbx_b200.codegen.shift import ShiftedTable
            sp = shifted_pip(name)
            body = head + ["#pragma once", '#include "%s.cuh"' % name,
                           "// %d monomials of the %s basis, %d coefficient orbits" %
                           (len(sp.monos), SHIFT_TYPES[name], sp.norb)]
            if name in COSET_TYPES:
                cfs, ctab_s = coset_of(name, shifted_basis=True)
                body.append("// coset form: %d terms of R x %d permutations" % (ctab_s.nterms, len(cfs.perms)))
                emit_pip_f32x2(Trie(ctab_s), nv, "%s_pip_s32" % name, body,
                               max(1, (ctab_s.nterms + COSET_PIECE_TERMS - 1) // COSET_PIECE_TERMS), perms=cfs.perms)
            else:
                # ~400 terms per piece: larger pieces spill in the paired form
                # (2048-water trimers, x/g in shared memory: 0.833/0.818/0.910 ms
                # at 330/400/480 terms per piece)
                strie = Trie(ShiftedTable(sp, name))
                emit_pip_f32x2(strie, nv, "%s_pip_s32" % name, body, max(1, (len(sp.monos) + 399) // 400))
            write_if_changed(os.path.join(OUT, "%s_pip_s32.cuh" % name), "\n".join(body) + "\n")
    return os.path.join(OUT, name + ".cuh"), leaves, inner


TU_HEAD = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// %(what)s for the %(name)s evaluator.
#include <cstring>
#include <vector>
#include "../holder_kernel.cuh"
#include "../launch_cache.cuh"
#include "%(name)s.cuh"
%(include)s
static __constant__ double c_%(name)s[%(ncoef)d];
static __constant__ float cf_%(name)s[%(ncoef)d];
struct %(name)s_CC {
    __device__ __forceinline__ double operator[](int k) const { return c_%(name)s[k]; }
    __device__ __forceinline__ float f(int k) const { return cf_%(name)s[k]; }
};

%(scale_decl)s
int mbx_set_coef_%(name)s_%(v)s(const double* a, int from_device, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    std::vector<double> h(%(ncoef)d);
    if (from_device) {
        e = cudaMemcpyAsync(h.data(), a, sizeof(double) * %(ncoef)d, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return (int)e;
    } else {
        for (int k = 0; k < %(ncoef)d; ++k) h[k] = a[k];
    }
%(scale_apply)s    e = cudaMemcpyToSymbolAsync(c_%(name)s, h.data(), sizeof(double) * %(ncoef)d, 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return (int)e;
    // FP32 copy for the mixed-precision leaf sums (a warp-uniform FFMA operand)
    std::vector<float> f(%(ncoef)d);
    for (int k = 0; k < %(ncoef)d; ++k) f[k] = (float)h[k];
    e = cudaMemcpyToSymbolAsync(cf_%(name)s, f.data(), sizeof(float) * %(ncoef)d, 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return (int)e;
}
"""

LOCK_LAUNCH = """
int mbx_launch_%(name)s_%(v)s(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // persistent grid of lockstep blocks: every resident block slot once
    // (blocks claim chunks of LOCK_THREADS n-mers dynamically); the
    // variables%(gtext)s of the block's n-mers in dynamic shared memory
    auto kern = holder_lock_kernel<%(name)s_T, %(name)s_CC, %(mode)s, false>;
    block = %(name)s_T::LOCK_THREADS;
    const int smem = %(ncol)d * %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS * (int)sizeof(double);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, block, smem, smem, &sms, &bps);
    if (r) return r;
    const long need = (A.n + block - 1) / block;
    grid = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    if (grid < 1) grid = 1;
    kern<<<grid, block, smem, s>>>(A);
    return (int)cudaGetLastError();
}

int mbx_prime_%(name)s_%(v)s(cudaStream_t s) {
    // code prefetch of the %(what2)s: a launch of the evaluation kernel itself in its
    // prefetch mode (prime_pieces), one warp per SM, every piece run by at
    // least four of them
    auto kern = holder_lock_kernel<%(name)s_T, %(name)s_CC, %(mode)s, false>;
    const int smem_full = %(ncol)d * %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS * (int)sizeof(double);
    const int smem = %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS * (int)sizeof(double);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, 0, smem_full, 0, &sms, &bps);
    if (r) return r;
    HolderArgs A;
    memset(&A, 0, sizeof(A));
    A.prime_npieces = %(name)s_%(pipname)s_NPIECES;
    A.prime_passes = (4 * A.prime_npieces + sms - 1) / sms;
    kern<<<sms, 32, smem, s>>>(A);
    return (int)cudaGetLastError();
}
"""

VARIANTS = {
    # variant: (description, body)
    "g": ("FP64 energy + gradient kernel", LOCK_LAUNCH % {
        "name": "%(name)s", "v": "g", "gtext": " and their gradient accumulators", "mode": "HM_GRAD_FP64",
        "ncol": 2, "what2": "FP64 gradient trie", "pipname": "pip"}),
    "e": ("FP64 energy-only kernel", LOCK_LAUNCH % {
        "name": "%(name)s", "v": "e", "gtext": "", "mode": "HM_ENERGY",
        "ncol": 1, "what2": "FP64 energy trie", "pipname": "pip_e"}),
}

# The table unit of every evaluator: the coefficient adjoint and, for the
# evaluators without straight-line code, the table-driven evaluation, both
# reading the polynomial's term table (csrc/term_table.cuh) and its
# coefficients from global memory.
TABLE_TU = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// Table-driven kernels (term table in global memory) of the %(name)s evaluator.
#include <cstring>
#include "../holder_kernel.cuh"
#include "../launch_cache.cuh"
#include "%(name)s.cuh"

int mbx_launch_%(name)s_c(const HolderArgs& A, const double* w, double* out, int grid, int block, cudaStream_t s) {
    // coefficient adjoint: dynamic shared memory = per-coefficient sums +
    // the variable columns of the block's four warps
    auto kern = holder_dcoef_table_kernel<%(name)s_T>;
    const int smem = (%(name)s_T::NCOEF + 4 * 32 * %(name)s_T::NVARS) * (int)sizeof(double);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, 0, smem, 0, &sms, &bps);
    if (r) return r;
    kern<<<grid, 128, smem, s>>>(A, w, out);
    return (int)cudaGetLastError();
}
%(warp)s"""

TABLE_WARP = """
int mbx_launch_%(name)s_w(const HolderArgs& A, int grads, int grid, cudaStream_t s) {
    if (%(name)s_T::NTERMS > 100000) {
        // very large table, few n-mers: a warp per n-mer
        holder_table_kernel<%(name)s_T, 4><<<grid, 128, 0, s>>>(A, grads);
        return (int)cudaGetLastError();
    }
    // a lane per n-mer; x and gradient columns of four warps in dynamic shared memory
    auto kern = holder_table_lane_kernel<%(name)s_T>;
    const int smem = 4 * 2 * %(name)s_T::NVARS * 32 * (int)sizeof(double);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, 128, smem, smem, &sms, &bps);
    if (r) return r;
    const long need = (A.n + 127) / 128;
    const int g = (int)(need < (long)sms * bps ? (need > 0 ? need : 1) : (long)sms * bps);
    kern<<<g, 128, smem, s>>>(A, grads);
    return (int)cudaGetLastError();
}
"""


ONEBODY_TU = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// Table-driven 1-body kernel of the %(name)s evaluator.
#include <cstring>
#include "../holder_kernel.cuh"
#include "../launch_cache.cuh"
#include "%(name)s.cuh"

int mbx_launch_%(name)s_o(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // a lane per monomer; x and gradient columns of four warps in dynamic shared memory
    auto kern = onebody_table_kernel<%(name)s_T>;
    const int smem = 4 * 2 * %(name)s_T::NVARS * 32 * (int)sizeof(double);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, 128, smem, smem, &sms, &bps);
    if (r) return r;
    if (A.n <= 0) return 0;
    const long need = (A.n + 127) / 128;
    const int g = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    kern<<<g, 128, smem, s>>>(A);
    return (int)cudaGetLastError();
}
"""


# Evaluators with straight-line (generated Horner trie) kernels: the water
# and methane-water polynomials of MB-pol / MB-nrg the timed path runs.  All
# others run the table-driven kernels: their tries would add minutes of
# compile time each for types no timed workload uses.
STRAIGHT_TYPES = ("mbpol2b", "mbpol3b", "ch4h2o2b", "ch4h2o3b")


def variants_of(name):
    from mbx_b200.specs import KERNEL_ALIASES
    if name in ONEBODY_SPECS:
        return "o"
    name = KERNEL_ALIASES.get(name, name)
    if name in STRAIGHT_TYPES:
        return "ge" + ("s" if name in SHIFT_TYPES else "") + "t"
    return "wt"


SHIFT_TU = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// Paired FP32 (%(basis)s basis) energy + gradient kernel for the %(name)s evaluator.
#include <cstring>
#include <vector>
#include "../holder_kernel.cuh"
#include "../launch_cache.cuh"
#include "%(name)s.cuh"
#include "%(name)s_pip_s32.cuh"

// one coefficient per monomial orbit of the basis, as an FP32 pair (c, c)
// for the paired instructions
static __constant__ f2_t cs_%(name)s[%(norb)d];
static __constant__ double cs0_%(name)s[1];        // constant term (FP64)
struct %(name)s_CS {
    __device__ __forceinline__ f2_t f2(int k) const { return cs_%(name)s[k]; }
    __device__ __forceinline__ double b0() const { return cs0_%(name)s[0]; }
};

// b = F a: the basis coefficients are linear in the fitted ones.  Row j of F
// (entries sF_row[j] .. sF_row[j+1]) lists (k, factor); sF0 is the constant.
static const int sF_row_%(name)s[%(norb1)d] = {%(rows)s};
static const int sF_k_%(name)s[%(nnz)d] = {%(ks)s};
static const double sF_f_%(name)s[%(nnz)d] = {%(fs)s};
static const int sF0_k_%(name)s[%(nnz0)d] = {%(k0)s};
static const double sF0_f_%(name)s[%(nnz0)d] = {%(f0)s};
// per-orbit factor of the kernel's coefficients (1, or the coset-form scale)
static const double sscale_%(name)s[%(norb)d] = {%(sscale)s};

int mbx_set_coef_%(name)s_s(const double* a, int from_device, cudaStream_t s) {
    std::vector<double> h(%(ncoef)d);
    cudaError_t e = cudaSuccess;
    if (from_device) {
        e = cudaMemcpyAsync(h.data(), a, sizeof(double) * %(ncoef)d, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return (int)e;
    } else {
        for (int k = 0; k < %(ncoef)d; ++k) h[k] = a[k];
    }
    std::vector<unsigned long long> b(%(norb)d);
    for (int j = 0; j < %(norb)d; ++j) {
        double acc = 0.0;
        for (int q = sF_row_%(name)s[j]; q < sF_row_%(name)s[j + 1]; ++q) acc += sF_f_%(name)s[q] * h[sF_k_%(name)s[q]];
        const float f = (float)(acc * sscale_%(name)s[j]);
        unsigned int u;
        memcpy(&u, &f, sizeof(u));
        b[j] = (unsigned long long)u | ((unsigned long long)u << 32);
    }
    double b0 = 0.0;
    for (int q = 0; q < %(nnz0)d; ++q) b0 += sF0_f_%(name)s[q] * h[sF0_k_%(name)s[q]];
    e = cudaMemcpyToSymbolAsync(cs_%(name)s, b.data(), sizeof(unsigned long long) * %(norb)d, 0,
                                cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbolAsync(cs0_%(name)s, &b0, sizeof(double), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return (int)e;
}

int mbx_launch_%(name)s_s(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // three kernels (holder_kernel.cuh): the FP64 variables at full
    // occupancy, the paired FP32 trie in a persistent grid of lockstep blocks
    // (two n-mers per thread, every resident block slot once, the paired
    // variables and gradient accumulators of the block in dynamic shared
    // memory), the FP64 chain rule and sums at full occupancy; A.ps holds the
    // scratch between them (capacity A.ps.cap >= A.n)
    if (!A.ps.dx || !A.ps.q || A.ps.cap < A.n) return (int)cudaErrorInvalidValue;
    auto kern = pair_trie_kernel<%(name)s_T, %(name)s_CS>;
    block = %(name)s_T::LOCK_THREADS_S;
    const int smem = 2 * %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS_S * (int)sizeof(f2_t);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, block, smem, smem, &sms, &bps);
    if (r) return r;
    const long wide = (long)sms * 16;
    const long gv = (A.n + 255) / 256, gf = (A.n + 127) / 128;
    pair_vars_kernel<%(name)s_T><<<(int)(gv < wide ? (gv > 0 ? gv : 1) : wide), 256, 0, s>>>(A);
    const long need = (A.n + 2 * block - 1) / (2 * block);
    grid = (int)(need < (long)sms * bps ? need : (long)sms * bps);
    if (grid < 1) grid = 1;
    kern<<<grid, block, smem, s>>>(A);
    pair_finish_kernel<%(name)s_T><<<(int)(gf < wide ? (gf > 0 ? gf : 1) : wide), 128, 0, s>>>(A);
    return (int)cudaGetLastError();
}

int mbx_prime_%(name)s_s(cudaStream_t s) {
    // code prefetch of the paired FP32 trie: a launch of the evaluation kernel itself in its
    // prefetch mode (prime_pieces), one warp per SM, every piece run by at
    // least four of them
    auto kern = pair_trie_kernel<%(name)s_T, %(name)s_CS>;
    const int smem_full = 2 * %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS_S * (int)sizeof(f2_t);
    const int smem = %(name)s_T::NVARS * %(name)s_T::LOCK_THREADS_S * (int)sizeof(f2_t);
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, 0, smem_full, 0, &sms, &bps);
    if (r) return r;
    HolderArgs A;
    memset(&A, 0, sizeof(A));
    A.prime_npieces = %(name)s_pip_s32_NPIECES;
    A.prime_passes = (4 * A.prime_npieces + sms - 1) / sms;
    kern<<<sms, 32, smem, s>>>(A);
    return (int)cudaGetLastError();
}
"""


QF_TU = """// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.
// Mixed-precision evaluation of the %(name)s polynomial on the tensor cores
// (quadratic form over the %(basis)s FP32 basis, csrc/qf_kernel.cuh).
#include <cmath>
#include <cstring>
#include <vector>
#include "../holder_kernel.cuh"
#include "../launch_cache.cuh"
#include "%(name)s.cuh"
#include "%(name)s_qf.cuh"

// b = F a: the basis coefficients are linear in the fitted ones.  Row j of F
// (entries sF_row[j] .. sF_row[j+1]) lists (k, factor); sF0 is the constant.
static const int sF_row_%(name)s[%(norb1)d] = {%(rows)s};
static const int sF_k_%(name)s[%(nnz)d] = {%(ks)s};
static const double sF_f_%(name)s[%(nnz)d] = {%(fs)s};
static const int sF0_k_%(name)s[%(nnz0)d] = {%(k0)s};
static const double sF0_f_%(name)s[%(nnz0)d] = {%(f0)s};
%(tables)s
// IEEE binary16 of x, rounded to nearest even (subnormals kept; |x| < 65504 here)
static unsigned short qf_half(double x) {
    const unsigned short sign = std::signbit(x) ? 0x8000 : 0;
    const double a = std::fabs(x);
    if (a == 0.0) return sign;
    int e;
    const double f = std::frexp(a, &e);   // a = f 2^e, f in [0.5, 1)
    if (e >= -13) {                        // normal: a >= 2^-14
        double m = std::nearbyint(std::ldexp(f, 11));
        if (m == 2048.0) {
            m = 1024.0;
            ++e;
        }
        return (unsigned short)(sign | ((e + 14) << 10) | ((int)m - 1024));
    }
    return (unsigned short)(sign | (int)std::nearbyint(std::ldexp(a, 24)));   // subnormal: m 2^-24
}

static double qf_half_value(unsigned short h) {
    const int e = (h >> 10) & 0x1f, m = h & 0x3ff;
    const double v = e ? std::ldexp(1024.0 + m, e - 25) : std::ldexp((double)m, -24);
    return (h & 0x8000) ? -v : v;
}

// The tensor-core operands for fitted coefficients a: the C' image in the
// kernel's layout (%(name)s_Q::IMAGE_BYTES bytes), the column factors
// 2^-(s_j + t_j) (NB floats) and the constant term.  Host only.
int mbx_qf_image_%(name)s(const double* a, unsigned char* img, float* colf, double* b0_out) {
    constexpr int NB = %(name)s_Q::NB;
    std::vector<double> b(%(norb)d);
    for (int j = 0; j < %(norb)d; ++j) {
        double acc = 0.0;
        for (int q = sF_row_%(name)s[j]; q < sF_row_%(name)s[j + 1]; ++q) acc += sF_f_%(name)s[q] * a[sF_k_%(name)s[q]];
        b[j] = acc;
    }
    double b0 = 0.0;
    for (int q = 0; q < %(nnz0)d; ++q) b0 += sF0_f_%(name)s[q] * a[sF0_k_%(name)s[q]];
    *b0_out = b0;
    // C (symmetric), then C' = D C D, D = diag(2^t)
    std::vector<double> C((size_t)NB * NB, 0.0);
    for (int q = 0; q < qf_nmono_%(name)s; ++q) {
        const int i = qf_mi_%(name)s[q], j = qf_mj_%(name)s[q];
        const double c = b[qf_mo_%(name)s[q]];
        if (i == j) {
            C[(size_t)i * NB + i] += c;
        } else {
            C[(size_t)i * NB + j] += 0.5 * c;
            C[(size_t)j * NB + i] += 0.5 * c;
        }
    }
    for (int i = 0; i < NB; ++i)
        for (int j = 0; j < NB; ++j) C[(size_t)i * NB + j] = std::ldexp(C[(size_t)i * NB + j], qf_t_%(name)s[i] + qf_t_%(name)s[j]);
    // column exponents: largest |C'_ij 2^s_j| of a column below 2^14
    std::vector<int> sj(NB, 0);
    for (int j = 0; j < NB; ++j) {
        double m = 0.0;
        for (int i = 0; i < NB; ++i) m = std::fmax(m, std::fabs(C[(size_t)i * NB + j]));
        if (m > 0.0) {
            int e;
            std::frexp(m, &e);        // floor(log2 m) = e - 1
            sj[j] = 14 - e;
        }
        colf[j] = (float)std::ldexp(1.0, -(sj[j] + qf_t_%(name)s[j]));
    }
    // K block s, pass p (columns pass_col(p) .. + pass_n(p)): B[n][k] =
    // C'_kn 2^s_n in hi, mid[, lo] FP16 parts of pass_n(p) rows x 16, core
    // matrix (n' / 8, k / 8) of a part at (n' / 8) 128 + (k / 8) (pass_n / 8) 128
    // (row groups contiguous), row n' %% 8 at 16 (n' %% 8), n' = n - pass_col(p)
    memset(img, 0, (size_t)%(name)s_Q::IMAGE_BYTES);
    for (int s = 0; s < %(name)s_Q::KS; ++s) {
        const int parts = %(name)s_Q::parts(s);
        for (int p = 0; p < %(name)s_Q::NPASS; ++p) {
            const int width = %(name)s_Q::pass_n(p), c0 = %(name)s_Q::pass_col(p);
            unsigned char* st = img + %(name)s_Q::chunk_offset(s, p);
            for (int nn = 0; nn < width; ++nn)
                for (int kk = 0; kk < 16; ++kk) {
                    const int k = 16 * s + kk, n = c0 + nn;
                    double x = std::ldexp(C[(size_t)k * NB + n], sj[n]);
                    const size_t off = (size_t)(nn / 8) * 128 + (size_t)(kk / 8) * (width / 8) * 128 + (nn %% 8) * 16 +
                                       (kk %% 8) * 2;
                    for (int pt = 0; pt < parts; ++pt) {
                        const unsigned short h = qf_half(x);
                        memcpy(st + (size_t)pt * width * 32 + off, &h, 2);
                        x -= qf_half_value(h);
                    }
                }
        }
    }
    return 0;
}

int mbx_set_coef_%(name)s_s(const double* a, int from_device, cudaStream_t s) {
    std::vector<double> h(%(ncoef)d);
    cudaError_t e = cudaSuccess;
    if (from_device) {
        e = cudaMemcpyAsync(h.data(), a, sizeof(double) * %(ncoef)d, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return (int)e;
    } else {
        for (int k = 0; k < %(ncoef)d; ++k) h[k] = a[k];
    }
    std::vector<unsigned char> img((size_t)%(name)s_Q::IMAGE_BYTES);
    std::vector<float> colf(%(name)s_Q::NB);
    double b0 = 0.0;
    mbx_qf_image_%(name)s(h.data(), img.data(), colf.data(), &b0);
    e = cudaMemcpyToSymbolAsync(qf_img_%(name)s, img.data(), img.size(), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbolAsync(qf_colf_%(name)s, colf.data(), sizeof(float) * colf.size(), 0,
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(qf_b0_%(name)s, &b0, sizeof(double), 0, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return (int)e;
}

int mbx_launch_%(name)s_s(const HolderArgs& A, int grid, int block, cudaStream_t s) {
    // three kernels: the FP64 variables shifted to the FP32 basis at full
    // occupancy (pair_vars_kernel), the quadratic form on the tensor cores
    // (qf_eval_kernel: one CTA per SM, persistent over tiles of 128 n-mers),
    // the FP64 chain rule and sums at full occupancy (pair_finish_kernel);
    // A.ps holds the scratch between them (capacity A.ps.cap >= A.n)
    if (!A.ps.dx || !A.ps.q || A.ps.cap < A.n) return (int)cudaErrorInvalidValue;
    auto kern = qf_eval_kernel<%(name)s_T, %(name)s_Q>;
    static LaunchCache lc;
    int sms = 0, bps = 0;
    const int r = launch_facts(lc, kern, qf::THREADS, qf::Layout<%(name)s_Q>::SMEM, qf::Layout<%(name)s_Q>::SMEM, &sms,
                               &bps);
    if (r) return r;
    const long wide = (long)sms * 16;
    const long gv = (A.n + 255) / 256, gf = (A.n + 127) / 128;
    pair_vars_kernel<%(name)s_T><<<(int)(gv < wide ? (gv > 0 ? gv : 1) : wide), 256, 0, s>>>(A);
    const long tiles = (A.n + 127) / 128;
    grid = (int)(tiles < (long)sms ? (tiles > 0 ? tiles : 1) : sms);
    kern<<<grid, qf::THREADS, qf::Layout<%(name)s_Q>::SMEM, s>>>(A);
    pair_finish_kernel<%(name)s_T><<<(int)(gf < wide ? (gf > 0 ? gf : 1) : wide), 128, 0, s>>>(A);
    return (int)cudaGetLastError();
}

int mbx_prime_%(name)s_s(cudaStream_t) {
    return 0;   // the tensor-core kernel's code is small: nothing to prefetch
}
"""


def write_qf_tu(name, path):
    from mbx_b200.codegen import qf
    sp = shifted_pip(name)
    q = qf.QuadForm(name, sp)
    rows, ks, fs = [0], [], []
    for row in sp.F:
        for k, f in sorted(row.items()):
            ks.append(k)
            fs.append(f)
        rows.append(len(ks))
    k0 = sorted(sp.const_F)
    d = {"name": name, "basis": SHIFT_TYPES[name], "norb": sp.norb, "norb1": sp.norb + 1,
         "ncoef": SPECS[name].ncoef, "nnz": len(ks), "nnz0": max(1, len(k0)),
         "rows": ",".join(map(str, rows)), "ks": ",".join(map(str, ks)),
         "fs": ",".join(repr(float(f)) for f in fs),
         "k0": ",".join(map(str, k0)) if k0 else "0",
         "f0": ",".join(repr(float(sp.const_F[k])) for k in k0) if k0 else "0.0",
         "tables": qf.emit_host_tables(q, name)}
    write_tu(path, QF_TU % d)


def write_shift_tu(name, path):
    sp = shifted_pip(name)
    rows, ks, fs = [0], [], []
    for row in sp.F:
        for k, f in sorted(row.items()):
            ks.append(k)
            fs.append(f)
        rows.append(len(ks))
    k0 = sorted(sp.const_F)
    d = {"name": name, "NAME": name.upper(), "basis": SHIFT_TYPES[name], "norb": sp.norb, "norb1": sp.norb + 1,
         "ncoef": SPECS[name].ncoef, "nnz": len(ks), "nnz0": max(1, len(k0)),
         "rows": ",".join(map(str, rows)), "ks": ",".join(map(str, ks)),
         "fs": ",".join(repr(float(f)) for f in fs),
         "k0": ",".join(map(str, k0)) if k0 else "0",
         "sscale": ",".join(repr(float(x)) for x in (coset_of(name, True)[0].scale if name in COSET_TYPES
                                                       else np.ones(sp.norb))),
         "f0": ",".join(repr(float(sp.const_F[k])) for k in k0) if k0 else "0.0"}
    write_tu(path, SHIFT_TU % d)


def write_tu(path, text):
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)


def write_kernels_cu(name):
    paths = []
    inc = {"g": "pip", "e": "pip_e"}
    if name in ONEBODY_SPECS:
        path = os.path.join(OUT, "%s_t.cu" % name)
        write_tu(path, ONEBODY_TU % {"name": name})
        return [path]
    spec = SPECS[name]
    for v in variants_of(name):
        if v == "w":
            continue   # part of the table unit
        if v == "s":
            path = os.path.join(OUT, "%s_s.cu" % name)
            if name in QF_TYPES:
                write_qf_tu(name, path)
            else:
                write_shift_tu(name, path)
            paths.append(path)
            continue
        path = os.path.join(OUT, "%s_%s.cu" % (name, v))
        if v == "t":
            d = {"name": name, "warp": TABLE_WARP % {"name": name} if "w" in variants_of(name) else ""}
            write_tu(path, TABLE_TU % d)
        else:
            what, body = VARIANTS[v]
            d = {"name": name, "NAME": name.upper(), "ncoef": spec.ncoef, "v": v, "what": what,
                 "include": '#include "%s_%s.cuh"\n' % (name, inc[v]), "scale_decl": "", "scale_apply": ""}
            if name in COSET_TYPES:
                cf, _ = coset_of(name)
                d["scale_decl"] = ("// coset form: the kernels take a_k * scale_k (codegen/coset.py)\n"
                                   "static const double coset_scale_%s[%d] = {%s};\n" %
                                   (name, spec.ncoef, ", ".join(repr(float(x)) for x in cf.scale)))
                d["scale_apply"] = "    for (int k = 0; k < %d; ++k) h[k] *= coset_scale_%s[k];\n" % (spec.ncoef, name)
            write_tu(path, (TU_HEAD + body) % d)
        paths.append(path)
    return paths


def term_runs(vars_):
    """(variable, exponent) runs of a term's variable list, in order."""
    runs = []
    for v in vars_:
        if runs and runs[-1][0] == v:
            runs[-1][1] += 1
        else:
            runs.append([v, 1])
    return runs


@__import__("functools").lru_cache(maxsize=None)
def _table_runs(table_name):
    t = load_pip(table_name)
    return [term_runs(t.var[q, :t.deg[q]].tolist()) for q in range(t.nterms)]


def term_pairs_max(table):
    return max(1, max(len(r) for r in _table_runs(table.name)))


def table_names():
    """Term tables in registry order (an evaluator sharing another's table
    refers to the same entry), then the 1-body evaluators' tables."""
    from mbx_b200.specs import KERNEL_ALIASES
    names = []
    for n in SPECS:
        t = SPECS[KERNEL_ALIASES.get(n, n)].pip_table
        if t not in names:
            names.append(t)
    for n, sp in ONEBODY_SPECS.items():
        if sp.pip_table not in names:
            names.append(sp.pip_table)
    return names


def write_term_tables():
    """Every evaluator's term table (csrc/term_table.cuh encoding) in one
    binary file, embedded in the library by terms_blob.cpp (.incbin), plus the
    index of the tables."""
    blob = bytearray()
    index = []
    for tname in table_names():
        t = load_pip(tname)
        runs = _table_runs(tname)
        words = np.zeros((t.nterms, 4), np.int32)
        words[:, 0] = t.k
        for q, rr in enumerate(runs):
            if len(rr) > 6:
                raise ValueError("%s term %d has more than six distinct variables" % (tname, q))
            packed = [0, 0, 0]
            for i in range(6):
                v, e = (rr[i] if i < len(rr) else (255, 0))
                if not (0 <= v < 255 and 0 < e < 256) and v != 255:
                    raise ValueError("%s term %d: variable %d exponent %d out of range" % (tname, q, v, e))
                packed[i >> 1] |= ((v & 255) | (e << 8)) << (16 * (i & 1))
            for j in range(3):
                words[q, 1 + j] = packed[j] - (1 << 32) if packed[j] >= 1 << 31 else packed[j]
        off_terms = len(blob)
        blob += words.tobytes()
        off_coef = len(blob)
        blob += np.ascontiguousarray(t.coef, np.float64).tobytes()
        pad = (-len(blob)) % 16
        blob += b"\0" * pad
        index.append((tname, off_terms, off_coef, t.nterms, term_pairs_max(t)))
    bin_path = os.path.join(OUT, "terms.bin")
    old = open(bin_path, "rb").read() if os.path.exists(bin_path) else None
    if old != bytes(blob):
        with open(bin_path, "wb") as f:
            f.write(bytes(blob))
    lines = ["// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.", "#pragma once",
             "// term tables in terms.bin: (name, byte offset of the int4 terms, of the",
             "// double multiplicities, number of terms, (variable, exponent) pairs per term at most)",
             "struct TermTableInfo { const char* name; long off_terms, off_tcoef, nterms; int pairs; };",
             "static const TermTableInfo mbx_term_tables[] = {"]
    for tname, ot, oc, nt, npair in index:
        lines.append('    {"%s", %d, %d, %d, %d},' % (tname, ot, oc, nt, npair))
    lines.append("};")
    lines.append("static const int mbx_num_term_tables = %d;" % len(index))
    lines.append("static const long mbx_terms_bytes = %d;" % len(blob))
    write_tu(os.path.join(OUT, "terms_index.inc"), "\n".join(lines) + "\n")
    # the binary is referenced by absolute path (generated per checkout)
    write_tu(os.path.join(OUT, "terms_blob.cpp"),
             "// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.\n"
             "// The term tables of every evaluator (terms.bin), embedded read-only.\n"
             "__asm__(\".section .rodata\\n\"\n"
             "        \".balign 16\\n\"\n"
             "        \".globl mbx_terms_blob\\n\"\n"
             "        \".type mbx_terms_blob, @object\\n\"\n"
             "        \"mbx_terms_blob:\\n\"\n"
             "        \".incbin \\\"%s\\\"\\n\"\n"
             "        \".size mbx_terms_blob, %d\\n\"\n"
             "        \".previous\\n\");\n" % (bin_path, len(blob)))


def write_ps1b():
    """The Partridge-Schwenke polynomial sums of the water 1-body term
    (mbx_b200/data/ps1b.json, extracted by codegen/onebody_extract.py) as
    straight-line code: for every term j of ps::pot_nasa's loop
    (potential/1b/ps.cpp:455-476) the four sums with the term's indices and
    coefficient as literals, every product and sum rounded on its own in the
    reference's operand order."""
    import json
    d = json.load(open(os.path.join(PKG, "data", "ps1b.json")))
    L = ["// Generated by mbx_b200/codegen/gen_kernels.py from mbx_b200/data/ps1b.json -- do not edit.",
         "#pragma once",
         "#define PS1B_REOH %s" % lit(d["reoh"]), "#define PS1B_B1 %s" % lit(d["b1"]),
         "#define PS1B_ROH %s" % lit(d["roh"]), "#define PS1B_ALPHAOH %s" % lit(d["alphaoh"]),
         "#define PS1B_PHH2 %s" % lit(d["phh2"]), "#define PS1B_DEOH %s" % lit(d["deoh"]),
         "#define PS1B_PHH1 %s" % lit(d["phh1"]), "#define PS1B_COSTHE %s" % lit(d["costhe"]),
         "#define PS1B_OFFSET %s" % lit(d["offset"]), "#define PS1B_CM1_KCALMOL %s" % lit(d["cm1_kcalmol"]),
         "#define PS1B_C0 %s" % lit(d["c5z"][0]),
         "__device__ __forceinline__ void ps1b_sums(const double (&f0)[16], const double (&f1)[16], "
         "const double (&f2)[16], double& s0, double& s1, double& s2, double& s3) {"]
    M, A = "__dmul_rn", "__dadd_rn"
    for j in range(1, len(d["c5z"])):
        I, J, K = d["idx1"][j], d["idx2"][j], d["idx3"][j]
        c = lit(d["c5z"][j])
        sym = "%s(%s(f0[%d], f1[%d]), %s(f0[%d], f1[%d]))" % (A, M, I, J, M, J, I)
        L.append("    { const double sym = %s;" % sym)
        L.append("      s0 = %s(s0, %s(%s(%s, sym), f2[%d]));" % (A, M, M, c, K))
        t1 = "%s(%s(%s(%s, f0[%d]), f1[%d]), %s(%s(%s, f0[%d]), f1[%d]))" % (
            A, M, M, lit(float(I - 1)), I - 1, J, M, M, lit(float(J - 1)), J - 1, I)
        L.append("      s1 = %s(s1, %s(%s(%s, %s), f2[%d]));" % (A, M, M, c, t1, K))
        t2 = "%s(%s(%s(%s, f0[%d]), f1[%d]), %s(%s(%s, f0[%d]), f1[%d]))" % (
            A, M, M, lit(float(J - 1)), I, J - 1, M, M, lit(float(I - 1)), J, I - 1)
        L.append("      s2 = %s(s2, %s(%s(%s, %s), f2[%d]));" % (A, M, M, c, t2, K))
        L.append("      s3 = %s(s3, %s(%s(%s(%s, sym), %s), f2[%d])); }" % (A, M, M, M, c, lit(float(K - 1)), K - 1))
    L.append("}")
    write_tu(os.path.join(OUT, "ps1b.inc"), "\n".join(L) + "\n")


def write_registry():
    """Host tables: evaluator descriptions and default coefficients."""
    from mbx_b200.tables import load_fit
    from mbx_b200.specs import KERNEL_ALIASES
    lines = ["// Generated by mbx_b200/codegen/gen_kernels.py -- do not edit.", "#pragma once",
             '#include "../holder_kernel.cuh"', ""]
    for name in SPECS:
        vs = variants_of(name)
        if name in KERNEL_ALIASES:
            vs = ""   # runs the kernels of KERNEL_ALIASES[name], declared there
        for v in "gesw":
            if v not in vs:
                continue
            if v in "ges":
                lines.append("int mbx_launch_%s_%s(const HolderArgs& A, int grid, int block, cudaStream_t s);" %
                             (name, v))
                lines.append("int mbx_prime_%s_%s(cudaStream_t s);" % (name, v))
                lines.append("int mbx_set_coef_%s_%s(const double* a, int from_device, cudaStream_t s);" % (name, v))
            else:
                lines.append("int mbx_launch_%s_w(const HolderArgs& A, int grads, int grid, cudaStream_t s);" % name)
        if "t" in vs:
            lines.append("int mbx_launch_%s_c(const HolderArgs& A, const double* w, double* out, int grid, "
                         "int block, cudaStream_t s);" % name)
        fit = load_fit(name)
        lines.append("static const double mbx_fit_%s[%d] = {" % (name, len(fit)))
        for i in range(0, len(fit), 4):
            lines.append("    " + ", ".join(repr(float(x)) for x in fit[i:i + 4]) + ",")
        lines.append("};")
    lines.append("")
    names = list(SPECS)
    tables = table_names()
    lines.append("static const EvaluatorInfo mbx_evaluators[] = {")
    for name, spec in SPECS.items():
        vs = variants_of(name)
        kern = KERNEL_ALIASES.get(name, name)
        ids = list(spec.monomers) + ["", ""][:3 - len(spec.monomers)]
        skip = {"pair_gt": 0, "two_of_three_gt": 1, "all_three_gt": 2}[spec.skip]

        def fn(v, kind):
            # the table unit ("t") holds the coefficient adjoint ("c")
            have = ("t" in vs) if v == "c" else (v in vs)
            return ("mbx_%s_%s_%s" % (kind, kern, v)) if have else "nullptr"
        lines.append('    {"%s", %d, {"%s", "%s", "%s"}, %s, %d, %d, %d, %d, mbx_fit_%s, %s, %s, %s, %s, %s, %s,' %
                     (name, spec.nbody, ids[0], ids[1], ids[2], lit(spec.rf), skip, spec.ncoef, spec.nreal,
                      spec.nvars, name, fn("g", "launch"), fn("e", "launch"), fn("c", "launch"),
                      fn("w", "launch"), fn("s", "launch"), lit(MIXED_FP64_RADIUS.get(name, 0.0))))
        lines.append("     %s, %s, %s," % (fn("g", "prime"), fn("e", "prime"), fn("s", "prime")))
        lines.append("     {%s, nullptr, nullptr, nullptr, nullptr}, %d, %d}," %
                     (", ".join(fn(v, "set_coef") for v in "ges"), tables.index(SPECS[kern].pip_table),
                      names.index(kern)))
    lines.append("};")
    lines.append("static const int mbx_num_evaluators = %d;" % len(SPECS))
    # host builders of the tensor-core operands of the mixed mode (QF_TYPES)
    from mbx_b200.codegen import qf as qfmod
    lines.append("struct QfInfo { const char* name; long image_bytes; int nb; "
                 "int (*build)(const double*, unsigned char*, float*, double*); };")
    for name in sorted(QF_TYPES):
        lines.append("int mbx_qf_image_%s(const double* a, unsigned char* img, float* colf, double* b0);" % name)
    lines.append("static const QfInfo mbx_qf_types[] = {")
    for name in sorted(QF_TYPES):
        q = qfmod.QuadForm(name, shifted_pip(name))
        lines.append('    {"%s", %dL, %d, mbx_qf_image_%s},' % (name, qfmod.image_bytes(q), q.npad, name))
    lines.append("};")
    lines.append("static const int mbx_num_qf_types = %d;" % len(QF_TYPES))
    # 1-body evaluators (table-driven), by monomer id
    from mbx_b200.specs import ONEBODY_DISPATCH
    lines.append("struct OneBodyInfo { const char* name; const char* mon; int ncoef; const double* fit; int table; "
                 "int (*launch)(const HolderArgs&, int, int, cudaStream_t); };")
    for name, sp in ONEBODY_SPECS.items():
        lines.append("int mbx_launch_%s_o(const HolderArgs& A, int grid, int block, cudaStream_t s);" % name)
        fit = load_fit(name)
        lines.append("static const double mbx_fit_%s[%d] = {%s};" %
                     (name, len(fit), ", ".join(repr(float(x)) for x in fit)))
    mon_of = {v: k for k, v in ONEBODY_DISPATCH.items()}
    lines.append("static const OneBodyInfo mbx_onebody[] = {%s};" % ", ".join(
        '{"%s", "%s", %d, mbx_fit_%s, %d, mbx_launch_%s_o}' %
        (name, mon_of[name], sp.ncoef, name, tables.index(sp.pip_table), name)
        for name, sp in ONEBODY_SPECS.items()))
    lines.append("static const int mbx_num_onebody = %d;" % len(ONEBODY_SPECS))
    # real atoms per monomer id (SetUpMonomers, bblock/sys_tools.cpp:133-254)
    from mbx_b200.specs import MONOMER_ATOMS
    lines.append("struct MonomerInfo { const char* id; int nat; };")
    lines.append("static const MonomerInfo mbx_monomers[] = {%s};" %
                 ", ".join('{"%s", %d}' % (m, n) for m, n in MONOMER_ATOMS.items()))
    lines.append("static const int mbx_num_monomers = %d;" % len(MONOMER_ATOMS))
    write_tu(os.path.join(OUT, "registry.inc"), "\n".join(lines) + "\n")


def main(argv=None, quiet=False):
    """Writes every generated file; returns the translation units to compile."""
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=list(SPECS))
    args = ap.parse_args(argv)
    os.makedirs(OUT, exist_ok=True)
    write_registry()
    write_term_tables()
    write_ps1b()
    from mbx_b200.specs import KERNEL_ALIASES
    keep = {"registry.inc", "terms_index.inc", "terms.bin", "terms_blob.cpp", "ps1b.inc"}
    if args.names == list(SPECS):
        args.names = list(SPECS) + list(ONEBODY_SPECS)
    for n in args.names:
        if n in KERNEL_ALIASES:
            continue
        path, leaves, inner = generate(n)
        keep.add(os.path.basename(path))
        if n in STRAIGHT_TYPES:
            for v in ("pip", "pip_e", "qf" if n in QF_TYPES else "pip_s32"):
                keep.add("%s_%s.cuh" % (n, v))
        keep.update(os.path.basename(p) for p in write_kernels_cu(n))
        if not quiet:
            print("%s: %d leaves, %d inner -> %s" % (n, leaves, inner, path))
    if args.names == list(SPECS) + list(ONEBODY_SPECS):
        # drop the units of an earlier generation (other variants or types)
        for f in os.listdir(OUT):
            if f not in keep:
                os.remove(os.path.join(OUT, f))
    return sorted(os.path.join(OUT, f) for f in os.listdir(OUT) if f.endswith((".cu", ".cpp")))


if __name__ == "__main__":
    main()
