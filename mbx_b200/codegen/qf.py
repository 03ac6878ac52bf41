"""Quadratic form of a degree-4 permutationally invariant polynomial, for
evaluation on the tensor cores.

The shifted polynomial P(d) = sum_m b_m prod_{v in m} d_v (``shift.py``,
d = x - x0) has monomials of degree <= 4.  Every monomial of degree 3 or 4 is
a product of two members of a basis B of monomials of degree <= 2 (the
constant, the 36 variables and a chosen set of products d_u d_v), so

    P(d) = m(d)^T C m(d),      m(d) = (prod_{v in beta} d_v)_{beta in B},

with C symmetric: the monomial m = beta_i beta_j puts b_m / 2 at (i, j) and
(j, i) (b_m at (i, i) when beta_i = beta_j).  For a tile of n-mers the
products y = C m(d) are one matrix product, Y = M C (M: n-mers x basis),
which the tcgen05 tensor cores compute; the energy is m . y and the gradient
dP/dd_u = 2 sum_j y_j d m_j / d d_u, both O(|B|) per n-mer.

The basis is chosen small: a greedy cover (each step adds the product d_u d_v
that completes the most uncovered monomials), then members whose removal
keeps every monomial covered are dropped.  For MB-pol 3b this gives 442
products, |B| = 479 (padded to 480), against 703 for all products of degree
<= 2, and the matrix product costs 2 x 480^2 multiply-adds per n-mer and
operand product (below).

Precision.  The tensor cores take FP16 operands with FP32 accumulation (one
rounding to nearest after every MMA, measured on the B200 to agree with this
model).  Both
operands are split into FP16 parts: m into hi + lo (22 bits), C into
hi + mid + lo (33 bits).  An error in C is the same for every n-mer and adds
up coherently over a box, so C needs the third part; an error in m is
n-mer-dependent and does not.  Per K block of 16 basis members the products
hi.hi + hi.mid + lo.hi are summed, and hi.lo on the K blocks of the members
that carry most of the coherent error (``NTHIRD`` members, ordered first).
Both operands are scaled by powers of two so that no FP16 value overflows and
few underflow: C symmetrically, C' = D C D with D = diag(2^t) (Ruiz
equilibration, from the fitted coefficients, fixed at generation time), then
every column of C' by 2^s_j so that its largest entry is below 2^14
(recomputed whenever the coefficients change); every n-mer's row of m D^-1 by
a power of two r so that its bound is below 2^14.

Test infrastructure and the library share this module: the generator writes
the basis and exponents to ``data/<name>.qf.json`` (computing them takes a
minute), and the kernels' straight-line code from it.
"""
import collections
import json
import os
import random

import numpy as np

from . import shift

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data")
NPAD = 16          # basis padded to a multiple of the K block (16)
NTHIRD = 128       # members whose K blocks take the third part of C (8 K blocks)
COLMAX_EXP = 14    # largest |C'| of a column below 2^14
ROWMAX_EXP = 14    # largest |m D^-1 r| of a row below 2^14
RUIZ_STEPS = 5


def _pairings(m):
    """Ways of writing a monomial (sorted variable tuple) as a product of two
    basis candidates of degree <= 2, best first."""
    if len(m) == 4:
        a, b, c, d = m
        return [((a, b), (c, d)), ((a, c), (b, d)), ((a, d), (b, c))]
    if len(m) == 3:
        a, b, c = m
        return [((a,), (b, c)), ((b,), (a, c)), ((c,), (a, b))]
    if len(m) == 2:
        return [((m[0],), (m[1],))]
    if len(m) == 1:
        return [((), m)]
    return [((), ())]


def _covered(m, B):
    return any(p in B and q in B for p, q in _pairings(m))


def select_basis(monos, nvars):
    """A small set of degree-2 products such that every monomial of degree 3
    or 4 is a product of two basis members (constant and variables always
    belong to the basis)."""
    base = {()} | {(v,) for v in range(nvars)}
    todo = [m for m in monos if len(m) >= 3]
    chosen = set()

    def basis():
        return base | chosen

    unc = [m for m in todo if not _covered(m, basis())]
    while unc:
        score = collections.Counter()
        B = basis()
        for m in unc:
            ps = _pairings(m)
            for p, q in ps:
                need = [x for x in (p, q) if x not in B]
                for x in set(need):
                    score[x] += 1.0 / (len(ps) * len(need))
        best = max(sorted(score), key=lambda x: score[x])
        chosen.add(best)
        B = basis()
        unc = [m for m in unc if not _covered(m, B)]
    # drop members that the rest already covers for
    order = sorted(chosen)
    random.Random(0).shuffle(order)
    for x in order:
        chosen.discard(x)
        B = basis()
        if not all(_covered(m, B) for m in todo):
            chosen.add(x)
    return [()] + [(v,) for v in range(nvars)] + sorted(chosen)


def assign(monos, basis):
    """(i, j) basis indices of every monomial, i <= j."""
    idx = {b: i for i, b in enumerate(basis)}
    out = []
    for m in monos:
        for p, q in _pairings(tuple(m)):
            if p in idx and q in idx:
                i, j = idx[p], idx[q]
                out.append((min(i, j), max(i, j)))
                break
        else:
            raise ValueError("monomial %r not covered by the basis" % (m,))
    return out


def c_matrix(nb, ij, orbit_of, b):
    """C (nb x nb, symmetric) for orbit coefficients b (constant term kept
    out: it is added in FP64)."""
    C = np.zeros((nb, nb))
    for (i, j), o in zip(ij, orbit_of):
        if i == j:
            C[i, i] += b[o]
        else:
            C[i, j] += 0.5 * b[o]
            C[j, i] += 0.5 * b[o]
    return C


def ruiz(C, steps=RUIZ_STEPS):
    t = np.zeros(C.shape[0])
    for _ in range(steps):
        S = np.abs(C) * (2.0 ** t)[:, None] * (2.0 ** t)[None, :]
        rm = S.max(axis=1)
        rm[rm == 0] = 1.0
        t = t - np.round(0.5 * np.log2(rm))
    return t.astype(int)


def column_exponents(Ce):
    """s_j with max_i |Ce_ij| 2^s_j < 2^COLMAX_EXP (0 for empty columns)."""
    cm = np.abs(Ce).max(axis=0)
    s = np.zeros(Ce.shape[1], int)
    nz = cm > 0
    s[nz] = COLMAX_EXP - 1 - np.floor(np.log2(cm[nz])).astype(int)
    return s


def split3(x):
    """Three FP16 parts of x (float64 array): hi + mid + lo."""
    h = x.astype(np.float16)
    m = (x - h.astype(np.float64)).astype(np.float16)
    lo = (x - h.astype(np.float64) - m.astype(np.float64)).astype(np.float16)
    return h, m, lo


def monomial_values(basis, d):
    """FP32 basis values m(d) for FP32 shifted variables d [n, nvars]: the
    products rounded as the kernel rounds them."""
    d = np.asarray(d, np.float32)
    out = np.empty((d.shape[0], len(basis)), np.float32)
    for j, b in enumerate(basis):
        if len(b) == 0:
            out[:, j] = 1.0
        elif len(b) == 1:
            out[:, j] = d[:, b[0]]
        else:
            out[:, j] = d[:, b[0]] * d[:, b[1]]
    return out


def order_by_importance(basis, ij, sp, b, d_sample):
    """Basis order for the kernel: the NTHIRD members whose third C part
    matters most (coherent contribution over liquid n-mers) first, then the
    rest in index order."""
    nb = len(basis)
    C = c_matrix(nb, ij, sp.orbit_of, b)
    t = ruiz(C)
    Ce = C * (2.0 ** t)[:, None] * (2.0 ** t)[None, :]
    cs = 2.0 ** column_exponents(Ce)
    Bs = Ce * cs[None, :]
    h, m, lo = split3(Bs)
    M = monomial_values(basis, d_sample).astype(np.float64)
    A = M * (2.0 ** -t)[None, :]
    W = M / (cs * 2.0 ** t)[None, :]
    contrib = np.abs(((A.T @ W) * lo.astype(np.float64)).sum(axis=1))
    first = sorted(np.argsort(-contrib, kind="stable")[:NTHIRD].tolist())
    rest = [i for i in range(nb) if i not in set(first)]
    return first + rest


def build(name, spec, table, a):
    """Basis (kernel order), per-member exponents t, for one polynomial."""
    sp = shift.shifted(spec, table)
    monos = [tuple(m) for m in sp.monos]
    basis = select_basis(monos, spec.nvars)
    ij = assign(monos, basis)
    _, b = shift.shifted_coefficients(sp, a)
    x = shift._variables(spec, shift.liquid_trimers(spec))
    d = (x - sp.x0).astype(np.float32)
    order = order_by_importance(basis, ij, sp, b, d)
    basis = [basis[i] for i in order]
    ij = assign(monos, basis)
    t = ruiz(c_matrix(len(basis), ij, sp.orbit_of, b))
    return {"name": name, "nvars": spec.nvars, "basis": [list(x) for x in basis], "t": t.tolist(),
            "nthird": NTHIRD, "npad": NPAD}


def path_of(name):
    return os.path.join(DATA, "%s.qf.json" % name)


def load(name):
    with open(path_of(name)) as f:
        q = json.load(f)
    q["basis"] = [tuple(x) for x in q["basis"]]
    return q


class QuadForm:
    """The quadratic form of one polynomial in the kernel's layout: basis in
    kernel order, padded size, the (i, j) entry of every shifted monomial."""

    def __init__(self, name, sp):
        q = load(name)
        self.name = name
        self.sp = sp
        self.basis = q["basis"]
        self.nb = len(self.basis)
        self.npad = -(-self.nb // q["npad"]) * q["npad"]
        self.t = np.zeros(self.npad, int)
        self.t[:self.nb] = q["t"]
        self.nthird = q["nthird"]
        self.ij = assign([tuple(m) for m in sp.monos], self.basis)

    def matrix(self, b):
        C = np.zeros((self.npad, self.npad))
        C[:self.nb, :self.nb] = c_matrix(self.nb, self.ij, self.sp.orbit_of, b)
        return C

    def operands(self, b):
        """(B parts hi/mid/lo [npad x npad] float16 with B[i, j] = C'_ij 2^s_j,
        column factors f_j = 2^-(s_j + t_j))."""
        Ce = self.matrix(b) * (2.0 ** self.t)[:, None] * (2.0 ** self.t)[None, :]
        s = column_exponents(Ce)
        Bs = Ce * (2.0 ** s)[None, :]
        return split3(Bs), 2.0 ** -(s + self.t)

    def row_scale(self, d):
        """Power of two r per row with |m_j(d) 2^-t_j| r < 2^ROWMAX_EXP for every j
        (a bound from max(1, max|d|)^2 and max_j 2^-t_j)."""
        dm = np.maximum(1.0, np.abs(np.asarray(d, np.float32)).max(axis=1).astype(np.float64))
        bound = dm * dm * 2.0 ** (-self.t.min())
        e = np.floor(np.log2(bound)).astype(int) + 1
        return 2.0 ** (ROWMAX_EXP - e)

    def emulate(self, b, d):
        """numpy restatement of the kernel's arithmetic: exact FP16 products,
        hi.hi summed into the main accumulator and the other products into
        the correction accumulator, FP32 rounding after every MMA (K block of
        16); returns (P without the constant term, dP/dd) for FP32 shifted
        variables d."""
        (bh, bm, bl), f = self.operands(b)
        bh, bm, bl = (x.astype(np.float64) for x in (bh, bm, bl))
        M = np.zeros((d.shape[0], self.npad), np.float32)
        M[:, :self.nb] = monomial_values(self.basis, d)
        r = self.row_scale(d)
        A = (M.astype(np.float64) * (2.0 ** -self.t)[None, :]) * r[:, None]
        ah = A.astype(np.float16).astype(np.float64)
        al = (A - ah).astype(np.float16).astype(np.float64)
        Ym = np.zeros((d.shape[0], self.npad), np.float32)
        Yc = np.zeros_like(Ym)
        for k0 in range(0, self.npad, 16):
            ks = slice(k0, k0 + 16)
            Ym = (Ym.astype(np.float64) + ah[:, ks] @ bh[ks]).astype(np.float32)
            corr = [ah[:, ks] @ bm[ks], al[:, ks] @ bh[ks]] + ([ah[:, ks] @ bl[ks]] if k0 < self.nthird else [])
            for p in corr:
                Yc = (Yc.astype(np.float64) + p).astype(np.float32)
        Y = (Ym + Yc).astype(np.float32)
        Z = Y.astype(np.float64) * f[None, :] / r[:, None]
        P = np.einsum("nj,nj->n", M.astype(np.float64), Z)
        g = np.zeros(d.shape, np.float64)
        dd = np.asarray(d, np.float32).astype(np.float64)
        for j, bb in enumerate(self.basis):
            if len(bb) == 1:
                g[:, bb[0]] += 2 * Z[:, j]
            elif len(bb) == 2:
                u, v = bb
                g[:, u] += 2 * Z[:, j] * dd[:, v]
                g[:, v] += 2 * Z[:, j] * dd[:, u]
        return P, g


def main(argv=None):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from mbx_b200.specs import SPECS
    from mbx_b200.tables import load_pip, load_fit
    names = argv or ["mbpol3b"]
    for name in names:
        q = build(name, SPECS[name], load_pip(name), load_fit(name))
        with open(path_of(name), "w") as f:
            json.dump(q, f, separators=(",", ":"))
        print("%s: basis %d (%d products), t %d..%d" % (name, len(q["basis"]), len(q["basis"]) - 1 - q["nvars"],
                                                         min(q["t"]), max(q["t"])))


if __name__ == "__main__":
    main()


# ---------------------------------------------------------------------------
# CUDA emission (the kernel is csrc/qf_kernel.cuh; this writes the
# polynomial-specific part: layout constants, row scales, A generation,
# epilogue, the host-side C assembly tables)

KB = 16                       # K block (tcgen05 kind::f16 K)
A_PART = 128 * KB * 2


def stage_bytes(q, s):
    return (3 if s * KB < q.nthird else 2) * q.npad * KB * 2


def stage_offset(q, s):
    return sum(stage_bytes(q, k) for k in range(s))


def image_bytes(q):
    return stage_offset(q, q.npad // KB)


# output columns of the kernel's passes, widest first.  Two passes of 240:
# one TMEM buffer (main + correction accumulator, 480 of the 512 columns),
# the read-back of a pass between its MMAs and the next pass's.  Passes of at
# most 128 columns (128, 128, 128, 96) get two buffers and overlap the
# read-back with the next pass, at twice the A generation: measured on the
# B200 (1.14 M trimers) 3.29 ms against 2.25 ms for two passes.
PASS_N = (240, 240)


def pass_col(p):
    return sum(PASS_N[:p])


def nparts(q, s):
    return 3 if s * KB < q.nthird else 2


def chunk_offset(q, s, p):
    """Offset of the (K block s, pass p) chunk: the passes' chunks of a block
    follow each other, each holding its FP16 parts (PASS_N[p] rows x 16)."""
    return stage_offset(q, s) + nparts(q, s) * pass_col(p) * KB * 2


def _f(x):
    return repr(float(x)) + "f" if float(x) != int(x) else "%d.0f" % int(x)


def emit_cuda(q, name, nvars):
    """Text of gen/<name>_qf.cuh for a QuadForm q."""
    assert q.npad == sum(PASS_N) == 480, "the kernel's passes cover 480 columns"
    ks = q.npad // KB
    kt = q.nthird // KB
    tmin, tmax = int(q.t[:q.nb].min()), int(q.t[:q.nb].max())
    nt = tmax - tmin + 1
    L = []
    w = L.append
    w("// Generated by mbx_b200/codegen/gen_kernels.py (codegen/qf.py) from mbx_b200/data/%s.qf.json -- do not edit." %
      name)
    w("// Quadratic form of the %s FP32-basis polynomial: %d basis members (padded to %d)," % (name, q.nb, q.npad))
    w("// K blocks of %d, the first %d with the third part of C." % (KB, kt))
    w("#pragma once")
    w('#include "../qf_kernel.cuh"')
    w("")
    w("// C' image (hi, mid[, lo] FP16 parts of every K block, K-major no-swizzle core")
    w("// matrices), written by mbx_set_coef_%s_s; per-column factors 2^-(s_j + t_j)" % name)
    w("__device__ __align__(128) unsigned char qf_img_%s[%d];" % (name, image_bytes(q)))
    w("__constant__ __align__(8) float qf_colf_%s[%d];   // read in pairs (colf2)" % (name, q.npad))
    w("__constant__ double qf_b0_%s[1];" % name)
    w("")
    w("struct %s_Q {" % name)
    w("    static constexpr int NB = %d, KS = %d, KT = %d, NT = %d, TMIN = %d;" % (q.npad, ks, kt, nt, tmin))
    w("    static constexpr long IMAGE_BYTES = %dL;" % image_bytes(q))
    w("    __host__ __device__ static constexpr long stage_offset(int s) {")
    w("        return s < KT ? s * %dL : %dL + (s - KT) * %dL;" % (3 * q.npad * KB * 2, kt * 3 * q.npad * KB * 2,
                                                               2 * q.npad * KB * 2))
    w("    }")
    w("    __host__ __device__ static constexpr int stage_bytes(int s) { return s < KT ? %d : %d; }" %
      (3 * q.npad * KB * 2, 2 * q.npad * KB * 2))
    w("    // passes over the output columns: pass p covers pass_n(p) columns from pass_col(p)")
    w("    static constexpr int NPASS = %d;" % len(PASS_N))
    sel_n = " : ".join("p == %d ? %d" % (i, n) for i, n in enumerate(PASS_N[:-1])) + " : %d" % PASS_N[-1]
    sel_c = " : ".join("p == %d ? %d" % (i, pass_col(i)) for i in range(len(PASS_N) - 1)) + \
        " : %d" % pass_col(len(PASS_N) - 1)
    w("    __host__ __device__ static constexpr int pass_n(int p) { return %s; }" % sel_n)
    w("    __host__ __device__ static constexpr int pass_col(int p) { return %s; }" % sel_c)
    w("    // the (K block s, pass p) chunk: the FP16 parts of pass_n(p) rows x 16")
    w("    __host__ __device__ static constexpr int parts(int s) { return s < KT ? 3 : 2; }")
    w("    __host__ __device__ static constexpr long chunk_offset(int s, int p) { return stage_offset(s) + "
      "(long)parts(s) * pass_col(p) * 32; }")
    w("    __host__ __device__ static constexpr int chunk_bytes(int s, int p) { return parts(s) * pass_n(p) * 32; }")
    w("    __device__ __forceinline__ static const unsigned char* image() { return qf_img_%s; }" % name)
    w("    __device__ __forceinline__ static double b0() { return qf_b0_%s[0]; }" % name)
    w("    // column scales of columns 2k and 2k + 1, for the paired FP32 multiply")
    w("    __device__ __forceinline__ static f2_t colf2(int k) { return reinterpret_cast<const f2_t*>(qf_colf_%s)[k]; }"
      % name)
    w("    // r = 2^(14 - e) with e = floor(log2(max(1, max|d|)^2 2^-TMIN)) + 1, so that every")
    w("    // |m_j(d) 2^-t_j| r < 2^14; sc[k] = r 2^-(TMIN + k); returns 1/r")
    w("    __device__ __forceinline__ static float row_scales(const float (&d)[%d], float (&sc)[NT]) {" % nvars)
    w("        float m = 1.0f;")
    w("#pragma unroll")
    w("        for (int v = 0; v < %d; ++v) m = fmaxf(m, fabsf(d[v]));" % nvars)
    w("        const float bound = m * m * %s;" % _f(2.0 ** (-tmin)))
    w("        const int e = ((__float_as_int(bound) >> 23) & 0xff) - 127 + 1;")
    w("#pragma unroll")
    w("        for (int k = 0; k < NT; ++k) sc[k] = __int_as_float((127 + 14 - e - (TMIN + k)) << 23);")
    w("        return __int_as_float((127 + e - 14) << 23);")
    w("    }")
    # A generation
    w("    // A values of K block s (basis members 16 s .. 16 s + 15): m_j(d) 2^-t_j r, hi/lo FP16")
    w("    __device__ __forceinline__ static void gen(int s, const float (&d)[%d], const float (&sc)[NT], "
      "uint32_t (&hi)[8], uint32_t (&lo)[8]) {" % nvars)
    w("        float a[16];")
    w("        switch (s) {")
    for s in range(ks):
        w("        case %d:" % s)
        for i in range(KB):
            j = s * KB + i
            if j >= q.nb:
                w("            a[%d] = 0.0f;" % i)
                continue
            b = q.basis[j]
            k = int(q.t[j]) - tmin
            if len(b) == 0:
                w("            a[%d] = sc[%d];" % (i, k))
            elif len(b) == 1:
                w("            a[%d] = d[%d] * sc[%d];" % (i, b[0], k))
            else:
                w("            a[%d] = (d[%d] * d[%d]) * sc[%d];" % (i, b[0], b[1], k))
        w("            break;")
    w("        default:")
    w("#pragma unroll")
    w("            for (int i = 0; i < 16; ++i) a[i] = 0.0f;")
    w("        }")
    w("#pragma unroll")
    w("        for (int i = 0; i < 8; ++i) qf::split2(a[2 * i], a[2 * i + 1], hi[i], lo[i]);")
    w("    }")
    # epilogue
    w("    // columns 16 c .. 16 c + 15 of Y, scaled: z_j = y_j 2^-(s_j + t_j) (y / r, scaled back by the")
    w("    // caller); adds z_j dm_j/dd to g and returns the chunk's share of the energy that g does not")
    w("    // carry: by Euler's identity for monomials of degree k, sum_u d_u dm/dd_u = k m, so")
    w("    // sum_j m_j z_j = z_const + (sum_{deg 1} d_u z_j + sum_u d_u g_u) / 2 over the pass,")
    w("    // and the degree-2 columns (all but 37) need no energy term of their own")
    w("    __device__ __forceinline__ static float epi(int c, const float (&z)[16], const float (&d)[%d], "
      "float (&g)[%d]) {" % (nvars, nvars))
    w("        float p = 0.0f;")
    w("        switch (c) {")
    for c in range(ks):
        w("        case %d:" % c)
        for i in range(KB):
            j = c * KB + i
            if j >= q.nb:
                continue
            b = q.basis[j]
            if len(b) == 0:
                w("            p += z[%d];" % i)
            elif len(b) == 1:
                w("            p = fmaf(0.5f * d[%d], z[%d], p);" % (b[0], i))
                w("            g[%d] += z[%d];" % (b[0], i))
            else:
                u, v = b
                w("            g[%d] = fmaf(z[%d], d[%d], g[%d]);" % (u, i, v, u))
                w("            g[%d] = fmaf(z[%d], d[%d], g[%d]);" % (v, i, u, v))
        w("            break;")
    w("        default:")
    w("            break;")
    w("        }")
    w("        return p;")
    w("    }")
    w("};")
    return "\n".join(L) + "\n"


def emit_host_tables(q, name):
    """C++ arrays for the host-side assembly of C from the orbit coefficients:
    per shifted monomial its (i, j) basis entry and orbit; the exponents t."""
    mi = ",".join(str(i) for i, _ in q.ij)
    mj = ",".join(str(j) for _, j in q.ij)
    mo = ",".join(str(int(o)) for o in q.sp.orbit_of)
    L = ["// quadratic form: entry (i, j) of every shifted monomial, its orbit; exponents t",
         "static const int qf_nmono_%s = %d;" % (name, len(q.ij)),
         "static const short qf_mi_%s[%d] = {%s};" % (name, len(q.ij), mi),
         "static const short qf_mj_%s[%d] = {%s};" % (name, len(q.ij), mj),
         "static const short qf_mo_%s[%d] = {%s};" % (name, len(q.ij), mo),
         "static const signed char qf_t_%s[%d] = {%s};" % (name, q.npad, ",".join(str(int(x)) for x in q.t))]
    return "\n".join(L) + "\n"


def image(q, b):
    """The kernel's B image (bytes) and column factors for orbit coefficients
    b: per K block s and pass p (columns pass_col(p) .. + PASS_N[p]), the FP16
    parts (hi, mid, and lo on the first nthird / 16 blocks) of
    B[n][k] = C'_kn 2^s_n, each part PASS_N[p] rows x 16, core matrix
    (n' / 8, k / 8) at (n' / 8) 128 + (k / 8) (PASS_N[p] / 8) 128 (row groups
    contiguous), row n' % 8 at 16 (n' % 8), n' = n - pass_col(p)."""
    (bh, bm, bl), f = q.operands(b)
    out = bytearray(image_bytes(q))
    kk = np.arange(KB)
    buf = np.frombuffer(out, np.uint8)
    for s in range(q.npad // KB):
        parts = (bh, bm, bl) if s * KB < q.nthird else (bh, bm)
        for pp, width in enumerate(PASS_N):
            n = np.arange(width)
            off = ((n[:, None] // 8) * 128 + (kk[None, :] // 8) * (width // 8) * 128 + (n[:, None] % 8) * 16 +
                   (kk[None, :] % 8) * 2)
            base = chunk_offset(q, s, pp)
            c0 = pass_col(pp)
            for p, part in enumerate(parts):
                vals = part[s * KB:(s + 1) * KB, c0:c0 + width].T.astype(np.float16).view(np.uint16)
                o = base + p * width * KB * 2 + off
                buf[o.ravel()] = (vals.ravel() & 0xff).astype(np.uint8)
                buf[(o + 1).ravel()] = (vals.ravel() >> 8).astype(np.uint8)
    return bytes(out), f.astype(np.float32)
