"""Coset form of a permutationally invariant polynomial: a small polynomial R
summed over a few variable permutations.

A PIP is P(x) = sum_k a_k sum_{m in O_k} m(x), every O_k an orbit of
monomials under the polynomial's permutation group G (48 permutations of the
MB-pol 3b variables: three waters times their two hydrogens).  For a subgroup
H of G and a left transversal T (G = union of t H over t in T),

    sum_{m in O} m(x) = |Stab_H(r)| / |Stab_G(r)| * sum_{t in T} sum_{m' in H r} m'(pi_t x)

for any representative r of O, where (pi_t x)_v = x_{p_t[v]}.  So

    P(x) = sum_{t in T} R(pi_t x),  R(y) = sum_k a'_k sum_{m' in H r_k} m'(y),
    a'_k = a_k * c_k * |Stab_H(r_k)| / |Stab_G(r_k)|,

(c_k the monomials' multiplicity in the table) and
grad P(x)_u = sum_t sum_{v : p_t[v] = u} (dR/dy_v)(pi_t x).

With r_k chosen to maximise |Stab_H(r_k)|, R of MB-pol 3b has 1,536 monomials
for an H of order 2 and |T| = 24, 1.10 times the 33,525 monomials of P in
total work -- but R's code is small enough to stay in the instruction cache
while it runs 24 times, where P's straight-line code (~10^5 instructions) is
fetched from L2 on every pass.

This is arithmetic of the polynomial, not of the reference's code: the
fitted coefficients and monomials are the same, only grouped differently.
"""
import collections

import numpy as np

from .shift import variable_group


def _act(p, mono):
    """Monomial m(pi x) as a monomial of x: variables v -> p[v]."""
    return tuple(sorted(p[v] for v in mono))


def _compose(a, b):
    return tuple(a[b[v]] for v in range(len(a)))


def _subgroups_of_order_2(group):
    ident = tuple(range(len(group[0])))
    return [frozenset((ident, g)) for g in group if g != ident and _compose(g, g) == ident]


CosetForm = collections.namedtuple("CosetForm", "perms monos k scale nterms_full order_h")


def coset_form(spec, table, group=None):
    """The coset form of table's polynomial with the best subgroup H of order
    2 (least total work): perms (the |T| permutations p_t), R's monomials and
    their coefficient index k, scale[k] (a'_k = a_k * scale[k])."""
    group = group or variable_group(spec, table)
    by_k = collections.defaultdict(list)
    mult = {}
    for t in range(table.nterms):
        k = int(table.k[t])
        m = tuple(sorted(table.var[t, :table.deg[t]].tolist()))
        by_k[k].append(m)
        if mult.setdefault(k, float(table.coef[t])) != float(table.coef[t]):
            raise ValueError("%s: coefficient %d has unequal multiplicities" % (table.name, k))
    orbits = {}
    for k, monos in by_k.items():
        o = set(monos)
        if {_act(g, monos[0]) for g in group} != o:
            raise ValueError("%s: coefficient %d is not one orbit of the group" % (table.name, k))
        orbits[k] = o
    best = None
    for H in _subgroups_of_order_2(list(group)):
        r_monos, r_k, scale = [], [], {}
        for k in sorted(orbits):
            o = orbits[k]
            rep = max(sorted(o), key=lambda m: sum(1 for h in H if _act(h, m) == m))
            stab_h = sum(1 for h in H if _act(h, rep) == rep)
            stab_g = len(group) // len(o)
            scale[k] = mult[k] * stab_h / stab_g
            for m in sorted({_act(h, rep) for h in H}):
                r_monos.append(m)
                r_k.append(k)
        work = len(r_monos) * (len(group) // 2)
        if best is None or work < best[0]:
            best = (work, H, r_monos, r_k, scale)
    _, H, r_monos, r_k, scale = best
    perms = []
    covered = set()
    for g in group:
        if g in covered:
            continue
        perms.append(g)
        covered |= {_compose(g, h) for h in H}
    if len(covered) != len(group):
        raise ValueError("transversal does not cover the group")
    ncoef = max(orbits) + 1
    sc = np.zeros(ncoef)
    for k, s in scale.items():
        sc[k] = s
    return CosetForm(perms, r_monos, r_k, sc, table.nterms, 2)


class CosetTable:
    """R of a coset form in the layout of tables.PipTable (k = coefficient
    index, multiplicity 1: the scale is folded into the coefficients)."""

    def __init__(self, cf, nvars, name):
        n = len(cf.monos)
        self.name = name
        self.nvars = nvars
        self.ncoef = len(cf.scale)
        self.nterms = n
        self.k = np.array(cf.k, np.int32)
        self.coef = np.ones(n)
        self.deg = np.array([len(m) for m in cf.monos], np.int32)
        width = max(4, int(self.deg.max()) if n else 4)
        self.var = np.full((n, width), -1, np.int32)
        for t, m in enumerate(cf.monos):
            self.var[t, :len(m)] = m


def evaluate(cf, a, x):
    """numpy check of the coset form: (P, dP/dx) at one point x."""
    a = np.asarray(a, float) * cf.scale
    e = 0.0
    g = np.zeros(len(x))
    for p in cf.perms:
        y = x[list(p)]
        for m, k in zip(cf.monos, cf.k):
            val = a[k] * np.prod(y[list(m)]) if m else a[k]
            e += val
            for i, v in enumerate(m):
                rest = [m[j] for j in range(len(m)) if j != i]
                g[p[v]] += a[k] * np.prod(y[rest])
    return e, g
