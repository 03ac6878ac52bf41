"""Shifted basis of a permutationally invariant polynomial, for FP32 evaluation.

The fitted MB-pol 3b polynomial P(x) = sum_k a_k sum_{m in orbit k} prod x_v
is evaluated as a sum of ~3e4 monomials whose values cancel to a small result:
summed over a liquid box, sum |a_k m(x)| exceeds |P| by ~10^5.  Products
rounded to FP32 (relative error ~1e-7) then leave ~1e-5 of the energy, too
much for a 1e-6 energy target.  Re-expanded around a reference point x0 in
the middle of the data,

    P(x) = sum_m b_m prod (x_v - x0_v),

the same polynomial has far smaller terms (the large constant and linear
parts are collected into a few coefficients), and FP32 monomials of
dx = x - x0 leave ~5e-8 of the 3b energy of a 2048-water box.

The reference point is chosen symmetric under the polynomial's permutation
group (the site permutations that map the term table onto itself), so the
shifted polynomial has the same symmetry: every monomial of one orbit of the
group carries one shared coefficient b_j, and the shifted coefficients fit in
constant memory (one per orbit) like the original ones.

``b = F a`` is linear in the fitted coefficients; F is kept as a sparse table
so that the library re-derives b whenever the coefficients change.
"""
import collections
import itertools

import numpy as np


def _element(site):
    return site[0]


def site_permutations(spec):
    """Candidate site permutations: identical monomers exchanged, identical
    elements exchanged within a monomer.  Only real sites are permuted."""
    first = [sum(spec.nat[:m]) for m in range(spec.nbody)]
    within = []
    for m in range(spec.nbody):
        idx = list(range(first[m], first[m] + spec.nat[m]))
        classes = collections.OrderedDict()
        for i in idx:
            classes.setdefault(_element(spec.sites[i]), []).append(i)
        perms = [dict()]
        for members in classes.values():
            perms = [{**p, **dict(zip(members, q))} for p in perms for q in itertools.permutations(members)]
        within.append(perms)
    out = []
    for order in itertools.permutations(range(spec.nbody)):
        if any(spec.monomers[order[m]] != spec.monomers[m] for m in range(spec.nbody)):
            continue
        if any(spec.nat[order[m]] != spec.nat[m] for m in range(spec.nbody)):
            continue
        for choice in itertools.product(*within):
            perm = {}
            for m in range(spec.nbody):
                # slot m takes the atoms of monomer order[m], relabelled within
                src = first[order[m]]
                for i, j in choice[m].items():
                    perm[src + (i - first[m])] = first[m] + (j - first[m])
            out.append(perm)
    return out


def variable_group(spec, table):
    """Permutations of the variables (tuples p with x'_v = x_{p[v]}) induced
    by site permutations that leave the term table invariant."""
    if spec.lp:
        raise NotImplementedError("%s: virtual sites" % spec.name)
    key = {}
    for v, (kind, s1, s2, k, d0) in enumerate(spec.variables):
        key[(kind, frozenset((s1, s2)), k, d0)] = v
    terms = set()
    for t in range(table.nterms):
        terms.add((int(table.k[t]), tuple(sorted(table.var[t, :table.deg[t]].tolist()))))
    group = []
    for perm in site_permutations(spec):
        p = []
        for kind, s1, s2, k, d0 in spec.variables:
            p.append(key.get((kind, frozenset((perm[s1], perm[s2])), k, d0)))
        if None in p:
            continue
        if all((k, tuple(sorted(p[v] for v in mono))) in terms for k, mono in terms):
            group.append(tuple(p))
    return group


def _variables(spec, xyz):
    """numpy restatement of the evaluator's variables for AoS n-mers."""
    out = np.empty((xyz.shape[0], spec.nvars))
    r = xyz.reshape(xyz.shape[0], -1, 3)
    for v, (kind, s1, s2, k, d0) in enumerate(spec.variables):
        d = np.linalg.norm(r[:, s1] - r[:, s2], axis=1)
        e = np.exp(k * (d0 - d))
        out[:, v] = e if kind == "exp" else e / d
    return out


def liquid_trimers(spec, seed=0):
    """Water trimers of a 256-molecule liquid box (1 g/cm3) that the
    evaluator's skip rule keeps, as AoS coordinates (minimum image)."""
    from mbx_b200 import workloads
    ids, xyz, box = workloads.water_256(seed)
    L = box[0]
    w = xyz.reshape(-1, 9)
    o = w[:, :3]
    n = len(w)
    d = o[:, None, :] - o[None, :, :]
    d -= L * np.round(d / L)
    r = np.linalg.norm(d, axis=2)
    near = r <= spec.rf
    np.fill_diagonal(near, False)
    out = set()
    for i in range(n):
        # i near both others: at most one of the three distances beyond rf
        for j, k in itertools.combinations(np.nonzero(near[i])[0].tolist(), 2):
            out.add(tuple(sorted((i, j, k))))
    res = []
    for i, j, k in sorted(out):
        a = w[i].reshape(3, 3)
        b = w[j].reshape(3, 3) - L * np.round((w[j][:3] - w[i][:3]) / L)
        c = w[k].reshape(3, 3) - L * np.round((w[k][:3] - w[i][:3]) / L)
        res.append(np.concatenate([a.reshape(-1), b.reshape(-1), c.reshape(-1)]))
    return np.array(res)


def reference_point(spec, table, group):
    """Per-variable medians over liquid trimers, averaged over each variable's
    orbit under the group (so that x0 is invariant)."""
    x = _variables(spec, liquid_trimers(spec))
    med = np.median(x, axis=0)
    x0 = np.zeros(spec.nvars)
    for v in range(spec.nvars):
        orbit = sorted({g[v] for g in group})
        x0[v] = np.mean(med[orbit])
    return x0


ShiftedPip = collections.namedtuple(
    "ShiftedPip", "nvars norb x0 monos orbit_of const_F F group")


def shifted(spec, table):
    """The shifted polynomial: monomials of dx with their orbit index, and the
    linear map from the fitted coefficients a to the orbit coefficients b
    (F[j] = {k: factor}; const_F = {k: factor} for the constant term)."""
    group = variable_group(spec, table)
    x0 = reference_point(spec, table, group)
    full = collections.defaultdict(lambda: collections.defaultdict(float))
    for t in range(table.nterms):
        k = int(table.k[t])
        c = float(table.coef[t])
        mono = table.var[t, :table.deg[t]].tolist()
        for r in range(len(mono) + 1):
            for keep in itertools.combinations(range(len(mono)), r):
                fac = c
                for i in range(len(mono)):
                    if i not in keep:
                        fac *= x0[mono[i]]
                full[tuple(sorted(mono[i] for i in keep))][k] += fac
    const_F = dict(full.pop((), {}))
    # orbits of the shifted monomials under the group
    orbit_id = {}
    reps = []
    for m in sorted(full, key=lambda m: (len(m), m)):
        if m in orbit_id:
            continue
        j = len(reps)
        reps.append(m)
        for g in group:
            orbit_id[tuple(sorted(g[v] for v in m))] = j
    monos = sorted(full, key=lambda m: (orbit_id[m], m))
    F = [dict(full[rep]) for rep in reps]
    return ShiftedPip(spec.nvars, len(reps), x0, monos, [orbit_id[m] for m in monos], const_F, F, group)


def shifted_coefficients(sp, a):
    """(b_const, b[norb]) for fitted coefficients a."""
    a = np.asarray(a, np.float64)
    b = np.array([sum(f * a[k] for k, f in row.items()) for row in sp.F])
    b0 = sum(f * a[k] for k, f in sp.const_F.items())
    return b0, b


class ShiftedTable:
    """The shifted monomials in the layout of tables.PipTable (k = orbit)."""

    def __init__(self, sp, name):
        n = len(sp.monos)
        self.name = name
        self.nvars = sp.nvars
        self.ncoef = sp.norb
        self.nterms = n
        self.k = np.array(sp.orbit_of, np.int32)
        self.coef = np.ones(n)
        self.deg = np.array([len(m) for m in sp.monos], np.int32)
        self.var = np.full((n, 4), -1, np.int32)
        for t, m in enumerate(sp.monos):
            self.var[t, :len(m)] = m
