"""CUDA path against the oracle and the reference's golden vectors (GPU).

Tolerances: FP64 path energies within 1e-10 relative and gradients within
1e-8 kcal/mol/A of the FP64 oracle.  Mixed path (MB-pol 3b in a paired FP32
trie over a shifted basis, everything else FP64): total 2b+3b energy of a
liquid box within 1e-6 relative, each term within 2e-6, forces within
1e-3 kcal/mol/A; gas-phase n-mers, away from the basis' reference point,
within 1e-5.  n-mer lists must be identical after canonicalisation.
"""
import os
import sys

import numpy as np
import pytest

import mbx_oracle as mo
from conftest import GOLDEN, golden
from mbx_b200 import system as msys, workloads
from mbx_b200.specs import ALKALI, HALIDES, SPECS
from mbx_b200.tables import load_fit

pytestmark = pytest.mark.gpu
sys.path.insert(0, GOLDEN)

E_REL = 1e-10
G_ABS = 1e-8
# A single n-mer's polynomial is a sum of terms up to ~1e6 times larger than
# the result (condition numbers median 8e5, max 2e10 for MB-pol 2b), so two
# FP64 evaluations in different orders agree to ~1e-9 kcal/mol per n-mer,
# not to 1e-10 relative; per-n-mer energies are compared absolutely.
E_ABS_NMER = 1e-8
# CO2 models whose intramolecular variables exp(k (d0 - r)) are far above 1
# (up to 32): their degree-5 polynomials sum terms up to ~1e8 times a
# dimer's energy, so FP64 evaluation orders differ by ~1e-16 of that sum:
# up to ~4e-8 kcal/mol per dimer between the oracle's term sums and the
# reference's Horner program (the trie here lands within 2e-9 of the
# reference on its co2cm580 golden, the oracle 4e-8 off).  These compare
# within 1e-6 kcal/mol per dimer (or 1e-8 relative) and 1e-6 kcal/mol/A, or
# 1e-8 of the largest force.
ILL_CONDITIONED = {"cm595co22b", "cm590co22b", "cm585co22b", "cm5875co22b", "cm580co22b"}
ILL_E_REL = 1e-8
ILL_E_ABS = 1e-6


def g_tol(name, go):
    return max(1e-6, 1e-8 * np.abs(go).max()) if name in ILL_CONDITIONED else G_ABS


def e_close(name, e, eo, n=1):
    if name in ILL_CONDITIONED:
        return rel(e, eo) < ILL_E_REL or abs(e - eo) < ILL_E_ABS * n
    return rel(e, eo) < E_REL or abs(e - eo) < E_ABS_NMER
MIXED_REL = 1e-6          # total 2b+3b energy of a liquid box; also each term's error against |E2B| + |E3B|
MIXED_REL_TERM = 2e-6     # one term (2b or 3b) of the 2048-water box, relative to itself
MIXED_REL_GAS = 1e-5      # sums over random gas-phase n-mers of accessible geometry (below)
MIXED_FORCE = 1e-3        # kcal/mol/A, largest force error of a liquid box
# The mixed MB-pol 3b kernel accumulates on the tensor cores, whose FP32
# accumulation aligns every addend of an MMA to the largest and truncates: its
# error grows with the cancellation of the polynomial, which is strongest when
# two waters are closer than liquid water ever brings them.
MIXED_RMIN = 2.5           # A: first-atom separations at and above this are "accessible" (liquid, clusters)
MIXED_NMER_ABS = 1.5e-4    # kcal/mol, one trimer of accessible geometry (B200: at most 8.8e-5 measured)
MIXED_NMER_ABS_CLOSE = 5e-4  # kcal/mol, one trimer with waters closer than MIXED_RMIN (B200: 2.1e-4 measured)
MIXED_NMER_GRAD = 3e-4     # kcal/mol/A, gradient of one trimer of accessible geometry (B200: at most 2.0e-4
                           # measured, a trimer at 2.51 A; 1.3e-6 on average)
FP32_TYPES = ("mbpol3b",)  # types with a mixed-precision kernel; the rest run FP64 when mixed


def canon(nm):
    nm = np.sort(np.asarray(nm, np.int64), axis=1)
    return nm[np.lexsort(nm.T[::-1])] if len(nm) else nm


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


# ------------------------------------------------------------------ polynomials
STRAIGHT = ["mbpol2b", "mbpol3b", "ch4h2o2b", "ch4h2o3b", "h2oli2b", "h2ocs2b", "h2ona3b"]


@pytest.mark.parametrize("name", STRAIGHT)
def test_poly_random_vs_oracle(ctx, name):
    nv = SPECS[name].nvars
    rng = np.random.default_rng(7)
    nd = 257
    x = rng.uniform(0.05, 1.2, size=(nv, nd))
    g = np.zeros((nv, nd))
    e = ctx.poly(name, np.ascontiguousarray(x), g)
    a = load_fit(name)
    for i in range(0, nd, 37):
        eo, go = mo.pip_eval(name, a, x[:, i])
        assert rel(e[i], eo) < E_REL or abs(e[i] - eo) < 1e-12
        np.testing.assert_allclose(g[:, i], go, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("fixture,name", [("poly_mbpol2b", "mbpol2b"), ("poly_ch4h2o2b", "ch4h2o2b"),
                                          ("poly_ch4h2o3b", "ch4h2o3b"), ("poly_mbpol3b", "mbpol3b"),
                                          ("poly_h2oion2b", "h2oli2b"), ("poly_h2oion3b", "h2oli3b")])
def test_poly_golden(ctx, fixture, name):
    gd = golden(fixture)
    nv = SPECS[name].nvars
    x = np.array(gd["x"])
    x = x.reshape(nv, -1)[:, 0] if len(x) != nv else x
    ctx.set_coefficients(name, np.array(gd["a"]))
    try:
        g = np.zeros((nv, 1))
        e = ctx.poly(name, np.ascontiguousarray(x.reshape(nv, 1)), g)
    finally:
        ctx.set_coefficients(name, None)
    gexp = np.array(gd["g_expected"])
    gexp = gexp.reshape(nv, -1)[:, 0] if len(gexp) != nv else gexp
    e_exp = gd["e_expected"][0] if isinstance(gd["e_expected"], list) else gd["e_expected"]
    assert abs(e[0] - e_exp) < 1e-8 * max(1, abs(e_exp))
    np.testing.assert_allclose(g[:, 0], gexp, rtol=1e-8, atol=1e-8)


# ------------------------------------------------------------------ evaluators
HOLDERS = [("holder2b_x2b_v9x", "mbpol2b"), ("holder2b_ch4_h2o", "ch4h2o2b"), ("holder2b_ch4_ch4", "ch4ch42b"),
           ("holder3b_x3b_v2x", "mbpol3b"), ("holder3b_ch4_h2o_h2o", "ch4h2o3b")]
HOLDERS += [("holder2b_h2o_%s" % ion, "h2o%s2b" % ion) for ion in ("li", "na", "k", "rb", "cs")]
HOLDERS += [("holder3b_h2o_h2o_%s" % ion, "h2o%s3b" % ion) for ion in ("li", "na", "k", "rb", "cs")]
HOLDERS += [("holder2b_%s_h2o" % h, "%sh2o2b" % h) for h in ("f", "cl", "br", "i")]
HOLDERS += [("holder3b_%s_h2o_h2o" % h, "%sh2o3b" % h) for h in ("f", "cl", "br", "i")]
HOLDERS += [("holder2b_ar_ar", "arar2b"), ("holder2b_cl_cl", "clcl2b"), ("holder2b_na_na", "nana2b"),
            ("holder2b_na_cl", "nacl2b"), ("holder2b_ar_cs", "csar2b"), ("holder2b_ar_h2o", "arh2o2b")]
HOLDERS += [("holder2b_h2_h2", "h2h22b"), ("holder2b_h2_h2o", "h2oh22b"), ("holder2b_nh3_nh3", "nh3nh32b"),
            ("holder2b_nh3pbe_nh3pbe", "nh3pbe2b"), ("holder2b_cs_h2", "csh22b"), ("holder2b_mbpbe_mbpbe", "mbpbe2b"),
            ("holder2b_ch4_co2", "ch4co22b"), ("holder3b_mbpbe_mbpbe_mbpbe", "mbpbe3b"),
            ("holder3b_co2_co2_co2", "co23b"), ("holder2b_co2a_co2a", "co2a2b"), ("holder2b_co2_co2", "co2co22b"),
            ("holder2b_h2o_co2", "h2oco22b")]
HOLDERS += [("holder2b_h2o_n2o5", "n2o5h2o2b"), ("holder3b_n2o5_h2o_h2o", "n2o5h2o3b")]
HOLDERS += [("holder2b_%s" % m, m[3:] + "co22b")
            for m in ("co2cm5100", "co2cm595", "co2cm590", "co2cm5875", "co2cm585", "co2cm580")]
HOLDERS += [("holder2b_h2o_co2a", "h2oco2a2b")]
# fixtures whose test passes the monomers to the holder in another order
# (holder slot i <- xyz(order[i] + 1))
HOLDER_ORDER = {"holder2b_h2_h2o": (1, 0), "holder2b_h2o_n2o5": (1, 0)}


@pytest.mark.parametrize("fixture,name", HOLDERS)
def test_evaluator_golden(ctx, fixture, name):
    gd = golden(fixture)
    s = SPECS[name]
    n = gd.get("ndim", gd.get("ntrim"))
    order = HOLDER_ORDER.get(fixture, range(s.nbody))
    blocks = [np.array(gd["xyz%d" % (k + 1)]).reshape(n, -1) for k in order]
    xyz = np.ascontiguousarray(np.concatenate(blocks, axis=1))
    grad = np.zeros_like(xyz)
    vir = np.zeros(9)
    e = ctx.evaluate(name, xyz, grad, vir)
    eo, go, vo, _ = mo.holder_eval(name, xyz)
    assert abs(e - gd["energy_expected"]) < 1e-6
    assert e_close(name, e, eo)
    np.testing.assert_allclose(grad, go, rtol=0, atol=g_tol(name, go))
    np.testing.assert_allclose(vir, vo, rtol=1e-10 if name not in ILL_CONDITIONED else 1e-7, atol=g_tol(name, go))
    off = 0
    for i, k in enumerate(order):
        w = blocks[i].shape[1]
        np.testing.assert_allclose(grad[:, off:off + w].reshape(-1), gd["grad%d_expected" % (k + 1)], atol=1e-6)
        off += w


def random_nmers(name, n, seed=3):
    """Gas-phase n-mers of the evaluator's types spanning its cutoff."""
    s = SPECS[name]
    rng = np.random.default_rng(seed)
    bodies = {m: f() for m, f in workloads.BODIES.items()}
    for ion in ALKALI + HALIDES + ("ar", "he"):
        bodies[ion] = np.zeros((1, 3))
    out = []
    for _ in range(n):
        parts = []
        centre0 = np.zeros(3)
        for k, m in enumerate(s.monomers):
            # first-atom separations from contact (3.2 A for the 2.3 A long CO2) to beyond the cutoff
            # He-He from 6 A: its degree-23 polynomial is ill-conditioned closer in; N2O5 (terminal O
            # 2.25 A from the bridging O) from 3 A
            # the ill-conditioned CO2 models from 4.5 A (ILL_CONDITIONED)
            rmin = (4.5 if name in ILL_CONDITIONED else 3.2 if any(m.startswith("co2") for m in s.monomers) else
                    6.0 if name == "hehe2b" else 3.0 if "n2o5" in s.monomers else 2.4)
            c = centre0 if k == 0 else workloads._random_directions(rng, 1)[0] * rng.uniform(rmin, s.rf + 0.5)
            parts.append(workloads.place(rng, bodies[m], c[None, :])[0].reshape(-1))
        out.append(np.concatenate(parts))
    return np.ascontiguousarray(np.array(out))


@pytest.mark.parametrize("name", list(SPECS))
def test_evaluator_random_vs_oracle(ctx, name):
    n = 64 if name == "ch4ch42b" else 512
    xyz = random_nmers(name, n)
    grad = np.zeros_like(xyz)
    vir = np.zeros(9)
    eper = np.zeros(n)
    e = ctx.evaluate(name, xyz, grad, vir, eper)
    eo, go, vo, epo = mo.holder_eval(name, xyz, per_nmer=True)
    ill = name in ILL_CONDITIONED
    assert e_close(name, e, eo, n)
    np.testing.assert_allclose(eper, epo, rtol=ILL_E_REL if ill else 0, atol=ILL_E_ABS if ill else E_ABS_NMER)
    np.testing.assert_allclose(grad, go, rtol=0, atol=g_tol(name, go))
    np.testing.assert_allclose(vir, vo, rtol=1e-7 if ill else 1e-9, atol=1e-6 if ill else 1e-8)


def first_atom_min_distance(name, xyz):
    """Smallest distance between the first atoms of the n-mer's monomers."""
    s = SPECS[name]
    first = np.cumsum([0] + list(s.nat[:-1]))
    r = xyz.reshape(len(xyz), -1, 3)[:, first, :]
    return np.min([np.linalg.norm(r[:, i] - r[:, j], axis=1)
                   for i in range(len(first)) for j in range(i + 1, len(first))], axis=0)


@pytest.mark.parametrize("name", ["mbpol2b", "mbpol3b", "ch4h2o2b", "ch4h2o3b"])
def test_evaluator_mixed(ctx, name):
    xyz = random_nmers(name, 512, seed=11)
    grad = np.zeros_like(xyz)
    eper = np.zeros(len(xyz))
    e = ctx.evaluate(name, xyz, grad, None, eper, mixed=True)
    eo, go, _, epo = mo.holder_eval(name, xyz, per_nmer=True)
    if name in FP32_TYPES:
        # The random generator places monomers 1 and 2 independently around
        # monomer 0, so some trimers have two waters closer than MIXED_RMIN
        # (overlapping, down to < 1 A): there the per-trimer bound is wider;
        # the budget on sums applies to the accessible trimers.
        acc = first_atom_min_distance(name, xyz) >= MIXED_RMIN
        err = np.abs(eper - epo)
        assert rel(eper[acc].sum(), epo[acc].sum()) < MIXED_REL_GAS, (eper[acc].sum(), epo[acc].sum())
        assert err[acc].max() < MIXED_NMER_ABS, err[acc].max()
        assert err.max() < MIXED_NMER_ABS_CLOSE, err.max()
        assert np.abs(grad - go).max() < 1e-5 * np.abs(go).max()
    else:
        # no FP32 kernel for this type: the mixed mode evaluates it in FP64
        assert rel(e, eo) < E_REL or abs(e - eo) < E_ABS_NMER
        np.testing.assert_allclose(grad, go, rtol=0, atol=G_ABS)


def accessible_nmers(name, n, seed):
    """n random gas-phase n-mers whose first atoms are all at least
    MIXED_RMIN apart."""
    xyz = random_nmers(name, 4 * n + 16, seed=seed)
    xyz = xyz[first_atom_min_distance(name, xyz) >= MIXED_RMIN]
    assert len(xyz) >= n
    return np.ascontiguousarray(xyz[:n])


def test_mixed_odd_counts(ctx):
    """Mixed kernel: n-mer counts that fill a tile of 128 partly, once or
    twice over; every n-mer evaluated, the total the sum of the per-n-mer
    energies."""
    for n in (1, 2, 3, 127, 129, 255, 257, 513):
        xyz = accessible_nmers("mbpol3b", n, seed=n)
        grad = np.zeros_like(xyz)
        eper = np.zeros(n)
        e = ctx.evaluate("mbpol3b", xyz, grad, None, eper, mixed=True)
        eo, go, _, epo = mo.holder_eval("mbpol3b", xyz, per_nmer=True)
        np.testing.assert_allclose(eper, epo, rtol=0, atol=MIXED_NMER_ABS)
        assert abs(e - eper.sum()) < 1e-12 * max(1.0, np.abs(eper).sum()), n
        assert np.abs(grad - go).max() < MIXED_NMER_GRAD, n


@pytest.mark.parametrize("name", ["mbpol2b", "mbpol3b", "ch4h2o2b", "ch4h2o3b"])
def test_dcoef_vs_oracle(ctx, name):
    xyz = random_nmers(name, 96, seed=5)
    w = np.random.default_rng(1).normal(size=len(xyz))
    out = ctx.evaluate_dcoef(name, xyz, w)
    ref = (mo.holder_dcoef(name, xyz) * w[:, None]).sum(0)
    np.testing.assert_allclose(out, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


# ------------------------------------------------------------------ systems
def compare_system(ids, xyz, box, c2, c3, ig2=(), ig3=(), mixed=False, lists=True, g_rtol=0.0, e_rtol=E_REL,
                   g_atol=G_ABS):
    o = mo.OracleSystem(ids, xyz, box, c2, c3, ig2, ig3)
    g = msys.from_arrays(ids, xyz, box, c2, c3, ig2, ig3, precision="mixed" if mixed else "fp64")
    etot, etot_o = 0.0, 0.0
    terms = []
    for nb in (2, 3):
        eo = o.energy(nb)
        go = o.real_grads()
        vo = o.virial.copy()
        e = g.TwoBodyEnergy(True) if nb == 2 else g.ThreeBodyEnergy(True)
        gr = g.GetRealGrads()
        vr = g.GetVirial()
        etot += e
        etot_o += eo
        terms.append((nb, e, eo))
        if mixed:
            assert np.abs(np.asarray(gr) - go).max() < MIXED_FORCE, nb
        else:
            assert rel(e, eo) < e_rtol, (nb, e, eo)
            np.testing.assert_allclose(gr, go, rtol=g_rtol, atol=g_atol)
            np.testing.assert_allclose(vr, vo, rtol=1e-9 if e_rtol < 1e-9 else 1e-7, atol=1e-7)
        if lists:
            cut = c2 if nb == 2 else c3
            assert np.array_equal(canon(g.GetPairList(nb, cut)), o.top.nmers_to_input(o.nmers(nb))), nb
            listed, _ = g.NmerCounts(nb)
            assert listed == len(o.nmers(nb))
    if mixed:
        # each term's error within the 1e-6 budget of the total energy, and
        # the total within 1e-6 (a small term, like E3B of a CH4-rich box,
        # may be off by more than 1e-6 of itself)
        scale = sum(abs(eo) for _, _, eo in terms)
        for nb, e, eo in terms:
            assert abs(e - eo) < MIXED_REL * scale, (nb, e, eo)
        assert rel(etot, etot_o) < MIXED_REL, (etot, etot_o)
    return g


def test_water_256_fp64():
    ids, xyz, box = workloads.water_256(0)
    compare_system(ids, xyz, box, 9.0, 7.0)


def test_water_256_mixed():
    ids, xyz, box = workloads.water_256(0)
    compare_system(ids, xyz, box, 9.0, 7.0, mixed=True, lists=False)


@pytest.mark.parametrize("fixture", ["system_256_h2o_cubic_box", "system_57_ch4_513_h2o"])
def test_published_fixtures(fixture):
    gd = golden(fixture)
    g = compare_system(gd["ids"], np.array(gd["xyz"]), gd["box"] or None, gd["cutoff2b"], gd["cutoff3b"],
                       gd["ignore_2b"], gd["ignore_3b"])
    e2 = g.TwoBodyEnergy(False)
    e3 = g.ThreeBodyEnergy(False)
    assert abs(e2 - gd["E2B"]) < 1e-9 * abs(gd["E2B"]) + 1e-8
    assert abs(e3 - gd["E3B"]) < 1e-9 * abs(gd["E3B"]) + 1e-8


def test_methane_water_box():
    ids, xyz, box = workloads.methane_water_box(seed=0)
    compare_system(ids, xyz, box, 9.0, 7.0)


def test_methane_water_box_mixed():
    """Mixed MB-nrg system (57 CH4 + 513 H2O): the water trimers go through the
    paired FP32 kernel, every CH4 type stays FP64."""
    ids, xyz, box = workloads.methane_water_box(seed=0)
    compare_system(ids, xyz, box, 9.0, 7.0, mixed=True, lists=False)


@pytest.mark.parametrize("ion", ALKALI + HALIDES)
def test_ion_water_box(ion):
    """256-site box with three alkali ions: the ion-water dimers and the
    water-water-ion trimers through the ion kernels (FP64 in both modes),
    lists, energies, gradients and virial against the oracle."""
    ids, xyz, box = workloads.ion_water_box([ion] * 3, seed=1)
    compare_system(ids, xyz, box, 9.0, 7.0)


@pytest.mark.parametrize("ions", [("na+", "cl-", "na+", "cl-", "na+", "cl-"), ("ar", "ar", "ar"),
                                  ("cs+", "ar", "cs+", "ar"), ("li+", "f-", "k+", "br-")])
def test_solution_box(ions):
    """Salt solutions and argon in water: every pair type of the box (ion-ion
    and atom-atom included) and the ion trimers on the GPU against the
    oracle; five monomer types in the last one."""
    ids, xyz, box = workloads.ion_water_box(list(ions), seed=4)
    compare_system(ids, xyz, box, 9.0, 7.0)


@pytest.mark.parametrize("ids,L", [(["nh3"] * 200, 19.72), (["nh3pbe0d3bj"] * 200, 19.72),
                                   (["h2"] * 60 + ["h2o"] * 150 + ["cs+"] * 2, 19.72), (["mbpbe"] * 220, 19.72),
                                   (["ch4"] + ["h2o"] * 180 + ["na+", "cl-"], 19.72), (["co2"] * 200, 26.0),
                                   (["co2_archive"] * 200, 26.0), (["co2"] * 30 + ["h2o"] * 250, 22.0),
                                   (["he"] + ["h2o"] * 220, 19.72), (["n2o5"] * 10 + ["h2o"] * 250, 26.0),
                                   (["co2cm590"] * 100 + ["co2cm585"] * 100, 30.0),
                                   (["co2cm5875"] * 100 + ["co2cm580"] * 100, 30.0),
                                   (["co2cm5100"] * 30 + ["co2cm595"] * 30 + ["h2o"] * 220, 22.0),
                                   (["co2_archive"] * 30 + ["h2o"] * 250, 22.0)])
def test_molecule_box(ids, L):
    """Liquids and mixtures of the MB-nrg types beyond water and ions on the
    GPU against the oracle (the boxes the oracle is checked on against the
    compiled reference).  Randomly oriented molecules on a lattice have close
    contacts with forces of 10^2-10^4 kcal/mol/A, where two FP64 summation
    orders differ by ~1e-11 of the force: gradients within 1e-8 absolute
    plus 1e-10 relative."""
    ids, xyz, box = workloads.molecule_box(ids, L=L, seed=3)
    if any(m in ("co2cm595", "co2cm590", "co2cm585", "co2cm5875", "co2cm580") for m in ids):
        # ill-conditioned CO2 models (ILL_CONDITIONED)
        compare_system(ids, xyz, box, 9.0, 7.0, e_rtol=ILL_E_REL, g_atol=1e-6)
    else:
        compare_system(ids, xyz, box, 9.0, 7.0, g_rtol=1e-10)


def test_helium_dilute():
    """He in water with He-He pairs at 6.5 A and more (the He-He polynomial
    is ill-conditioned at shorter range)."""
    ids, xyz, box = workloads.dilute_box("he", 10, seed=1)
    compare_system(ids, xyz, box, 9.0, 7.0)


def test_ion_water_box_mixed():
    ids, xyz, box = workloads.ion_water_box(["na+", "cl-", "k+"], seed=2)
    compare_system(ids, xyz, box, 9.0, 7.0, mixed=True, lists=False)


def test_gas_phase_cluster():
    ids, xyz = workloads.water_cluster(40, seed=2)
    compare_system(ids, xyz, None, 9.0, 7.0)


def test_edge_cases(ctx):
    # one monomer: no n-mers, zero energy
    ids, xyz, box = workloads.water_256(0)
    one = msys.from_arrays(ids[:1], xyz[:9], box, 9.0, 7.0)
    assert one.TwoBodyEnergy(True) == 0.0 and one.ThreeBodyEnergy(True) == 0.0
    # two monomers far apart: listed but not evaluated
    far = np.concatenate([xyz[:9], xyz[:9] + np.array([8.0, 0, 0] * 3)])
    s = msys.from_arrays(["h2o", "h2o"], far, box, 9.0, 7.0)
    assert s.TwoBodyEnergy(True) == 0.0
    assert s.NmerCounts(2) == (1, 0)
    # cutoff beyond half the box: the reference assumes it never happens; here it is an error
    with pytest.raises(msys.CUException):
        msys.from_arrays(ids, xyz, box, 11.0, 7.0)
    # ignored type tuples contribute nothing
    ig = msys.from_arrays(ids, xyz, box, 9.0, 7.0, ignore_3b=[["h2o", "h2o", "h2o"]])
    assert ig.ThreeBodyEnergy(True) == 0.0
    assert ig.NmerCounts(3)[0] > 0


def test_ghost_monomers():
    """use_ghost: ghosts join the search, only n-mers owned by a local monomer count."""
    ids, xyz, box = workloads.water_256(0)
    is_local = np.ones(len(ids), int)
    is_local[::3] = 0
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0, is_local=is_local)
    g = msys.System()
    names = ["O", "H", "H"]
    for i in range(len(ids)):
        g.AddMonomer(xyz[9 * i:9 * i + 9], names, "h2o", int(is_local[i]))
        g.AddMolecule([i])
    g.Initialize()
    g.SetUpFromJson({"MBX": {"box": list(box), "twobody_cutoff": 9.0, "threebody_cutoff": 7.0}})
    for nb in (2, 3):
        eo = o.energy(nb, use_ghost=True)
        e = g.TwoBodyEnergy(True, True) if nb == 2 else g.ThreeBodyEnergy(True, True)
        assert rel(e, eo) < E_REL
        np.testing.assert_allclose(g.GetRealGrads(), o.real_grads(), atol=G_ABS)


def ref_fixture(name):
    """The reference's own results on a seeded workload (tests/golden/ref_<name>.npz,
    written by tests/golden/make_ref_fixtures.py from the compiled reference)."""
    from make_ref_fixtures import WORKLOADS, xyz_hash
    make_fn, c2, c3 = WORKLOADS[name]
    ids, xyz, box = make_fn()
    d = np.load(os.path.join(GOLDEN, "ref_%s.npz" % name))
    assert str(d["xyz_sha256"]) == xyz_hash(xyz), "workload %s no longer matches its fixture" % name
    return ids, xyz, box, c2, c3, d


@pytest.mark.parametrize("name", ["water_256", "water_2048", "methane_water"])
def test_fp64_vs_reference(name):
    """The FP64 path against the reference's own TwoBodyEnergy(true) /
    ThreeBodyEnergy(true) (bblock/system.cpp:2403-2423, 2727-2745): energies
    within 1e-10 relative, gradients within 1e-8 kcal/mol/A, virials, and the
    n-mer lists identical to the reference's (same length, same canonical
    hash).  2048 waters is the bench workload at full size."""
    from make_ref_fixtures import list_hash
    ids, xyz, box, c2, c3, d = ref_fixture(name)
    g = msys.from_arrays(ids, xyz, box, c2, c3)
    for nb, cut in ((2, c2), (3, c3)):
        e = g.TwoBodyEnergy(True) if nb == 2 else g.ThreeBodyEnergy(True)
        gr = np.asarray(g.GetRealGrads())
        vr = np.asarray(g.GetVirial())
        er = float(d["e%d" % nb])
        assert rel(e, er) < E_REL, (nb, e, er)
        np.testing.assert_allclose(gr, d["g%d" % nb], rtol=0, atol=G_ABS)
        np.testing.assert_allclose(vr, d["v%d" % nb], rtol=1e-10, atol=1e-7)
        nm = canon(g.GetPairList(nb, cut))
        assert len(nm) == int(d["n%d" % nb]) and list_hash(nm) == str(d["l%d_sha256" % nb]), nb


@pytest.mark.parametrize("name", ["water_256", "water_256_bead", "water_2048", "methane_water"])
def test_onebody_vs_reference(name):
    """System::OneBodyEnergy(true) (bblock/system.cpp:2140): the GPU
    Partridge-Schwenke term against the reference's, energy within 1e-10
    relative (or 1e-9 kcal/mol per water: a near-equilibrium water's energy
    is a small difference of terms ~10^5 times larger), gradients within
    1e-8 kcal/mol/A, virial."""
    ids, xyz, box, c2, c3, d = ref_fixture(name)
    g = msys.from_arrays(ids, xyz, box, c2, c3)
    for do_grads in (True, False):
        e = g.OneBodyEnergy(do_grads)
        er = float(d["e1"])
        assert rel(e, er) < E_REL or abs(e - er) < 1e-9 * len(ids), (e, er)
    g.OneBodyEnergy(True)
    np.testing.assert_allclose(g.GetRealGrads(), d["g1"], rtol=0, atol=G_ABS)
    np.testing.assert_allclose(g.GetVirial(), d["v1"], rtol=1e-10, atol=1e-8)
    assert g.NmerCounts(1)[0] == len(ids)


def test_onebody_refuses_cpu_only_types():
    """A monomer type whose 1-body term the reference has but the GPU path
    does not (NH3) makes the 1-body call fail loudly, unless ignored; the
    ignored type then contributes nothing."""
    rng = np.random.default_rng(4)
    ids = ["h2o"] * 6 + ["nh3"] * 2
    parts = []
    for k, m in enumerate(ids):
        centre = np.array([4.0 * (k % 4), 4.0 * (k // 4), 0.0])
        parts.append(workloads.place(rng, workloads.BODIES[m](), centre[None, :])[0].reshape(-1))
    xyz = np.concatenate(parts)
    g = msys.from_arrays(ids, xyz, None, 9.0, 7.0)
    with pytest.raises(Exception, match="1-body"):
        g.OneBodyEnergy(True)
    g.ignore_1b = ["nh3"]
    g._push_config()
    e = g.OneBodyEnergy(True)
    w = msys.from_arrays(ids[:6], np.concatenate(parts[:6]), None, 9.0, 7.0)
    assert abs(e - w.OneBodyEnergy(True)) <= 1e-12 * abs(e)


def test_water_box_three_cells_per_axis():
    """A box with exactly 3 cells per axis for both cutoffs (27.5 A: 9.17 A
    cells), the tightest case of the neighbour search's one-copy test (every
    cell a neighbour of every other, each member reached through exactly the
    copy its cell's wrap names): lists, energies, gradients and virials
    against the restatement."""
    ids, xyz, box = workloads.water_box(n_side=9, n_mol=694, L=27.5, seed=5)
    compare_system(ids, xyz, box, 9.0, 7.0)


def triclinic_water_box(n_side=9, n_mol=700, L=30.0, shear=(0.15, 0.1, 0.12), seed=6, jitter=0.3):
    """Waters on a lattice in the fractional coordinates of a triclinic box
    (lattice vectors a = (L, 0, 0), b = (s0 L, L, 0), c = (s1 L, s2 L, L), the
    lower-triangular form the reference's fractional coordinates assume), so
    that periodic images keep the lattice spacing."""
    rng = np.random.default_rng(seed)
    B = np.array([[L, 0, 0], [shear[0] * L, L, 0], [shear[1] * L, shear[2] * L, L]], float)
    g = (np.arange(n_side) + 0.5) / n_side - 0.5
    frac = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pick = rng.choice(len(frac), size=n_mol, replace=False)
    centres = frac[pick] @ B + rng.uniform(-jitter, jitter, size=(n_mol, 3))
    xyz = workloads.place(rng, workloads.water_body(), centres)
    return ["h2o"] * n_mol, xyz.reshape(-1), B.reshape(-1)


def test_water_box_triclinic():
    """A triclinic box (perpendicular widths 29.6-30 A: 3 cells per axis for
    the 2b cutoff, 4 for the 3b one), where the neighbour search's cells are
    parallelepipeds and its one-copy test rests on their perpendicular
    widths: lists, energies, gradients and virials against the restatement."""
    ids, xyz, box = triclinic_water_box()
    compare_system(ids, xyz, box, 9.0, 7.0)


def test_water_2048_lists_vs_restatement():
    """The full-size lists also equal the oracle restatement's, n-mer by n-mer."""
    ids, xyz, box = workloads.water_2048(0)
    g = msys.from_arrays(ids, xyz, box, 9.0, 7.0)
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0)
    for nb in (2, 3):
        cut = 9.0 if nb == 2 else 7.0
        assert np.array_equal(canon(g.GetPairList(nb, cut)), o.top.nmers_to_input(o.nmers(nb)))


def test_water_2048_mixed():
    """The mixed path (MB-pol 3b in the paired FP32 kernel) on the bench
    workload against the reference: each term within 2e-6 of itself, the
    2b+3b total within 1e-6."""
    ids, xyz, box, c2, c3, d = ref_fixture("water_2048")
    r2, r3 = float(d["e2"]), float(d["e3"])
    m = msys.from_arrays(ids, xyz, box, c2, c3, precision="mixed")
    e2 = m.TwoBodyEnergy(True)
    e3 = m.ThreeBodyEnergy(True)
    assert rel(e2, r2) < MIXED_REL_TERM and rel(e3, r3) < MIXED_REL_TERM
    assert rel(e2 + e3, r2 + r3) < MIXED_REL


@pytest.mark.parametrize("mixed", [False, True])
def test_energy_2b3b_matches_separate_terms(mixed):
    """mbx_energy_2b3b (both terms side by side) against the separate calls,
    host arrays through the System mirror and device arrays through the C ABI."""
    torch = pytest.importorskip("torch")
    from mbx_b200 import capi
    ids, xyz, box = workloads.water_256(0)
    prec = "mixed" if mixed else "fp64"
    a = msys.from_arrays(ids, xyz, box, 9.0, 7.0, precision=prec)
    e2 = a.TwoBodyEnergy(True)
    g2 = np.asarray(a.GetRealGrads())
    v2 = a.GetVirial()
    e3 = a.ThreeBodyEnergy(True)
    g3 = np.asarray(a.GetRealGrads())
    v3 = a.GetVirial()
    b = msys.from_arrays(ids, xyz, box, 9.0, 7.0, precision=prec)
    f2, f3 = b.TwoAndThreeBodyEnergy(True)
    tol = 1e-12 if not mixed else 1e-9
    assert abs(f2 - e2) <= tol * abs(e2) + 1e-10 and abs(f3 - e3) <= tol * abs(e3) + 1e-10
    np.testing.assert_allclose(b.GetRealGrads(), g2 + g3, rtol=0, atol=1e-9)
    np.testing.assert_allclose(b.GetVirial(), v2 + v3, rtol=1e-10, atol=1e-8)
    assert b.NmerCounts(2) == a.NmerCounts(2) and b.NmerCounts(3) == a.NmerCounts(3)
    # device arrays, twice in a row (the child context is reused)
    ctx = capi.Context(0)
    c = msys.from_arrays(ids, xyz, box, 9.0, 7.0, context=ctx)
    sites = torch.tensor(c.sites, device="cuda")
    for _ in range(2):
        g = torch.zeros_like(sites)
        d2, d3 = ctx.energy_2b3b(sites, g, np.zeros(9), mixed=mixed)
        assert abs(d2 - e2) <= tol * abs(e2) + 1e-10 and abs(d3 - e3) <= tol * abs(e3) + 1e-10
