"""The oracle restatement against the reference's own golden vectors (CPU)."""
import os
import sys

import numpy as np
import pytest

import mbx_oracle as mo
from conftest import golden
from mbx_b200.tables import load_fit, load_pip
from mbx_b200 import workloads
from mbx_b200.specs import ALKALI, HALIDES, SPECS, check

# the reference's unit tests use an absolute margin of 1e-6
# (unittest-energy2b.cpp:45, tools/testutils.h:46-54); this oracle must do better
TOL = 1e-8


def test_specs_consistent():
    assert check()
    for name, s in SPECS.items():
        t = load_pip(name)
        assert t.nvars == s.nvars and t.ncoef == s.ncoef
        assert len(load_fit(name)) == s.ncoef


POLY = [("poly_mbpol2b", "mbpol2b"), ("poly_ch4h2o2b", "ch4h2o2b"), ("poly_ch4ch42b", "ch4ch42b"),
        ("poly_ch4h2o3b", "ch4h2o3b"), ("poly_mbpol3b", "mbpol3b"), ("poly_h2oion2b", "h2oli2b"),
        ("poly_h2oion3b", "h2oli3b"), ("poly_arh2o2b", "arh2o2b"), ("poly_co2co22b", "co2co22b"),
        ("poly_h2oco22b", "h2oco22b")]


@pytest.mark.parametrize("fixture,name", POLY)
def test_poly_golden(fixture, name):
    g = golden(fixture)
    nv = SPECS[name].nvars
    a = np.array(g["a"])
    x = np.array(g["x"])
    if name == "mbpol3b":
        x = x.reshape(nv, -1)[:, 0] if len(x) != nv else x   # 8-lane API, lane 0
    if name == "mbpol2b":
        e, gr = mo.pip_eval(name, a, x)
    else:
        e, gr = mo.pip_eval(name, a, x[:nv])
    e_exp = g["e_expected"][0] if isinstance(g["e_expected"], list) else g["e_expected"]
    assert abs(e - e_exp) < TOL * max(1.0, abs(e_exp))
    gexp = np.array(g["g_expected"])
    if name == "mbpol3b" and len(gexp) != nv:
        gexp = gexp.reshape(nv, -1)[:, 0]
    np.testing.assert_allclose(gr, gexp[:nv], rtol=1e-8, atol=TOL)


def test_poly_h2oion2b_six_configs():
    g = golden("poly_h2oion2b")
    a = np.array(g["a"])
    x6 = np.array(g["x_6"]).reshape(8, 6)   # variable-major, nd = 6
    gexp = np.array(g["g_6_expected"]).reshape(8, 6)
    for i in range(6):
        e, gr = mo.pip_eval("h2oli2b", a, x6[:, i])
        assert abs(e - g["e_6_expected"][i]) < TOL * max(1.0, abs(e))
        np.testing.assert_allclose(gr, gexp[:, i], rtol=1e-8, atol=TOL)


def test_poly_mbpol2b_two_configs():
    g = golden("poly_mbpol2b")
    a = np.array(g["a"])
    x2 = np.array(g["x_2"]).reshape(31, 2)   # variable-major, nd = 2
    gexp = np.array(g["g_2_expected"]).reshape(31, 2)
    for i in range(2):
        e, gr = mo.pip_eval("mbpol2b", a, x2[:, i])
        assert abs(e - g["e_2_expected"][i]) < TOL * max(1.0, abs(e))
        np.testing.assert_allclose(gr, gexp[:, i], rtol=1e-8, atol=TOL)


DISPATCH = ["energy2b_h2o_h2o", "energy2b_ch4_ch4", "energy2b_ch4_h2o", "energy3b_h2o_h2o_h2o",
            "energy3b_ch4_h2o_h2o", "energy2b_cs_h2o", "energy2b_li_h2o", "energy3b_li_h2o_h2o",
            "energy3b_cs_h2o_h2o"]
DISPATCH += ["energy2b_%s_h2o" % h for h in ("f", "cl", "br", "i")]
DISPATCH += ["energy3b_%s_h2o_h2o" % h for h in ("f", "cl", "br", "i")]
DISPATCH += ["energy2b_%s" % p for p in ("ar_ar", "cl_cl", "na_na", "ar_cs", "na_cl", "ar_h2o")]
DISPATCH += ["energy2b_%s" % p for p in ("h2_h2", "h2_h2o", "nh3_nh3", "nh3pbe_nh3pbe", "h2_cs", "mbpbe_mbpbe",
                                         "ch4_co2")]
DISPATCH += ["energy3b_mbpbe_mbpbe_mbpbe", "energy3b_co2_co2_co2", "energy2b_co2a_co2a", "energy2b_co2_co2",
             "energy2b_h2o_co2"]
DISPATCH += ["energy2b_n2o5_h2o", "energy3b_n2o5_h2o_h2o"]
CO2CM = ("co2cm5100", "co2cm595", "co2cm590", "co2cm5875", "co2cm585", "co2cm580")
DISPATCH += ["energy2b_%s" % m for m in CO2CM] + ["energy2b_co2a_h2o"]


@pytest.mark.parametrize("fixture", DISPATCH)
def test_dispatch_golden(fixture):
    g = golden(fixture)
    nb = 3 if "xyz3" in g else 2
    ids = [g["mon%d" % (i + 1)] for i in range(nb)]
    xyzs = [np.array(g["xyz%d" % (i + 1)]) for i in range(nb)]
    e, grads, vir = mo.get_nb_energy(ids, xyzs, g["nm"])
    assert abs(e - g["energy_expected"]) < 1e-6   # the golden is printed to 11 digits
    for i in range(nb):
        np.testing.assert_allclose(grads[i].reshape(-1), g["grad%d_expected" % (i + 1)], rtol=1e-7, atol=1e-6)
    np.testing.assert_allclose(vir, g["virial_expected"], rtol=1e-7, atol=1e-6)


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
HOLDERS += [("holder2b_%s" % m, m[3:] + "co22b") for m in CO2CM] + [("holder2b_h2o_co2a", "h2oco2a2b")]


# fixtures whose test passes the monomers to the holder in another order
# (unittest-poly-holder-2b.cpp:1098: eval(xyz2, xyz1, ...)): holder slot i <- xyz(order[i] + 1)
HOLDER_ORDER = {"holder2b_h2_h2o": (1, 0), "holder2b_h2o_n2o5": (1, 0)}


@pytest.mark.parametrize("fixture,name", HOLDERS)
def test_holder_golden(fixture, name):
    g = golden(fixture)
    s = SPECS[name]
    n = g.get("ndim", g.get("ntrim"))
    order = HOLDER_ORDER.get(fixture, range(s.nbody))
    blocks = [np.array(g["xyz%d" % (k + 1)]).reshape(n, -1) for k in order]
    xyz = np.concatenate(blocks, axis=1)
    e, grad, vir, _ = mo.holder_eval(name, xyz)
    assert abs(e - g["energy_expected"]) < 1e-6
    off = 0
    for i, k in enumerate(order):
        w = blocks[i].shape[1]
        np.testing.assert_allclose(grad[:, off:off + w].reshape(-1), g["grad%d_expected" % (k + 1)], rtol=1e-7,
                                   atol=1e-6)
        off += w
    np.testing.assert_allclose(vir, g["virial_expected"], rtol=1e-7, atol=1e-6)


@pytest.mark.parametrize("fixture", ["system_256_h2o_cubic_box", "system_57_ch4_513_h2o"])
def test_system_published_energies(fixture):
    """timing/*/output holds E2B and E3B to 11 significant digits."""
    g = golden(fixture)
    s = mo.OracleSystem(g["ids"], np.array(g["xyz"]), g["box"] or None, g["cutoff2b"], g["cutoff3b"],
                        g["ignore_2b"], g["ignore_3b"])
    e2 = s.energy(2, do_grads=False)
    e3 = s.energy(3, do_grads=False)
    assert abs(e2 - g["E2B"]) < 1e-10 * abs(g["E2B"]) + 1e-9 * 10
    assert abs(e3 - g["E3B"]) < 1e-9 * abs(g["E3B"]) + 1e-8


# the reference's generated program for each extracted table (harness kind)
REF_PROGRAM = {"mbpol2b": 0, "mbpol3b": 1, "ch4h2o2b": 2, "ch4ch42b": 3, "ch4h2o3b": 4, "h2oli2b": 5, "h2oli3b": 6,
               "fh2o2b": 7, "fh2o3b": 8, "nana2b": 9, "nacl2b": 10, "arh2o2b": 11, "h2h22b": 12, "h2oh22b": 13,
               "csh22b": 14, "nh3nh32b": 15, "ch4co22b": 16, "mbpbe2b": 17, "co23b": 18, "mbpbe3b": 19,
               "co2co22b": 20, "h2oco22b": 21, "hehe2b": 22, "h2ohe2b": 23, "n2o5h2o2b": 24, "n2o5h2o3b": 25}


@pytest.mark.parametrize("name", list(REF_PROGRAM))
def test_table_vs_reference_program(name):
    """The extracted term table (through the oracle's evaluation) against the
    compiled reference program it came from, value and gradient at random
    variables with the type's fitted coefficients (CH4-CH4: value only, the
    reference ships no gradient program for it)."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    nv = SPECS[name].nvars
    a = load_fit(name)
    rng = np.random.default_rng(11)
    grad = name != "ch4ch42b"
    for _ in range(4):
        x = rng.uniform(0.05, 1.2, size=nv)
        if grad:
            e_r, g_r = mo.RefSystem.poly(REF_PROGRAM[name], a, x)
            e_o, g_o = mo.pip_eval(name, a, x)
            np.testing.assert_allclose(g_o, g_r, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(g_r).max()))
        else:
            e_r = mo.RefSystem.poly(REF_PROGRAM[name], a, x, want_grad=False)
            e_o = mo.pip_eval(name, a, x, want_grad=False)
        assert abs(e_o - e_r) < 1e-9 * max(1.0, abs(e_r))


@pytest.mark.parametrize("ion", ALKALI + HALIDES)
@pytest.mark.parametrize("nb", [2, 3])
def test_ion_water_vs_reference(ion, nb):
    """Get2B / Get3B of a 256-site box holding ions: the oracle against the
    compiled reference (oracle/_ref), every n-mer type of the box (one Na+ or
    Cl-, whose like-ion pairs have a polynomial in the reference that is not
    on this path; three of the others)."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    ids, xyz, box = workloads.ion_water_box([ion] * (1 if ion in ("na+", "cl-") else 3), seed=1)
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0)
    r = mo.RefSystem(ids, xyz, box, 9.0, 7.0)
    e_o, e_r = o.energy(nb), r.energy(nb)
    assert abs(e_o - e_r) < 1e-10 * abs(e_r)
    np.testing.assert_allclose(o.real_grads(), r.real_grads(), rtol=0, atol=1e-8)
    np.testing.assert_allclose(o.virial, r.virial(), rtol=1e-9, atol=1e-7)


@pytest.mark.parametrize("ions", [("na+", "cl-", "na+", "cl-", "na+", "cl-"), ("ar", "ar", "ar"),
                                  ("cs+", "ar", "cs+", "ar"), ("li+", "f-", "k+", "br-")])
@pytest.mark.parametrize("nb", [2, 3])
def test_solution_vs_reference(ions, nb):
    """Salt solutions and argon in water (every pair type of the box has an
    evaluator here, ion-ion and atom-atom included): the oracle against the
    compiled reference."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    ids, xyz, box = workloads.ion_water_box(list(ions), seed=4)
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0)
    r = mo.RefSystem(ids, xyz, box, 9.0, 7.0)
    e_o, e_r = o.energy(nb), r.energy(nb)
    assert abs(e_o - e_r) < 1e-10 * abs(e_r)
    np.testing.assert_allclose(o.real_grads(), r.real_grads(), rtol=0, atol=1e-8)
    np.testing.assert_allclose(o.virial, r.virial(), rtol=1e-9, atol=1e-7)


MOLECULE_BOXES = [
    # (ids, terms compared): every n-mer type of the box has an evaluator on this path
    (["nh3"] * 200, (2, 3)),
    (["nh3pbe0d3bj"] * 200, (2, 3)),
    (["h2"] * 60 + ["h2o"] * 150 + ["cs+"] * 2, (2, 3)),
    (["mbpbe"] * 220, (2, 3)),
    # one CH4: the reference ships no CH4-CH4 gradient program (its stand-in here differentiates numerically)
    (["ch4"] + ["h2o"] * 180 + ["na+", "cl-"], (2, 3)),
    # CO2 at liquid-CO2 spacing (a 26 A box; the water lattice of 19.72 A
    # overlaps the 2.3 A long molecules)
    (["co2"] * 200, (2, 3), 26.0),
    (["co2_archive"] * 200, (2,), 26.0),
    # CO2 in water
    (["co2"] * 30 + ["h2o"] * 250, (2, 3), 22.0),
    # helium: water with a single He (He-He pairs in test_helium_dilute_vs_reference)
    (["he"] + ["h2o"] * 220, (2, 3)),
    # the co2cm* CO2 models, alone and in water.  Their intramolecular
    # variables exp(k (d0 - r)) are far above 1 (co2cm580: O-O d0 = 10 A,
    # x = 32; co2cm595: C-O x = 29; co2cm5875 and co2cm585: O-O x = 6), so
    # every dimer's degree-5 polynomial sums terms up to ~1e7 times the
    # result: two FP64 evaluation orders (the reference's Horner program, the
    # oracle's term sums) differ by up to ~3e-9 of the energy and ~1e-8 of a
    # force.  Tolerances (energy relative, gradient absolute) 1e-8 and 1e-6.
    (["co2cm595"] * 200, (2,), 30.0, (1e-8, 1e-6)),
    (["co2cm590"] * 100 + ["co2cm585"] * 100, (2,), 30.0, (1e-8, 1e-6)),
    (["co2cm5875"] * 100 + ["co2cm580"] * 100, (2,), 30.0, (1e-8, 1e-6)),
    (["co2cm5100"] * 30 + ["co2cm580"] * 30 + ["h2o"] * 220, (2,), 22.0, (1e-8, 1e-6)),
    # co2_archive in water
    (["co2_archive"] * 30 + ["h2o"] * 250, (2,), 22.0),
    # N2O5 in water (a 26 A box: the molecule spans 4.5 A)
    (["n2o5"] * 10 + ["h2o"] * 250, (2, 3), 26.0),
]


@pytest.mark.parametrize("case", range(len(MOLECULE_BOXES)))
def test_molecule_box_vs_reference(case):
    """Liquids and mixtures of the template MB-nrg types (NH3, H2 in water
    with Cs+, MB-pbe water, CO2 3b) and methane in salt water: the oracle
    against the compiled reference."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    ids, nbs = MOLECULE_BOXES[case][:2]
    L = MOLECULE_BOXES[case][2] if len(MOLECULE_BOXES[case]) > 2 else 19.72
    e_rtol, g_atol = MOLECULE_BOXES[case][3] if len(MOLECULE_BOXES[case]) > 3 else (1e-10, 1e-8)
    ids, xyz, box = workloads.molecule_box(ids, L=L, seed=case)
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0)
    r = mo.RefSystem(ids, xyz, box, 9.0, 7.0)
    for nb in nbs:
        e_o, e_r = o.energy(nb), r.energy(nb)
        assert abs(e_o - e_r) < e_rtol * max(1.0, abs(e_r)), (nb, e_o, e_r)
        # close contacts of randomly oriented molecules carry forces up to
        # ~1e4 kcal/mol/A: 1e-10 of the force on top of the absolute bound
        np.testing.assert_allclose(o.real_grads(), r.real_grads(), rtol=1e-10, atol=g_atol)
        np.testing.assert_allclose(o.virial, r.virial(), rtol=1e-9 if e_rtol < 1e-9 else 1e-7, atol=1e-7)


def test_helium_dilute_vs_reference():
    """He in water at He-He distances of 6.5 A and more.  The He-He
    polynomial (degree 23 in x = exp(k (d0 - r)), x > 1 below 5.7 A) is
    ill-conditioned at short range: there two FP64 evaluation orders (the
    reference's Horner program, the oracle's term sums) differ by up to 1e-8
    relative and neither is closer to the exact value, so parity is pinned
    where x < 1."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    ids, xyz, box = workloads.dilute_box("he", 10, seed=1)
    o = mo.OracleSystem(ids, xyz, box, 9.0, 7.0)
    r = mo.RefSystem(ids, xyz, box, 9.0, 7.0)
    e_o, e_r = o.energy(2), r.energy(2)
    assert abs(e_o - e_r) < 1e-10 * abs(e_r)
    np.testing.assert_allclose(o.real_grads(), r.real_grads(), rtol=0, atol=1e-8)


@pytest.mark.parametrize("name", ["water_256", "water_2048", "methane_water", "water_256_bead"])
def test_reference_fixtures_match_the_reference(name):
    """The committed reference fixtures (tests/golden/ref_*.npz) are what the
    compiled reference computes now, on the workload the recipe makes now."""
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_ref_fixtures import WORKLOADS, list_hash, xyz_hash
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    make_fn, c2, c3 = WORKLOADS[name]
    ids, xyz, box = make_fn()
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_%s.npz" % name))
    assert str(d["xyz_sha256"]) == xyz_hash(xyz)
    r = mo.RefSystem(ids, xyz, box, c2, c3)
    if "e1" in d:
        assert abs(r.energy(1) - float(d["e1"])) <= 1e-12 * abs(float(d["e1"])) + 1e-12
        np.testing.assert_allclose(r.real_grads(), d["g1"], rtol=0, atol=1e-10)
    for nb, cut in ((2, c2), (3, c3)):
        # the reference's OpenMP reduction order may vary between runs
        assert abs(r.energy(nb) - float(d["e%d" % nb])) <= 1e-12 * abs(float(d["e%d" % nb]))
        np.testing.assert_allclose(r.real_grads(), d["g%d" % nb], rtol=0, atol=1e-10)
        nm = r.pair_list(nb, cut)
        assert len(nm) == int(d["n%d" % nb]) and list_hash(nm) == str(d["l%d_sha256" % nb])


def _ref_root():
    r = os.environ.get("MBX_REFERENCE", "")
    if not os.path.isdir(os.path.join(r, "src")):
        pytest.skip("reference sources absent (MBX_REFERENCE)")
    return r


def test_fit_files_match_reference_sources():
    """Every committed fitted-coefficient file (mbx_b200/data/*.fit), which the
    oracle and the kernels both read, is the coefficient array of the
    reference's source it names (parsed afresh from the reference's text)."""
    from mbx_b200.codegen import pip_extract as px
    ref = _ref_root()
    from mbx_b200.specs import ONEBODY_SPECS
    for name in sorted(px.FITS):
        vals = px.extract_fit(ref, name, (SPECS[name] if name in SPECS else ONEBODY_SPECS[name]).ncoef)
        np.testing.assert_array_equal(load_fit(name), np.array(vals), err_msg=name)


@pytest.mark.parametrize("name", list(REF_PROGRAM))
def test_table_vs_reference_program_random_coefficients(name):
    """The term tables, which the oracle and the kernels both read, against the
    compiled reference programs with random coefficients (not the fitted ones
    the other checks use): agreement at random points pins every term."""
    if not mo.RefSystem.available():
        pytest.fail("reference library not built here (python oracle/build_ref.py)")
    nv = SPECS[name].nvars
    rng = np.random.default_rng(17)
    a = rng.normal(size=SPECS[name].ncoef)
    for _ in range(3):
        x = rng.uniform(0.05, 1.2, size=nv)
        if name != "ch4ch42b":
            e_r, g_r = mo.RefSystem.poly(REF_PROGRAM[name], a, x)
            e_o, g_o = mo.pip_eval(name, a, x)
            np.testing.assert_allclose(g_o, g_r, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(g_r).max()))
        else:
            e_r = mo.RefSystem.poly(REF_PROGRAM[name], a, x, want_grad=False)
            e_o = mo.pip_eval(name, a, x, want_grad=False)
        assert abs(e_o - e_r) < 1e-9 * max(1.0, abs(e_r))
