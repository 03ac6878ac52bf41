"""Declarative description of the 2-body and 3-body evaluators on the path.

Each evaluator of the reference ("polynomial holder": variables built from
inter-site distances, virtual sites, a switching function, the chain rule to
atoms and the virial) follows one template.  This module states every
evaluator as data -- its sites, its polynomial variables, its switch and its
skip rule -- so that the CUDA generator (``codegen/gen_kernels.py``) and the
CPU oracle restatement (``oracle/``) are produced from one description.  The
numbers below are the fitted model constants of the reference and must be
identical to it; each block cites where they are defined.

Variable kinds (r = |p1 - p2|):

* ``exp``   v = exp(k * (d0 - r))
            (``variable::v_exp0``, potential/2b/x2b-v9x.cpp:54-69;
            ``var``, potential/3b/x3b-v2x.cpp:52-59 writes the same value as
            exp(-k (r - d0)); ``variable::v_exp`` in tools/variable.cpp:68 is
            the case d0 = 0)
* ``coul``  v = exp(k * (d0 - r)) / r   (``variable::v_coul``,
            potential/2b/x2b-v9x.cpp:73-92)

Virtual sites ``lp``: the two MB-pol lone-pair sites of a water (O, H1, H2),
``monomer::setup`` potential/2b/x2b-v9x.cpp:119-135:
    X(+/-) = O + 0.5 * g_in * (OH1 + OH2) +/- g_out * (OH1 x OH2)
with g_in = -9.721486914088159e-02, g_out = 9.859272078406150e-02
(x2b-v9x.cpp:1341-1342; the same numbers are w12/wcross in
x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:1003-1005).

Switches (cosine, ``f_switch``):
    s(r) = 1 for r <= ri, (1 + cos(pi (r - ri)/(rf - ri)))/2 for ri < r <= rf,
           0 for r > rf
* ``pair``: s(r12) on the first-atom distance of the two monomers
  (x2b-v9x.cpp:1349-1362, x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:804-818,
  x2b_A1B4_A1B4_deg4_exp0_v1x.cpp:1453-1466)
* ``triple``: s12 s13 + s12 s23 + s13 s23 on the three first-atom distances
  (x3b-v2x.cpp:1275-1288,1690; mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp:1318-1333)
* ``triple2``: s12 s13 + s12 s23 + s13 s23 - 2 s12 s13 s23
  (mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp:12927,13127,13181-13183)

Skip rules (n-mers not evaluated; their energy and gradient are exactly 0):
* ``pair_gt``: r12 > rf  (x2b-v9x.cpp:1563)
* ``two_of_three_gt``: at least two of r12, r13, r23 > rf (x3b-v2x.cpp:1515)
* ``all_three_gt``: all of r12, r13, r23 > rf
  (mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp:1561)
"""
from dataclasses import dataclass, field, replace
from typing import List, Tuple

LP_GAMMA_IN = -9.721486914088159e-02
LP_GAMMA_OUT = 9.859272078406150e-02


@dataclass(frozen=True)
class Spec:
    name: str                  # also the PIP table name in mbx_b200/data
    monomers: Tuple[str, ...]  # monomer ids in evaluator (holder) order
    nat: Tuple[int, ...]       # real atoms per monomer
    sites: Tuple[str, ...]     # real atoms in holder order, then virtual sites
    lp: Tuple[Tuple[int, int, int, int], ...]  # (monomer, first real site, X+ site, X- site)
    variables: Tuple[Tuple[str, int, int, float, float], ...]  # (kind, site1, site2, k, d0)
    switch: str                # "pair", "triple", "triple2" or "cos2"
    ri: float
    rf: float
    skip: str                  # "pair_gt", "two_of_three_gt", "all_three_gt"
    nvars: int
    ncoef: int
    degree: int
    ref: str                   # reference evaluator (file:line)
    table: str = ""            # PIP table in mbx_b200/data when shared by several evaluators ("": name)
    # "raw": the evaluator's virial sums -r . g over the polynomial gradient
    # alone (no switch factor, no switch gradient), as the reference's
    # x2b_A1B2C4_D1E2_v1x does; "": over the switched gradient
    virial: str = ""

    @property
    def pip_table(self):
        return self.table or self.name

    @property
    def nbody(self):
        return len(self.monomers)

    @property
    def nreal(self):
        return sum(self.nat)

    def site(self, name):
        return self.sites.index(name)


def _vars(sites, table):
    out = []
    for kind, a, b, k, d0 in table:
        out.append((kind, sites.index(a), sites.index(b), float(k), float(d0)))
    return tuple(out)


# ---------------------------------------------------------------------------
# MB-pol 2b: x2o::x2b_v9x, potential/2b/x2b-v9x.cpp:1514-1819 (constants
# :1330-1346, variables :1600-1650)
# ---------------------------------------------------------------------------
_S = ("Oa", "Ha1", "Ha2", "Ob", "Hb1", "Hb2", "Xa1", "Xa2", "Xb1", "Xb2")
_kHHi, _kOHi = -6.480884773303821e-01, 1.674518993682975e+00
_kHHc, _kOHc, _kOOc = 1.148231864355956e+00, 1.205989761123099e+00, 1.395357065790959e+00
_kXH, _kXO, _kXX = 7.347036852042255e-01, 7.998249864422826e-01, 7.960663960630585e-01
MBPOL2B = Spec(
    name="mbpol2b", monomers=("h2o", "h2o"), nat=(3, 3), sites=_S,
    lp=((0, 0, 6, 7), (1, 3, 8, 9)),
    variables=_vars(_S, [
        ("exp", "Ha1", "Ha2", _kHHi, 1.0), ("exp", "Hb1", "Hb2", _kHHi, 1.0),
        ("exp", "Oa", "Ha1", _kOHi, 1.0), ("exp", "Oa", "Ha2", _kOHi, 1.0),
        ("exp", "Ob", "Hb1", _kOHi, 1.0), ("exp", "Ob", "Hb2", _kOHi, 1.0),
        ("coul", "Ha1", "Hb1", _kHHc, 4.0), ("coul", "Ha1", "Hb2", _kHHc, 4.0),
        ("coul", "Ha2", "Hb1", _kHHc, 4.0), ("coul", "Ha2", "Hb2", _kHHc, 4.0),
        ("coul", "Oa", "Hb1", _kOHc, 4.0), ("coul", "Oa", "Hb2", _kOHc, 4.0),
        ("coul", "Ob", "Ha1", _kOHc, 4.0), ("coul", "Ob", "Ha2", _kOHc, 4.0),
        ("coul", "Oa", "Ob", _kOOc, 4.0),
        ("exp", "Xa1", "Hb1", _kXH, 4.0), ("exp", "Xa1", "Hb2", _kXH, 4.0),
        ("exp", "Xa2", "Hb1", _kXH, 4.0), ("exp", "Xa2", "Hb2", _kXH, 4.0),
        ("exp", "Xb1", "Ha1", _kXH, 4.0), ("exp", "Xb1", "Ha2", _kXH, 4.0),
        ("exp", "Xb2", "Ha1", _kXH, 4.0), ("exp", "Xb2", "Ha2", _kXH, 4.0),
        ("exp", "Oa", "Xb1", _kXO, 4.0), ("exp", "Oa", "Xb2", _kXO, 4.0),
        ("exp", "Ob", "Xa1", _kXO, 4.0), ("exp", "Ob", "Xa2", _kXO, 4.0),
        ("exp", "Xa1", "Xb1", _kXX, 4.0), ("exp", "Xa1", "Xb2", _kXX, 4.0),
        ("exp", "Xa2", "Xb1", _kXX, 4.0), ("exp", "Xa2", "Xb2", _kXX, 4.0),
    ]),
    switch="pair", ri=4.5, rf=6.5, skip="pair_gt",
    nvars=31, ncoef=1153, degree=4, ref="potential/2b/x2b-v9x.cpp:1514",
)

# ---------------------------------------------------------------------------
# MB-pol 3b: x2o::x3b_v2x, potential/3b/x3b-v2x.cpp:1403-1808 (constants
# :1256-1271, variables :1548-1584)
# ---------------------------------------------------------------------------
_S = ("Oa", "Ha1", "Ha2", "Ob", "Hb1", "Hb2", "Oc", "Hc1", "Hc2")
_kHHi3, _dHHi3 = -2.254303257872797e+00, 1.690594510379166e+00
_kOHi3, _dOHi3 = -2.564771901404151e-01, -2.999999868517452e+00
_kHH3, _dHH3 = 4.247920544074333e-01, 3.499031358429095e+00
_kOH3, _dOH3 = 8.128985941165371e-01, 4.854042963514281e+00
_kOO3, _dOO3 = 3.749457984616480e-02, 4.816312044947604e-08
_pairs3 = [
    ("Ha1", "Ha2", _kHHi3, _dHHi3), ("Hb1", "Hb2", _kHHi3, _dHHi3), ("Hc1", "Hc2", _kHHi3, _dHHi3),
    ("Oa", "Ha1", _kOHi3, _dOHi3), ("Oa", "Ha2", _kOHi3, _dOHi3), ("Ob", "Hb1", _kOHi3, _dOHi3),
    ("Ob", "Hb2", _kOHi3, _dOHi3), ("Oc", "Hc1", _kOHi3, _dOHi3), ("Oc", "Hc2", _kOHi3, _dOHi3),
    ("Ha1", "Hb1", _kHH3, _dHH3), ("Ha1", "Hb2", _kHH3, _dHH3), ("Ha1", "Hc1", _kHH3, _dHH3),
    ("Ha1", "Hc2", _kHH3, _dHH3), ("Ha2", "Hb1", _kHH3, _dHH3), ("Ha2", "Hb2", _kHH3, _dHH3),
    ("Ha2", "Hc1", _kHH3, _dHH3), ("Ha2", "Hc2", _kHH3, _dHH3), ("Hb1", "Hc1", _kHH3, _dHH3),
    ("Hb1", "Hc2", _kHH3, _dHH3), ("Hb2", "Hc1", _kHH3, _dHH3), ("Hb2", "Hc2", _kHH3, _dHH3),
    ("Oa", "Hb1", _kOH3, _dOH3), ("Oa", "Hb2", _kOH3, _dOH3), ("Oa", "Hc1", _kOH3, _dOH3),
    ("Oa", "Hc2", _kOH3, _dOH3), ("Ob", "Ha1", _kOH3, _dOH3), ("Ob", "Ha2", _kOH3, _dOH3),
    ("Ob", "Hc1", _kOH3, _dOH3), ("Ob", "Hc2", _kOH3, _dOH3), ("Oc", "Ha1", _kOH3, _dOH3),
    ("Oc", "Ha2", _kOH3, _dOH3), ("Oc", "Hb1", _kOH3, _dOH3), ("Oc", "Hb2", _kOH3, _dOH3),
    ("Oa", "Ob", _kOO3, _dOO3), ("Oa", "Oc", _kOO3, _dOO3), ("Ob", "Oc", _kOO3, _dOO3),
]
MBPOL3B = Spec(
    name="mbpol3b", monomers=("h2o", "h2o", "h2o"), nat=(3, 3, 3), sites=_S, lp=(),
    variables=_vars(_S, [("exp", a, b, k, d) for a, b, k, d in _pairs3]),
    switch="triple", ri=0.0, rf=4.5, skip="two_of_three_gt",
    nvars=36, ncoef=1163, degree=4, ref="potential/3b/x3b-v2x.cpp:1403",
)

# ---------------------------------------------------------------------------
# CH4-H2O 2b: x2b_A1B2Z2_C1D4_v1x("h2o","ch4"), water first,
# potential/2b/x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:954-1250 (constants :778-800,
# variables :1007-1044)
# ---------------------------------------------------------------------------
_S = ("A1", "B1", "B2", "C1", "D1", "D2", "D3", "D4", "Z1", "Z2")
_c = dict(
    kAB=(7.981769253199138e-01, 4.040819683827504e+00), kBB=(2.579463880579890e-01, 2.377019586697373e+00),
    kCD=(3.688427221099756e-01, 4.333852019203771e+00), kDD=(7.091344939292101e-01, 3.168984322065454e+00),
    AC=(1.564512113339641e+00, 3.257864349051078e+00), AD=(6.622458897222858e-01, 3.893753782478246e+00),
    BC=(1.206761651281590e+00, 2.837093011555366e+00), BD=(7.972437249347342e-01, 5.352114146493275e+00),
    CZ=(1.291962400963017e+00, 4.726091329507012e+00), DZ=(4.825788863998004e-01, 5.184523093153075e+00),
)


def _v(kind, a, b, key):
    k, d = _c[key]
    return (kind, a, b, k, d)


_tab = [_v("exp", "A1", "B1", "kAB"), _v("exp", "A1", "B2", "kAB"), _v("exp", "B1", "B2", "kBB")]
_tab += [_v("exp", "C1", "D%d" % i, "kCD") for i in range(1, 5)]
_tab += [_v("exp", "D%d" % i, "D%d" % j, "kDD") for i in range(1, 5) for j in range(i + 1, 5)]
_tab += [_v("exp", "A1", "C1", "AC")] + [_v("exp", "A1", "D%d" % i, "AD") for i in range(1, 5)]
_tab += [_v("exp", "B1", "C1", "BC")] + [_v("exp", "B1", "D%d" % i, "BD") for i in range(1, 5)]
_tab += [_v("exp", "B2", "C1", "BC")] + [_v("exp", "B2", "D%d" % i, "BD") for i in range(1, 5)]
_tab += [_v("coul", "Z1", "C1", "CZ")] + [_v("coul", "Z1", "D%d" % i, "DZ") for i in range(1, 5)]
_tab += [_v("coul", "Z2", "C1", "CZ")] + [_v("coul", "Z2", "D%d" % i, "DZ") for i in range(1, 5)]
CH4H2O2B = Spec(
    name="ch4h2o2b", monomers=("h2o", "ch4"), nat=(3, 5), sites=_S, lp=((0, 0, 8, 9),),
    variables=_vars(_S, _tab), switch="pair", ri=8.0, rf=9.0, skip="pair_gt",
    nvars=38, ncoef=603, degree=3, ref="potential/2b/x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:954",
)

# ---------------------------------------------------------------------------
# CH4-CH4 2b: x2b_A1B4_A1B4_v1x, potential/2b/x2b_A1B4_A1B4_deg4_exp0_v1x.cpp
# :1600-1760 (constants :1436-1449, variables :1515-1559)
# ---------------------------------------------------------------------------
_S = ("Aa", "B1a", "B2a", "B3a", "B4a", "Ab", "B1b", "B2b", "B3b", "B4b")
_kABi = (3.188848769154688e+00, 1.993909788871820e+00)
_kBBi = (1.204263123667977e+00, 2.367262478707738e+00)
_kAA = (3.280825850503320e+00, 1.705786899598748e+00)
_kAB = (6.515735442121080e-01, 4.621435907700928e+00)
_kBB = (1.345128916678614e+00, 5.411919409835622e+00)
_tab = []
for m in "ab":
    _tab += [("exp", "A" + m, "B%d%s" % (i, m)) + _kABi for i in range(1, 5)]
    _tab += [("exp", "B%d%s" % (i, m), "B%d%s" % (j, m)) + _kBBi for i in range(1, 5) for j in range(i + 1, 5)]
_tab += [("exp", "Aa", "Ab") + _kAA]
_tab += [("exp", "Aa", "B%db" % i) + _kAB for i in range(1, 5)]
for i in range(1, 5):
    _tab += [("exp", "B%da" % i, "Ab") + _kAB]
    _tab += [("exp", "B%da" % i, "B%db" % j) + _kBB for j in range(1, 5)]
CH4CH42B = Spec(
    name="ch4ch42b", monomers=("ch4", "ch4"), nat=(5, 5), sites=_S, lp=(),
    variables=_vars(_S, _tab), switch="pair", ri=8.0, rf=9.0, skip="pair_gt",
    nvars=45, ncoef=1345, degree=4, ref="potential/2b/x2b_A1B4_A1B4_deg4_exp0_v1x.cpp:1600",
)

# ---------------------------------------------------------------------------
# CH4-H2O-H2O 3b: mbnrg_A1B4_C1D2_C1D2_deg3_v1, methane first,
# potential/3b/mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp:1481-1863 (constants
# :1301-1313, variables :1617-1671; v_exp has d0 = 0)
# ---------------------------------------------------------------------------
_S = ("A1", "B1", "B2", "B3", "B4", "C1", "D1", "D2", "C2", "D3", "D4")
_k = dict(
    AB1=1.531189404203529e+00, AC0=4.745721065911203e+00, AD0=5.125853420719423e-01,
    BB1=2.388453487869389e+00, BC0=8.378927200873254e-01, BD0=1.429945481869194e+00,
    CC0=5.000000078438228e-01, CD1=5.359930384592185e+00, CD0=1.064344403260153e+00,
    DD1=2.264354654848907e+00, DD0=5.000020400292975e-01,
)
_tab = [
    ("A1", "B1", "AB1"), ("A1", "B2", "AB1"), ("A1", "B3", "AB1"), ("A1", "B4", "AB1"),
    ("A1", "C1", "AC0"), ("A1", "C2", "AC0"),
    ("A1", "D1", "AD0"), ("A1", "D2", "AD0"), ("A1", "D3", "AD0"), ("A1", "D4", "AD0"),
]
for i in range(1, 5):
    _tab += [("B%d" % i, "B%d" % j, "BB1") for j in range(i + 1, 5)]
    _tab += [("B%d" % i, "C1", "BC0"), ("B%d" % i, "C2", "BC0")]
    _tab += [("B%d" % i, "D%d" % j, "BD0") for j in range(1, 5)]
_tab += [("C1", "C2", "CC0"), ("C1", "D1", "CD1"), ("C1", "D2", "CD1"), ("C1", "D3", "CD0"), ("C1", "D4", "CD0"),
         ("C2", "D1", "CD0"), ("C2", "D2", "CD0"), ("C2", "D3", "CD1"), ("C2", "D4", "CD1"),
         ("D1", "D2", "DD1"), ("D1", "D3", "DD0"), ("D1", "D4", "DD0"), ("D2", "D3", "DD0"), ("D2", "D4", "DD0"),
         ("D3", "D4", "DD1")]
CH4H2O3B = Spec(
    name="ch4h2o3b", monomers=("ch4", "h2o", "h2o"), nat=(5, 3, 3), sites=_S, lp=(),
    variables=_vars(_S, [("exp", a, b, _k[key], 0.0) for a, b, key in _tab]),
    switch="triple", ri=5.0, rf=6.0, skip="all_three_gt",
    nvars=55, ncoef=1254, degree=3, ref="potential/3b/mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp:1481",
)

# ---------------------------------------------------------------------------
# Alkali-metal ion - water 2b: h2o_ion::x2b_h2o_ion_v2x(mon1 = "h2o", ion),
# water first, potential/2b/x2b-A1B2Z2_C-v1x.cpp:2604-2770 (variables
# :2637-2649; lone pairs from monomer::setup :121-135 with the MB-pol gammas;
# switch f_switch :2418-2430 on the O-ion distance, dimers beyond r2f
# skipped :2600).  One polynomial (poly_2b_h2o_ion_v1x, 8 variables, degree
# 5, 429 coefficients) for all five ions; the non-linear constants, the
# switch radii and the coefficients are per ion (constructor blocks
# :181-625 li+, :628-1072 na+, :1075-1519 k+, :1522-1966 rb+, :1969-2413
# cs+).
# ---------------------------------------------------------------------------
_S_ION2B = ("O", "H1", "H2", "X", "Xp", "Xm")
_ION2B = {
    # ion: (k_HH_intra, k_OH_intra, k_XH_coul, k_XO_coul, k_xlp_main,
    #       d_HH_intra, d_OH_intra, d_XH_coul, d_XO_coul, d_xlp_main, r2i, r2f)
    "li+": (2.841179733353343e-01, 1.999999982813816e+00, 1.221694270779757e-01, 8.277382286185307e-01,
            1.168420032277624e+00, 1.999965084185145e+00, 1.138547391709435e+00, 4.576629521685452e+00,
            3.210235763647789e+00, 3.611985038328086e+00, 5.0, 6.0),
    "na+": (7.823878977486063e-01, 1.999999957825146e+00, 7.950431747693237e-02, 6.680682051951390e-01,
            8.311885364375440e-01, 1.999918468032695e+00, 5.269425988634360e-01, 6.287228652758436e+00,
            6.242799339695940e+00, 3.872159916140287e+00, 5.5, 6.5),
    "k+": (3.377427362895352e-01, 1.999994321311263e+00, 1.986401977927494e-01, 1.373943653398614e+00,
           7.815071238402381e-01, 5.669440892013204e-01, 7.466617529933223e-01, 4.662999403661182e+00,
           3.646598993078812e+00, 3.748049151082972e+00, 6.0, 7.0),
    "rb+": (3.195475762417059e-01, 6.446164826239851e-01, 5.104027836124081e-01, 1.273907587244391e+00,
            7.482531727951891e-01, 1.431386688762102e+00, 1.999530480711730e+00, 4.312600876869783e+00,
            4.872074227770685e+00, 3.821777646259915e+00, 6.0, 7.0),
    "cs+": (3.418356162428376e-01, 3.760948616075574e-01, 4.355574735817115e-01, 9.970388969117101e-01,
            6.771893256000681e-01, 1.998465969152339e+00, 1.999745711872710e+00, 6.331169164351936e+00,
            6.050756912670806e+00, 4.309622503190793e+00, 6.0, 7.0),
}


def _ion2b(ion, name):
    kHH, kOH, kXH, kXO, kXL, dHH, dOH, dXH, dXO, dXL, ri, rf = _ION2B[ion]
    tab = [("exp", "H1", "H2", kHH, dHH),
           ("exp", "O", "H1", kOH, dOH), ("exp", "O", "H2", kOH, dOH),
           ("coul", "X", "H1", kXH, dXH), ("coul", "X", "H2", kXH, dXH),
           ("coul", "X", "O", kXO, dXO),
           ("exp", "X", "Xp", kXL, dXL), ("exp", "X", "Xm", kXL, dXL)]
    return Spec(name=name, monomers=("h2o", ion), nat=(3, 1), sites=_S_ION2B, lp=((0, 0, 4, 5),),
                variables=_vars(_S_ION2B, tab), switch="pair", ri=ri, rf=rf, skip="pair_gt",
                nvars=8, ncoef=429, degree=5, ref="potential/2b/x2b-A1B2Z2_C-v1x.cpp:2604", table="h2oion2b")


H2OLI2B = _ion2b("li+", "h2oli2b")
H2ONA2B = _ion2b("na+", "h2ona2b")
H2OK2B = _ion2b("k+", "h2ok2b")
H2ORB2B = _ion2b("rb+", "h2orb2b")
H2OCS2B = _ion2b("cs+", "h2ocs2b")
ALKALI = ("li+", "na+", "k+", "rb+", "cs+")

# ---------------------------------------------------------------------------
# Alkali-metal ion - water - water 3b: x3b_h2o_ion_v1x_deg4_filtered(ion),
# waters first, potential/3b/x3b-h2o-ion-v1x-deg4-filtered.cpp:206-480
# (variables :309-337, all exp(-k (r - r0)) = ``exp`` with d0 = r0;
# f_switch :98-111 on the three first-atom distances, trimers with two of
# them beyond r3f skipped :296).  One polynomial
# (poly_3b_h2o_ion_v1x_deg4_filtered, 21 variables, degree 4, 1016
# coefficients); constants and coefficients per ion (constructor blocks
# :485-1521 li+, :1522-2560 na+, :2561-3601 k+, :3602-4638 rb+,
# :4639-5677 cs+).
# ---------------------------------------------------------------------------
_S_ION3B = ("Oa", "Ha1", "Ha2", "Ob", "Hb1", "Hb2", "X")
_ION3B = {
    # ion: (kOH_intra, dOH_intra, kHH_intra, dHH_intra, kHH, dHH, kOH, dOH,
    #       kOO, dOO, kXH, dXH, kXO, dXO, r3i, r3f)
    "li+": (3.699637401847997e-01, 1.068868829761452e+01, 1.679876695401232e-01, 1.975171570009532e+00,
            1.684254969412778e-01, 1.129172172428989e+00, 9.935182415951276e-01, 4.802676630871010e+00,
            8.505367453684953e-01, 9.078259767894229e+00, 4.576806684033723e-02, 3.739394864987378e+00,
            1.919355248053607e-01, 6.346405495344363e+00, 0.0, 4.5),
    "na+": (1.079285891981862e+00, 2.493557848672918e+00, -2.009859067711048e-01, 4.331575675326020e+00,
            4.884318738475223e-01, 1.003637515624313e+01, 6.109404006641794e-01, 7.677682294461052e+00,
            6.521263121174117e-01, 4.789256072989140e+00, 4.772422237444002e-02, 6.916712361001890e+00,
            1.252130248577817e-01, 9.920052988243551e+00, 0.0, 4.5),
    "k+": (5.465082839032473e-01, 3.154303998006160e+00, 1.505534948596776e+00, 9.488236920987529e+00,
           5.669173309079441e-01, 1.023524681458323e+01, 7.149221098880705e-01, 5.287618686287184e+00,
           5.877602499345129e-01, 4.432532991705378e+00, 4.399022736050681e-02, 1.561826519728719e+00,
           4.772570648100866e-01, 3.541346877424266e+00, 0.0, 4.5),
    "rb+": (2.571848425019958e-01, 7.619101258901348e-01, 4.935811847841025e+00, 2.117837104002506e+00,
            6.641539139948633e-01, 1.127561151275100e+01, 8.262323078009421e-01, 6.835848274082730e+00,
            4.657013878889721e-01, 7.037153931329832e+00, 1.973569678997551e-02, 6.299823660916497e-01,
            3.504015211699528e-01, 1.112494982897995e+01, 0.0, 4.5),
    "cs+": (8.068929184027878e-01, 2.035944886211303e-04, 2.343614900390014e-01, 5.101199357764126e-01,
            2.580358900220996e-01, 7.186210165587381e+00, 7.063990540733522e-01, 1.142220902170943e+01,
            2.374997393974423e-02, 3.021128948742693e+00, 4.022139878389860e-01, 8.914038895157681e+00,
            5.995683887693093e-02, 2.398846003968965e+00, 0.0, 4.5),
}


def _ion3b(ion, name):
    kOHi, dOHi, kHHi, dHHi, kHH, dHH, kOH, dOH, kOO, dOO, kXH, dXH, kXO, dXO, ri, rf = _ION3B[ion]
    tab = [("Oa", "Ha1", kOHi, dOHi), ("Oa", "Ha2", kOHi, dOHi), ("Ha1", "Ha2", kHHi, dHHi),
           ("Ob", "Hb1", kOHi, dOHi), ("Ob", "Hb2", kOHi, dOHi), ("Hb1", "Hb2", kHHi, dHHi),
           ("Ha1", "Hb1", kHH, dHH), ("Ha1", "Hb2", kHH, dHH), ("Ha2", "Hb1", kHH, dHH), ("Ha2", "Hb2", kHH, dHH),
           ("Oa", "Hb1", kOH, dOH), ("Oa", "Hb2", kOH, dOH), ("Ob", "Ha1", kOH, dOH), ("Ob", "Ha2", kOH, dOH),
           ("Oa", "Ob", kOO, dOO),
           ("Ha1", "X", kXH, dXH), ("Ha2", "X", kXH, dXH), ("Hb1", "X", kXH, dXH), ("Hb2", "X", kXH, dXH),
           ("Oa", "X", kXO, dXO), ("Ob", "X", kXO, dXO)]
    return Spec(name=name, monomers=("h2o", "h2o", ion), nat=(3, 3, 1), sites=_S_ION3B, lp=(),
                variables=_vars(_S_ION3B, [("exp", a, b, k, d) for a, b, k, d in tab]),
                switch="triple", ri=ri, rf=rf, skip="two_of_three_gt", nvars=21, ncoef=1016, degree=4,
                ref="potential/3b/x3b-h2o-ion-v1x-deg4-filtered.cpp:206", table="h2oion3b")


H2OLI3B = _ion3b("li+", "h2oli3b")
H2ONA3B = _ion3b("na+", "h2ona3b")
H2OK3B = _ion3b("k+", "h2ok3b")
H2ORB3B = _ion3b("rb+", "h2orb3b")
H2OCS3B = _ion3b("cs+", "h2ocs3b")

# ---------------------------------------------------------------------------
# Halide - water 2b: mbnrg_A1_B1C2X2_deg6_v1(halide, "h2o"), halide first,
# potential/2b/mbnrg_2b_A1_B1C2X2_deg6_v1.cpp:3789-3980 (variables
# :3865-3872, tools/variable.cpp v_exp/v_coul with d0 = 0; MB-pol lone pairs
# :3853-3856; f_switch :3685-3699 on the halide-O distance, dimers beyond ro
# skipped :3810).  One polynomial (poly_A1_B1C2X2_deg6_v1, 8 variables,
# degree 6, 906 coefficients); constants and coefficients per halide
# (constructor blocks :12-927 f-, :929-1844 cl-, :1846-2761 br-,
# :2763-3678 i-).
# ---------------------------------------------------------------------------
_S_HAL2B = ("A", "B", "C1", "C2", "X1", "X2")
_HAL2B = {
    # halide: (k_AB (coul), k_AC (coul), k_AX, k_BC intra, k_CC intra, ri, ro)
    "f-": (6.235116852837913e-08, 3.545923893694392e-01, 3.507638336966289e-01, 4.131876960255009e-01,
           3.616986527314591e-01, 5.3, 7.3),
    "cl-": (4.434101301397339e-07, 3.581531291002636e-08, 3.220935488191130e-01, 2.809297687850453e-01,
            3.015683487617984e-01, 5.8, 7.8),
    "br-": (4.363632730909749e-06, 6.538608932949625e-07, 2.834802070784692e-01, 1.238561725021965e-01,
            3.140346943732611e-01, 5.9, 7.9),
    "i-": (7.590595972237534e-07, 3.470400079944597e-06, 2.480149059099078e-01, 3.002335368068454e-01,
           2.183115173238724e-01, 6.2, 8.2),
}


def _hal2b(ion, name):
    kAB, kAC, kAX, kBC, kCC, ri, ro = _HAL2B[ion]
    tab = [("coul", "A", "B", kAB, 0.0), ("coul", "A", "C1", kAC, 0.0), ("coul", "A", "C2", kAC, 0.0),
           ("exp", "A", "X1", kAX, 0.0), ("exp", "A", "X2", kAX, 0.0),
           ("exp", "B", "C1", kBC, 0.0), ("exp", "B", "C2", kBC, 0.0), ("exp", "C1", "C2", kCC, 0.0)]
    return Spec(name=name, monomers=(ion, "h2o"), nat=(1, 3), sites=_S_HAL2B, lp=((1, 1, 4, 5),),
                variables=_vars(_S_HAL2B, tab), switch="pair", ri=ri, rf=ro, skip="pair_gt",
                nvars=8, ncoef=906, degree=6, ref="potential/2b/mbnrg_2b_A1_B1C2X2_deg6_v1.cpp:3789",
                table="halh2o2b")


FH2O2B = _hal2b("f-", "fh2o2b")
CLH2O2B = _hal2b("cl-", "clh2o2b")
BRH2O2B = _hal2b("br-", "brh2o2b")
IH2O2B = _hal2b("i-", "ih2o2b")
HALIDES = ("f-", "cl-", "br-", "i-")

# ---------------------------------------------------------------------------
# Halide - water - water 3b: mbnrg_A1_B1C2X2_B1C2X2_deg4_v1(halide, "h2o",
# "h2o"), halide first, potential/3b/mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp:
# 12956-13282 (variables :13072-13112, d0 = 0; MB-pol lone pairs on both
# waters; switch ``triple2`` :13127; trimers with all three first-atom
# distances beyond ro skipped :12990).  One polynomial
# (poly_A1_B1C2X2_B1C2X2_deg4_v1, 41 variables, degree 4, 3173 coefficients);
# constants and coefficients per halide (constructor blocks :13-3202 f-,
# :3204-6393 cl-, :6395-9584 br-, :9586-12775 i-).
# ---------------------------------------------------------------------------
_S_HAL3B = ("A", "B1", "C1", "C2", "B2", "C3", "C4", "X1", "X2", "X3", "X4")
_HAL3B = {
    # halide: (kAB c, kAC c, kAX, kBB c, kBC intra, kBC c, kBX, kCC intra, kCC c, kCX, kXX, ri, ro)
    "f-": (1.683174003900960e-02, 1.462488339952361e-01, 1.495490093533567e-01, 3.398373799669774e+00,
           8.390335120106681e-01, 3.159841858407245e-09, 4.996257547423549e-01, 2.635206665339118e+00,
           4.004058684253884e-02, 2.561129825500117e-01, 3.703274677292788e-01, 0.0, 5.8),
    "cl-": (3.050780499728952e+00, 2.317377443605641e-02, 2.360729625543786e-01, 3.864106971541486e+00,
            1.994298755795063e-01, 9.464531078609996e-02, 4.009804221983941e+00, 1.933213969741414e+00,
            1.271399144654976e-01, 2.092270464467735e-01, 5.164915204892290e-01, 0.0, 5.8),
    "br-": (4.934350368264340e-09, 8.053864705533755e-05, 1.767787145924113e-01, 4.808245301601014e+00,
            3.132138118081313e-01, 1.315368607065956e+00, 6.791698758407823e-01, 6.865835071774395e+00,
            6.324551383433107e-02, 2.549642769697353e-01, 2.245436992967047e+00, 0.0, 5.9),
    "i-": (5.157227102182063e-09, 1.983825013735218e-06, 3.818504443080583e-01, 9.683345246557618e-02,
           1.267839872255443e-01, 2.540217377512282e-01, 1.570538875818527e+00, 1.652271352978735e+00,
           2.456950872841040e-02, 2.124956943635082e-01, 1.036383352473932e+00, 0.0, 6.0),
}


def _hal3b(ion, name):
    kAB, kAC, kAX, kBB, kBCi, kBC, kBX, kCCi, kCC, kCX, kXX, ri, ro = _HAL3B[ion]
    c, e = "coul", "exp"
    tab = [(c, "A", "B1", kAB), (c, "A", "B2", kAB),
           (c, "A", "C1", kAC), (c, "A", "C2", kAC), (c, "A", "C3", kAC), (c, "A", "C4", kAC),
           (e, "A", "X1", kAX), (e, "A", "X2", kAX), (e, "A", "X3", kAX), (e, "A", "X4", kAX),
           (c, "B1", "B2", kBB), (e, "B1", "C1", kBCi), (e, "B1", "C2", kBCi),
           (c, "B1", "C3", kBC), (c, "B1", "C4", kBC), (e, "B1", "X3", kBX), (e, "B1", "X4", kBX),
           (c, "B2", "C1", kBC), (c, "B2", "C2", kBC), (e, "B2", "C3", kBCi), (e, "B2", "C4", kBCi),
           (e, "B2", "X1", kBX), (e, "B2", "X2", kBX),
           (e, "C1", "C2", kCCi), (c, "C1", "C3", kCC), (c, "C1", "C4", kCC),
           (e, "C1", "X3", kCX), (e, "C1", "X4", kCX),
           (c, "C2", "C3", kCC), (c, "C2", "C4", kCC), (e, "C2", "X3", kCX), (e, "C2", "X4", kCX),
           (e, "C3", "C4", kCCi), (e, "C3", "X1", kCX), (e, "C3", "X2", kCX), (e, "C4", "X1", kCX),
           (e, "C4", "X2", kCX),
           (e, "X1", "X3", kXX), (e, "X1", "X4", kXX), (e, "X2", "X3", kXX), (e, "X2", "X4", kXX)]
    return Spec(name=name, monomers=(ion, "h2o", "h2o"), nat=(1, 3, 3), sites=_S_HAL3B,
                lp=((1, 1, 7, 8), (2, 4, 9, 10)),
                variables=_vars(_S_HAL3B, [(kind, a, b, k, 0.0) for kind, a, b, k in tab]), switch="triple2",
                ri=ri, rf=ro, skip="all_three_gt", nvars=41, ncoef=3173, degree=4,
                ref="potential/3b/mbnrg_3b_A1_B1C2X2_B1C2X2_deg4_v1.cpp:12956", table="halh2o3b")


# ---------------------------------------------------------------------------
# Atom - atom 2b (like ions, argon): mbnrg_A1_A1_deg9_v1(m, m) and
# mbnrg_A1_B1_deg9_v1(a, b): one variable exp(k (d0 - r)) (variable::v_exp0,
# tools/variable.cpp:49), a degree-9 polynomial, cosine switch 7 -> 9 A
# (potential/2b/mbnrg_2b_A1_A1_deg9_v1.cpp:138-235, constructor blocks :11-25
# na+, :27-41 cl-, :43-57 ar; potential/2b/mbnrg_2b_A1_B1_deg9_v1.cpp:121-220,
# blocks :11-25 (na+, cl-), :27-41 (cs+, ar)).
# ---------------------------------------------------------------------------
_ATOM2B = {
    # (first, second): (k, d0, ri, ro, name, table)
    ("na+", "na+"): (4.380148617370266e-01, 7.568203895545039e+00, 7.0, 9.0, "nana2b", "a1a12b"),
    ("cl-", "cl-"): (3.397551018612796e-01, 1.015131833802185e+01, 7.0, 9.0, "clcl2b", "a1a12b"),
    ("ar", "ar"): (6.511296783204924e-01, 5.457946966470896e+00, 7.0, 9.0, "arar2b", "a1a12b"),
    ("na+", "cl-"): (7.325513873941363e-01, 5.045021050700971e+00, 7.0, 9.0, "nacl2b", "a1b12b"),
    ("cs+", "ar"): (7.020794887920050e-01, 5.319522241193717e+00, 7.0, 9.0, "csar2b", "a1b12b"),
}


def _atom2b(pair):
    k, d0, ri, ro, name, table = _ATOM2B[pair]
    src = "potential/2b/mbnrg_2b_A1_A1_deg9_v1.cpp:138" if table == "a1a12b" else \
        "potential/2b/mbnrg_2b_A1_B1_deg9_v1.cpp:121"
    return Spec(name=name, monomers=pair, nat=(1, 1), sites=("A", "B"), lp=(),
                variables=_vars(("A", "B"), [("exp", "A", "B", k, d0)]), switch="pair", ri=ri, rf=ro,
                skip="pair_gt", nvars=1, ncoef=9, degree=9, ref=src, table=table)


ATOM2B = tuple(_atom2b(p) for p in _ATOM2B)

# Argon - water 2b: mbnrg_A1_B1C2X2_deg5_v1("ar", "h2o"), argon first; the
# halide-water template at degree 5 (potential/2b/mbnrg_2b_A1_B1C2X2_deg5_v1.cpp
# :616-760, variables :684-691, switch 6 -> 8 A, constructor block :11-516).
_k = (2.024685536820054e-07, 1.081497729997992e-01, 5.088638473248670e-01, 5.831588251891519e-01,
      1.961512707948666e-01)
ARH2O2B = Spec(
    name="arh2o2b", monomers=("ar", "h2o"), nat=(1, 3), sites=_S_HAL2B, lp=((1, 1, 4, 5),),
    variables=_vars(_S_HAL2B, [("coul", "A", "B", _k[0], 0.0), ("coul", "A", "C1", _k[1], 0.0),
                         ("coul", "A", "C2", _k[1], 0.0), ("exp", "A", "X1", _k[2], 0.0),
                         ("exp", "A", "X2", _k[2], 0.0), ("exp", "B", "C1", _k[3], 0.0),
                         ("exp", "B", "C2", _k[3], 0.0), ("exp", "C1", "C2", _k[4], 0.0)]),
    switch="pair", ri=6.0, rf=8.0, skip="pair_gt", nvars=8, ncoef=496, degree=5,
    ref="potential/2b/mbnrg_2b_A1_B1C2X2_deg5_v1.cpp:616",
)

# ---------------------------------------------------------------------------
# Template-generated MB-nrg evaluators (H2, NH3, CH4-CO2, MB-pbe water, CO2
# 3b): their specs are read from the reference's sources by
# codegen/mbnrg_spec.py into data/<name>.spec.json (same fields as above).
# ---------------------------------------------------------------------------
EXTRACTED = ("h2h22b", "h2oh22b", "csh22b", "nh3nh32b", "nh3pbe2b", "ch4co22b", "mbpbe2b", "co23b", "mbpbe3b",
             "n2o5h2o3b")


def _load_extracted(name):
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", name + ".spec.json")) as f:
        d = json.load(f)
    return Spec(name=d["name"], monomers=tuple(d["monomers"]), nat=tuple(d["nat"]), sites=tuple(d["sites"]),
                lp=tuple(tuple(x) for x in d["lp"]),
                variables=tuple((v[0], int(v[1]), int(v[2]), float(v[3]), float(v[4])) for v in d["variables"]),
                switch=d["switch"], ri=float(d["ri"]), rf=float(d["rf"]), skip=d["skip"], nvars=int(d["nvars"]),
                ncoef=int(d["ncoef"]), degree=int(d["degree"]), ref=d["ref"], table=d["table"])


TEMPLATE_SPECS = tuple(_load_extracted(n) for n in EXTRACTED)

# ---------------------------------------------------------------------------
# CO2 - CO2 2b: x2b_A1B2_A1B2_v1x(m, m) for the CO2 models co2_archive, co2
# and co2cm5100 .. co2cm580, potential/2b/x2b_A1B2_A1B2_v1x.cpp:18485-18700
# (variables :18562-18580, local variable::v_exp(r0, k) = exp(k (r0 - r))
# :62-77; f_switch :18373-18386 on the C-C distance, dimers beyond r2f
# skipped :18541).  One polynomial (poly_2b_A1B2_A1B2_v1x, 15 variables,
# degree 5, 2269 coefficients); constants and coefficients per model
# (constructor blocks at the lines given below).
# ---------------------------------------------------------------------------
_S_CO22B = ("Aa", "B1a", "B2a", "Ab", "B1b", "B2b")
_CO22B = {
    # model: (evaluator, d_intra_AB, k_intra_AB, d_intra_BB, k_intra_BB, d_AA, k_AA, d_AB, k_AB, d_BB, k_BB, r2i,
    #         r2f), constructor block line
    "co2_archive": ("co2a2b", 2.533470783111825e+00, 1.772445777810116e+00, 1.299246633223584e+00,
                    1.546435354569379e+00, 4.042621705776338e+00, 1.375890559471216e+00, 4.893559114105628e+00,
                    7.248440685272545e-01, 2.785825083032128e+00, 2.691866638221668e+00, 8.0, 9.0),  # :88
    "co2": ("co2co22b", 3.098180719521002e+00, 1.267379326287500e+00, 2.152649569148020e+00, 6.904623477544016e-01,
            4.195717132005157e+00, 6.959794865790364e-02, 6.633057823695092e+00, 9.311550654726656e-01,
            5.614642310195038e+00, 1.053234040860423e+00, 7.0, 9.0),  # :2373
    "co2cm5100": ("cm5100co22b", 3.098180719521002e+00, 1.267379326287500e+00, 2.152649569148020e+00,
                  6.904623477544016e-01, 4.195717132005157e+00, 6.959794865790364e-02, 6.633057823695092e+00,
                  9.311550654726656e-01, 5.614642310195038e+00, 1.053234040860423e+00, 7.0, 9.0),  # :4657
    "co2cm595": ("cm595co22b", 4.903036747511356e+00, 9.019913232531600e-01, 2.703937855283358e+00,
                 1.004834209745757e+00, 4.537101521312326e+00, 9.163852883742113e-02, 6.300498483648834e+00,
                 9.021417601624032e-01, 5.827456239776177e+00, 1.089701616045492e+00, 7.0, 9.0),  # :6941
    "co2cm590": ("cm590co22b", 2.329138487337566e+00, 1.434391663074755e+00, 3.229816367099317e+00,
                 9.702035861774958e-01, 4.006166160264772e+00, 1.117857009888089e-01, 5.789451971684920e+00,
                 8.757387756335298e-01, 5.798891302817732e+00, 1.133531479542603e+00, 7.0, 9.0),  # :9226
    "co2cm585": ("cm585co22b", 2.165524277685071e+00, 2.061892967817994e+00, 2.835603377312035e+00,
                 3.459793262493814e+00, 4.235604053709159e+00, 1.141488887995241e-01, 4.667583436073858e+00,
                 8.691887001880019e-01, 5.473818228420447e+00, 1.157204319628839e+00, 7.0, 9.0),  # :11513
    "co2cm5875": ("cm5875co22b", 3.134332315833306e+00, 1.282904902772805e+00, 4.434199799497058e+00,
                  8.407363065419096e-01, 1.800437262469989e+00, 1.216397961826567e-01, 6.926666442517130e+00,
                  8.810761305307210e-01, 4.127797348559158e+00, 1.148765431751049e+00, 7.0, 9.0),  # :13798
    "co2cm580": ("cm580co22b", 4.158829702809511e+00, 8.744952741703924e-01, 9.999985981119849e+00,
                 4.486543492998215e-01, 3.899891165573160e+00, 1.074038746629509e+00, 4.292889407717251e+00,
                 6.400679425638476e-01, 4.386671648943636e+00, 1.326376079648352e+00, 7.0, 9.0),  # :16083
}
# On this path: co2 and co2_archive.  The six co2cm* models share the
# polynomial with their own constants; each would be another ~10 MB of
# kernel code, and they are left out (their dimers evaluate to 0 here).
CO2_MODELS = ("co2", "co2_archive", "co2cm5100", "co2cm595", "co2cm590", "co2cm585", "co2cm5875", "co2cm580")
# evaluators that run another evaluator's kernels (and coefficients): the
# reference's co2cm5100 block (x2b_A1B2_A1B2_v1x.cpp:4657) repeats the co2
# block's constants and coefficients exactly (:2373), so its dimers run the
# co2 kernels; water with any CO2 model but co2_archive runs the H2O - CO2
# evaluator with the co2 constants (energy2b.cpp:140-145, :318-321), one
# alias per model so that each carries its monomer ids
KERNEL_ALIASES = {"cm5100co22b": "co2co22b"}
KERNEL_ALIASES.update({"h2o%sco22b" % m[3:]: "h2oco22b" for m in CO2_MODELS if m.startswith("co2cm")})


def _co22b(model):
    name, dAB_i, kAB_i, dBB_i, kBB_i, dAA, kAA, dAB, kAB, dBB, kBB, ri, rf = _CO22B[model]
    tab = [("Aa", "B1a", kAB_i, dAB_i), ("Aa", "B2a", kAB_i, dAB_i), ("B1a", "B2a", kBB_i, dBB_i),
           ("Ab", "B1b", kAB_i, dAB_i), ("Ab", "B2b", kAB_i, dAB_i), ("B1b", "B2b", kBB_i, dBB_i),
           ("Aa", "Ab", kAA, dAA), ("Aa", "B1b", kAB, dAB), ("Aa", "B2b", kAB, dAB),
           ("B1a", "Ab", kAB, dAB), ("B1a", "B1b", kBB, dBB), ("B1a", "B2b", kBB, dBB),
           ("B2a", "Ab", kAB, dAB), ("B2a", "B1b", kBB, dBB), ("B2a", "B2b", kBB, dBB)]
    return Spec(name=name, monomers=(model, model), nat=(3, 3), sites=_S_CO22B, lp=(),
                variables=_vars(_S_CO22B, [("exp", a, b, k, d) for a, b, k, d in tab]), switch="pair", ri=ri,
                rf=rf, skip="pair_gt", nvars=15, ncoef=2269, degree=5,
                ref="potential/2b/x2b_A1B2_A1B2_v1x.cpp:18485", table="co2co22btab")


CO22B = tuple(_co22b(m) for m in CO2_MODELS)

# ---------------------------------------------------------------------------
# H2O - CO2 2b: x2b_A1B2Z2_C1D2_v1x("h2o", "co2"), water first,
# potential/2b/x2b_A1B2Z2_C1D2_v1x.cpp:3635-3891 (variables :3685-3711,
# local variable::v_exp(r0, k) = exp(k (r0 - r)) :63-77; MB-pol lone pairs
# :3683; f_switch :3503-3516 on the O-C distance, dimers beyond r2f skipped
# :3690; constructor block :1821-3498).  The reference evaluates every CO2
# model but co2_archive against water with these constants
# (energy2b.cpp:318-321); co2_archive has a block of its own (H2OCO2A2B).
# ---------------------------------------------------------------------------
_S_H2OCO2 = ("A", "B1", "B2", "C", "D1", "D2", "Z1", "Z2")
_hc = dict(iAB=(4.592278064081765e-01, 4.092695741312179e-01), iBB=(1.797813612275968e+00, 2.515176186264408e+00),
           iCD=(1.231347340156158e+00, 1.752314332686619e+00), iDD=(1.094966061053114e+00, 2.988285212499331e+00),
           AC=(2.896045802044917e+00, 3.685742424189701e+00), AD=(1.353339012220006e+00, 3.527920970445803e+00),
           BC=(9.715865977702702e-01, 2.782062426936132e+00), BD=(7.363939494330982e-01, 8.005028705768890e-01),
           CZ=(8.336695227449923e-01, 5.744059557046924e+00), DZ=(1.053500025566689e+00, 3.961598744247630e+00))
_tab = [("A", "B1", "iAB"), ("A", "B2", "iAB"), ("B1", "B2", "iBB"), ("C", "D1", "iCD"), ("C", "D2", "iCD"),
        ("D1", "D2", "iDD"), ("A", "C", "AC"), ("A", "D1", "AD"), ("A", "D2", "AD"), ("B1", "C", "BC"),
        ("B1", "D1", "BD"), ("B1", "D2", "BD"), ("B2", "C", "BC"), ("B2", "D1", "BD"), ("B2", "D2", "BD"),
        ("Z1", "C", "CZ"), ("Z1", "D1", "DZ"), ("Z1", "D2", "DZ"), ("Z2", "C", "CZ"), ("Z2", "D1", "DZ"),
        ("Z2", "D2", "DZ")]
H2OCO22B = Spec(
    name="h2oco22b", monomers=("h2o", "co2"), nat=(3, 3), sites=_S_H2OCO2, lp=((0, 0, 6, 7),),
    variables=_vars(_S_H2OCO2, [("exp", a, b) + _hc[key] for a, b, key in _tab]), switch="pair", ri=8.0, rf=9.0,
    skip="pair_gt", nvars=21, ncoef=1653, degree=4, ref="potential/2b/x2b_A1B2Z2_C1D2_v1x.cpp:3635",
)
# water - co2_archive: the same evaluator with the constants of its own block
# (x2b_A1B2Z2_C1D2_v1x.cpp:144-1802; the switch radii are the header's
# defaults 8 and 9 A, x2b_A1B2Z2_C1D2_v1x.h:129-132)
_hca = dict(iAB=(2.991129377354730e+00, 9.711475336203186e-01), iBB=(1.776076592672980e+00, 2.247507043695376e+00),
            iCD=(8.784095840943548e-01, 2.930193028642861e+00), iDD=(2.220694581661451e+00, 2.481043684198385e+00),
            AC=(9.760814515633827e-01, 2.730468459200360e+00), AD=(2.671217176193513e+00, 2.711874357778875e+00),
            BC=(1.206205856757539e+00, 4.665335309987695e+00), BD=(2.879622692196830e-01, 6.043660542816871e+00),
            CZ=(1.382134149600439e+00, 4.584956529773560e+00), DZ=(3.624833784927413e+00, 4.021523821428722e+00))
H2OCO2A2B = replace(H2OCO22B, name="h2oco2a2b", monomers=("h2o", "co2_archive"), table="h2oco22b",
                    variables=_vars(_S_H2OCO2, [("exp", a, b) + _hca[key] for a, b, key in _tab]))
H2OCO2CM2B = tuple(replace(H2OCO22B, name="h2o%sco22b" % m[3:], monomers=("h2o", m), table="h2oco22b")
                   for m in CO2_MODELS if m.startswith("co2cm"))

# ---------------------------------------------------------------------------
# Helium: He - He 2b x2b_A1_A1_v1x (potential/2b/x2b_A1_A1_deg23_v1x.cpp:398,
# one variable exp(k (d0 - r)) :441, degree-23 polynomial, switch 7 -> 8 A on
# the He-He distance, block :283-316) and H2O - He 2b x2b_A1B2Z2_C1_v1x
# (potential/2b/x2b_A1B2Z2_C1_deg5_v1x.cpp:896, water first, MB-pol lone
# pairs :948, local v_exp / v_coul with d0 = 0 :76-122, variables :953-960,
# switch 9.5 -> 10.5 A on the O-He distance, block :283-291).
# ---------------------------------------------------------------------------
HEHE2B = Spec(
    name="hehe2b", monomers=("he", "he"), nat=(1, 1), sites=("A", "B"), lp=(),
    variables=_vars(("A", "B"), [("exp", "A", "B", 3.224372466704150e-01, 5.731623745108086e+00)]),
    switch="pair", ri=7.0, rf=8.0, skip="pair_gt", nvars=1, ncoef=23, degree=23,
    ref="potential/2b/x2b_A1_A1_deg23_v1x.cpp:398",
)
_S_H2OHE = ("A", "B1", "B2", "C", "Z1", "Z2")
_kAB, _kBB, _kAC, _kBC, _kCZ = (3.508775028719293e-03, 2.754491059307637e-02, 2.291365738385344e-01,
                                7.249481919751055e-01, 1.496283150810939e-01)
H2OHE2B = Spec(
    name="h2ohe2b", monomers=("h2o", "he"), nat=(3, 1), sites=_S_H2OHE, lp=((0, 0, 4, 5),),
    variables=_vars(_S_H2OHE, [("exp", "A", "B1", _kAB, 0.0), ("exp", "A", "B2", _kAB, 0.0),
                               ("exp", "B1", "B2", _kBB, 0.0), ("exp", "A", "C", _kAC, 0.0),
                               ("exp", "B1", "C", _kBC, 0.0), ("exp", "B2", "C", _kBC, 0.0),
                               ("coul", "Z1", "C", _kCZ, 0.0), ("coul", "Z2", "C", _kCZ, 0.0)]),
    switch="pair", ri=9.5, rf=10.5, skip="pair_gt", nvars=8, ncoef=496, degree=5,
    ref="potential/2b/x2b_A1B2Z2_C1_deg5_v1x.cpp:896",
)

# ---------------------------------------------------------------------------
# N2O5 - H2O 2b: x2b_A1B2C4_D1E2_v1x("h2o", "n2o5"), N2O5 first (sites A =
# bridging O, B = N, C = terminal O; water D = O, E = H),
# potential/2b/x2b_A1B2C4_D1E2_deg3_v1x.cpp:1183 (variables exp(-k r) with the
# local variable::v_exp :19-34, listed :1226-1270; switch 8 -> 9 A on the
# bridging-O - water-O distance, dimers beyond r2f skipped :1200; constructor
# block :59-1060).  Its virial sums -r . g over the polynomial's own gradient,
# before the switch factor and without the switch gradient (:1353-1391), so
# it differs from -r . (total gradient) for dimers between 8 and 9 A.
# N2O5 - H2O - H2O 3b is the template evaluator
# mbnrg_3b_A1B2C4_D1E2_D1E2_deg3_v1 with the cos2 switch (extracted spec).
# ---------------------------------------------------------------------------
_S_N2O5H2O = ("A", "B1", "B2", "C1", "C2", "C3", "C4", "D", "E1", "E2")
_kn = dict(AD=7.286306346099436e-01, AE=7.828602981218888e-01, BD=3.351348473713356e-01, BE=3.639320594943890e-01,
           CD=6.858079184494418e-01, CE=6.808310453124187e-01, BB=6.196445062175264e-01, CC=3.302260758676124e-01,
           AB=8.129813213030901e-01, AC=4.872207055177465e-01, BC=9.817144022006012e-01, EE=1.532053819248005e-01,
           DE=1.268361659534204e+00)
_C4 = ("C1", "C2", "C3", "C4")
_tab = ([("B1", "B2", "BB")] + [(a, b, "CC") for i, a in enumerate(_C4) for b in _C4[i + 1:]] +
        [("A", b, "AB") for b in ("B1", "B2")] + [("A", c, "AC") for c in _C4] +
        [(b, c, "BC") for b in ("B1", "B2") for c in _C4] + [("E1", "E2", "EE"), ("D", "E1", "DE"), ("D", "E2", "DE"),
                                                             ("A", "D", "AD"), ("A", "E1", "AE"), ("A", "E2", "AE"),
                                                             ("B1", "D", "BD"), ("B2", "D", "BD")] +
        [(b, e, "BE") for b in ("B1", "B2") for e in ("E1", "E2")] + [(c, "D", "CD") for c in _C4] +
        [(c, e, "CE") for c in _C4 for e in ("E1", "E2")])
N2O5H2O2B = Spec(
    name="n2o5h2o2b", monomers=("n2o5", "h2o"), nat=(7, 3), sites=_S_N2O5H2O, lp=(),
    variables=_vars(_S_N2O5H2O, [("exp", a, b, _kn[key], 0.0) for a, b, key in _tab]), switch="pair", ri=8.0,
    rf=9.0, skip="pair_gt", nvars=45, ncoef=983, degree=3, ref="potential/2b/x2b_A1B2C4_D1E2_deg3_v1x.cpp:1183",
    virial="raw",
)

FH2O3B = _hal3b("f-", "fh2o3b")
CLH2O3B = _hal3b("cl-", "clh2o3b")
BRH2O3B = _hal3b("br-", "brh2o3b")
IH2O3B = _hal3b("i-", "ih2o3b")

SPECS = {s.name: s for s in (MBPOL2B, MBPOL3B, CH4H2O2B, CH4CH42B, CH4H2O3B,
                             H2OLI2B, H2ONA2B, H2OK2B, H2ORB2B, H2OCS2B,
                             H2OLI3B, H2ONA3B, H2OK3B, H2ORB3B, H2OCS3B,
                             FH2O2B, CLH2O2B, BRH2O2B, IH2O2B, FH2O3B, CLH2O3B, BRH2O3B, IH2O3B,
                             ARH2O2B, H2OCO22B, H2OCO2A2B, HEHE2B, H2OHE2B, N2O5H2O2B) + H2OCO2CM2B + ATOM2B + TEMPLATE_SPECS + CO22B}

# Dispatch by sorted monomer ids (e2b::get_2b_energy, potential/2b/energy2b.cpp:
# 240-254,258-281,282,323; e3b::get_3b_energy, potential/3b/energy3b.cpp:185-216,
# 220-228,243).  Any other tuple evaluates to 0, as in the reference's else branch.
DISPATCH_2B = {("h2o", "h2o"): "mbpol2b", ("ch4", "h2o"): "ch4h2o2b", ("ch4", "ch4"): "ch4ch42b",
               ("h2o", "li+"): "h2oli2b", ("h2o", "na+"): "h2ona2b", ("h2o", "k+"): "h2ok2b",
               ("h2o", "rb+"): "h2orb2b", ("cs+", "h2o"): "h2ocs2b",
               ("f-", "h2o"): "fh2o2b", ("cl-", "h2o"): "clh2o2b", ("br-", "h2o"): "brh2o2b", ("h2o", "i-"): "ih2o2b",
               ("na+", "na+"): "nana2b", ("cl-", "cl-"): "clcl2b", ("ar", "ar"): "arar2b", ("cl-", "na+"): "nacl2b",
               ("ar", "cs+"): "csar2b", ("ar", "h2o"): "arh2o2b",
               ("h2", "h2"): "h2h22b", ("h2", "h2o"): "h2oh22b", ("cs+", "h2"): "csh22b", ("nh3", "nh3"): "nh3nh32b",
               ("nh3pbe0d3bj", "nh3pbe0d3bj"): "nh3pbe2b", ("ch4", "co2"): "ch4co22b", ("mbpbe", "mbpbe"): "mbpbe2b"}
DISPATCH_2B.update({(m, m): _CO22B[m][0] for m in CO2_MODELS})
# water with any CO2 model but co2_archive: the co2 constants
# (energy2b.cpp:140-145 and :318-321)
DISPATCH_2B[("co2", "h2o")] = "h2oco22b"
DISPATCH_2B[("co2_archive", "h2o")] = "h2oco2a2b"
DISPATCH_2B.update({(m, "h2o"): "h2o%sco22b" % m[3:] for m in CO2_MODELS if m.startswith("co2cm")})
DISPATCH_2B[("he", "he")] = "hehe2b"
DISPATCH_2B[("h2o", "he")] = "h2ohe2b"
DISPATCH_2B[("h2o", "n2o5")] = "n2o5h2o2b"
DISPATCH_3B = {("h2o", "h2o", "h2o"): "mbpol3b", ("ch4", "h2o", "h2o"): "ch4h2o3b",
               ("h2o", "h2o", "li+"): "h2oli3b", ("h2o", "h2o", "na+"): "h2ona3b", ("h2o", "h2o", "k+"): "h2ok3b",
               ("h2o", "h2o", "rb+"): "h2orb3b", ("cs+", "h2o", "h2o"): "h2ocs3b",
               ("f-", "h2o", "h2o"): "fh2o3b", ("cl-", "h2o", "h2o"): "clh2o3b", ("br-", "h2o", "h2o"): "brh2o3b",
               ("h2o", "h2o", "i-"): "ih2o3b", ("co2", "co2", "co2"): "co23b", ("mbpbe", "mbpbe", "mbpbe"): "mbpbe3b",
               ("h2o", "h2o", "n2o5"): "n2o5h2o3b"}

# Real atoms and total sites (real + electrostatic virtual sites) per monomer
# type, as the reference's monomer table sets them (bblock/sys_tools.cpp
# SetUpMonomers:133-254: h2o has 3 atoms + the M site, ch4 5 atoms, the
# alkali-metal and halide ions and argon one atom, :210-225, h2 two, nh3
# four, co2 three, mbpbe like h2o three atoms and four sites, :191-233).
# ---------------------------------------------------------------------------
# 1-body MB-nrg: CH4, x1b_A1B4_deg5_exp0::x1b_A1B4_v1x,
# potential/1b/x1b_A1B4_deg5_exp0_v1x.cpp:309-419 (constants :302-305,
# variables v_exp0(d0, k) = exp(k (d0 - r)) :67-80, :327-336).  No switch, no
# cutoff: every local CH4 is evaluated (System::Get1B, system.cpp:2269).
# ---------------------------------------------------------------------------
_S = ("A1", "B1", "B2", "B3", "B4")
_kAB1, _dAB1 = 9.118575345478506e-01, 4.848036021821232e+00
_kBB1, _dBB1 = 3.397786901029656e-01, 6.999341954887242e+00
CH41B = Spec(
    name="ch41b", monomers=("ch4",), nat=(5,), sites=_S, lp=(),
    variables=_vars(_S, [("exp", "A1", "B%d" % i, _kAB1, _dAB1) for i in range(1, 5)] +
                    [("exp", "B%d" % i, "B%d" % j, _kBB1, _dBB1) for i in range(1, 5) for j in range(i + 1, 5)]),
    switch="none", ri=0.0, rf=0.0, skip="none",
    nvars=10, ncoef=207, degree=5, ref="potential/1b/x1b_A1B4_deg5_exp0_v1x.cpp:361",
)
# 1-body evaluators with a GPU kernel other than water's Partridge-Schwenke
# term, by monomer id (e1b::get_1b_energy, potential/1b/energy1b.cpp:53-56)
ONEBODY_SPECS = {CH41B.name: CH41B}
ONEBODY_DISPATCH = {"ch4": "ch41b"}

MONOMER_ATOMS = {"h2o": 3, "ch4": 5, "li+": 1, "na+": 1, "k+": 1, "rb+": 1, "cs+": 1,
                 "f-": 1, "cl-": 1, "br-": 1, "i-": 1, "ar": 1, "h2": 2, "nh3": 4, "nh3pbe0d3bj": 4, "co2": 3,
                 "mbpbe": 3, "co2_archive": 3, "co2cm5100": 3, "co2cm595": 3, "co2cm590": 3, "co2cm585": 3,
                 "co2cm5875": 3, "co2cm580": 3, "he": 1, "n2o5": 7}
MONOMER_SITES = dict(MONOMER_ATOMS, h2o=4, mbpbe=4)
# atom names a caller passes to AddMonomer for each id (input order)
MONOMER_ATOM_NAMES = {"h2o": ("O", "H", "H"), "ch4": ("C", "H", "H", "H", "H"), "li+": ("Li",), "na+": ("Na",),
                      "k+": ("K",), "rb+": ("Rb",), "cs+": ("Cs",), "f-": ("F",), "cl-": ("Cl",), "br-": ("Br",),
                      "i-": ("I",), "ar": ("Ar",), "h2": ("H", "H"), "nh3": ("N", "H", "H", "H"),
                      "nh3pbe0d3bj": ("N", "H", "H", "H"), "co2": ("C", "O", "O"), "mbpbe": ("O", "H", "H")}
MONOMER_ATOM_NAMES["he"] = ("He",)
# n2o5: bridging O, the two N, then the four terminal O (bonds 0-1, 0-2, 1-3,
# 1-4, 2-5, 2-6, bblock/sys_tools.cpp:725-733)
MONOMER_ATOM_NAMES["n2o5"] = ("O", "N", "N", "O", "O", "O", "O")
MONOMER_ATOM_NAMES.update({m: ("C", "O", "O") for m in ("co2_archive", "co2cm5100", "co2cm595", "co2cm590",
                                                         "co2cm585", "co2cm5875", "co2cm580")})


def check():
    for s in SPECS.values():
        assert len(s.variables) == s.nvars, (s.name, len(s.variables))
        assert len(s.sites) == s.nreal + 2 * len(s.lp), s.name
    return True


def sorted_slots(ids):
    """Slot order into which the reference's dispatch sorts monomer ids
    (potential/2b/energy2b.cpp:240-254; potential/3b/energy3b.cpp:185-216)."""
    m = list(ids)
    if len(m) == 2:
        return (1, 0) if m[1] < m[0] else (0, 1)
    k = [0, 1, 2]
    if m[2] < m[0] and m[2] < m[1]:
        m[0], m[2] = m[2], m[0]
        k[0], k[2] = k[2], k[0]
    if m[0] > m[1] and m[0] > m[2]:
        m[0], m[2] = m[2], m[0]
        k[0], k[2] = k[2], k[0]
    elif m[1] > m[0] and m[1] > m[2]:
        m[1], m[2] = m[2], m[1]
        k[1], k[2] = k[2], k[1]
    if m[0] > m[1]:
        m[0], m[1] = m[1], m[0]
        k[0], k[1] = k[1], k[0]
    return tuple(k)


def dispatch(ids):
    """(evaluator name or None, evaluator slot -> original slot) for an n-mer
    whose monomers, in n-mer order, have the given ids."""
    so = sorted_slots(ids)
    sorted_ids = [ids[s] for s in so]
    table = DISPATCH_2B if len(ids) == 2 else DISPATCH_3B
    name = table.get(tuple(sorted_ids))
    if name is None:
        return None, None
    used = [False] * len(ids)
    order = []
    for h in SPECS[name].monomers:
        for s in range(len(ids)):
            if not used[s] and sorted_ids[s] == h:
                used[s] = True
                order.append(so[s])
                break
    return name, tuple(order)
