#!/usr/bin/env python3
"""Extract the reference's golden vectors for the 2b/3b path into JSON fixtures.

Reads the reference's own Catch2 unit tests and timing fixtures (from a
reference checkout: --ref or MBX_REFERENCE) and writes ``tests/golden/*.json``:

* evaluator / dispatch goldens: ``unittest-energy2b.cpp`` (h2o-h2o :48-97,
  ch4-ch4 :314-360, ch4-h2o :361-427), ``unittest-energy3b.cpp`` (h2o x3
  :48-145, ch4-h2o-h2o :472-571), ``unittest-poly-holder-2b.cpp``
  (x2b_A1B2Z2_C1D4_v1x :659-706, x2b_A1B4_A1B4_v1x :935-974,
  x2b_v9x :975-1018), ``unittest-poly-holder-3b.cpp`` (mbnrg_3b_A1B4_C1D2_C1D2
  :337-383, x3b-v2x :910-954);
* alkali-ion - water 2b: ``unittest-energy2b.cpp`` (cs-h2o :166-236, li-h2o
  :237-313), ``unittest-poly-holder-2b.cpp`` (x2b_h2o_ion_v2x :707-934, one
  fixture per ion), ``unittest-poly-2b.cpp`` (poly_2b_A1B2Z2_C_deg5_v1x
  :2327-2536);
* halide - water 2b / halide - water - water 3b: ``unittest-energy2b.cpp``
  (f--h2o :1322, cl-h2o :1380, br-h2o :1438, i-h2o :1498),
  ``unittest-energy3b.cpp`` (f-h2o-h2o :1010, cl- :1104, br- :1198, i- :1292),
  ``unittest-poly-holder-2b.cpp`` (mbnrg_A1_B1C2X2_deg6_v1 sections :64-219),
  ``unittest-poly-holder-3b.cpp`` (mbnrg_A1_B1C2X2_B1C2X2_deg4_v1 :174-336);
* atom - atom 2b and argon - water 2b: ``unittest-energy2b.cpp`` (ar-ar :820,
  cl-cl :867, na-na :914, ar-cs :965, na-cl :1012, ar-h2o :1063),
  ``unittest-poly-holder-2b.cpp`` (mbnrg_A1_A1_deg9_v1 :1229-1312,
  mbnrg_A1_B1_deg9_v1 :1313-1370, mbnrg_A1_B1C2X2_deg5_v1 ar-h2o :220),
  ``unittest-poly-2b.cpp`` (poly_2b_A1_B1C2X2_deg5_v1 :53-204);
* template MB-nrg types: ``unittest-energy2b.cpp`` (h2-h2 :544, h2-h2o :607,
  nh3-nh3 :674, nh3pbe0d3bj :741, h2-cs :1126, mbpbe-mbpbe :1250, ch4-co2
  :1943), ``unittest-energy3b.cpp`` (mbpbe x3 :911, co2 x3 :1386),
  ``unittest-poly-holder-2b.cpp`` (:1019-1546), ``unittest-poly-holder-3b.cpp``
  (:84-173);
* CO2 - CO2 2b: ``unittest-energy2b.cpp`` (co2_archive :99, co2 :1558, the
  co2cm* models :1613-1942), ``unittest-poly-holder-2b.cpp``
  (x2b_A1B2_A1B2_v1x :263-560),
  ``unittest-poly-2b.cpp`` (poly_2b_A1B2_A1B2_v1x :205-993);
* H2O - CO2 2b: ``unittest-energy2b.cpp`` (h2o-co2 :2000, co2_archive-h2o
  :428), ``unittest-poly-holder-2b.cpp`` (x2b_A1B2Z2_C1D2_v1x h2o-co2 :562,
  h2o-co2_archive :596),
  ``unittest-poly-2b.cpp`` (poly_2b_A1B2Z2_C1D2_v1x :994-1580);
* N2O5 - water 2b and 3b: ``unittest-energy2b.cpp`` (n2o5-h2o :1180),
  ``unittest-poly-holder-2b.cpp`` (x2b_A1B2C4_D1E2_v1x h2o-n2o5 :1407),
  ``unittest-energy3b.cpp`` (n2o5-h2o-h2o :808), ``unittest-poly-holder-3b.cpp``
  (mbnrg_A1B2C4_D1E2_D1E2_deg3_v1 :956);
* water - water - alkali-ion 3b: ``unittest-energy3b.cpp`` (li-h2o-h2o
  :146-357, cs-h2o-h2o :358-471), ``unittest-poly-holder-3b.cpp``
  (x3b_h2o_ion_v1x_deg4_filtered :384-909, one fixture per ion),
  ``unittest-poly-3b.cpp`` (poly_3b_h2o_ion_v1x_deg4_filtered :1350-1719);
* polynomial goldens: ``unittest-poly-2b.cpp`` (poly_2b_v6x :2537-3012,
  poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x :1581-1827, poly_2b_A1B4_A1B4_deg4_exp0_v1x
  :1828-2326), ``unittest-poly-3b.cpp`` (poly_3b_A1B4_C1D2_C1D2_deg3_v1
  :879-1349, poly-3b-v2x :1720-2160);
* system fixtures: the coordinates of ``timing/256_h2o_cubic_box`` and
  ``timing/57_ch4_513_h2o_rectangular`` with their published E2B/E3B
  (``timing/*/output:5-6``) and configuration (``mbx.json``).

Every array is copied verbatim (as numbers); nothing else of the reference is
kept.  Run: ``python tests/golden/make_golden.py [--ref DIR] (or MBX_REFERENCE)``.
"""
import argparse
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))

BLOCKS = [
    # (fixture name, file, header regex)
    ("energy2b_h2o_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)', r'SECTION\("h2o-h2o"\)'),
    ("energy2b_ch4_ch4", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)', r'SECTION\("ch4-ch4"\)'),
    ("energy2b_ch4_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)', r'SECTION\("ch4-h2o"\)'),
    ("energy3b_h2o_h2o_h2o", "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("h2o-h2o-h2o"\)'),
    ("energy3b_ch4_h2o_h2o", "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("ch4-h2o-h2o"\)'),
    ("holder2b_x2b_v9x", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_v9x::struct"\)', None),
    ("holder2b_ch4_h2o", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2Z2_C1D4_v1x::struct"\)', None),
    ("holder2b_ch4_ch4", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B4_A1B4_v1x::struct"\)', None),
    ("holder3b_x3b_v2x", "src/unittests/unittest-poly-holder-3b.cpp", r'TEST_CASE\("x3b-v2x::class"\)', None),
    ("holder3b_ch4_h2o_h2o", "src/unittests/unittest-poly-holder-3b.cpp", r'TEST_CASE\("mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1::class"\)', None),
    ("poly_mbpol2b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_v6x:struct"\)', None),
    ("poly_ch4h2o2b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x:struct"\)', None),
    ("poly_ch4ch42b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\("poly_2b_A1B4_A1B4_deg4_exp0_v1x:struct"\)', None),
    ("poly_ch4h2o3b", "src/unittests/unittest-poly-3b.cpp", r'TEST_CASE\("poly_3b_A1B4_C1D2_C1D2_deg3_v1.h"\)', None),
    ("poly_mbpol3b", "src/unittests/unittest-poly-3b.cpp", r'TEST_CASE\("poly-3b-v2x::class"\)', None),
    # alkali-metal ion - water 2b
    ("energy2b_cs_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)', r'SECTION\("cs-h2o"\)'),
    ("energy2b_li_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)', r'SECTION\("li-h2o"\)'),
    ("poly_h2oion2b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_A1B2Z2_C_deg5_v1x:struct"\)', None),
] + [("holder2b_h2o_%s" % ion, "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_h2o_ion_v2x::struct"\)',
      r'SECTION\("h2o-%s"\)' % ion) for ion in ("li", "na", "k", "rb", "cs")]
# water - water - alkali-ion 3b
BLOCKS += [
    ("energy3b_li_h2o_h2o", "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("li-h2o-h2o"\)'),
    ("energy3b_cs_h2o_h2o", "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("cs-h2o-h2o"\)'),
    ("poly_h2oion3b", "src/unittests/unittest-poly-3b.cpp", r'TEST_CASE\("poly-3b-h2o-ion-v1x_deg4_filtered::class"\)',
     None),
] + [("holder3b_h2o_h2o_%s" % ion, "src/unittests/unittest-poly-holder-3b.cpp",
      r'TEST_CASE\("x3b-3b-h2o-ion-v1x_deg4_filtered::class"\)', r'SECTION\("h2o-h2o-%s"\)' % ion)
     for ion in ("li", "na", "k", "rb", "cs")]
# halide - water 2b and halide - water - water 3b
_HAL = (("f", "f--h2o", "f-h2o-h2o"), ("cl", "cl-h2o", "cl-h2o-h2o"), ("br", "br-h2o", "br-h2o-h2o"),
        ("i", "i-h2o", "i-h2o-h2o"))
BLOCKS += [("energy2b_%s_h2o" % h, "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
            r'SECTION\("%s"\)' % s2) for h, s2, _ in _HAL]
BLOCKS += [("energy3b_%s_h2o_h2o" % h, "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("%s"\)' % s3)
           for h, _, s3 in _HAL]
BLOCKS += [("holder2b_%s_h2o" % h, "src/unittests/unittest-poly-holder-2b.cpp",
            r'TEST_CASE\("mbnrg_A1_B1C2X2_deg5_v1::struct"\)', r'SECTION\("%s--h2o"\)' % h) for h, _, _ in _HAL]
BLOCKS += [("holder3b_%s_h2o_h2o" % h, "src/unittests/unittest-poly-holder-3b.cpp",
            r'TEST_CASE\("mbnrg_A1_B1C2X2_B1C2X2_deg4_v1::struct"\)', r'SECTION\("%s--h2o-h2o"\)' % h)
           for h, _, _ in _HAL]
# atom - atom 2b and argon - water 2b
BLOCKS += [("energy2b_%s" % f, "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
            r'SECTION\("%s"\)' % sec) for f, sec in (("ar_ar", "ar-ar"), ("cl_cl", "cl-cl"), ("na_na", "na-na"),
                                                      ("ar_cs", "ar-cs"), ("na_cl", "na-cl"), ("ar_h2o", "ar-h2o"))]
BLOCKS += [("holder2b_%s" % f, "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("%s"\)' % tc,
            r'SECTION\("%s"\)' % sec) for f, tc, sec in (
    ("ar_ar", "mbnrg_A1_A1_deg9_v1::struct", "ar-ar"), ("cl_cl", "mbnrg_A1_A1_deg9_v1::struct", "cl-cl"),
    ("na_na", "mbnrg_A1_A1_deg9_v1::struct", "na-na"), ("na_cl", "mbnrg_A1_B1_deg9_v1::struct", "na-cl"),
    ("ar_cs", "mbnrg_A1_B1_deg9_v1::struct", "ar-cs"), ("ar_h2o", "mbnrg_A1_B1C2X2_deg5_v1::struct", "ar-h2o"))]
BLOCKS += [("poly_arh2o2b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_A1_B1C2X2_deg5_v1:struct"\)',
            None)]
# template MB-nrg evaluators (H2, NH3, CH4-CO2, MB-pbe, CO2 3b)
BLOCKS += [("energy2b_%s" % f, "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
            r'SECTION\("%s"\)' % sec) for f, sec in (
    ("h2_h2", "h2-h2"), ("h2_h2o", "h2-h2o"), ("nh3_nh3", "nh3-nh3"), ("nh3pbe_nh3pbe", "nh3pbe0d3bj-nh3pbe0d3bj"),
    ("h2_cs", "h2-cs"), ("mbpbe_mbpbe", "mbpbe-mbpbe"), ("ch4_co2", "ch4-co2"))]
BLOCKS += [("energy3b_%s" % f, "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("%s"\)' % sec)
           for f, sec in (("mbpbe_mbpbe_mbpbe", "mbpbe-mbpbe-mbpbe"), ("co2_co2_co2", "co2-co2-co2"))]
BLOCKS += [("holder2b_%s" % f, "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("%s"\)' % tc,
            r'SECTION\("%s"\)' % sec) for f, tc, sec in (
    ("h2_h2", "mbnrg_A2_A2_deg6_v1::struct", "h2-h2"), ("h2_h2o", "mbnrg_2b_A1B2Z2_C2_deg5_v1::struct", "h2-h2o"),
    ("nh3_nh3", "mbnrg_A1B3_A1B3_deg4_v1::struct", "nh3-nh3"),
    ("nh3pbe_nh3pbe", "mbnrg_A1B3_A1B3_deg4_v1::struct", "nh3pbe0d3bj-nh3pbe0d3bj"),
    ("cs_h2", "mbnrg_A1_B2_deg7_v1::struct", "cs-h2"), ("mbpbe_mbpbe", "mbnrg_A1B2Z2_A1B2Z2_deg4_vmbpbe::struct",
                                                       "mbpbe-mbpbe"),
    ("ch4_co2", "mbnrg_A1B4_C1D2_deg4_v1::struct", "ch4-co2"))]
BLOCKS += [("holder3b_%s" % f, "src/unittests/unittest-poly-holder-3b.cpp", r'TEST_CASE\("%s"\)' % tc,
            r'SECTION\("%s"\)' % sec) for f, tc, sec in (
    ("mbpbe_mbpbe_mbpbe", "mbnrg_A1B2_A1B2_A1B2_deg4_vmbpbe::struct", "mbpbe-mbpbe-mbpbe"),
    ("co2_co2_co2", "mbnrg_A1B2_A1B2_A1B2_deg4_v1::struct", "co2-co2-co2"))]
# CO2 - CO2 2b (co2_archive and co2 models)
BLOCKS += [
    ("energy2b_co2a_co2a", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
     r'SECTION\("co2-co2"\)'),
    ("energy2b_co2_co2", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
     (r'SECTION\("co2-co2"\)', 1)),
    ("holder2b_co2a_co2a", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2_A1B2_v1x::struct"\)',
     r'SECTION\("co2_archive-co2_archive"\)'),
    ("holder2b_co2_co2", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2_A1B2_v1x::struct"\)',
     r'SECTION\("co2-co2"\)'),
    ("poly_co2co22b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_A1B2_A1B2_v1x:struct"\)', None),
    # H2O - CO2 2b (co2 model)
    ("energy2b_h2o_co2", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
     r'SECTION\("h2o-co2"\)'),
    ("holder2b_h2o_co2", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2Z2_C1D2_v1x::struct"\)',
     r'SECTION\("h2o-co2"\)'),
    ("poly_h2oco22b", "src/unittests/unittest-poly-2b.cpp", r'TEST_CASE\(":poly_2b_A1B2Z2_C1D2_v1x:struct"\)', None),
]
# CO2 - CO2 2b of the co2cm* models
CO2CM = ("co2cm5100", "co2cm595", "co2cm590", "co2cm5875", "co2cm585", "co2cm580")
BLOCKS += [("energy2b_%s" % m, "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
            r'SECTION\("%s-%s"\)' % (m, m)) for m in CO2CM]
BLOCKS += [("holder2b_%s" % m, "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2_A1B2_v1x::struct"\)',
            r'SECTION\("%s-%s"\)' % (m, m)) for m in CO2CM]
# H2O - CO2 2b, co2_archive model
BLOCKS += [
    ("energy2b_co2a_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
     r'SECTION\("co2-h2o"\)'),
    ("holder2b_h2o_co2a", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2Z2_C1D2_v1x::struct"\)',
     r'SECTION\("h2o-co2_archive"\)'),
]
# N2O5 - H2O 2b and N2O5 - H2O - H2O 3b
BLOCKS += [
    ("energy2b_n2o5_h2o", "src/unittests/unittest-energy2b.cpp", r'TEST_CASE\("energy2b::get_2b_energy"\)',
     r'SECTION\("n2o5-h2o"\)'),
    ("holder2b_h2o_n2o5", "src/unittests/unittest-poly-holder-2b.cpp", r'TEST_CASE\("x2b_A1B2C4_D1E2_v1x::struct"\)',
     r'SECTION\("h2o-n2o5"\)'),
    ("energy3b_n2o5_h2o_h2o", "src/unittests/unittest-energy3b.cpp", r'TEST_CASE', r'SECTION\("n2o5-h2o-h2o"\)'),
    ("holder3b_n2o5_h2o_h2o", "src/unittests/unittest-poly-holder-3b.cpp", r'TEST_CASE\("::struct"\)',
     r'SECTION\("n2o5-h2o-h2o"\)'),
]

SYSTEMS = [
    ("system_256_h2o_cubic_box", "timing/256_h2o_cubic_box"),
    ("system_57_ch4_513_h2o", "timing/57_ch4_513_h2o_rectangular"),
]


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def block_after(text, header, start=0):
    m = re.compile(header).search(text, start)
    if not m:
        raise ValueError("header %s not found" % header)
    i = text.index("{", m.end())
    depth, j = 1, i + 1
    while depth:
        depth += (text[j] == "{") - (text[j] == "}")
        j += 1
    return m.start(), text[i + 1:j - 1]


def parse_block(body):
    out = {}
    for m in re.finditer(r"std::vector<double>\s+(\w+)\s*=\s*\{([^}]*)\}\s*;", body):
        out[m.group(1)] = [float(v) for v in m.group(2).replace(",", " ").split()]
    for m in re.finditer(r"std::vector<double>\s+(\w+)\s*\(\s*([^)]*)\)\s*;", body):
        out.setdefault(m.group(1) + "__size", m.group(2).strip())
    for m in re.finditer(r"(?<![\w:])double\s+(\w+)\s*=\s*([-+0-9.eE]+)\s*;", body):
        out[m.group(1)] = float(m.group(2))
    for m in re.finditer(r"std::string\s+(\w+)\s*=\s*\"([^\"]*)\"\s*;", body):
        out[m.group(1)] = m.group(2)
    for m in re.finditer(r"(?:size_t|int)\s+(\w+)\s*=\s*(\d+)\s*;", body):
        out[m.group(1)] = int(m.group(2))
    return out


def extract_blocks(ref):
    for name, rel, case, section in BLOCKS:
        text = strip_comments(open(os.path.join(ref, rel)).read())
        pos, body = block_after(text, case)
        if section:
            # (regex, n): the n-th section with that header (0 = the first)
            sec, nth = section if isinstance(section, tuple) else (section, 0)
            start = 0
            for _ in range(nth):
                start = re.compile(sec).search(body, start).end()
            _, body = block_after(body, sec, start)
        data = parse_block(body)
        data["_source"] = rel
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(data, f)
        print(name, sorted(k for k in data if not k.startswith("_")))


def read_nrg(path):
    ids, xyz = [], []
    for line in open(path):
        w = line.split()
        if not w:
            continue
        if w[0].upper() == "MONOMER":
            ids.append(w[1])
        elif len(w) == 4 and w[0].isalpha() and w[0].upper() not in ("SYSTEM", "MOLECULE"):
            try:
                xyz += [float(v) for v in w[1:]]
            except ValueError:
                pass
    return ids, xyz


def extract_systems(ref):
    for name, rel in SYSTEMS:
        ids, xyz = read_nrg(os.path.join(ref, rel, "input.nrg"))
        cfg = json.load(open(os.path.join(ref, rel, "mbx.json")))["MBX"]
        out = {}
        for line in open(os.path.join(ref, rel, "output")):
            m = re.match(r"\s*(2B|3B)\s*=\s*([-+0-9.eE]+)", line)
            if m:
                out[m.group(1)] = float(m.group(2))
        data = {"ids": ids, "xyz": xyz, "box": cfg.get("box", []), "cutoff2b": cfg["twobody_cutoff"],
                "cutoff3b": cfg["threebody_cutoff"], "ignore_2b": cfg.get("ignore_2b_poly", []),
                "ignore_3b": cfg.get("ignore_3b_poly", []), "E2B": out["2B"], "E3B": out["3B"],
                "_source": rel}
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(data, f)
        print(name, len(ids), "monomers", data["E2B"], data["E3B"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MBX_REFERENCE"), required=not os.environ.get("MBX_REFERENCE"))
    a = ap.parse_args()
    extract_blocks(a.ref)
    extract_systems(a.ref)


if __name__ == "__main__":
    main()
