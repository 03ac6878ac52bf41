"""The spec extractor of the template-generated MB-nrg evaluators
(codegen/mbnrg_spec.py) against the specs written by hand for the same
template, and the committed extracted specs against a fresh extraction (CPU;
needs the reference's sources, skipped where they are absent)."""
import json
import os

import pytest

from mbx_b200.codegen import mbnrg_spec as ms
from mbx_b200.specs import SPECS

REF = "/root/reference"
needs_ref = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference sources absent")


@needs_ref
@pytest.mark.parametrize("name", list(ms.HANDWRITTEN))
def test_extractor_reproduces_handwritten(name):
    d = ms.extract(REF, name, *ms.HANDWRITTEN[name])
    s = SPECS[name]
    assert tuple(d["monomers"]) == s.monomers and tuple(d["nat"]) == s.nat
    assert len(d["sites"]) == len(s.sites)
    assert [tuple(x) for x in d["lp"]] == list(s.lp)
    assert [tuple(v) for v in d["variables"]] == list(s.variables)
    assert (d["switch"], d["skip"], d["ri"], d["rf"]) == (s.switch, s.skip, s.ri, s.rf)
    assert (d["nvars"], d["ncoef"], d["degree"]) == (s.nvars, s.ncoef, s.degree)
    assert d["table"] == s.pip_table


@needs_ref
@pytest.mark.parametrize("name", list(ms.SOURCES))
def test_committed_specs_match_extraction(name):
    d = ms.extract(REF, name, *ms.SOURCES[name])
    with open(os.path.join(ms.DATA, name + ".spec.json")) as f:
        c = json.load(f)
    assert json.loads(json.dumps(d)) == c
