"""The spec extractor of the template-generated MB-nrg evaluators
(codegen/mbnrg_spec.py) against the specs written by hand for the same
template, and the committed extracted specs against a fresh extraction (CPU;
needs the reference's sources, skipped where they are absent)."""
import json
import os

import pytest

from mbx_b200.codegen import mbnrg_spec as ms
from mbx_b200.specs import SPECS

REF = os.environ.get("MBX_REFERENCE", "")
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


def _reference_tuples(path, nb):
    """Sorted monomer-id tuples the reference's get_2b_energy / get_3b_energy
    dispatch on (their if/else-if chains, one tuple per alternative of an
    'a || b' slot)."""
    import itertools
    import re
    text = open(path).read()
    out = set()
    for cond in re.findall(r"if\s*\((.*?)\)\s*\{", text, re.S):
        slots = {}
        for i, m in re.findall(r'mon(\d)\s*==\s*"([^"]+)"', cond):
            slots.setdefault(int(i), []).append(m)
        if len(slots) == nb:
            out.update(itertools.product(*[slots[k] for k in sorted(slots)]))
    return out


@needs_ref
@pytest.mark.parametrize("nb", [2, 3])
def test_every_reference_tuple_has_an_evaluator(nb):
    """Every monomer tuple the reference dispatches to a polynomial
    (potential/2b/energy2b.cpp, potential/3b/energy3b.cpp) has an evaluator
    here, with the reference's monomer ids."""
    from mbx_b200.specs import DISPATCH_2B, DISPATCH_3B, dispatch
    path = os.path.join(REF, "src", "potential", "2b/energy2b.cpp" if nb == 2 else "3b/energy3b.cpp")
    table = DISPATCH_2B if nb == 2 else DISPATCH_3B
    tuples = _reference_tuples(path, nb)
    assert len(tuples) >= (40 if nb == 2 else 14)
    for t in tuples:
        assert t in table, t
        name, order = dispatch(t)
        assert name == table[t] and sorted(order) == list(range(nb)), t
