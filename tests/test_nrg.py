"""The .nrg reader (io_tools/read_nrg.cpp) and the System it builds (CPU).

Checked against the reference's own input files (timing/*/input.nrg, read
where the reference checkout is present) through the golden extraction of
tests/golden/make_golden.py, and by a format -> parse round trip of seeded
workloads; malformed files raise with the line number, as the reference's
ReadNrg does."""
import glob
import os

import numpy as np
import pytest

from conftest import golden
from mbx_b200 import nrg, workloads
from mbx_b200.system import CUException


def _workload_nrg(ids, xyz):
    from mbx_b200.specs import MONOMER_ATOMS
    from mbx_b200.system import MONOMER_ATOM_NAMES
    s = nrg.NrgSystem("0")
    xyz = np.asarray(xyz).reshape(-1)
    off = 0
    for i, m in enumerate(ids):
        n = 3 * MONOMER_ATOMS[m]
        s.ids.append(m)
        s.atoms.append(list(MONOMER_ATOM_NAMES[m]))
        s.xyz.append(list(xyz[off:off + n]))
        s.molecules.append([i])
        off += n
    return s


@pytest.mark.parametrize("maker", [lambda: workloads.water_256(0), lambda: workloads.methane_water_box(seed=0)])
def test_round_trip(maker):
    from mbx_b200.specs import MONOMER_ATOMS
    ids, xyz, box = maker()
    n10 = sum(3 * MONOMER_ATOMS[m] for m in ids[:10])
    text = nrg.format_nrg([_workload_nrg(ids, xyz), _workload_nrg(ids[:10], np.asarray(xyz).reshape(-1)[:n10])])
    systems = nrg.parse_nrg(text)
    assert len(systems) == 2
    assert systems[0].ids == list(ids)
    np.testing.assert_array_equal(np.array(systems[0].coordinates()), np.asarray(xyz).reshape(-1))
    assert systems[0].molecules == [[i] for i in range(len(ids))]


def test_molecule_with_two_monomers_keeps_first_id():
    """As in the reference: a second MONOMER line inside one MOLECULE is not
    re-read for its id (read_nrg.cpp:206-216)."""
    text = ("SYSTEM\nMOLECULE\nMONOMER h2o\nO 0 0 0\nH 0.9 0 0\nH 0 0.9 0\nENDMON\n"
            "MONOMER h2o\nO 3 0 0\nH 3.9 0 0\nH 3 0.9 0\nENDMON\nENDMOL\nENDSYS\n")
    s = nrg.parse_nrg(text)[0]
    assert s.ids == ["h2o", "h2o"] and s.molecules == [[0, 1]]


@pytest.mark.parametrize("text,line", [
    ("MOLECULE\n", 1),
    ("SYSTEM\nMONOMER h2o\n", 2),
    ("SYSTEM\nMOLECULE\nMONOMER h2o\nO a b c\n", 4),
])
def test_errors_name_the_line(text, line):
    with pytest.raises(CUException, match="line  %d" % line):
        nrg.parse_nrg(text)


def test_reference_input_files():
    """Every timing/*/input.nrg of the reference reads to the monomers and
    coordinates of its golden extraction."""
    ref = os.environ.get("MBX_REFERENCE", "")
    files = sorted(glob.glob(os.path.join(ref, "timing", "*", "input.nrg")))
    if not files:
        pytest.skip("reference checkout absent (MBX_REFERENCE)")
    for f in files:
        systems = nrg.read_nrg(f)
        assert len(systems) == 1 and systems[0].ids, f
    for fixture, sub in (("system_256_h2o_cubic_box", "256_h2o_cubic_box"),
                         ("system_57_ch4_513_h2o", "57_ch4_513_h2o_rectangular")):
        gd = golden(fixture)
        s = nrg.read_nrg(os.path.join(ref, "timing", sub, "input.nrg"))[0]
        assert s.ids == gd["ids"]
        np.testing.assert_array_equal(np.array(s.coordinates()), np.array(gd["xyz"]))
