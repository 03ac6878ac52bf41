"""Host-side bookkeeping: internal monomer order, tags, dispatch (CPU)."""
import numpy as np

from mbx_b200.specs import dispatch, sorted_slots
from mbx_b200.topology import Topology


def test_internal_order_types_by_count():
    # OrderMonomers: types by ascending count, ties by first appearance
    t = Topology(["h2o", "ch4", "h2o", "h2o", "ch4", "h2o"])
    assert t.ids == ["ch4", "ch4", "h2o", "h2o", "h2o", "h2o"]
    assert list(t.internal_to_input) == [1, 4, 0, 2, 3, 5]
    # first sites: ch4 has 5 sites, h2o 4 (O H H M)
    assert list(t.first_index) == [0, 5, 10, 14, 18, 22]
    # tags are input atom positions of each monomer's first atom
    assert list(t.tag) == [3, 14, 0, 8, 11, 19]


def test_sites_round_trip():
    t = Topology(["h2o", "ch4", "h2o"])
    xyz = np.arange(3 * t.numat, dtype=float)
    s = t.sites_from_input(xyz)
    assert len(s) == 3 * t.numsites
    np.testing.assert_array_equal(t.input_from_sites(s), xyz)


def test_dispatch_matches_reference_sorting():
    assert sorted_slots(("ch4", "h2o")) == (0, 1)
    assert sorted_slots(("h2o", "ch4")) == (1, 0)
    assert dispatch(("ch4", "h2o")) == ("ch4h2o2b", (1, 0))   # water first in the evaluator
    assert dispatch(("h2o", "h2o", "ch4")) == ("ch4h2o3b", (2, 1, 0))
    assert dispatch(("ch4", "ch4", "h2o")) == (None, None)      # no polynomial: energy 0


def test_nmers_to_input_canonical():
    t = Topology(["h2o", "ch4", "h2o"])
    nm = np.array([[2, 0], [1, 0]])
    out = t.nmers_to_input(nm)
    assert out.tolist() == sorted(out.tolist())
