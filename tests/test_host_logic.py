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


def test_registered_torch_ops_shapes():
    """torch.ops.mbxgpu.* are registered at import and their fake (meta)
    implementations give the shapes of the CUDA ones, so graph capture and
    tracing see the right outputs without a GPU."""
    import torch
    from torch._subclasses.fake_tensor import FakeTensorMode
    from mbx_b200 import torch_ops  # noqa: F401  (registers the ops)
    with FakeTensorMode():
        s = torch.empty(100, 3, dtype=torch.float64)
        e2, e3, g, v = torch.ops.mbxgpu.energy_2b3b(s, 0, False)
        assert (e2.shape, e3.shape, g.shape, v.shape) == ((), (), (100, 3), (9,))
        x = torch.empty(32, 27, dtype=torch.float64)
        c = torch.empty(1163, dtype=torch.float64)
        e = torch.ops.mbxgpu.nmer_energies(x, c, "mbpol3b", False)
        assert e.shape == (32,) and e.dtype == torch.float64
        gx, gc = torch.ops.mbxgpu.nmer_energies_backward(e, x, c, "mbpol3b", False)
        assert gx.shape == x.shape and gc.shape == c.shape
