"""Batched configurations (mbx_set_batch / mbx_batch_energy / mbx_tune), GPU.

No counterpart in the reference: each configuration of a batch must give the
energies, gradients and virial of the same configuration evaluated alone
(single-system path, itself pinned to the oracle), whatever else is in the
batch; graph replay must repeat the plain sequence; the autotuner must leave
the results unchanged.
"""
import numpy as np
import pytest

import mbx_oracle as mo
from mbx_b200 import system as msys, workloads
from mbx_b200.batch import Batch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

E_REL = 1e-10
G_ABS = 1e-8


def small_batch():
    """Two 256-water boxes (different seeds), a bead of one of them and two
    gas-phase clusters of uneven size."""
    ids0, x0, box = workloads.water_256(0)
    ids1, x1, _ = workloads.water_256(1)
    bead = workloads.beads(x0, 1, 0.05, seed=7)[0]
    c1 = workloads.water_cluster(40, seed=3)
    c2 = workloads.water_cluster(9, seed=4)
    return [(ids0, x0, box), (ids1, x1, box), (ids0, bead, box), (c1[0], c1[1], None), (c2[0], c2[1], None)]


def single(cfg, nbody, mixed=False):
    ids, xyz, box = cfg
    s = msys.from_arrays(ids, xyz, box, 9.0, 7.0, precision="mixed" if mixed else "fp64")
    e = s.TwoBodyEnergy(True) if nbody == 2 else s.ThreeBodyEnergy(True)
    return e, np.asarray(s.GetRealGrads()), np.asarray(s.GetVirial())


@pytest.mark.parametrize("nbody", [2, 3])
def test_batch_matches_single_configurations(nbody):
    cfgs = small_batch()
    b = Batch(cfgs)
    e, v = b.energy(nbody, graph=False, virials=True)
    for k, cfg in enumerate(cfgs):
        es, gs, vs = single(cfg, nbody)
        assert abs(e[k] - es) <= E_REL * abs(es) + 1e-9, (k, e[k], es)
        np.testing.assert_allclose(b.real_grads(k), gs, rtol=0, atol=G_ABS)
        np.testing.assert_allclose(v[k], vs, rtol=1e-9, atol=1e-7)


@pytest.mark.parametrize("nbody", [2, 3])
def test_batch_tiny_configurations(nbody):
    """Configurations too small for some terms (one water, two waters, three
    waters) between larger ones and a periodic box: the batched search runs
    over all of them at once, and each must still give what it gives alone
    (no dimer or trimer across configurations, zero where none exists)."""
    ids0, x0, box = workloads.water_256(0)
    one = workloads.water_cluster(1, seed=21)
    two = workloads.water_cluster(2, seed=22)
    three = workloads.water_cluster(3, seed=23)
    c = workloads.water_cluster(30, seed=24)
    cfgs = [(one[0], one[1], None), (c[0], c[1], None), (two[0], two[1], None), (ids0, x0, box),
            (three[0], three[1], None), (one[0], one[1], None)]
    b = Batch(cfgs)
    e, v = b.energy(nbody, graph=False, virials=True)
    for k, cfg in enumerate(cfgs):
        n = len(cfg[0])
        if n < nbody:
            assert e[k] == 0.0, (k, e[k])
            assert not np.any(b.real_grads(k)), k
            continue
        es, gs, vs = single(cfg, nbody)
        assert abs(e[k] - es) <= E_REL * abs(es) + 1e-9, (k, e[k], es)
        np.testing.assert_allclose(b.real_grads(k), gs, rtol=0, atol=G_ABS)
        np.testing.assert_allclose(v[k], vs, rtol=1e-9, atol=1e-7)


def test_batch_cluster_vs_oracle():
    cfgs = small_batch()
    b = Batch(cfgs)
    e3 = b.energy(3, graph=False)
    ids, xyz, _ = cfgs[3]
    o = mo.OracleSystem(ids, xyz, None, 9.0, 7.0)
    eo = o.energy(3)
    assert abs(e3[3] - eo) <= E_REL * abs(eo) + 1e-9
    np.testing.assert_allclose(b.real_grads(3), o.real_grads(), rtol=0, atol=G_ABS)


@pytest.mark.parametrize("mixed", [False, True])
def test_graph_replay_repeats_plain_sequence(mixed):
    b = Batch(small_batch())
    # the first call wraps the coordinates in place (FixMonomerCoordinates);
    # the FP32 basis sees the last-bit differences of the wrapped variables
    # (~1e-7 of an energy), so every compared call starts from wrapped input
    b.energy(3, mixed=mixed, graph=False)
    e_plain = b.energy(3, mixed=mixed, graph=False)
    b.grad.zero_()
    e_first = b.energy(3, mixed=mixed, graph=True)      # plain run, then capture
    g_first = b.grad.clone()
    for _ in range(3):
        b.grad.zero_()
        e_rep = b.energy(3, mixed=mixed, graph=True)    # replays
        np.testing.assert_allclose(e_rep, e_plain, rtol=1e-12, atol=1e-10)
        torch.testing.assert_close(b.grad, g_first, rtol=0, atol=1e-10)
    np.testing.assert_allclose(e_first, e_plain, rtol=1e-12, atol=1e-10)


def test_graph_recaptures_after_coordinates_move():
    b = Batch(small_batch())
    b.energy(3, graph=True)
    b.energy(3, graph=True)
    # new coordinates in the same device array: the graph reads them
    x0 = b.sites.clone()
    b.sites.add_(0.01 * torch.sin(torch.arange(b.sites.numel(), device=b.sites.device, dtype=torch.float64)))
    b.energy(3, graph=False)   # wraps the moved coordinates
    e_graph = b.energy(3, graph=True)
    e_plain = b.energy(3, graph=False)
    np.testing.assert_allclose(e_graph, e_plain, rtol=1e-12, atol=1e-10)
    b.sites.copy_(x0)


def test_graph_follows_a_cutoff_change():
    """A replayed graph must not keep the cutoffs it was captured with: after
    set_config, the next graph call gives the plain sequence's result for the
    new cutoffs."""
    b = Batch(small_batch())
    e_old = b.energy(2, grads=False, graph=True)
    e_old = b.energy(2, grads=False, graph=True)   # replayed
    b.ctx.set_config(5.0, 7.0, None)   # drops dimers the 2b switch still weighs
    e_graph = b.energy(2, grads=False, graph=True)
    e_plain = b.energy(2, grads=False, graph=False)
    np.testing.assert_allclose(e_graph, e_plain, rtol=1e-12, atol=1e-10)
    assert np.abs(np.asarray(e_graph) - np.asarray(e_old)).max() > 1e-6


def test_batch_mixed_errors():
    cfgs = small_batch()[:3]
    b = Batch(cfgs)
    e64 = b.energy(2, graph=False) + b.energy(3, graph=False)
    emx = b.energy(2, mixed=True, graph=False) + b.energy(3, mixed=True, graph=False)
    assert np.all(np.abs(emx - e64) <= 1e-6 * np.abs(e64))


def test_tune_keeps_results():
    b = Batch(small_batch())
    e_before = b.energy(3, graph=False)
    knobs, ms = b.tune(3)
    assert knobs["nb_warps"] in (1, 4) and knobs["nb_unroll"] in (1, 2, 4)
    assert knobs["tri_threads"] in (64, 128, 256)
    assert ms > 0
    e_after = b.energy(3, graph=True)
    np.testing.assert_allclose(e_after, e_before, rtol=1e-12, atol=1e-10)
    knobs2, _ = b.tune(2)
    assert knobs2["dim_threads"] in (64, 128, 256)
    assert b.ctx.knobs(3) == knobs


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_2b3b_matches_separate_terms(mixed):
    """Both terms side by side (child context mirroring the batch) against the
    separate term calls; plain run, graph capture and replays."""
    cfgs = small_batch()
    b = Batch(cfgs)
    b.energy(2, mixed=mixed, graph=False)          # wraps the coordinates
    b.grad.zero_()
    e2, v2 = b.energy(2, mixed=mixed, graph=False, virials=True)
    e3, v3 = b.energy(3, mixed=mixed, graph=False, virials=True)
    g_sep = b.grad.clone()
    for graph in (False, True, True, True):
        b.grad.zero_()
        f2, f3, v = b.energy_2b3b(mixed=mixed, graph=graph, virials=True)
        np.testing.assert_allclose(f2, e2, rtol=1e-12, atol=1e-10)
        np.testing.assert_allclose(f3, e3, rtol=1e-12, atol=1e-10)
        np.testing.assert_allclose(v, v2 + v3, rtol=1e-10, atol=1e-8)
        torch.testing.assert_close(b.grad, g_sep, rtol=0, atol=1e-9)
