"""Refitting path: torch.autograd over the evaluators (GPU).

Workload of the differentiation config: gas-phase water trimers (O-O 2.4-6.5 A)
and dimers (O-O 2.2-9 A), random orientations, synthetic targets from the
polynomial with coefficients perturbed by 1% Gaussian noise.  Checks: the
coordinate gradient against central finite differences (step 1e-5 A) and the
oracle's analytic gradient, the coefficient gradient against the oracle's
design matrix.
"""
import numpy as np
import pytest

import mbx_oracle as mo
from mbx_b200 import workloads
from mbx_b200.tables import load_fit

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("name,maker", [("mbpol2b", workloads.gas_dimers), ("mbpol3b", workloads.gas_trimers)])
def test_coordinate_gradient_fd(name, maker):
    from mbx_b200 import torch_ops
    xyz_np = maker(64, seed=4)
    xyz = torch.tensor(xyz_np, device="cuda", requires_grad=True)
    coef = torch_ops.fitted_coefficients(name)
    e = torch_ops.nmer_energies(name, xyz, coef)
    w = torch.linspace(0.5, 1.5, len(xyz_np), dtype=torch.float64, device="cuda")
    (e * w).sum().backward()
    g = xyz.grad.cpu().numpy()
    # analytic gradients of the oracle
    _, go, _, _ = mo.holder_eval(name, xyz_np)
    np.testing.assert_allclose(g, go * w.cpu().numpy()[:, None], atol=1e-8)
    # central finite differences, step 1e-5 A, a few coordinates
    h = 1e-5
    rng = np.random.default_rng(0)
    for _ in range(12):
        i, j = rng.integers(len(xyz_np)), rng.integers(xyz_np.shape[1])
        xp, xm = xyz_np.copy(), xyz_np.copy()
        xp[i, j] += h
        xm[i, j] -= h
        with torch.no_grad():
            ep = torch_ops.nmer_energies(name, torch.tensor(xp, device="cuda"), coef)[i].item()
            em = torch_ops.nmer_energies(name, torch.tensor(xm, device="cuda"), coef)[i].item()
        fd = (ep - em) / (2 * h) * w[i].item()
        assert abs(fd - g[i, j]) < 1e-5 * max(1.0, abs(g[i, j]))


@pytest.mark.parametrize("name,maker", [("mbpol2b", workloads.gas_dimers), ("mbpol3b", workloads.gas_trimers)])
def test_coefficient_gradient_refit_loss(name, maker):
    from mbx_b200 import torch_ops
    xyz_np = maker(200, seed=9)
    a0 = load_fit(name)
    rng = np.random.default_rng(2)
    a_pert = a0 * (1 + 0.01 * rng.normal(size=a0.shape))
    # synthetic targets from the perturbed polynomial (oracle)
    _, _, _, target = mo.holder_eval(name, xyz_np, do_grads=False, a=a_pert, per_nmer=True)
    coef = torch.tensor(a0, device="cuda", requires_grad=True)
    xyz = torch.tensor(xyz_np, device="cuda")
    e = torch_ops.nmer_energies(name, xyz, coef)
    t = torch.tensor(target, device="cuda")
    loss = ((e - t) ** 2).sum()
    loss.backward()
    D = mo.holder_dcoef(name, xyz_np)                       # dE_n/da
    _, _, _, e0 = mo.holder_eval(name, xyz_np, do_grads=False, per_nmer=True)
    ref = 2 * ((e0 - target)[:, None] * D).sum(0)
    got = coef.grad.cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-8, atol=1e-9 * np.abs(ref).max())
    # E is linear in a: dE/da is exact, so one gradient step along -grad lowers the loss
    with torch.no_grad():
        step = 1e-3 / max(1e-300, float((coef.grad ** 2).sum()) ** 0.5)
        e2 = torch_ops.nmer_energies(name, xyz, coef - step * coef.grad)
        assert float(((e2 - t) ** 2).sum()) < float(loss)
    torch_ops.context().set_coefficients(name, None)


def test_mixed_refit_forward():
    """Mixed forward of the refitting workload (gas-phase trimers, off the FP32
    basis' liquid reference point: 1e-5 of the summed energy), and the
    coefficient gradient through it (the shifted coefficients follow a)."""
    from mbx_b200 import torch_ops
    xyz_np = workloads.gas_trimers(500, seed=1)
    coef = torch_ops.fitted_coefficients("mbpol3b")
    e64 = torch_ops.nmer_energies("mbpol3b", torch.tensor(xyz_np, device="cuda"), coef)
    e32 = torch_ops.nmer_energies("mbpol3b", torch.tensor(xyz_np, device="cuda"), coef, mixed=True)
    assert abs(float(e32.sum() - e64.sum())) / float(e64.abs().sum()) < 1e-5
    # custom coefficients reach the FP32 basis (b = F a recomputed)
    c2 = (coef * 1.01).detach()
    e64b = torch_ops.nmer_energies("mbpol3b", torch.tensor(xyz_np, device="cuda"), c2)
    e32b = torch_ops.nmer_energies("mbpol3b", torch.tensor(xyz_np, device="cuda"), c2, mixed=True)
    assert abs(float(e32b.sum() - e64b.sum())) / float(e64b.abs().sum()) < 1e-5
    assert abs(float(e64b.sum()) - 1.01 * float(e64.sum())) < 1e-9 * float(e64.abs().sum())
    torch_ops.context().set_coefficients("mbpol3b", None)


@pytest.mark.parametrize("name,maker", [("mbpol2b", workloads.gas_dimers), ("mbpol3b", workloads.gas_trimers)])
def test_gradcheck(name, maker):
    """torch.autograd.gradcheck (central differences) of the FP64 n-mer
    energies with respect to coordinates and coefficients, 16 n-mers."""
    from mbx_b200 import torch_ops
    xyz = torch.tensor(maker(16, seed=3), device="cuda", requires_grad=True)
    coef = torch_ops.fitted_coefficients(name).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x, a: torch_ops.nmer_energies(name, x, a), (xyz, coef),
                                    eps=1e-6, atol=1e-5, rtol=1e-4)
    torch_ops.context().set_coefficients(name, None)


def test_second_derivative_is_refused():
    """A force-matching refit needs d loss(F) / d a, a second derivative: the
    backward pass is not differentiable and says so."""
    from mbx_b200 import torch_ops
    xyz = torch.tensor(workloads.gas_dimers(8, seed=2), device="cuda", requires_grad=True)
    coef = torch_ops.fitted_coefficients("mbpol2b").requires_grad_(True)
    e = torch_ops.nmer_energies("mbpol2b", xyz, coef)
    with pytest.raises(RuntimeError, match="second derivatives"):
        torch.autograd.grad(e.sum(), xyz, create_graph=True)
    # the first derivative alone still works
    e = torch_ops.nmer_energies("mbpol2b", xyz, coef)
    (f,) = torch.autograd.grad(e.sum(), xyz)
    assert f.shape == xyz.shape and not f.requires_grad


@pytest.mark.parametrize("name,maker", [("mbpol2b", workloads.gas_dimers), ("mbpol3b", workloads.gas_trimers)])
def test_virial_and_energy_only_forward(name, maker):
    """virial=True gives the evaluators' virial (the oracle's), the plain
    forward the same energies as the gradient path."""
    from mbx_b200 import torch_ops
    xyz_np = maker(100, seed=6)
    xyz = torch.tensor(xyz_np, device="cuda")
    coef = torch_ops.fitted_coefficients(name)
    e, v = torch_ops.nmer_energies(name, xyz, coef, virial=True)
    e_only = torch_ops.nmer_energies(name, xyz, coef)
    eo, _, vo, epo = mo.holder_eval(name, xyz_np, per_nmer=True)
    np.testing.assert_allclose(e.cpu().numpy(), epo, rtol=0, atol=1e-8)
    np.testing.assert_allclose(e_only.cpu().numpy(), e.cpu().numpy(), rtol=0, atol=1e-8)
    np.testing.assert_allclose(v.cpu().numpy(), np.asarray(vo).reshape(-1), rtol=1e-9, atol=1e-8)
    assert not v.requires_grad


def test_system_energy_backward_recomputes():
    """system_energy: energy-only forward, the gradient kernels in backward;
    equal to the System's own gradient, virial as the second result."""
    from mbx_b200 import system as msys, torch_ops
    ids, xyz, box = workloads.water_256(0)
    s = msys.from_arrays(ids, xyz, box, 9.0, 7.0)
    e_ref = s.ThreeBodyEnergy(True)
    g_ref = np.asarray(s.GetRealGrads())
    v_ref = np.asarray(s.GetVirial())
    s2 = msys.from_arrays(ids, xyz, box, 9.0, 7.0)
    sites = torch.tensor(s2.sites, device="cuda", requires_grad=True)
    e, v = torch_ops.system_energy(s2, 3, sites, virial=True)
    e.backward()
    assert abs(float(e) - e_ref) < 1e-10 * abs(e_ref)
    g = sites.grad.detach().cpu().numpy()
    s2.grad = g
    np.testing.assert_allclose(s2.GetRealGrads(), g_ref, rtol=0, atol=1e-8)
    np.testing.assert_allclose(v.cpu().numpy(), v_ref, rtol=1e-10, atol=1e-8)


def test_registered_torch_ops():
    """torch.ops.mbxgpu.* (torch.library custom ops): energy_2b3b against the
    System path, nmer_energies with its registered autograd against the
    autograd.Function path."""
    from mbx_b200 import capi, system as msys, torch_ops
    ids, xyz, box = workloads.water_256(0)
    a = msys.from_arrays(ids, xyz, box, 9.0, 7.0)
    e2, e3 = a.TwoAndThreeBodyEnergy(True)
    g_ref = np.asarray(a.GetGrads())
    ctx = capi.Context(0)
    b = msys.from_arrays(ids, xyz, box, 9.0, 7.0, context=ctx)
    sites = torch.tensor(b.sites, device="cuda")
    s0 = sites.clone()
    o2, o3, g, v = torch.ops.mbxgpu.energy_2b3b(sites, ctx.h.value, False)
    assert torch.equal(sites, s0)
    assert abs(float(o2) - e2) < 1e-10 * abs(e2) and abs(float(o3) - e3) < 1e-10 * abs(e3)
    np.testing.assert_allclose(g.cpu().numpy(), g_ref, rtol=0, atol=1e-9)
    np.testing.assert_allclose(v.cpu().numpy(), a.GetVirial(), rtol=1e-10, atol=1e-8)
    # nmer_energies as a registered op with autograd
    x = torch.tensor(workloads.gas_trimers(32, seed=8), device="cuda", requires_grad=True)
    coef = torch_ops.fitted_coefficients("mbpol3b").requires_grad_(True)
    e = torch.ops.mbxgpu.nmer_energies(x, coef, "mbpol3b", False)
    (e * torch.linspace(0.5, 1.5, 32, dtype=torch.float64, device="cuda")).sum().backward()
    x2 = x.detach().clone().requires_grad_(True)
    c2 = coef.detach().clone().requires_grad_(True)
    e_ref = torch_ops.nmer_energies("mbpol3b", x2, c2)
    (e_ref * torch.linspace(0.5, 1.5, 32, dtype=torch.float64, device="cuda")).sum().backward()
    np.testing.assert_allclose(e.detach().cpu().numpy(), e_ref.detach().cpu().numpy(), rtol=0, atol=1e-12)
    np.testing.assert_allclose(x.grad.cpu().numpy(), x2.grad.cpu().numpy(), rtol=0, atol=1e-12)
    np.testing.assert_allclose(coef.grad.cpu().numpy(), c2.grad.cpu().numpy(), rtol=1e-12, atol=1e-12)
    ctx.close()
