"""torch.autograd wrappers over the CUDA evaluators (the python plugin's extension).

``nmer_energies(name, xyz, coef)`` returns the switched energy of every n-mer
(``xyz``: [n, nreal*3] float64 CUDA tensor, monomers in evaluator order,
already imaged; ``coef``: [ncoef] float64 CUDA tensor of linear coefficients).

* forward: the energy-only kernel (no gradient is formed);
* backward, d/dxyz: the reverse pass as a kernel of its own -- the gradient
  kernel recomputes variables and monomials from the coordinates (nothing
  is stored by the forward pass) and its per-n-mer gradients are scaled by
  the upstream gradient;
* backward, d/dcoef: the adjoint with respect to the linear coefficients,
  sum_n w_n dE_n/da, computed by a kernel that recomputes the monomials from
  the coordinates (they are never stored).

With ``virial=True`` the call also returns the virial of the n-mers
(-sum r (x) dE/dr, 9 components, the evaluators' convention; computed by the
gradient kernel, not differentiable).

The backward pass is itself not differentiable: a second derivative (for
instance d loss(forces) / d coef, which a force-matching refit needs) raises
an error instead of returning a wrong value.

``system_energy(system, nbody, sites)`` is the same for a whole System term
(Get2B/Get3B) with respect to the site coordinates: energy-only forward, the
gradient recomputed by the gradient kernels in backward.

Everything runs on the library's CUDA kernels; the tensors are passed by
device pointer on torch's current stream.
"""
import numpy as np
import torch

from . import capi

_contexts = {}


# cudaStreamLegacy: the handle that names the legacy default stream (a null
# stream handle would make mbx_create give the context a stream of its own,
# unordered with torch's work on the default stream)
_LEGACY_STREAM = 1


def context(device=None):
    """The library context of the current device and torch's current stream
    (kernels are ordered with torch's work on that stream)."""
    dev = torch.cuda.current_device() if device is None else device
    key = (dev, torch.cuda.current_stream(dev).cuda_stream)
    if key not in _contexts:
        _contexts[key] = capi.Context(dev, key[1] or _LEGACY_STREAM)
    return _contexts[key]


def _no_second_derivative():
    """The backward kernels are not themselves differentiable: a backward
    pass that builds a graph (create_graph=True, e.g. for d loss(forces) /
    d coef) is refused here instead of silently dropping the second-order
    terms."""
    if torch.is_grad_enabled():
        raise RuntimeError("mbx_b200: second derivatives of the 2b/3b energies are not supported "
                           "(the backward pass is a kernel, not a differentiable graph; use create_graph=False)")


class _NmerEnergies(torch.autograd.Function):
    @staticmethod
    def forward(fctx, xyz, coef, name, mixed, want_virial):
        if not (xyz.is_cuda and coef.is_cuda):
            raise TypeError("xyz and coef must be CUDA tensors")
        xyz = xyz.contiguous()
        coef = coef.contiguous()
        c = context(xyz.device.index)
        c.set_coefficients(name, coef)
        n = xyz.shape[0]
        e = torch.empty(n, dtype=torch.float64, device=xyz.device)
        vir = np.zeros(9)
        if want_virial:
            g = torch.zeros_like(xyz)
            c.evaluate(name, xyz, g, vir, e, mixed=mixed, grads=True)
        else:
            c.evaluate(name, xyz, None, None, e, mixed=mixed, grads=False)
        fctx.save_for_backward(xyz, coef)
        fctx.name = name
        fctx.mixed = mixed
        v = torch.tensor(vir, dtype=torch.float64, device=xyz.device)
        fctx.mark_non_differentiable(v)
        return e, v

    @staticmethod
    def backward(fctx, ge, gv):
        _no_second_derivative()
        xyz, coef = fctx.saved_tensors
        ge = ge.contiguous()
        c = context(xyz.device.index)
        c.set_coefficients(fctx.name, coef)
        dxyz = dcoef = None
        if fctx.needs_input_grad[0]:
            # reverse pass: the gradient kernel, everything recomputed from xyz
            g = torch.zeros_like(xyz)
            c.evaluate(fctx.name, xyz, g, None, None, mixed=fctx.mixed, grads=True)
            dxyz = g * ge[:, None]
        if fctx.needs_input_grad[1]:
            dcoef = torch.zeros_like(coef)
            c.evaluate_dcoef(fctx.name, xyz, ge, dcoef)
        return dxyz, dcoef, None, None, None


def nmer_energies(name, xyz, coef, mixed=False, virial=False):
    """Per-n-mer energies (and, with virial=True, the virial as a second
    result)."""
    e, v = _NmerEnergies.apply(xyz, coef, name, mixed, virial)
    return (e, v) if virial else e


def fitted_coefficients(name, device="cuda"):
    from .tables import load_fit
    return torch.tensor(load_fit(name), dtype=torch.float64, device=device)


class _SystemEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, sites, system, nbody, want_virial):
        sites = sites.contiguous()
        vir = np.zeros(9)
        mixed = system.precision == "mixed"
        if want_virial:
            g = torch.zeros_like(sites)
            e = system._ctx.energy(nbody, sites, g, vir, mixed=mixed)
        else:
            e = system._ctx.energy(nbody, sites, None, None, mixed=mixed, grads=False)
        fctx.save_for_backward(sites)
        fctx.system = system
        fctx.nbody = nbody
        v = torch.tensor(vir, dtype=torch.float64, device=sites.device)
        fctx.mark_non_differentiable(v)
        return torch.tensor(e, dtype=torch.float64, device=sites.device), v

    @staticmethod
    def backward(fctx, ge, gv):
        _no_second_derivative()
        (sites,) = fctx.saved_tensors
        s = fctx.system
        g = torch.zeros_like(sites)
        s._ctx.energy(fctx.nbody, sites, g, np.zeros(9), mixed=s.precision == "mixed")
        return g * ge, None, None, None


def system_energy(system, nbody, sites, virial=False):
    """Get2B/Get3B of an initialised mbx_b200.system.System on device site
    coordinates (and, with virial=True, the term's virial as a second result).

    Note: like System::SetPBC, the call wraps the coordinates in place."""
    e, v = _SystemEnergy.apply(sites, system, nbody, virial)
    return (e, v) if virial else e


# ---------------------------------------------------------------------------
# Registered torch operators (torch.ops.mbxgpu.*): the same CUDA kernels as
# dispatcher ops, usable from TorchScript-free graphs and by name from C++
# torch code.  A context is passed by its handle (capi.Context.h.value).

@torch.library.custom_op("mbxgpu::energy_2b3b", mutates_args=())
def _op_energy_2b3b(sites: torch.Tensor, handle: int, mixed: bool) -> tuple[torch.Tensor, torch.Tensor,
                                                                             torch.Tensor, torch.Tensor]:
    """Get2B and Get3B of a context's system on device site coordinates
    (System::TwoBodyEnergy/ThreeBodyEnergy): (E2B, E3B, dE/dsites of both
    terms, virial[9]).  The coordinates are not modified (the op works on a
    copy, wrapped as SetPBC does)."""
    c = capi.Context.from_handle(handle)
    x = sites.detach().clone().contiguous()
    g = torch.zeros_like(x)
    vir = np.zeros(9)
    e2, e3 = c.energy_2b3b(x, g, vir, mixed=mixed)
    dev = sites.device
    return (torch.tensor(e2, dtype=torch.float64, device=dev), torch.tensor(e3, dtype=torch.float64, device=dev), g,
            torch.tensor(vir, dtype=torch.float64, device=dev))


@_op_energy_2b3b.register_fake
def _(sites, handle, mixed):
    s = sites.new_empty(())
    return s, sites.new_empty(()), torch.empty_like(sites), sites.new_empty(9)


@torch.library.custom_op("mbxgpu::nmer_energies", mutates_args=())
def _op_nmer_energies(xyz: torch.Tensor, coef: torch.Tensor, name: str, mixed: bool) -> torch.Tensor:
    """Switched energy of every n-mer (evaluator calling convention, AoS
    coordinates already imaged), energy-only kernel."""
    c = context(xyz.device.index)
    c.set_coefficients(name, coef.contiguous())
    x = xyz.contiguous()
    e = torch.empty(x.shape[0], dtype=torch.float64, device=x.device)
    c.evaluate(name, x, None, None, e, mixed=mixed, grads=False)
    return e


@_op_nmer_energies.register_fake
def _(xyz, coef, name, mixed):
    return xyz.new_empty(xyz.shape[0])


@torch.library.custom_op("mbxgpu::nmer_energies_backward", mutates_args=())
def _op_nmer_energies_backward(ge: torch.Tensor, xyz: torch.Tensor, coef: torch.Tensor, name: str,
                               mixed: bool) -> tuple[torch.Tensor, torch.Tensor]:
    """Reverse pass of mbxgpu::nmer_energies: (dL/dxyz, dL/dcoef) for upstream
    dL/dE_n = ge, from the gradient kernel and the coefficient adjoint kernel
    (monomials recomputed from the coordinates)."""
    c = context(xyz.device.index)
    c.set_coefficients(name, coef.contiguous())
    x = xyz.contiguous()
    g = torch.zeros_like(x)
    c.evaluate(name, x, g, None, None, mixed=mixed, grads=True)
    dcoef = torch.zeros_like(coef)
    c.evaluate_dcoef(name, x, ge.contiguous(), dcoef)
    return g * ge[:, None], dcoef


@_op_nmer_energies_backward.register_fake
def _(ge, xyz, coef, name, mixed):
    return torch.empty_like(xyz), torch.empty_like(coef)


def _nmer_setup(ctx, inputs, output):
    xyz, coef, name, mixed = inputs
    ctx.save_for_backward(xyz, coef)
    ctx.name = name
    ctx.mixed = mixed


def _nmer_backward(ctx, ge):
    _no_second_derivative()
    xyz, coef = ctx.saved_tensors
    dxyz, dcoef = torch.ops.mbxgpu.nmer_energies_backward(ge, xyz, coef, ctx.name, ctx.mixed)
    return dxyz, dcoef, None, None


torch.library.register_autograd("mbxgpu::nmer_energies", _nmer_backward, setup_context=_nmer_setup)
