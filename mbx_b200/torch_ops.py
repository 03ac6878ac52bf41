"""torch.autograd wrappers over the CUDA evaluators (the python plugin's extension).

``nmer_energies(name, xyz, coef)`` returns the switched energy of every n-mer
(``xyz``: [n, nreal*3] float64 CUDA tensor, monomers in evaluator order,
already imaged; ``coef``: [ncoef] float64 CUDA tensor of linear coefficients).
Its backward pass gives

* d/dxyz: the analytic reverse pass (the per-n-mer gradients the forward
  kernel produced), scaled by the upstream gradient;
* d/dcoef: the adjoint with respect to the linear coefficients,
  sum_n w_n dE_n/da, computed by a kernel that recomputes the monomials from
  the coordinates (they are never stored).

``system_energy(system, nbody, sites)`` is the same for a whole System term
(Get2B/Get3B) with respect to the site coordinates.

Everything runs on the library's CUDA kernels; the tensors are passed by
device pointer on the current stream.
"""
import numpy as np
import torch

from . import capi

_contexts = {}


def context(device=None):
    dev = torch.cuda.current_device() if device is None else device
    key = (dev, torch.cuda.current_stream(dev).cuda_stream)
    if key not in _contexts:
        _contexts[key] = capi.Context(dev, key[1])
    return _contexts[key]


class _NmerEnergies(torch.autograd.Function):
    @staticmethod
    def forward(fctx, xyz, coef, name, mixed):
        if not (xyz.is_cuda and coef.is_cuda):
            raise TypeError("xyz and coef must be CUDA tensors")
        xyz = xyz.contiguous()
        coef = coef.contiguous()
        c = context(xyz.device.index)
        c.set_coefficients(name, coef)
        n = xyz.shape[0]
        e = torch.empty(n, dtype=torch.float64, device=xyz.device)
        g = torch.zeros_like(xyz)
        c.evaluate(name, xyz, g, None, e, mixed=mixed, grads=True)
        fctx.save_for_backward(xyz, coef, g)
        fctx.name = name
        return e

    @staticmethod
    def backward(fctx, ge):
        xyz, coef, g = fctx.saved_tensors
        ge = ge.contiguous()
        dxyz = g * ge[:, None] if fctx.needs_input_grad[0] else None
        dcoef = None
        if fctx.needs_input_grad[1]:
            c = context(xyz.device.index)
            c.set_coefficients(fctx.name, coef)
            dcoef = torch.zeros_like(coef)
            c.evaluate_dcoef(fctx.name, xyz, ge, dcoef)
        return dxyz, dcoef, None, None


def nmer_energies(name, xyz, coef, mixed=False):
    return _NmerEnergies.apply(xyz, coef, name, mixed)


def fitted_coefficients(name, device="cuda"):
    from .tables import load_fit
    return torch.tensor(load_fit(name), dtype=torch.float64, device=device)


class _SystemEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, sites, system, nbody):
        sites = sites.contiguous()
        g = torch.zeros_like(sites)
        vir = np.zeros(9)
        e = system._ctx.energy(nbody, sites, g, vir, mixed=system.precision == "mixed")
        fctx.save_for_backward(g)
        return torch.tensor(e, dtype=torch.float64, device=sites.device)

    @staticmethod
    def backward(fctx, ge):
        (g,) = fctx.saved_tensors
        return g * ge, None, None


def system_energy(system, nbody, sites):
    """Get2B/Get3B of an initialised mbx_b200.system.System on device site coordinates.

    Note: like System::SetPBC, the call wraps the coordinates in place."""
    return _SystemEnergy.apply(sites, system, nbody)
