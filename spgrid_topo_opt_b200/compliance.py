"""Differentiable compliance for the PyTorch layer.

``Compliance(inputs)(rho)`` solves K(rho) u = f on the GPU and returns the
compliance C = f.u (the work of the loads on the converged displacement).  Its
backward is the self-adjoint SIMP sensitivity computed by the library's
sensitivity kernel (topo_opt/objective/minimal_compliance.cpp:86-146):

    dC/drho_e = -dx * p * rho_e^(p-1) * (1 - E_min) * u_e^T K0 u_e

with K0 = mu0*K_mu + lambda0*K_la the unit-stiffness element matrix.  The
reference's objective omits the dx of the solver's stiffness
(minimal_compliance.cpp:158, hex_fem.cpp:52-82); here C is the true f.u of the
solver's system, so its gradient carries dx.  The relation holds for loads on
free nodes with homogeneous Dirichlet conditions, and for densities above
``minimum_density`` (where the SIMP map is differentiable).

``rho`` has the shape of the input density blocks, [nblocks, 64] (in-block index
i*16 + j*4 + k), on the GPU or the host.  The problem stays resident on the GPU
between calls; only the densities change (the set of material cells, rho > 0,
must not).  Everything runs on the device: the densities go to the solver
device to device, f.u is summed there, and the backward's sensitivity kernel
writes the gradient tensor directly; under ``torch.no_grad()`` (or for a rho
that does not require a gradient) no solution copy is kept.
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import fem_interface as fi
from . import native


def force_work(inputs: fi.FEMInputs, disp: np.ndarray) -> float:
    """f.u over the force list, reading u from the per-input-block displacements."""
    lookup = {tuple(b): i for i, b in enumerate(np.asarray(inputs.density.base))}
    total = 0.0
    for rec in inputs.forces:
        c = np.asarray(rec["coord"])
        base = (c // 4) * 4
        b = lookup.get(tuple(base))
        if b is None:
            continue
        o = c - base
        total += float(np.dot(disp[b, o[0] * 16 + o[1] * 4 + o[2], :3], rec["f"]))
    return total


class _ComplianceFn(torch.autograd.Function):
    """Forward: densities to the session (device to device), solve, f.u on the
    device.  When a gradient will be needed the forward keeps a device copy of
    the solution; the backward launches the sensitivity kernel on it, scaled by
    -dx and the incoming gradient (a device scalar), straight into the gradient
    tensor.  No array crosses to the host in either pass."""

    @staticmethod
    def forward(ctx, rho: torch.Tensor, model: "Compliance", keep: bool):
        dev = torch.device("cuda", torch.cuda.current_device())
        r = rho.detach().to(dev, torch.float64).reshape(-1, 64).contiguous()
        model.session.set_density_device(r)
        model.last_stats = model.session.solve(tolerance=model.tolerance)
        c = torch.empty(1, dtype=torch.float64, device=dev)
        model.session.compliance_device(c)
        if keep:
            u = torch.empty(model.session.solution_size(), dtype=torch.float64, device=dev)
            model.session.solution_device(u)
            ctx.save_for_backward(r, u)
        ctx.dx = float(model.inputs.dx)
        ctx.model = model
        ctx.shape, ctx.dtype, ctx.device = rho.shape, rho.dtype, rho.device
        return c.reshape(()).to(rho.device, rho.dtype)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        r, u = ctx.saved_tensors
        g = grad_out.detach().to(r.device, torch.float64).reshape(1).contiguous()
        grad = torch.empty_like(r)
        ctx.model.session.sensitivity_device(u, r, -ctx.dx, g, grad)
        return grad.reshape(ctx.shape).to(ctx.device, ctx.dtype), None, None


class Compliance:
    """C(rho) = f.u with u = K(rho)^-1 f on the GPU, differentiable in rho."""

    def __init__(self, inputs: fi.FEMInputs, precision: int = native.PRECISION_FP64, tolerance: float = 1e-10):
        self.inputs = copy.deepcopy(inputs)
        self.tolerance = tolerance
        self.session = native.Session(self.inputs, precision=precision)
        self.last_stats = None

    def __call__(self, rho: torch.Tensor) -> torch.Tensor:
        keep = torch.is_grad_enabled() and rho.requires_grad
        return _ComplianceFn.apply(rho, self, keep)

    def displacements(self) -> np.ndarray:
        """The last solve's displacements per input block, [nblocks, 64, 4] (host copy)."""
        return self.session.displacements()

    def close(self):
        self.session.close()
