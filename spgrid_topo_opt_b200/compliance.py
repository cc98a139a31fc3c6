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
i*16 + j*4 + k).  The problem stays resident on the GPU between calls; only the
densities change (the set of material cells, rho > 0, must not).
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
    @staticmethod
    def forward(ctx, rho: torch.Tensor, model: "Compliance"):
        r = rho.detach().to("cpu", torch.float64).numpy().reshape(-1, 64)
        model.session.set_density(r)
        model.last_stats = model.session.solve(tolerance=model.tolerance)
        disp = model.session.displacements()
        _, dc, _ = model.session.sensitivity(r)
        model.displacements = disp
        ctx.dx = float(model.inputs.dx)
        ctx.save_for_backward(torch.as_tensor(dc.reshape(rho.shape), dtype=rho.dtype, device=rho.device))
        return torch.tensor(force_work(model.inputs, disp), dtype=rho.dtype, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (dc,) = ctx.saved_tensors
        return -ctx.dx * dc * grad_out, None


class Compliance:
    """C(rho) = f.u with u = K(rho)^-1 f on the GPU, differentiable in rho."""

    def __init__(self, inputs: fi.FEMInputs, precision: int = native.PRECISION_FP64, tolerance: float = 1e-10):
        self.inputs = copy.deepcopy(inputs)
        self.tolerance = tolerance
        self.session = native.Session(self.inputs, precision=precision)
        self.displacements = None
        self.last_stats = None

    def __call__(self, rho: torch.Tensor) -> torch.Tensor:
        return _ComplianceFn.apply(rho, self)

    def close(self):
        self.session.close()
