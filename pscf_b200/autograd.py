"""torch.autograd binding of the engine's density and its adjoint.

SCFDensity.apply(omega, engine) returns (rho, lnQ) for omega of shape
[n_inst, n_monomer, nr] (float64, CPU or CUDA); its backward calls the C
ABI adjoint (pscfg_density_adjoint[_device]) to give dL/domega for any
scalar L of rho and lnQ.  SCFDensityCell also takes the cell parameters
as an input and returns dL/dcell (pscfg_density_adjoint_cell).  The backward first re-runs density on the saved
omega, so other engine calls between forward and backward do not change
the result.  PyTorch only carries the tensors; all arithmetic runs in the
engine's kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .engine import Engine, _ptr


def _density(engine: Engine, omega: torch.Tensor):
    n, M, nr = engine.n_inst, engine.M, engine.nr
    nch = max(len(s.chains) for s in engine.systems)
    if omega.is_cuda:
        w = omega.detach().contiguous()
        rho = torch.empty_like(w)
        q = engine.density_device(w.data_ptr(), rho.data_ptr())
    else:
        r, q = engine.density(omega.detach().cpu().numpy())
        rho = torch.from_numpy(r)
    lnq = torch.from_numpy(np.log(np.maximum(q[:, :nch], 1e-300))).to(omega.device)
    return rho.reshape(n, M, nr), lnq


class SCFDensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, engine):
        rho, lnq = _density(engine, omega)
        ctx.engine = engine
        ctx.save_for_backward(omega.detach())
        return rho, lnq

    @staticmethod
    def backward(ctx, grad_rho, grad_lnq):
        engine = ctx.engine
        (omega,) = ctx.saved_tensors
        _density(engine, omega)
        n = engine.n_inst
        gq = np.zeros((n, 4))
        if grad_lnq is not None:
            a = grad_lnq.detach().cpu().numpy().reshape(n, -1)
            gq[:, : a.shape[1]] = a
        if grad_rho is None:
            grad_rho = torch.zeros_like(omega)
        if omega.is_cuda:
            G = grad_rho.detach().contiguous().to(torch.float64)
            out = torch.empty_like(G)
            engine._check(engine.lib.pscfg_density_adjoint_device(engine._h, C.c_void_p(G.data_ptr()), _ptr(gq),
                                                                  C.c_void_p(out.data_ptr())))
            return out, None
        g = engine.density_adjoint(grad_rho.detach().cpu().numpy(), gq)
        return torch.from_numpy(g), None


class SCFDensityCell(torch.autograd.Function):
    """(rho, lnQ) as functions of omega and of the cell parameters
    [n_inst, n_cell_param] (float64, CPU): forward sets the engine's cells,
    backward returns dL/domega and dL/dcell through
    pscfg_density_adjoint_cell."""

    @staticmethod
    def forward(ctx, omega, cell, engine):
        c = cell.detach().cpu().numpy()
        for i in range(engine.n_inst):
            engine.set_cell_param(i, list(c[i]))
        rho, lnq = _density(engine, omega)
        ctx.engine = engine
        ctx.save_for_backward(omega.detach(), cell.detach())
        return rho, lnq

    @staticmethod
    def backward(ctx, grad_rho, grad_lnq):
        engine = ctx.engine
        omega, cell = ctx.saved_tensors
        c = cell.cpu().numpy()
        for i in range(engine.n_inst):
            engine.set_cell_param(i, list(c[i]))
        _density(engine, omega)
        n = engine.n_inst
        gq = np.zeros((n, 4))
        if grad_lnq is not None:
            a = grad_lnq.detach().cpu().numpy().reshape(n, -1)
            gq[:, : a.shape[1]] = a
        if grad_rho is None:
            grad_rho = torch.zeros_like(omega)
        g, gc = engine.density_adjoint(grad_rho.detach().cpu().numpy(), gq, want_cell=True)
        return (torch.from_numpy(g).to(omega.device), torch.from_numpy(gc).to(cell.device), None)


def density(omega: torch.Tensor, engine: Engine, cell: torch.Tensor = None):
    """(rho, lnQ) = density(omega) with gradients through the adjoint; with
    `cell` ([n_inst, n_cell_param] tensor) also differentiable in the cell
    parameters."""
    if cell is None:
        return SCFDensity.apply(omega, engine)
    return SCFDensityCell.apply(omega, cell, engine)
