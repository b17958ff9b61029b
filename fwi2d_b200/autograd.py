"""torch.autograd.Function over the device FWI gradient.

FWIMisfit.apply(model, propagator, kind, src_blocks, obs_blocks[, seismotype])
returns the L2 misfit 0.5 dt sum_t w_t r_t^2 of the propagator's shots for
the raw model (vp, vs, rho[, delta, eps]) as a 0-d float64 tensor; backward
returns the gradient with respect to (vp, vs, rho) computed by the library's
adjoint-state pipeline (fwi2d_fwi_gradient: forward with snapshots,
residual, adjoint propagation with the imaging condition, H quadrature and
chain rule; src/include/optimization.hpp:590-915, src/cpp/we_op.cpp:1057-1239).
The anisotropy parameters of a VTI model get a zero gradient, as in the
reference (we_op.cpp:1521-1522).
"""
import numpy as np
import torch

from . import workloads as W


class FWIMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, model, prop, kind, src_blocks, obs_blocks, seismotype=1):
        m = model.detach().to("cpu", torch.float32).numpy()
        g, phi = prop.fwi_gradient(W.convert(kind, m), src_blocks, obs_blocks, seismotype)
        full = np.zeros(m.shape, np.float32)
        full[: g.shape[0]] = g
        ctx.save_for_backward(torch.from_numpy(full).to(model.device))
        return torch.tensor(phi, dtype=torch.float64, device=model.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out.to(g.dtype) * g, None, None, None, None, None
