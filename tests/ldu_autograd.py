"""A thin torch.autograd.Function over the C ABI (test harness only).

forward: x = A(diag, upper, lower)^{-1} b with cf_solve (FP32 inner, FP64
refinement on the GPU); backward: cf_solve_adjoint gives lambda = A^{-T} gx
and the face-parallel gradients.  Tensors are FP64 on the CPU; the library
moves them to and from the device.
"""
import numpy as np
import torch

from metal4foam_b200 import _lib


class LduSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, diag, upper, lower, b, context, addr, options, solver,
                adjoint_options=None):
        a = addr
        context.set_topology(a.n, a.nf, *a.arrays())
        context.set_coeffs(diag.detach().numpy(), upper.detach().numpy(),
                           None if lower is None else lower.detach().numpy())
        x = np.zeros(a.n)
        perf = context.solve(solver, x, np.ascontiguousarray(b.detach().numpy()), options)
        if not perf.converged:
            raise RuntimeError(f"forward solve did not converge: {perf.as_dict()}")
        xt = torch.from_numpy(x)
        ctx.context = context
        ctx.addr = addr
        ctx.options = options if adjoint_options is None else adjoint_options
        ctx.solver = solver
        ctx.has_lower = lower is not None
        ctx.coeffs = (diag.detach().numpy(), upper.detach().numpy(),
                      None if lower is None else lower.detach().numpy())
        ctx.save_for_backward(xt)
        return xt

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        c = ctx.context
        a = ctx.addr
        # the forward's coefficients may have been replaced by another call
        c.set_topology(a.n, a.nf, *a.arrays())
        c.set_coeffs(*ctx.coeffs)
        lam, dU, dL, dD, perf = c.solve_adjoint(ctx.solver, x.numpy(),
                                                np.ascontiguousarray(gx.numpy()), a.nf,
                                                ctx.options)
        if not perf.converged:
            raise RuntimeError(f"adjoint solve did not converge: {perf.as_dict()}")
        t = torch.from_numpy
        g_lower = t(dL) if ctx.has_lower else None
        g_upper = t(dU) if ctx.has_lower else t(dU + dL)   # symmetric: lower is upper
        return t(dD), g_upper, g_lower, t(lam), None, None, None, None, None


def solve(diag, upper, lower, b, context, addr, options, solver=_lib.CF_SOLVER_PCG,
          adjoint_options=None):
    return LduSolve.apply(diag, upper, lower, b, context, addr, options, solver,
                          adjoint_options)
