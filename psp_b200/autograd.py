"""Differentiable sweeping-preconditioned Helmholtz solves for torch.

``helmholtz_solve(solver, velocity, f)`` returns u = A(velocity)^{-1} f for a
CUDA float64 velocity (natural order, nx*ny*nz) and CUDA complex128 sources
f (nx*ny*nz x k, natural order, right-hand sides interleaved per point), and
is differentiable in both.  The backward pass is the adjoint-state method:
the operator is complex symmetric (A^T = A: PML stretching scales each row
by s1 s2 s3, initialize_finalize.hpp:527-587), so one more solve with the
forward factors, z = A^{-1} conj(dL/dconj(u)), gives

    dL/dconj(f) = conj(z)
    dL/dvel_i   = -Re( dA_ii/dvel_i * sum_r z[i,r] u[i,r] ),
    dA_ii/dvel_i = 2 omega^2 / vel_i^3 * s1 s2 s3   (the centre term),

the last computed on the device by psp_cu_gradient_device.  Complex
gradients follow torch's convention (the gradient of a real loss with
respect to a complex tensor is dL/dconj(z)).  The reference has no adjoint;
this module is the differentiation layer of the rebuild.
"""
import torch

from . import FP64, MIXED, LogicError  # noqa: F401  (re-exported precision names)


def _after_torch(solver, device):
    """The solver issues its work on its own stream (and synchronizes it
    before returning); make that stream wait for torch's pending work."""
    torch.cuda.ExternalStream(solver.stream_ptr(), device=device).wait_stream(torch.cuda.current_stream(device))


class _HelmholtzSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, velocity, f, solver, m, rel_tol, precision):
        if not (velocity.is_cuda and f.is_cuda):
            raise LogicError("helmholtz_solve needs CUDA tensors")
        if velocity.dtype != torch.float64 or f.dtype != torch.complex128:
            raise LogicError("velocity must be float64 and f complex128")
        vel = velocity.detach().reshape(-1).contiguous()
        u = f.detach().contiguous().clone()
        _after_torch(solver, f.device)
        solver.Initialize(vel, precision=precision)
        solver.Solve(u, m, rel_tol)
        ctx.solver, ctx.m, ctx.rel_tol, ctx.precision = solver, m, rel_tol, precision
        ctx.version = solver.factor_version
        ctx.shape = velocity.shape
        ctx.save_for_backward(vel, u)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        vel, u = ctx.saved_tensors
        solver = ctx.solver
        if solver.factor_version != ctx.version:  # re-factored since the forward solve
            solver.Initialize(vel, precision=ctx.precision)
            ctx.version = solver.factor_version
        z = grad_u.detach().conj().contiguous().clone()
        _after_torch(solver, z.device)
        solver.Solve(z, ctx.m, ctx.rel_tol)
        grad_f = z.conj() if ctx.needs_input_grad[1] else None
        grad_vel = solver.gradient_device(u, z).reshape(ctx.shape) if ctx.needs_input_grad[0] else None
        return grad_vel, grad_f, None, None, None, None


def helmholtz_solve(solver, velocity, f, m=20, rel_tol=1e-4, precision=FP64):
    """u = A(velocity)^{-1} f, factoring ``solver`` (a DistHelmholtz) at
    ``velocity``; differentiable in ``velocity`` and ``f``."""
    return _HelmholtzSolve.apply(velocity, f, solver, m, rel_tol, precision)


def misfit_and_gradient(solver, velocity, sources, receivers, data, m=20, rel_tol=1e-4, precision=FP64):
    """J = 1/2 sum |u[receivers] - data|^2 and dJ/dvelocity for one velocity
    model: an Initialize, a forward solve of all sources, an adjoint solve and
    the gradient kernel.  ``receivers`` indexes grid points (natural order);
    ``data`` is (len(receivers), k)."""
    vel = velocity.detach().clone().requires_grad_(True)
    u = helmholtz_solve(solver, vel, sources, m, rel_tol, precision)
    r = u[receivers.long()] - data
    J = 0.5 * (r.real.square() + r.imag.square()).sum()
    J.backward()
    return J.detach(), vel.grad
