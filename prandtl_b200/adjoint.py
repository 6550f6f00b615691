"""Differentiable right-hand side and SSP-RK3 trajectories for torch.

* ``rhs(op, u)`` — ``op.Mult`` as a ``torch.autograd.Function``; its backward
  is the CUDA vector-Jacobian product ``pdg_rhs_vjp``.
* ``rk3(op, u0, dt, nsteps, every)`` — ``nsteps`` fused SSP-RK3 steps whose
  backward recomputes each segment of ``every`` steps from a stored
  checkpoint and runs the discrete adjoint of the Shu-Osher stages through it,
  so memory holds ``nsteps / every`` states plus one segment's stages.
* ``kinetic_energy(mesh, u)`` — total kinetic energy with the LGL quadrature
  (sum over nodes of J w_i |m|^2 / (2 rho)), a differentiable objective.

The reference has no adjoint; these wrap the operator the reference's
``DGSEMOperator::Mult`` (src/Operators/DGSEMOperator.cpp:537-591) defines, in
its fixed form (``compat=0``), and MFEM's RK3SSPSolver stages
(src/Simulation/Simulation.cpp:1010).
"""
from __future__ import annotations

import numpy as np

from .mesh import CartesianMesh, gll_nodes


def _torch():
    import torch
    return torch


def _rhs_function():
    torch = _torch()

    class RHSFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u, op):
            out = torch.empty_like(u)
            op.Mult(u, out)
            ctx.save_for_backward(u)
            ctx.op = op
            return out

        @staticmethod
        def backward(ctx, g):
            (u,) = ctx.saved_tensors
            return ctx.op.vjp(u, g.contiguous()), None

    return RHSFunction


def _rk3_function():
    torch = _torch()

    class CheckpointedRK3(torch.autograd.Function):
        @staticmethod
        def forward(ctx, u0, op, dt, nsteps, every):
            x = u0.detach().clone()
            checkpoints = []
            for n in range(nsteps):
                if n % every == 0:
                    checkpoints.append(x.clone())
                op.rk3_step(x, dt)
            ctx.op, ctx.dt, ctx.nsteps, ctx.every = op, dt, nsteps, every
            ctx.checkpoints = checkpoints
            return x

        @staticmethod
        def backward(ctx, gN):
            op, dt, nsteps, every = ctx.op, ctx.dt, ctx.nsteps, ctx.every
            ubar = gN.contiguous().clone()
            tmp = torch.empty_like(ubar)
            # fused stage adjoints (pdg_rk_stage_vjp) on meshes without boundary faces
            fused = not getattr(op.mesh, "boundaries", None)
            if fused:
                b1, b2, bx = torch.empty_like(ubar), torch.empty_like(ubar), torch.empty_like(ubar)
            for seg in reversed(range(len(ctx.checkpoints))):
                first = seg * every
                last = min(first + every, nsteps)
                # recompute the segment's stage inputs (u, u1, u2) per step
                stages = []
                x = ctx.checkpoints[seg].clone()
                for _ in range(first, last):
                    u1, u2, u3 = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
                    op.rk_stage(0, dt, x, x, u1)
                    op.rk_stage(1, dt, x, u1, u2)
                    op.rk_stage(2, dt, x, u2, u3)
                    stages.append((x, u1, u2))
                    x = u3
                # u3 = u/3 + 2/3 (u2 + dt L(u2)); u2 = 3/4 u + 1/4 (u1 + dt L(u1)); u1 = u + dt L(u)
                for x, u1, u2 in reversed(stages):
                    if fused:
                        # the stage algebra runs inside the VJP's last kernel
                        op.rk_stage_vjp(2, dt, u2, ubar, b2, bx)
                        op.rk_stage_vjp(1, dt, u1, b2, b1, bx)
                        op.rk_stage_vjp(0, dt, x, b1, b2, bx)
                        ubar, bx = bx, ubar
                        continue
                    op.vjp(u2, ubar, out=tmp)
                    b2 = (2.0 / 3.0) * (ubar + dt * tmp)
                    bxs = (1.0 / 3.0) * ubar
                    op.vjp(u1, b2, out=tmp)
                    b1 = 0.25 * (b2 + dt * tmp)
                    bxs += 0.75 * b2
                    op.vjp(x, b1, out=tmp)
                    bxs += b1 + dt * tmp
                    ubar = bxs
            ctx.checkpoints = None
            return ubar, None, None, None, None

    return CheckpointedRK3


_RHS = None
_RK3 = None


def rhs(op, u):
    """Differentiable dudt = L(u) (op built with compat=0)."""
    global _RHS
    if _RHS is None:
        _RHS = _rhs_function()
    return _RHS.apply(u, op)


def rk3(op, u0, dt: float, nsteps: int, every: int = 5):
    """Differentiable state after nsteps SSP-RK3 steps, checkpointing every `every` steps."""
    global _RK3
    if _RK3 is None:
        _RK3 = _rk3_function()
    if every < 1 or nsteps < 0:
        raise ValueError("every >= 1 and nsteps >= 0 are required")
    return _RK3.apply(u0, op, float(dt), int(nsteps), int(every))


def node_weights(mesh: CartesianMesh) -> np.ndarray:
    """Quadrature weight J w_i (w_j w_k) of every node, byNODES order (one variable)."""
    _, w = gll_nodes(mesh.Np)
    w = np.asarray(w)
    J = float(np.prod(mesh.h))
    if mesh.dim == 2:
        we = np.outer(w, w).reshape(-1)
    else:
        we = np.einsum("k,j,i->kji", w, w, w).reshape(-1)
    return np.tile(J * we, mesh.num_elements)


def kinetic_energy(mesh: CartesianMesh, u, weights=None):
    """sum_nodes J w |m|^2 / (2 rho) of a device or host tensor u."""
    torch = _torch()
    nn = mesh.num_nodes
    if weights is None:
        weights = torch.as_tensor(node_weights(mesh), dtype=u.dtype, device=u.device)
    rho = u[:nn]
    m2 = sum(u[(1 + d) * nn:(2 + d) * nn] ** 2 for d in range(mesh.dim))
    return (weights * 0.5 * m2 / rho).sum()
