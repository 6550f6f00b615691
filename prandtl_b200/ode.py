"""Explicit Runge-Kutta solvers around ``DGSEMOperator.Mult``: the reference's
other ``ode_solver`` choices (src/Simulation/Simulation.cpp:176-199, MFEM's
``ODESolver`` interface: ``Init(op)``, ``Step(x, t, dt)``).

The right-hand side of every stage is the operator's own kernels; the stage
combinations are torch operations on the same device (SSP-RK3, the
benchmark's solver, keeps its fused stages in ``RK3SSPSolver``).  Tableaux:

* ``ForwardEulerSolver``: x += dt L(x).
* ``RK2Solver(a)``: c = (0, a), A = (a), b = (1 - 1/(2a), 1/(2a)); MFEM's
  ``RK2Solver`` defaults to a = 2/3 (Ralston's method), the value the
  reference gets from ``std::make_shared<RK2Solver>()``.
* ``RK4Solver``: the classical fourth-order method (b = 1/6, 1/3, 1/3, 1/6),
  used by the backward-facing-step case (TestCases/Euler/2D/
  BackwardFacingStep/config.json).

MFEM is an external dependency of the reference and is not vendored with
it, so these are the published methods, not restated MFEM code; the RHS is
autonomous here (no boundary data depend on time), so the stage times c do
not enter.  The reference's ``RK6`` and ``RK8`` (Verner's tableaux in MFEM)
are not provided.
"""
from __future__ import annotations

from contextlib import nullcontext


class ExplicitRKSolver:
    """x_{n+1} = x_n + dt sum_i b_i k_i, k_i = L(x_n + dt sum_{j<i} A_ij k_j)."""

    def __init__(self, A, b, c):
        s = len(b)
        if len(A) != s - 1 or len(c) != s or any(len(A[i]) != i + 1 for i in range(s - 1)):
            raise ValueError("tableau: A holds rows 1..s-1 of the strictly lower triangle")
        self.A, self.b, self.c = [list(r) for r in A], list(b), list(c)
        self.op = None
        self._k = []
        self._y = None

    def Init(self, op):
        self.op = op
        self._k = []

    def Step(self, x, t: float, dt: float, stream=None) -> float:
        """One step of a device state (torch CUDA tensor) in place; returns t + dt."""
        import torch
        if self.op is None:
            raise RuntimeError("Init(op) first")
        s = len(self.b)
        if len(self._k) != s or self._k[0].shape != x.shape or self._k[0].device != x.device:
            self._k = [torch.empty_like(x) for _ in range(s)]
            self._y = torch.empty_like(x)
        ctx = torch.cuda.stream(stream) if stream is not None else nullcontext()
        with ctx:
            for i in range(s):
                if i == 0:
                    y = x
                else:
                    y = self._y
                    y.copy_(x)
                    for j, a in enumerate(self.A[i - 1]):
                        if a != 0.0:
                            y.add_(self._k[j], alpha=dt * a)
                self.op.Mult(y, self._k[i], stream=stream)
            for j, bj in enumerate(self.b):
                if bj != 0.0:
                    x.add_(self._k[j], alpha=dt * bj)
        return t + dt


class ForwardEulerSolver(ExplicitRKSolver):
    def __init__(self):
        super().__init__([], [1.0], [0.0])


class RK2Solver(ExplicitRKSolver):
    def __init__(self, a: float = 2.0 / 3.0):
        if a == 0.0:
            raise ValueError("RK2Solver: a must be non-zero")
        super().__init__([[a]], [1.0 - 1.0 / (2.0 * a), 1.0 / (2.0 * a)], [0.0, a])


class RK4Solver(ExplicitRKSolver):
    def __init__(self):
        super().__init__([[0.5], [0.0, 0.5], [0.0, 0.0, 1.0]],
                         [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0], [0.0, 0.5, 0.5, 1.0])


def make_solver(name: str):
    """The solver a reference configuration's ``ode_solver`` names."""
    from . import RK3SSPSolver
    table = {"ForwardEuler": ForwardEulerSolver, "RK2": RK2Solver, "RK3SSP": RK3SSPSolver, "RK4": RK4Solver}
    if name not in table:
        raise ValueError(f"ode_solver {name!r}: one of {sorted(table)} (RK6 and RK8 are not provided)")
    return table[name]()
