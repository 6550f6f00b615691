"""The differentiable torch restatement (reference gradient of the adjoint)
against the C oracle's fixed (compat = 0) operator, and its autograd against
finite differences of itself."""
import numpy as np
import pytest
import torch

import oracle
from oracle.torch_rhs import TorchDGSEM
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import rel_maxnorm, rough

CASES = [("vortex", 2, 3, 0), ("rough2d", 2, 4, 0), ("rough2dns", 2, 3, 1), ("tgv", 3, 3, 1),
         ("rough3d", 3, 2, 1), ("rough3d", 3, 3, 0), ("rough3d", 3, 1, 1), ("rough2d", 2, 5, 0)]


def make(kind, dim, order):
    if kind == "vortex":
        m = cases.vortex_mesh(4, order)
        return m, cases.isentropic_vortex(m)
    if dim == 2:
        m = periodic_box(2, order, (4, 5), -1.0, 1.0)
        return m, rough(cases.kelvin_helmholtz(m), m, 3)
    m = periodic_box(3, order, (3, 2, 4), 0.0, 2 * np.pi)
    u = cases.taylor_green(m)
    return m, (u if kind == "tgv" else rough(u, m, 5))


@pytest.mark.parametrize("kind,dim,order,par", CASES)
def test_torch_rhs_matches_oracle_fixed(kind, dim, order, par):
    m, u = make(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71)
    want = oracle.Oracle(m, compat=0, **kw).rhs(u)
    got = TorchDGSEM(m, **kw).rhs(torch.tensor(u)).numpy()
    assert rel_maxnorm(got, want) < 1e-13


def with_mean_flow(u, m, U=(0.3, -0.2, 0.25)):
    """Adds a uniform velocity U to a state (keeps rho and p)."""
    nn = m.num_nodes
    u = u.copy()
    rho = u[:nn]
    e = u[(m.nv - 1) * nn:]
    for d in range(m.dim):
        mom = u[(1 + d) * nn:(2 + d) * nn]
        e += rho * U[d] * (mom / rho) + 0.5 * rho * U[d] ** 2
        mom += rho * U[d]
    return u


# Two kinks of the operator defeat a central difference of step 1e-6: the
# blending sigmoid (slope ~ 9.2 / T, T ~ 4e-3), which roughened states reach,
# and the wave speed |v| + c of the Lax-Friedrichs term at |v| = 0, which
# Taylor-Green nodes on stagnation planes sit on (harmless there while the
# face jumps are as small as for the smooth state).  The roughened cases
# therefore run with blending off and a mean flow; TGV with blending on.
@pytest.mark.parametrize("kind,dim,order,par,blend", [("rough3d", 3, 2, 1, 0), ("rough2d", 2, 4, 0, 0),
                                                      ("tgv", 3, 3, 1, 1), ("rough3d", 3, 3, 0, 0)])
def test_torch_vjp_matches_finite_differences(kind, dim, order, par, blend):
    """<c, (L(u + e v) - L(u - e v)) / 2e> = <J^T c, v> on random directions."""
    m, u = make(kind, dim, order)
    if kind == "rough3d":
        u = with_mean_flow(u, m)
    T = TorchDGSEM(m, parabolic=par, blending=bool(blend), mu=0.01 if par else 0.0, Pr=0.71)
    rng = np.random.default_rng(2)
    c = rng.standard_normal(u.size)
    ut = torch.tensor(u, requires_grad=True)
    g, = torch.autograd.grad(T.rhs(ut), ut, torch.tensor(c))
    for k in range(4):
        v = rng.standard_normal(u.size) * np.abs(u)  # relative steps: no kink within reach
        eps = 1e-6
        with torch.no_grad():
            fd = (T.rhs(torch.tensor(u + eps * v)) - T.rhs(torch.tensor(u - eps * v))).numpy() / (2 * eps)
        lhs, rhs = float(c @ fd), float(g.numpy() @ v)
        assert abs(lhs - rhs) <= 1e-6 * (abs(c) @ np.abs(fd))
