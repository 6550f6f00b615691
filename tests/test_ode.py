"""The explicit Runge-Kutta solvers (prandtl_b200.ode): tableaux, the host
logic on a linear test operator (CPU), and on the GPU against the same
tableau driven by the oracle's right-hand side."""
import numpy as np
import pytest

from prandtl_b200 import ode


class LinearOp:
    """L(x) = lam x on CPU tensors (the host logic only)."""

    def __init__(self, lam):
        self.lam = lam

    def Mult(self, u, dudt, stream=None):
        dudt.copy_(u * self.lam)


@pytest.mark.parametrize("name,poly", [
    ("ForwardEuler", [1, 1]),
    ("RK2", [1, 1, 0.5]),
    ("RK4", [1, 1, 0.5, 1 / 6, 1 / 24]),
])
def test_linear_amplification(name, poly):
    """On x' = lam x one step multiplies x by the method's stability
    polynomial sum_k (lam dt)^k / k! up to its order."""
    import torch
    lam, dt = -1.3, 0.2
    s = ode.make_solver(name)
    s.Init(LinearOp(lam))
    x = torch.ones(5, dtype=torch.float64)
    t = s.Step(x, 0.0, dt)
    z = lam * dt
    want = sum(c * z ** k for k, c in enumerate(poly))
    assert t == pytest.approx(dt)
    assert np.allclose(x.numpy(), want, rtol=1e-15, atol=0)


def test_tableaux():
    for s in (ode.ForwardEulerSolver(), ode.RK2Solver(), ode.RK2Solver(0.5), ode.RK4Solver()):
        assert sum(s.b) == pytest.approx(1.0)
        for i, row in enumerate(s.A):
            assert sum(row) == pytest.approx(s.c[i + 1])
    assert ode.RK2Solver().b == pytest.approx([0.25, 0.75])        # a = 2/3
    with pytest.raises(ValueError, match="RK8"):
        ode.make_solver("RK8")
    with pytest.raises(ValueError):
        ode.ExplicitRKSolver([[1.0, 2.0]], [0.5, 0.5], [0.0, 1.0])


def oracle_rk(orc, tab, u, dt):
    ks = []
    for i in range(len(tab.b)):
        y = u.copy()
        if i > 0:
            for j, a in enumerate(tab.A[i - 1]):
                y = y + dt * a * ks[j]
        ks.append(orc.rhs(y))
    out = u.copy()
    for j, b in enumerate(tab.b):
        out = out + dt * b * ks[j]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ForwardEuler", "RK2", "RK4"])
@pytest.mark.parametrize("parabolic", [0, 1])
def test_gpu_solvers_match_oracle(name, parabolic, cuda_device):
    import torch
    import oracle
    import prandtl_b200 as pb
    from helpers import rel_maxnorm, rough
    from test_boundaries import layout_case
    mesh, u = layout_case("2d_in_out_walls", 3)
    if parabolic:
        from test_boundaries import ns_layout_case
        mesh, u = ns_layout_case("ns_2d_subsonic", 3)
    kw = dict(compat=0, parabolic=parabolic, mu=0.02 if parabolic else 0.0, Pr=0.71)
    orc = oracle.Oracle(mesh, **kw)
    orc.rhs(u)
    dt = 0.1 * min(mesh.h) / (orc.max_char_speed() * 16)
    op = pb.DGSEMOperator(mesh, **kw)
    s = ode.make_solver(name)
    s.Init(op)
    x = torch.from_numpy(u.copy()).to(cuda_device)
    y = u
    t = 0.0
    for _ in range(2):
        t = s.Step(x, t, dt)
        y = oracle_rk(orc, s, y, dt)
    torch.cuda.synchronize()
    assert rel_maxnorm(x.cpu().numpy(), y) < 1e-11
    assert t == pytest.approx(2 * dt)
