"""Adjoint (vector-Jacobian product) of the right-hand side on the GPU.

Reference gradient: torch autograd through oracle/torch_rhs.py, the
differentiable restatement of the fixed operator (itself checked against the
C oracle).  Checks: the VJP against autograd (relative max norm, TOL_VJP);
the dot-product identity <c, J v> = <J^T c, v> with J v from central finite
differences of the GPU right-hand side (step 1e-6 relative per entry);
the torch.autograd.Function wrapper; and the gradient of the kinetic energy
after 20 SSP-RK3 steps with checkpoints every 5 steps against autograd
through 20 torch steps.
"""
import numpy as np
import pytest
import torch

import prandtl_b200 as pb
from oracle.torch_rhs import TorchDGSEM
from prandtl_b200 import adjoint, cases
from prandtl_b200.mesh import periodic_box

from helpers import rel_maxnorm, rough

# The VJP sums many terms of both signs (every two-point flux feeds two
# nodes); its rounding differs from autograd's summation order.
TOL_VJP = 1e-11
pytestmark = pytest.mark.gpu


def mean_flow(u, m, U=(0.3, -0.2, 0.25)):
    nn = m.num_nodes
    u = u.copy()
    rho = u[:nn]
    e = u[(m.nv - 1) * nn:]
    for d in range(m.dim):
        mom = u[(1 + d) * nn:(2 + d) * nn]
        e += rho * U[d] * (mom / rho) + 0.5 * rho * U[d] ** 2
        mom += rho * U[d]
    return u


def make(kind, dim, order):
    if kind == "vortex":
        m = cases.vortex_mesh(4, order)
        return m, cases.isentropic_vortex(m)
    if dim == 2:
        m = periodic_box(2, order, (4, 5), -1.0, 1.0)
        u = cases.kelvin_helmholtz(m)
        return m, (u if kind == "kh" else rough(u, m, 3))
    m = periodic_box(3, order, (3, 2, 4), 0.0, 2 * np.pi)
    u = cases.taylor_green(m)
    return m, (u if kind == "tgv" else mean_flow(rough(u, m, 5), m))


CASES = [("vortex", 2, 3, 0), ("kh", 2, 4, 0), ("rough2d", 2, 2, 0), ("rough2d", 2, 5, 0), ("rough2d", 2, 3, 1),
         ("tgv", 3, 3, 1), ("rough3d", 3, 3, 1), ("rough3d", 3, 2, 0), ("rough3d", 3, 1, 1), ("rough3d", 3, 4, 1),
         ("rough3d", 3, 5, 0)]


def params(par):
    return dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=0)


@pytest.mark.parametrize("blending", [1, 0])
@pytest.mark.parametrize("kind,dim,order,par", CASES)
def test_vjp_matches_autograd(kind, dim, order, par, blending, cuda_device):
    m, u = make(kind, dim, order)
    kw = params(par)
    rng = np.random.default_rng(1)
    c = rng.standard_normal(u.size)
    T = TorchDGSEM(m, parabolic=par, blending=bool(blending), mu=kw["mu"], Pr=0.71)
    ut = torch.tensor(u, requires_grad=True)
    (want,) = torch.autograd.grad(T.rhs(ut), ut, torch.tensor(c))
    op = pb.DGSEMOperator(m, blending=blending, **kw)
    got = op.vjp(torch.from_numpy(u).to(cuda_device), torch.from_numpy(c).to(cuda_device)).cpu().numpy()
    assert rel_maxnorm(got, want.numpy()) < TOL_VJP
    assert op.check() == 0


def test_vjp_rejects_compat_operator(cuda_device):
    m, u = make("tgv", 3, 2)
    op = pb.DGSEMOperator(m, parabolic=1, mu=0.01, compat=1)
    ud = torch.from_numpy(u).to(cuda_device)
    with pytest.raises(pb.PdgError):
        op.vjp(ud, ud.clone())


def test_dot_product_identity_tgv16(cuda_device):
    """TGV 16^3, N=3: <c, (L(u + e v) - L(u - e v)) / 2e> against <J^T c, v>
    on 32 random directions (cotangent seed 1, directions seed 2)."""
    m = cases.tgv_mesh(16, 3)
    u = cases.taylor_green(m)
    op = pb.DGSEMOperator(m, **params(1), blending=1)
    ud = torch.from_numpy(u).to(cuda_device)
    c = torch.from_numpy(np.random.default_rng(1).standard_normal(u.size)).to(cuda_device)
    g = op.vjp(ud, c)
    rng = np.random.default_rng(2)
    a, b = torch.empty_like(ud), torch.empty_like(ud)
    eps = 1e-6
    worst = 0.0
    for _ in range(32):
        v = torch.from_numpy(rng.standard_normal(u.size) * np.abs(u)).to(cuda_device)
        op.Mult(ud + eps * v, a)
        op.Mult(ud - eps * v, b)
        fd = (a - b) / (2 * eps)
        lhs, rhs = float((c * fd).sum()), float((g * v).sum())
        worst = max(worst, abs(lhs - rhs) / float((c.abs() * fd.abs()).sum()))
    assert worst < 1e-6


def test_autograd_function_wrapper(cuda_device):
    m, u = make("rough3d", 3, 2)
    op = pb.DGSEMOperator(m, **params(1))
    ud = torch.from_numpy(u).to(cuda_device).requires_grad_(True)
    c = torch.from_numpy(np.random.default_rng(4).standard_normal(u.size)).to(cuda_device)
    (g,) = torch.autograd.grad((adjoint.rhs(op, ud) * c).sum(), ud)
    want = op.vjp(ud.detach(), c)
    assert torch.equal(g, want)


def _torch_rk3(T, u, dt, nsteps):
    for _ in range(nsteps):
        u1 = u + dt * T.rhs(u)
        u2 = 0.75 * u + 0.25 * (u1 + dt * T.rhs(u1))
        u = u / 3.0 + 2.0 / 3.0 * (u2 + dt * T.rhs(u2))
    return u


@pytest.mark.parametrize("par", [1, 0])
def test_kinetic_energy_gradient_checkpointed(par, cuda_device):
    """d KE(u_20) / d u_0 with checkpoints every 5 steps against autograd
    through 20 torch steps; checkpoint spacing does not change the result."""
    m = periodic_box(3, 2, (3, 3, 2), 0.0, 2 * np.pi)
    u0 = mean_flow(cases.taylor_green(m), m)
    kw = params(par)
    op = pb.DGSEMOperator(m, **kw)
    ud = torch.from_numpy(u0).to(cuda_device)
    tmp = torch.empty_like(ud)
    op.Mult(ud, tmp)
    dt = op.cfl_dt(0.5)
    grads = []
    for every in (5, 1, 20):
        x0 = ud.clone().requires_grad_(True)
        ke = adjoint.kinetic_energy(m, adjoint.rk3(op, x0, dt, 20, every))
        (g,) = torch.autograd.grad(ke, x0)
        grads.append(g.cpu().numpy())
    assert np.array_equal(grads[0], grads[1]) and np.array_equal(grads[0], grads[2])
    T = TorchDGSEM(m, parabolic=par, mu=kw["mu"], Pr=0.71)
    ut = torch.tensor(u0, requires_grad=True)
    ke_t = adjoint.kinetic_energy(m, _torch_rk3(T, ut, dt, 20))
    (gt,) = torch.autograd.grad(ke_t, ut)
    assert rel_maxnorm(grads[0], gt.numpy()) < 1e-9


@pytest.mark.parametrize("kind,dim,order,par", [("rough2d", 2, 3, 0), ("rough3d", 3, 3, 1), ("rough3d", 3, 2, 0),
                                                ("rough2d", 2, 4, 1)])
def test_stage_vjp_fuses_the_stage_algebra(kind, dim, order, par, cuda_device):
    """pdg_rk_stage_vjp equals the VJP followed by the stage algebra in torch:
    stage 2 out = 2/3 (lam + dt g), bx = 1/3 lam; stage 1 out = 1/4 (lam + dt g),
    bx += 3/4 lam; stage 0 bx += lam + dt g (1e-13: one rounding of each term)."""
    m, u = make(kind, dim, order)
    op = pb.DGSEMOperator(m, **params(par))
    us = torch.from_numpy(u).to(cuda_device)
    rng = np.random.default_rng(11)
    lam = torch.from_numpy(rng.standard_normal(u.size)).to(cuda_device)
    bx0 = torch.from_numpy(rng.standard_normal(u.size)).to(cuda_device)
    dt = 1e-3
    g = op.vjp(us, lam)
    z = lam + dt * g
    want = {2: (2.0 / 3.0 * z, 1.0 / 3.0 * lam), 1: (0.25 * z, bx0 + 0.75 * lam), 0: (None, bx0 + z)}
    for stage in (2, 1, 0):
        out = torch.full_like(us, float("nan"))
        bx = bx0.clone()
        op.rk_stage_vjp(stage, dt, us, lam, out, bx)
        w_out, w_bx = want[stage]
        if w_out is not None:
            assert rel_maxnorm(out.cpu().numpy(), w_out.cpu().numpy()) < 1e-13, f"stage {stage} out"
        assert rel_maxnorm(bx.cpu().numpy(), w_bx.cpu().numpy()) < 1e-13, f"stage {stage} bx"
    assert op.check() == 0


def test_stage_vjp_rejects_boundary_meshes(cuda_device):
    mesh, u = cases.forward_facing_step(order=2, cells_per_unit=4)
    op = pb.DGSEMOperator(mesh, compat=0)
    x = torch.from_numpy(u).to(cuda_device)
    a, b = torch.empty_like(x), torch.zeros_like(x)
    with pytest.raises(pb.PdgError):
        op.rk_stage_vjp(1, 1e-3, x, x.clone(), a, b)
