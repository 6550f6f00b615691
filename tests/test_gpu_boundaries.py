"""Boundary faces on the GPU (Euler) against the oracle, whose boundary
conditions are pinned to the reference's own integrators
(tests/test_boundaries.py): both face paths (element-side for the fixed
operator, separate face kernels + boundary_kernel for the reference-value
operator), RK stages, graph-replayed steps, the filter, and the errors."""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200.mesh import box

from helpers import rel_maxnorm, rough
from test_boundaries import freestream_box, layout_case, layouts, uniform

pytestmark = pytest.mark.gpu
TOL = 1e-12


def dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("order", [1, 3, 4])
@pytest.mark.parametrize("name", sorted(layouts()))
def test_gpu_boundaries_match_oracle(name, order, compat, cuda_device):
    import torch
    mesh, u = layout_case(name, order)
    op = pb.DGSEMOperator(mesh, compat=compat)
    orc = oracle.Oracle(mesh, compat=compat)
    ref = orc.rhs(u)
    out = torch.empty(u.size, dtype=torch.float64, device=cuda_device)
    op.Mult(dev(u, cuda_device), out)
    torch.cuda.synchronize()
    assert rel_maxnorm(out.cpu().numpy(), ref) < TOL
    assert abs(op.GetMaxCharSpeed() - orc.max_char_speed()) <= 1e-12 * orc.max_char_speed()
    assert op.check() == 0


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("name", ["2d_in_out_walls", "3d_all"])
def test_gpu_boundary_stages_and_graph_steps(name, compat, cuda_device):
    import torch
    mesh, u = layout_case(name, 3)
    op = pb.DGSEMOperator(mesh, compat=compat)
    orc = oracle.Oracle(mesh, compat=compat)
    orc.rhs(u)
    dt = 0.2 * min(mesh.h) / (orc.max_char_speed() * 16)
    un = dev(u, cuda_device)
    us = dev(rough(u, mesh, 5, 0.01, 0.001), cuda_device)
    for stage in (0, 1, 2):
        out = torch.empty_like(un)
        op.rk_stage(stage, dt, un, us, out)
        torch.cuda.synchronize()
        assert rel_maxnorm(out.cpu().numpy(), orc.rk_stage(stage, dt, un.cpu().numpy(), us.cpu().numpy())) < TOL
    a = un.clone()
    b = un.clone()
    op.rk3_step(a, dt, nsteps=3)
    op.rk3_step(b, dt, nsteps=3, graph=True)
    y = u
    for _ in range(3):
        y = orc.rk3_step(y, dt)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert rel_maxnorm(a.cpu().numpy(), y) < 1e-11


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 2)])
def test_gpu_freestream_is_preserved(dim, order, cuda_device):
    import torch
    mesh = freestream_box(dim, order)
    u = uniform(mesh)
    for compat in (0, 1):
        op = pb.DGSEMOperator(mesh, compat=compat)
        out = torch.empty(u.size, dtype=torch.float64, device=cuda_device)
        op.Mult(dev(u, cuda_device), out)
        torch.cuda.synchronize()
        assert np.abs(out.cpu().numpy()).max() < 1e-12 * np.abs(u).max()


def test_gpu_filter_with_boundaries(cuda_device):
    import torch
    mesh, u = layout_case("2d_in_out_walls", 3)
    u = rough(u, mesh, 3, 0.2, 0.05)   # rougher, still positive
    assert u[:mesh.num_nodes].min() > 0
    op = pb.DGSEMOperator(mesh, compat=0, filter=1)
    orc = oracle.Oracle(mesh, compat=0, filter=1)
    orc.rhs(u)
    dt = 0.2 * min(mesh.h) / (orc.max_char_speed() * 16)
    x = dev(u, cuda_device)
    op.rk3_step(x, dt)
    torch.cuda.synchronize()
    y = orc.rk3_step(u, dt)
    assert np.isfinite(y).all()
    assert rel_maxnorm(x.cpu().numpy(), y) < 1e-11
    assert op.filter_count() == orc.filtered_elements()


def test_boundary_errors(cuda_device):
    import torch
    mesh, u = layout_case("2d_symmetry_state", 2)
    bcs = mesh.boundaries
    mesh.boundaries = {0: bcs[0]}              # condition 1 left unset
    op = pb.DGSEMOperator(mesh)
    out = torch.empty(u.size, dtype=torch.float64, device=cuda_device)
    with pytest.raises(pb.PdgError) as ei:
        op.Mult(dev(u, cuda_device), out)
    assert ei.value.code == 1 and "not set" in str(ei.value)
    with pytest.raises(pb.PdgError):
        op.set_boundary(1, 9)                  # unknown type
    with pytest.raises(pb.PdgError):
        op.set_boundary(1, pb.BC_SPECIFIED_STATE)  # a state is needed
    with pytest.raises(pb.PdgError):
        op.set_boundary(1, pb.BC_SPECIFIED_STATE, [1.0, 0.0, 0.0, -1.0])  # p < 0
    with pytest.raises(pb.PdgError):
        op.set_boundary(pb.MAX_BOUNDARIES, pb.BC_SLIP_WALL)
    op.set_boundary(1, *bcs[1])
    op.Mult(dev(u, cuda_device), out)
    mesh.boundaries = bcs
    op_ns = pb.DGSEMOperator(mesh, parabolic=1, mu=0.01)   # symmetry plane: no viscous flux
    with pytest.raises(pb.PdgError) as ei:
        op_ns.Mult(dev(u, cuda_device), out)
    assert ei.value.code == 5
    mesh3, _ = layout_case("3d_subsonic", 1)
    op3 = pb.DGSEMOperator(mesh3)
    with pytest.raises(pb.PdgError) as ei:      # total-pressure inflow: 2D only
        op3.set_boundary(0, pb.BC_SUBSONIC_INFLOW_PTTT, [3.5, 3.0, 2.0, 0.0, 0.0])
    assert ei.value.code == 5
    with pytest.raises(pb.PdgError):            # outflow pressure must be positive
        op3.set_boundary(1, pb.BC_SUBSONIC_OUTFLOW_P, [-1.0])


@pytest.mark.parametrize("blending", [1, 0])
@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("name", sorted(layouts()))
def test_gpu_vjp_with_boundaries_matches_autograd(name, order, blending, cuda_device):
    """pdg_rhs_vjp on meshes with boundary conditions (every type) against
    torch autograd through the differentiable restatement (fixed operator)."""
    import torch
    from oracle.torch_rhs import TorchDGSEM
    mesh, u = layout_case(name, order)
    c = np.random.default_rng(2).standard_normal(u.size)
    ut = torch.tensor(u, requires_grad=True)
    (want,) = torch.autograd.grad(TorchDGSEM(mesh, blending=bool(blending)).rhs(ut), ut, torch.tensor(c))
    op = pb.DGSEMOperator(mesh, compat=0, blending=blending)
    got = op.vjp(dev(u, cuda_device), dev(c, cuda_device)).cpu().numpy()
    assert rel_maxnorm(got, want.numpy()) < 1e-11
    assert op.check() == 0


@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("name", ["ns_2d_channel", "ns_2d_cavity", "ns_2d_isothermal", "ns_3d_channel",
                                  "ns_2d_subsonic", "ns_3d_subsonic", "ns_2d_riemann", "ns_2d_pttt"])
def test_gpu_ns_boundaries_match_oracle(name, order, compat, cuda_device):
    """Navier-Stokes boundary faces (BR1 boundary lifting, viscous boundary
    fluxes, no-slip walls) of both operators against the oracle, whose
    boundary code is pinned to the reference's (tests/test_boundaries.py);
    the reference-value operator runs the separate face passes and the
    boundary kernel, the fixed one its element-side faces."""
    import torch
    from test_boundaries import NS_KW, ns_layout_case
    if compat and name == "ns_2d_riemann":
        pytest.skip("Riemann invariants with Navier-Stokes: fixed operator only")
    mesh, u = ns_layout_case(name, order)
    op = pb.DGSEMOperator(mesh, compat=compat, **NS_KW)
    orc = oracle.Oracle(mesh, compat=compat, **NS_KW)
    ref = orc.rhs(u)
    x = dev(u, cuda_device)
    out = torch.empty_like(x)
    op.Mult(x, out)
    torch.cuda.synchronize()
    assert rel_maxnorm(out.cpu().numpy(), ref) < TOL
    g = op.gradients(x).cpu().numpy()
    assert rel_maxnorm(g, orc.gradients()) < 1e-11
    dt = 0.2 * min(mesh.h) / (orc.max_char_speed() * (order + 1) ** 2)
    us = dev(rough(u, mesh, 8, 0.01, 0.001), cuda_device)
    for stage in (0, 1, 2):
        y = torch.empty_like(x)
        op.rk_stage(stage, dt, x, us, y)
        torch.cuda.synchronize()
        assert rel_maxnorm(y.cpu().numpy(), orc.rk_stage(stage, dt, u, us.cpu().numpy())) < TOL
    a, b = x.clone(), x.clone()
    op.rk3_step(a, dt, nsteps=2)
    op.rk3_step(b, dt, nsteps=2, graph=True)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert op.check() == 0


def test_ns_boundary_errors(cuda_device):
    import torch
    from test_boundaries import NS_KW, ns_layout_case
    mesh, u = ns_layout_case("ns_2d_channel", 2)
    op = pb.DGSEMOperator(mesh, compat=0, **NS_KW)
    x = dev(u, cuda_device)
    with pytest.raises(pb.PdgError) as ei:          # no adjoint of NS boundary faces
        op.vjp(x, x)
    assert ei.value.code == 5
    op.set_boundary(2, pb.BC_SLIP_WALL)             # no viscous flux in the reference
    with pytest.raises(pb.PdgError) as ei:
        op.Mult(x, torch.empty_like(x))
    assert ei.value.code == 5
    for name in ("ns_2d_riemann",):              # reference-value operator: not built
        mr, ur = ns_layout_case(name, 2)
        opr = pb.DGSEMOperator(mr, compat=1, **NS_KW)
        with pytest.raises(pb.PdgError) as ei:
            opr.Mult(dev(ur, cuda_device), torch.empty(ur.size, dtype=torch.float64, device=cuda_device))
        assert ei.value.code == 5


@pytest.mark.parametrize("which", ["ffs", "cavity"])
def test_gpu_case_builders_match_oracle(which, cuda_device):
    """A few SSP-RK3 steps of the forward-facing step (Euler) and the
    lid-driven cavity (Navier-Stokes) against the oracle."""
    import torch
    from prandtl_b200 import cases
    if which == "ffs":
        mesh, u = cases.forward_facing_step(2, 5)
        kw = dict(compat=0)
    else:
        mesh, u = cases.lid_driven_cavity(4, 3)
        kw = dict(compat=0, parabolic=1, mu=0.01, Pr=0.71)
    op = pb.DGSEMOperator(mesh, **kw)
    orc = oracle.Oracle(mesh, **kw)
    orc.rhs(u)
    dt = 0.2 * min(mesh.h) / (orc.max_char_speed() * (mesh.order + 1) ** 2)
    x = dev(u, cuda_device)
    op.rk3_step(x, dt, nsteps=3)
    y = u
    for _ in range(3):
        y = orc.rk3_step(y, dt)
    torch.cuda.synchronize()
    assert rel_maxnorm(x.cpu().numpy(), y) < 1e-11
    assert op.check() == 0


@pytest.mark.parametrize("name", ["ns_2d_subsonic", "ns_3d_channel", "ns_2d_riemann", "ns_2d_pttt"])
def test_gpu_ns_boundary_face_paths_agree(name, cuda_device, monkeypatch):
    """The fixed operator's element-side faces and its separate face passes
    (PDG_ELEMENT_FACES=0: lifting, face kernels, boundary_kernel) give the
    same Navier-Stokes result on meshes with boundary faces."""
    import torch
    from test_boundaries import NS_KW, ns_layout_case
    mesh, u = ns_layout_case(name, 3)
    op = pb.DGSEMOperator(mesh, compat=0, **NS_KW)
    monkeypatch.setenv("PDG_ELEMENT_FACES", "0")
    op_sep = pb.DGSEMOperator(mesh, compat=0, **NS_KW)
    monkeypatch.delenv("PDG_ELEMENT_FACES")
    un = dev(u, cuda_device)
    us = dev(rough(u, mesh, 9, 0.01, 0.001), cuda_device)
    for stage in (-1, 0, 2):
        a, b = torch.empty_like(un), torch.empty_like(un)
        if stage < 0:
            op.Mult(us, a)
            op_sep.Mult(us, b)
        else:
            op.rk_stage(stage, 1e-3, un, us, a)
            op_sep.rk_stage(stage, 1e-3, un, us, b)
        torch.cuda.synchronize()
        assert rel_maxnorm(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    assert op.check() == 0 and op_sep.check() == 0
