"""General geometry on the GPU: geo_rhs_kernel against the oracle.

Meshes: curved (warped boxes, degree-N elements), skewed (an affine shear),
perturbed (bilinear / trilinear elements with moved vertices), rotated
element frames (faces meeting in other orientations, as in an unstructured
mesh) and perturbed boxes with boundary faces (inflow, outflow, slip wall,
symmetry; 3D adds Riemann invariants and a subsonic pressure outflow), in 2D
and 3D, both operators.  The oracle's general path matches the reference's
own sources to 1e-12 (tests/test_geometry.py).  Tolerance: 1e-12 relative in
max norm, or four times the rounding floor of the case (the spread between
the oracle's plain and fused-multiply-add builds) where that is larger.
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import geometry as G

from helpers import GEO_CASES, NS_GEO_CASES, geometry_case, ns_geometry_case, rel_maxnorm, smooth_state

pytestmark = pytest.mark.gpu

TOL = 1e-12
FLOOR_FACTOR = 4.0


def _tol(mesh, kw, fn):
    """max(TOL, FLOOR_FACTOR x the plain-vs-fma spread of the oracle's fn)."""
    a = fn(oracle.Oracle(mesh, **kw))
    b = fn(oracle.Oracle(mesh, fma=True, **kw))
    return max(TOL, FLOOR_FACTOR * rel_maxnorm(b, a)), a


@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("name", GEO_CASES)
def test_gpu_rhs_matches_oracle(name, compat, cuda_device):
    import torch
    g = geometry_case(name)
    u = smooth_state(g, 21)
    kw = dict(compat=compat, parabolic=0)
    tol, want = _tol(g, kw, lambda o: o.rhs(u))
    op = pb.DGSEMOperator(g, **kw)
    x = torch.from_numpy(u).to(cuda_device)
    out = torch.full_like(x, float("nan"))
    n0 = op.launch_count()
    op.Mult(x, out)
    assert op.launch_count() - n0 == 1
    assert rel_maxnorm(out.cpu().numpy(), want) < tol
    orc = oracle.Oracle(g, **kw)
    orc.rhs(u)
    eta_g, alpha_g = op.blending()
    eta_o, alpha_o = orc.blending()
    np.testing.assert_allclose(eta_g, eta_o, rtol=1e-12, atol=1e-14)
    # alpha = sigmoid(9.21 (eta - T) / T) amplifies eta's rounding by up to 9.2 eta / T
    np.testing.assert_allclose(alpha_g, alpha_o, rtol=1e-10, atol=1e-14)
    assert (alpha_o > 0).any()
    assert abs(op.GetMaxCharSpeed() - orc.max_char_speed()) <= 1e-12 * orc.max_char_speed()
    assert op.check() == 0


@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("name", ["warped2d", "rotated2d", "boundary2d", "warped3d", "rotated3d", "boundary3d"])
def test_gpu_rk_stages_and_graph_steps(name, compat, cuda_device):
    import torch
    g = geometry_case(name)
    u = smooth_state(g, 22)
    kw = dict(compat=compat, parabolic=0)
    op = pb.DGSEMOperator(g, **kw)
    x = torch.from_numpy(u).to(cuda_device)
    op.Mult(x, torch.empty_like(x))
    dt = op.cfl_dt(0.3)
    orc = oracle.Oracle(g, **kw)
    us = u
    for stage in range(3):
        tol, want = _tol(g, kw, lambda o: o.rk_stage(stage, dt, u, us))
        out = torch.empty_like(x)
        op.rk_stage(stage, dt, x, torch.from_numpy(us).to(cuda_device), out)
        assert rel_maxnorm(out.cpu().numpy(), want) < tol, f"stage {stage}"
        us = want
    want = u
    for _ in range(3):
        want = orc.rk3_step(want, dt)
    fma = u
    of = oracle.Oracle(g, fma=True, **kw)
    for _ in range(3):
        fma = of.rk3_step(fma, dt)
    y = x.clone()
    op.rk3_step(y, dt, nsteps=3, graph=True)
    assert rel_maxnorm(y.cpu().numpy(), want) < max(TOL, FLOOR_FACTOR * rel_maxnorm(fma, want))
    assert op.check() == 0


@pytest.mark.parametrize("name", ["warped2d", "skewed2d", "perturbed2d", "rotated2d"])
def test_gpu_free_stream_preservation_2d(name, cuda_device):
    import torch
    g = geometry_case(name)
    nn = g.num_nodes
    u = np.empty(g.size)
    u[:nn], u[nn:2 * nn], u[2 * nn:3 * nn], u[3 * nn:] = 1.2, 0.6, -0.3, 3.0
    op = pb.DGSEMOperator(g, compat=0, parabolic=0)
    x = torch.from_numpy(u).to(cuda_device)
    out = torch.empty_like(x)
    op.Mult(x, out)
    assert float(out.abs().max()) < 1e-11


@pytest.mark.parametrize("dim", [2, 3])
def test_gpu_rotation_invariance(dim, cuda_device):
    import torch
    base = geometry_case("perturbed2d" if dim == 2 else "perturbed3d")
    rt = G.rotate_frames(base, range(1, base.num_elements, 3), seed=9)
    u = smooth_state(base, 5)
    a_op = pb.DGSEMOperator(base, compat=0, parabolic=0)
    b_op = pb.DGSEMOperator(rt, compat=0, parabolic=0)
    xa = torch.from_numpy(u).to(cuda_device)
    xb = torch.from_numpy(G.permute_nodes(rt, u)).to(cuda_device)
    ra, rb = torch.empty_like(xa), torch.empty_like(xb)
    a_op.Mult(xa, ra)
    b_op.Mult(xb, rb)
    assert rel_maxnorm(rb.cpu().numpy(), G.permute_nodes(rt, ra.cpu().numpy())) < 1e-12


def test_gpu_geometry_errors(cuda_device):
    import torch
    g = geometry_case("rotated2d")
    # a wrong orientation code: the neighbour's normals do not match
    bad = G._copy(g)
    bad.coords = g.coords
    fo = np.array(g.face_orient, copy=True)
    e, f = 0, 1
    fo[e, f] ^= 2 << 3
    bad.face_orient = fo
    with pytest.raises(pb.PdgError) as ei:
        pb.DGSEMOperator(bad, compat=0, parabolic=0)
    assert ei.value.code == 1  # PDG_ERR_ARG
    # an inverted element
    inv = G._copy(g)
    Np = g.Np
    X = g.coords.reshape(2, g.num_elements, Np, Np).copy()
    X[:, 3] = X[:, 3, :, ::-1].copy()
    inv.coords = X.reshape(2, -1)
    inv.face_orient = g.face_orient
    with pytest.raises(pb.PdgError) as ei:
        pb.DGSEMOperator(inv, compat=0, parabolic=0)
    assert ei.value.code == 1  # PDG_ERR_ARG
    # the reference-value Navier-Stokes operator and the adjoint are box-mesh only
    with pytest.raises(pb.PdgError) as ei:
        pb.DGSEMOperator(g, compat=1, parabolic=1, mu=0.01)
    assert ei.value.code == 5  # PDG_ERR_UNSUPPORTED
    op = pb.DGSEMOperator(g, compat=0, parabolic=0)
    x = torch.from_numpy(smooth_state(g, 1)).to(cuda_device)
    with pytest.raises(pb.PdgError):
        op.vjp(x, torch.ones_like(x))
    # the geometry must be set before the first evaluation (a captured step
    # would otherwise replay the box kernels)
    from prandtl_b200.mesh import periodic_box
    bm = periodic_box(2, 3, (4, 5), 0.0, 1.0)
    opb = pb.DGSEMOperator(bm, compat=0, parabolic=0)
    xb = torch.from_numpy(smooth_state(bm, 1)).to(cuda_device)
    opb.Mult(xb, torch.empty_like(xb))
    with pytest.raises(pb.PdgError) as ei:
        opb._set_geometry(G.warped(bm, 0.01))
    assert ei.value.code == 1  # PDG_ERR_ARG


NS = dict(mu=0.01, Pr=0.71)


@pytest.mark.parametrize("name", NS_GEO_CASES + ["riemann2d_ns"])
def test_gpu_navier_stokes_matches_oracle(name, cuda_device):
    """Navier-Stokes on general geometry (fixed operator): the lifting
    kernel's primitive gradients, the right-hand side, the three RK stages
    and graph-replayed steps against the oracle (whose general NS path
    matches the reference's own NS build, tests/test_geometry.py)."""
    import torch
    g = ns_geometry_case(name)
    u = smooth_state(g, 31)
    kw = dict(compat=0, parabolic=1, **NS)
    op = pb.DGSEMOperator(g, **kw)
    x = torch.from_numpy(u).to(cuda_device)
    out = torch.empty_like(x)
    n0 = op.launch_count()
    op.Mult(x, out)
    assert op.launch_count() - n0 == 2
    tol, want = _tol(g, kw, lambda o: o.rhs(u))
    assert rel_maxnorm(out.cpu().numpy(), want) < tol
    orc = oracle.Oracle(g, **kw)
    orc.rhs(u)
    fma = oracle.Oracle(g, fma=True, **kw)
    fma.rhs(u)
    gw = orc.gradients()
    gtol = max(TOL, FLOOR_FACTOR * rel_maxnorm(fma.gradients(), gw))
    assert rel_maxnorm(op.gradients(x).cpu().numpy().reshape(-1), gw) < gtol
    dt = op.cfl_dt(0.3)
    us = u
    for stage in range(3):
        tol, want = _tol(g, kw, lambda o: o.rk_stage(stage, dt, u, us))
        o = torch.empty_like(x)
        op.rk_stage(stage, dt, x, torch.from_numpy(us).to(cuda_device), o)
        assert rel_maxnorm(o.cpu().numpy(), want) < tol, f"stage {stage}"
        us = want
    want, fw = u, u
    of = oracle.Oracle(g, fma=True, **kw)
    for _ in range(2):
        want = orc.rk3_step(want, dt)
        fw = of.rk3_step(fw, dt)
    y = x.clone()
    op.rk3_step(y, dt, nsteps=2, graph=True)
    assert rel_maxnorm(y.cpu().numpy(), want) < max(TOL, FLOOR_FACTOR * rel_maxnorm(fw, want))
    assert op.check() == 0


def test_gpu_navier_stokes_geometry_rejects_other_conditions(cuda_device):
    """Slip walls and symmetry planes have no viscous flux (as on box meshes)."""
    import torch
    from helpers import GEO_BCS_2D
    g = G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=5, bdr=[(0, 1), (2, 3)], boundaries=GEO_BCS_2D)
    op = pb.DGSEMOperator(g, compat=0, parabolic=1, **NS)   # a slip wall and a symmetry plane
    x = torch.from_numpy(smooth_state(g, 2)).to(cuda_device)
    with pytest.raises(pb.PdgError) as ei:
        op.Mult(x, torch.empty_like(x))
    assert ei.value.code == 5  # PDG_ERR_UNSUPPORTED
