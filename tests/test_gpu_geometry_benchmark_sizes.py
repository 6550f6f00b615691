"""General geometry at the geometry benchmark's full sizes: parity with the
oracle and discrete entropy conservation of the CUDA right-hand side.

Meshes (the ones the geometry bench cases time):
* curved Taylor-Green 32^3, N = 3: the periodic box [0, 2 pi]^3 with its DG
  nodes moved by a smooth periodic field of amplitude 0.02 (2.1 M nodes);
  Euler (both operators) and Navier-Stokes (mu = 1/1600, Pr = 0.71, fixed
  operator), on the Taylor-Green state and on a roughened state where every
  element blends in the subcell scheme;
* unstructured Kelvin-Helmholtz 128^2, N = 4: bilinear elements with randomly
  moved vertices and every other element's frame rotated (faces meeting in
  other orientations), Euler, both operators.

The oracle's general path is pinned to the reference's own integrators on
small meshes (tests/test_geometry.py); here the GPU runs the right-hand side
and the three SSP-RK3 stages at the full size.  Tolerance: 1e-12 relative in
max norm, or four times the rounding floor of the state (the spread between
the oracle's plain and fused-multiply-add builds) where that is larger.

Entropy conservation: with the face dissipation off and no blending, the
flux-differencing operator with mean metrics conserves entropy on a periodic
mesh whose metric terms meet the discrete metric identities (both meshes
here: 2D, and a warped box whose displacement is one scalar field in every
component, see tests/test_geometry.py), sum_i J_i w_i w(u_i) . du_i/dt = 0
(J_i the node's Jacobian determinant, w_i its LGL weight); the oracle meets
it at 1e-16 relative.  The
test checks the CUDA right-hand side at 1e-12 of sum_i J_i w_i |w . du/dt|,
and that the sum is negative with the dissipation on.
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200 import geometry as G
from prandtl_b200.mesh import periodic_box

from helpers import entropy_production, rel_maxnorm, rough

pytestmark = pytest.mark.gpu

TOL = 1e-12
FLOOR_FACTOR = 4.0
NS = dict(mu=1.0 / 1600.0, Pr=0.71)


def _curved_tgv(rough_state):
    g = G.warped(periodic_box(3, 3, 32, 0.0, 2 * np.pi), 0.02)
    u = cases.taylor_green(g)
    return g, (rough(u, g, 11, 0.02, 0.002) if rough_state else u)


def _unstructured_kh(rough_state):
    n = 128
    g = G.rotate_frames(G.perturbed_box(2, 4, n, -1.0, 1.0, 0.2, seed=1), range(0, n * n, 2), seed=2)
    u = cases.kelvin_helmholtz(g)
    return g, (rough(u, g, 13, 0.1, 0.02) if rough_state else u)


def _case(name):
    rough_state = name.endswith("_rough")
    return _curved_tgv(rough_state) if name.startswith("tgv") else _unstructured_kh(rough_state)


def _dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


def _rhs(op, u, device):
    import torch
    ud = _dev(u, device)
    out = torch.full_like(ud, float("nan"))
    op.Mult(ud, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _stage(op, stage, dt, un, us, device):
    import torch
    a, b = _dev(un, device), _dev(us, device)
    out = torch.full_like(a, float("nan"))
    op.rk_stage(stage, dt, a, b, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _check(mesh, u, kw, rough_state, device):
    op = pb.DGSEMOperator(mesh, **kw)
    orc = oracle.Oracle(mesh, **kw)
    ref = orc.rhs(u)
    floor = rel_maxnorm(oracle.Oracle(mesh, fma=True, **kw).rhs(u), ref)
    tol = max(TOL, FLOOR_FACTOR * floor)
    err = rel_maxnorm(_rhs(op, u, device), ref)
    assert err < tol, f"relative error {err:.3e}, rounding floor {floor:.3e}"
    eta_g, alpha_g = op.blending()
    eta_o, alpha_o = orc.blending()
    np.testing.assert_allclose(eta_g, eta_o, rtol=1e-10, atol=1e-13)
    # alpha = sigmoid(9.21 (eta - T) / T) amplifies eta's rounding
    np.testing.assert_allclose(alpha_g, alpha_o, rtol=1e-9, atol=1e-10)
    if rough_state:
        assert (alpha_o > 0).any(), "the roughened state must switch the subcell blending on"
    lam = orc.max_char_speed()
    assert abs(op.GetMaxCharSpeed() - lam) <= 1e-12 * lam
    dt = op.cfl_dt(0.3)
    us = u
    for stage in (0, 1, 2):
        want = orc.rk_stage(stage, dt, u, us)
        got = _stage(op, stage, dt, u, us, device)
        assert rel_maxnorm(got, want) < TOL, f"stage {stage}"
        us = want
    assert op.check() == 0


@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("name", ["tgv32", "tgv32_rough", "kh128", "kh128_rough"])
def test_geometry_benchmark_mesh_euler(name, compat, cuda_device):
    mesh, u = _case(name)
    _check(mesh, u, dict(parabolic=0, compat=compat), name.endswith("_rough"), cuda_device)


@pytest.mark.parametrize("name", ["tgv32", "tgv32_rough"])
def test_geometry_benchmark_mesh_navier_stokes(name, cuda_device):
    mesh, u = _case(name)
    _check(mesh, u, dict(parabolic=1, compat=0, **NS), name.endswith("_rough"), cuda_device)


@pytest.mark.parametrize("name", ["tgv32_rough", "kh128_rough"])
def test_geometry_entropy_conservation_on_gpu(name, cuda_device):
    mesh, u = _case(name)
    op = pb.DGSEMOperator(mesh, parabolic=0, blending=0, compat=0, face_dissipation=0.0)
    prod, scale = entropy_production(mesh, u, _rhs(op, u, cuda_device))
    assert scale > 0
    assert abs(prod) < 1e-12 * scale, f"entropy production {prod:.3e} against scale {scale:.3e}"
    op_d = pb.DGSEMOperator(mesh, parabolic=0, blending=0, compat=0)
    prod_d, _ = entropy_production(mesh, u, _rhs(op_d, u, cuda_device))
    assert prod_d < 0
