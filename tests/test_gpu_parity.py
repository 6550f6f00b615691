"""GPU right-hand side and RK stages against the oracle, through the C ABI.

Tolerance: 1e-12 relative in max norm per RHS; the CUDA
kernels compute in FP64 with fused multiply-adds, the oracle without.
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import golden_cases, load_golden, rel_maxnorm, rough

TOL = 1e-12
# The BR1 gradient field is an intermediate, not an RHS.  Its density row is
# rho*dw0 - dw_last*(KE - p/(g-1)) + ...: O(p/(g-1)) terms cancelling to a small
# gradient, so for nearly constant density it carries ~1e-14 absolute noise;
# 1e-11 relative to the field's max covers that.
TOL_GRAD = 1e-11

pytestmark = pytest.mark.gpu


def dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


def gpu_rhs(op, u, device):
    import torch
    ud = dev(u, device)
    out = torch.empty_like(ud)
    op.Mult(ud, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", golden_cases())
def test_gpu_matches_reference_fixture(name, cuda_device):
    mesh, params, z = load_golden(name)
    op = pb.DGSEMOperator(mesh, compat=1, **params)
    got = gpu_rhs(op, z["u"], cuda_device)
    assert rel_maxnorm(got, z["dudt"]) < TOL
    eta, alpha = op.blending()
    np.testing.assert_allclose(eta, z["eta"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(alpha, z["alpha"], rtol=0, atol=1e-10)
    assert abs(op.GetMaxCharSpeed() - float(z["lam"])) <= 1e-12 * float(z["lam"])
    if params["parabolic"]:
        g = op.gradients(dev(z["u"], cuda_device)).cpu().numpy()
        assert rel_maxnorm(g, z["grads"]) < TOL_GRAD
    assert op.check() == 0


CASES = [
    ("vortex", 2, 3, 0), ("kh", 2, 4, 0), ("rough2d", 2, 2, 0), ("rough2d", 2, 5, 0), ("rough2d", 2, 1, 0),
    ("tgv", 3, 3, 1), ("rough3d", 3, 3, 1), ("rough3d", 3, 2, 1), ("rough3d", 3, 4, 1), ("rough3d", 3, 1, 1),
    ("rough3d", 3, 3, 0), ("rough2dns", 2, 3, 1), ("rough2dns", 2, 4, 1),
]


def make_case(kind, dim, order, n=4):
    if kind == "vortex":
        m = cases.vortex_mesh(n, order)
        return m, cases.isentropic_vortex(m)
    if kind in ("kh", "rough2d", "rough2dns"):
        m = periodic_box(2, order, (n, n + 1), -1.0, 1.0)
        u = cases.kelvin_helmholtz(m)
        return m, (rough(u, m, 3) if kind != "kh" else u)
    m = periodic_box(3, order, (n, n - 1, n + 1), 0.0, 2 * np.pi)
    u = cases.taylor_green(m)
    return m, (rough(u, m, 5) if kind != "tgv" else u)


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("kind,dim,order,par", CASES)
def test_gpu_rhs_matches_oracle(kind, dim, order, par, compat, cuda_device):
    mesh, u = make_case(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=compat)
    op = pb.DGSEMOperator(mesh, **kw)
    orc = oracle.Oracle(mesh, **kw)
    ref = orc.rhs(u)
    got = gpu_rhs(op, u, cuda_device)
    assert rel_maxnorm(got, ref) < TOL
    e1, a1 = op.blending()
    e0, a0 = orc.blending()
    np.testing.assert_allclose(a1, a0, rtol=0, atol=1e-10)
    if par:
        g = op.gradients(dev(u, cuda_device)).cpu().numpy()
        assert rel_maxnorm(g, orc.gradients()) < TOL_GRAD
    assert abs(op.GetMaxCharSpeed() - orc.max_char_speed()) <= 1e-12 * orc.max_char_speed()


def test_host_path_matches_device_path(cuda_device):
    mesh, u = make_case("rough2d", 2, 3)
    op = pb.DGSEMOperator(mesh)
    a = gpu_rhs(op, u, cuda_device)
    b = np.empty_like(u)
    op.Mult(u, b)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("kind,dim,order,par", [("vortex", 2, 3, 0), ("rough3d", 3, 3, 1), ("kh", 2, 4, 0)])
def test_rk_stages_match_oracle(kind, dim, order, par, compat, cuda_device):
    import torch
    mesh, u = make_case(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=compat)
    op = pb.DGSEMOperator(mesh, **kw)
    orc = oracle.Oracle(mesh, **kw)
    orc.rhs(u)
    dt = 0.3 * min(mesh.h) / (orc.max_char_speed() * (order + 1) ** 2)
    un = dev(u, cuda_device)
    us = dev(rough(u, mesh, 9, 0.01, 0.001), cuda_device)
    for stage in (0, 1, 2):
        out = torch.empty_like(un)
        op.rk_stage(stage, dt, un, us, out)
        ref = orc.rk_stage(stage, dt, un.cpu().numpy(), us.cpu().numpy())
        torch.cuda.synchronize()
        assert rel_maxnorm(out.cpu().numpy(), ref) < TOL
    x = un.clone()
    op.rk3_step(x, dt)
    ref = orc.rk3_step(u, dt)
    torch.cuda.synchronize()
    assert rel_maxnorm(x.cpu().numpy(), ref) < TOL


def test_ten_steps_track_oracle(cuda_device):
    """A short trajectory with the reference dt rule stays within 1e-10."""
    mesh = cases.vortex_mesh(8, 3)
    u = cases.isentropic_vortex(mesh)
    op = pb.DGSEMOperator(mesh)
    orc = oracle.Oracle(mesh)
    x = dev(u, cuda_device)
    tmp = dev(np.zeros_like(u), cuda_device)
    op.Mult(x, tmp)
    orc.rhs(u)
    y = u.copy()
    for _ in range(10):
        dt = op.cfl_dt(0.5)
        dt_o = 0.5 * min(mesh.h) / (orc.max_char_speed() * 16)
        assert abs(dt - dt_o) <= 1e-12 * dt_o
        op.rk3_step(x, dt)
        y = orc.rk3_step(y, dt)
    assert rel_maxnorm(x.cpu().numpy(), y) < 1e-10


def test_error_word_flags_negative_density(cuda_device):
    mesh, u = make_case("vortex", 2, 3)
    u = u.copy()
    u[5] = -1.0  # rho < 0 at one node, set on the host
    op = pb.DGSEMOperator(mesh)
    gpu_rhs(op, u, cuda_device)
    with pytest.raises(pb.PdgError) as ei:
        op.check()
    assert ei.value.code == 4
    assert op.check() == 0  # the word was cleared


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("kind,dim,order,par", [("vortex", 2, 3, 0), ("tgv", 3, 2, 1)])
def test_graph_replayed_steps_equal_plain_steps(kind, dim, order, par, compat, cuda_device):
    """pdg_rk3_steps (one captured step, replayed) gives pdg_rk3_step's values."""
    import torch
    mesh, u = make_case(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=compat)
    op = pb.DGSEMOperator(mesh, **kw)
    a = torch.from_numpy(u).to(cuda_device)
    b = a.clone()
    tmp = torch.empty_like(a)
    op.Mult(a, tmp)
    dt = op.cfl_dt(0.5)
    op.rk3_step(a, dt, nsteps=4)
    l0 = op.launch_count()
    op.rk3_step(b, dt, nsteps=4, graph=True)
    per_step = (op.launch_count() - l0) / 4
    assert torch.equal(a, b)
    if compat:   # (face jumps,) volume, (lifting,) face passes per stage
        assert per_step == (6 if par else 1 + dim) * 3
    else:        # face fluxes (with the jumps), (lifting,) volume with faces per stage
        assert per_step == (3 if par else 2) * 3
    op.rk3_step(b, dt, nsteps=2, graph=True)   # replay without capture
    op.rk3_step(a, dt, nsteps=2)
    assert torch.equal(a, b)
    assert op.check() == 0


@pytest.mark.parametrize("kind,dim,order,par", [("rough2d", 2, 3, 0), ("rough3d", 3, 3, 1), ("rough2dns", 2, 4, 1),
                                                ("rough3d", 3, 2, 0)])
def test_element_side_faces_equal_face_kernels(kind, dim, order, par, cuda_device, monkeypatch):
    """The fixed operator's volume kernel with both sides' face terms gives the
    separate face kernels' outputs (PDG_ELEMENT_FACES=0 selects those)."""
    import torch
    mesh, u = make_case(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=0)
    op = pb.DGSEMOperator(mesh, **kw)
    monkeypatch.setenv("PDG_ELEMENT_FACES", "0")
    op_sep = pb.DGSEMOperator(mesh, **kw)
    monkeypatch.delenv("PDG_ELEMENT_FACES")
    un = dev(u, cuda_device)
    us = dev(rough(u, mesh, 9, 0.01, 0.001), cuda_device)
    for stage in (-1, 0, 1, 2):
        a = torch.empty_like(un)
        b = torch.empty_like(un)
        if stage < 0:
            op.Mult(us, a)
            op_sep.Mult(us, b)
        else:
            op.rk_stage(stage, 1e-3, un, us, a)
            op_sep.rk_stage(stage, 1e-3, un, us, b)
        torch.cuda.synchronize()
        assert rel_maxnorm(a.cpu().numpy(), b.cpu().numpy()) < 1e-14
    assert op.check() == 0 and op_sep.check() == 0


@pytest.mark.parametrize("kind,dim,order,par", [("rough2d", 2, 3, 0), ("rough3d", 3, 3, 1), ("rough2dns", 2, 4, 1),
                                                ("rough3d", 3, 2, 0), ("rough2d", 2, 5, 0), ("rough3d", 3, 4, 1)])
def test_face_buffer_equals_element_faces(kind, dim, order, par, cuda_device, monkeypatch):
    """Each face's inviscid flux evaluated once into the face buffer gives the
    values of both elements evaluating it themselves (PDG_FACE_BUFFER=0): the
    same arithmetic on the same inputs, inlined into different kernels, so
    equal up to the compiler's choice of fused multiply-adds (1e-14)."""
    import torch
    mesh, u = make_case(kind, dim, order)
    kw = dict(parabolic=par, mu=0.01 if par else 0.0, Pr=0.71, compat=0)
    op = pb.DGSEMOperator(mesh, **kw)
    monkeypatch.setenv("PDG_FACE_BUFFER", "0")
    op_el = pb.DGSEMOperator(mesh, **kw)
    monkeypatch.delenv("PDG_FACE_BUFFER")
    un = dev(u, cuda_device)
    us = dev(rough(u, mesh, 9, 0.01, 0.001), cuda_device)
    for stage in (-1, 0, 1, 2):
        a = torch.empty_like(un)
        b = torch.empty_like(un)
        if stage < 0:
            op.Mult(us, a)
            op_el.Mult(us, b)
        else:
            op.rk_stage(stage, 1e-3, un, us, a)
            op_el.rk_stage(stage, 1e-3, un, us, b)
        torch.cuda.synchronize()
        assert rel_maxnorm(a.cpu().numpy(), b.cpu().numpy()) < 1e-14, f"stage {stage}"
    assert op.GetMaxCharSpeed() == op_el.GetMaxCharSpeed()
    assert op.check() == 0 and op_el.check() == 0


@pytest.mark.parametrize("kind", ["tgv16_ns", "tgv16_euler", "vortex64"])
def test_host_step_pipeline_equals_device_step(kind, cuda_device, monkeypatch):
    """pdg_rk3_step_host pipelines its copies with stages 0 and 2 on meshes of
    4096 elements and more; two host steps equal two device steps bit for bit,
    and the unpipelined host step (PDG_HOST_PIPELINE=0) as well."""
    import torch
    if kind == "vortex64":
        mesh = cases.vortex_mesh(64, 3)
        u = rough(cases.isentropic_vortex(mesh), mesh, 7, 0.05, 0.01)
        kw = dict(parabolic=0, compat=0)
    else:
        mesh = cases.tgv_mesh(16, 3)
        u = rough(cases.taylor_green(mesh), mesh, 7, 0.02, 0.002)
        kw = dict(parabolic=1 if kind.endswith("ns") else 0, mu=1.0 / 1600.0, Pr=0.71, compat=0)
    assert mesh.num_elements >= 32 * 128
    op = pb.DGSEMOperator(mesh, **kw)
    x = dev(u, cuda_device)
    op.Mult(x, torch.empty_like(x))
    dt = op.cfl_dt(0.5)
    ref = x.clone()
    op.rk3_step(ref, dt, nsteps=2)
    lam = op.GetMaxCharSpeed()
    host = torch.from_numpy(u.copy()).pin_memory().numpy()
    for _ in range(2):
        op.rk3_step_host(host, dt)
    assert np.array_equal(host, ref.cpu().numpy())
    assert op.GetMaxCharSpeed() == lam
    monkeypatch.setenv("PDG_HOST_PIPELINE", "0")
    op2 = pb.DGSEMOperator(mesh, **kw)
    monkeypatch.delenv("PDG_HOST_PIPELINE")
    host2 = torch.from_numpy(u.copy()).pin_memory().numpy()
    for _ in range(2):
        op2.rk3_step_host(host2, dt)
    assert np.array_equal(host2, host)
    pageable = u.copy()  # the pipeline also serves pageable memory (without overlap)
    op.rk3_step_host(pageable, dt)
    op.rk3_step_host(pageable, dt)
    assert np.array_equal(pageable, host)
    assert op.check() == 0
