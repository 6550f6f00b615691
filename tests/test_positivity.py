"""Positivity-preserving limiter (params.filter & 2) after RK stages.

The reference's MinmodLimiter limits nothing (src/Limiters/MinmodLimiter.cpp:
22-77) and it has no positivity limiter, so the oracle restates the published
limiter of Zhang & Shu (2010), with its pressure step taken from the
concavity of the pressure.  CPU tests check the oracle's limiter for what the method guarantees:
element means unchanged (conservation), positive density and pressure at
every node afterwards, and elements without a violation left bit for bit.
GPU tests compare the CUDA limiter with the oracle after RK stages that
produce negative densities and pressures (rough states at large CFL), at
1e-12 relative in max norm (or four times the rounding floor of the stage, the
spread between the oracle's plain and fused-multiply-add builds, where that
is larger) with equal limiting counts, alone and after the
entropy filter, and on the Kelvin-Helmholtz benchmark mesh (64 x 64, N = 4),
whose configuration runs both.
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import gll_nodes, periodic_box

from helpers import rel_maxnorm, rough

TOL = 1e-12
GAMMA = 1.4


def _pressure(u, dim, nn):
    U = u.reshape(dim + 2, nn)
    return (GAMMA - 1.0) * (U[-1] - 0.5 * np.sum(U[1:1 + dim] ** 2, axis=0) / U[0])


def _means(u, mesh):
    _, w1 = gll_nodes(mesh.Np)
    wq = w1
    for _ in range(mesh.dim - 1):
        wq = np.kron(w1, wq)
    U = u.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    return np.einsum("ven,n->ve", U, wq) / wq.sum()


def _case(kind, order):
    if kind == "kh2d":
        m = periodic_box(2, order, (8, 9), -1.0, 1.0)
        return m, rough(cases.kelvin_helmholtz(m), m, 3, 0.15, 0.03), dict(parabolic=0)
    m = periodic_box(3, order, (4, 3, 5), 0.0, 2 * np.pi)
    u = rough(cases.taylor_green(m), m, 5, 0.15, 0.05)
    par = dict(parabolic=1, mu=0.01, Pr=0.71) if kind == "tgv3dns" else dict(parabolic=0)
    return m, u, par


# The CUDA kernels evaluate the fluxes in other algebraic forms than the
# oracle (shared reciprocals, the log-mean series expanded), so their rounding
# differs from the oracle's by a few times what fused multiply-adds alone
# change: the floor-based tolerance allows four times the floor.
FLOOR_FACTOR = 4.0


def _stage_tol(mesh, kw, stage, dt, un, us, want):
    """max(1e-12, FLOOR_FACTOR x the spread between the oracle's plain and
    fused-multiply-add builds on the same stage): near-vacuum nodes that the
    limiter leaves behind make a later stage's right-hand side very sensitive
    to rounding."""
    fma = oracle.Oracle(mesh, fma=True, **kw).rk_stage(stage, dt, un, us)
    return max(TOL, FLOOR_FACTOR * rel_maxnorm(fma, want))


def _dt(mesh, u, par, cfl):
    o = oracle.Oracle(mesh, compat=0, **par)
    o.rhs(u)
    return cfl * min(mesh.h) / (o.max_char_speed() * (mesh.order + 1) ** 2)


@pytest.mark.parametrize("kind,order,cfl", [("kh2d", 3, 10.0), ("kh2d", 4, 8.0), ("tgv3d", 3, 8.0)])
def test_oracle_limiter_conserves_and_restores_positivity(kind, order, cfl):
    mesh, u, par = _case(kind, order)
    orc = oracle.Oracle(mesh, compat=0, **par)
    y = orc.rk_stage(0, _dt(mesh, u, par, cfl), u, u)
    nn = mesh.num_nodes
    bad = (y[:nn] <= 0) | (_pressure(y, mesh.dim, nn) <= 0)
    assert bad.any(), "the case must produce non-positive nodes"
    z = oracle.Oracle(mesh, compat=0, filter=2, **par).positivity(y)
    np.testing.assert_allclose(_means(z, mesh), _means(y, mesh), rtol=1e-13, atol=1e-13)
    assert (z[:nn] > 0).all() and (_pressure(z, mesh.dim, nn) > 0).all()
    # elements with no violation keep their bits
    bad_el = bad.reshape(mesh.num_elements, mesh.ndof).any(axis=1)
    Y = y.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    Z = z.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    assert np.array_equal(Y[:, ~bad_el], Z[:, ~bad_el])
    assert not np.array_equal(Y[:, bad_el], Z[:, bad_el])


def test_oracle_limiter_leaves_positive_states():
    mesh = cases.vortex_mesh(8, 3)
    u = cases.isentropic_vortex(mesh)
    o = oracle.Oracle(mesh, compat=0, filter=2)
    assert np.array_equal(o.positivity(u), u)
    y = o.rk_stage(0, 1e-3, u, u)
    assert o.limited_elements() == 0
    assert np.array_equal(y, oracle.Oracle(mesh, compat=0).rk_stage(0, 1e-3, u, u))


# (kind, order, CFL, stages): a CFL at which the unlimited stage output has
# non-positive nodes while the limited stages stay finite; the Navier-Stokes
# case is run for its first stage only (its later stages, from near-vacuum
# nodes, are not finite at any CFL that limits)
LIMITED = [("kh2d", 3, 3.0, 3), ("kh2d", 4, 5.0, 3), ("kh2d", 2, 3.0, 3), ("tgv3d", 3, 5.0, 3), ("tgv3d", 2, 3.0, 3),
           ("tgv3d", 3, 10.0, 3), ("tgv3dns", 3, 4.0, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("filt", [2, 3])
@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("kind,order,cfl,stages", LIMITED)
def test_gpu_limited_stages_match_oracle(kind, order, cfl, stages, compat, filt, cuda_device):
    import torch
    mesh, u, par = _case(kind, order)
    dt = _dt(mesh, u, par, cfl)
    orc = oracle.Oracle(mesh, filter=filt, compat=compat, **par)
    op = pb.DGSEMOperator(mesh, filter=filt, compat=compat, **par)
    un = torch.from_numpy(u).to(cuda_device)
    us = u
    for stage in range(stages):
        want = orc.rk_stage(stage, dt, u, us)
        assert np.isfinite(want).all()
        out = torch.full_like(un, float("nan"))
        op.rk_stage(stage, dt, un, torch.from_numpy(us).to(cuda_device), out)
        got = out.cpu().numpy()
        tol = _stage_tol(mesh, dict(filter=filt, compat=compat, **par), stage, dt, u, us, want)
        assert rel_maxnorm(got, want) < tol, f"stage {stage}"
        assert op.limiter_count() == orc.limited_elements()
        if filt & 1:
            assert op.filter_count() == orc.filtered_elements()
        us = want
    if filt == 2:
        assert orc.limited_elements() > 0, "the case must exercise the limiter"
    # every element whose mean is admissible has positive nodes (at these
    # CFLs, beyond the scheme's positivity condition, a mean can leave the
    # admissible set, and then the limiter has nothing to contract towards)
    nn = mesh.num_nodes
    M = _means(us, mesh)
    ok_el = (M[0] > 0) & ((GAMMA - 1.0) * (M[-1] - 0.5 * np.sum(M[1:1 + mesh.dim] ** 2, axis=0) / M[0]) > 0)
    pos = ((us[:nn] > 0) & (_pressure(us, mesh.dim, nn) > 0)).reshape(mesh.num_elements, mesh.ndof).all(axis=1)
    assert pos[ok_el].all()


@pytest.mark.gpu
@pytest.mark.parametrize("rough_state", [False, True])
def test_gpu_kelvin_helmholtz_64_filter_and_limiter(rough_state, cuda_device):
    """The Kelvin-Helmholtz benchmark mesh (64 x 64, N = 4) with the entropy
    filter and the positivity limiter after every stage: one step's stages."""
    import torch
    mesh = cases.kh_mesh(64, 4)
    u = cases.kelvin_helmholtz(mesh)
    if rough_state:
        u = rough(u, mesh, 13, 0.15, 0.05)
    dt = _dt(mesh, u, dict(parabolic=0), 4.0 if rough_state else 0.5)
    kw = dict(parabolic=0, filter=3, compat=0)
    orc = oracle.Oracle(mesh, **kw)
    op = pb.DGSEMOperator(mesh, **kw)
    un = torch.from_numpy(u).to(cuda_device)
    us = u
    for stage in (0, 1, 2):
        want = orc.rk_stage(stage, dt, u, us)
        out = torch.empty_like(un)
        op.rk_stage(stage, dt, un, torch.from_numpy(us).to(cuda_device), out)
        tol = _stage_tol(mesh, kw, stage, dt, u, us, want)
        assert rel_maxnorm(out.cpu().numpy(), want) < tol, f"stage {stage}"
        assert op.limiter_count() == orc.limited_elements()
        assert op.filter_count() == orc.filtered_elements()
        us = want
    if rough_state:
        assert orc.limited_elements() > 0, "the roughened state must exercise the limiter"


# ---- general geometry: the limiter contracts towards J-weighted means ----

def _geo_case(kind):
    from prandtl_b200 import geometry as G
    if kind == "kh2d_curved":
        m = G.warped(periodic_box(2, 3, (8, 9), -1.0, 1.0), 0.03)
        return m, rough(cases.kelvin_helmholtz(m), m, 3, 0.15, 0.03)
    m = G.perturbed_box(3, 3, (4, 3, 5), 0.0, 2 * np.pi, 0.2, seed=2)
    return m, rough(cases.taylor_green(m), m, 5, 0.15, 0.05)


def _geo_means(u, mesh):
    """J-weighted element means (J from the LGL derivative of the node coordinates)."""
    _, w1 = gll_nodes(mesh.Np)
    wq = w1
    for _ in range(mesh.dim - 1):
        wq = np.kron(w1, wq)
    J = _node_jacobians(mesh)
    U = u.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    wt = J * wq[None, :]
    return np.einsum("ven,en->ve", U, wt) / wt.sum(axis=1)


def _node_jacobians(mesh):
    """det of dx/dxi at every node: the LGL derivative of the node coordinates."""
    x1, _ = gll_nodes(mesh.Np)
    Np, dim = mesh.Np, mesh.dim
    bw = np.array([1.0 / np.prod([x1[l] - x1[q] for q in range(Np) if q != l]) for l in range(Np)])
    D = np.zeros((Np, Np))
    for i in range(Np):
        for l in range(Np):
            if l != i:
                D[i, l] = bw[l] / bw[i] / (x1[i] - x1[l])
        D[i, i] = -D[i].sum()
    X = np.asarray(mesh.coords).reshape((dim, mesh.num_elements) + (Np,) * dim)
    cols = []
    for r in range(dim):
        ax = X.ndim - 1 - r  # reference axis r (x fastest) is array axis -1 - r
        cols.append(np.moveaxis(np.tensordot(D, X, axes=([1], [ax])), 0, ax))
    Jm = np.stack(cols, axis=-1)            # (dim_k, ne, ..., r)
    Jm = np.moveaxis(Jm, 0, -2)             # (ne, ..., k, r)
    return np.linalg.det(Jm).reshape(mesh.num_elements, -1)


@pytest.mark.parametrize("kind,cfl", [("kh2d_curved", 8.0), ("tgv3d_perturbed", 5.0)])
def test_oracle_limiter_on_general_geometry(kind, cfl):
    mesh, u = _geo_case(kind)
    par = dict(parabolic=0)
    o = oracle.Oracle(mesh, compat=0, **par)
    o.rhs(u)
    dt = cfl * min(mesh.h) / (o.max_char_speed() * (mesh.order + 1) ** 2)
    y = o.rk_stage(0, dt, u, u)
    nn = mesh.num_nodes
    bad = (y[:nn] <= 0) | (_pressure(y, mesh.dim, nn) <= 0)
    assert bad.any()
    z = oracle.Oracle(mesh, compat=0, filter=2, **par).positivity(y)
    np.testing.assert_allclose(_geo_means(z, mesh), _geo_means(y, mesh), rtol=1e-12, atol=1e-12)
    M = _geo_means(y, mesh)
    ok_el = (M[0] > 0) & ((GAMMA - 1.0) * (M[-1] - 0.5 * np.sum(M[1:1 + mesh.dim] ** 2, axis=0) / M[0]) > 0)
    pos = ((z[:nn] > 0) & (_pressure(z, mesh.dim, nn) > 0)).reshape(mesh.num_elements, mesh.ndof).all(axis=1)
    assert pos[ok_el].all()
    bad_el = bad.reshape(mesh.num_elements, mesh.ndof).any(axis=1)
    Y = y.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    Z = z.reshape(mesh.nv, mesh.num_elements, mesh.ndof)
    assert np.array_equal(Y[:, ~bad_el], Z[:, ~bad_el])


@pytest.mark.gpu
@pytest.mark.parametrize("filt", [2, 3])
@pytest.mark.parametrize("kind,cfl", [("kh2d_curved", 3.0), ("tgv3d_perturbed", 3.0)])
def test_gpu_limited_stages_on_general_geometry(kind, cfl, filt, cuda_device):
    """The entropy filter and the positivity limiter after each stage on a
    curved 2D and a perturbed 3D mesh, GPU against the oracle."""
    import torch
    mesh, u = _geo_case(kind)
    par = dict(parabolic=0)
    o = oracle.Oracle(mesh, compat=0, **par)
    o.rhs(u)
    dt = cfl * min(mesh.h) / (o.max_char_speed() * (mesh.order + 1) ** 2)
    kw = dict(filter=filt, compat=0, **par)
    orc = oracle.Oracle(mesh, **kw)
    op = pb.DGSEMOperator(mesh, **kw)
    un = torch.from_numpy(u).to(cuda_device)
    us = u
    for stage in range(3):
        want = orc.rk_stage(stage, dt, u, us)
        out = torch.empty_like(un)
        op.rk_stage(stage, dt, un, torch.from_numpy(us).to(cuda_device), out)
        tol = _stage_tol(mesh, kw, stage, dt, u, us, want)
        assert rel_maxnorm(out.cpu().numpy(), want) < tol, f"stage {stage}"
        assert op.limiter_count() == orc.limited_elements()
        if filt & 1:
            assert op.filter_count() == orc.filtered_elements()
        us = want
    if filt == 2:
        assert orc.limited_elements() > 0
