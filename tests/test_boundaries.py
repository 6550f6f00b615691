"""Boundary faces of the oracle (Euler; src/Integrators/BoundaryConditions/):
freestream preservation and mirror equivalence of the symmetry condition."""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import box, periodic_box

from helpers import rough

GAMMA = 1.4


def uniform(mesh, rho=1.0, vel=(2.0, 0.0, 0.0), p=1.0):
    u = np.zeros((mesh.nv, mesh.num_nodes))
    u[0] = rho
    for d in range(mesh.dim):
        u[1 + d] = rho * vel[d]
    u[-1] = p / (GAMMA - 1) + 0.5 * rho * sum(v * v for v in vel[:mesh.dim])
    return u.reshape(-1)


def freestream_box(dim, order):
    """Supersonic flow along x: inflow at -x, outflow at +x, slip walls on y,
    symmetry on z."""
    fs = uniform(periodic_box(dim, 1, 1, 0.0, 1.0))[:: (2 ** dim)]  # one node per variable
    bdr = [(0, 1), (2, 2)] + ([(3, 3)] if dim == 3 else [])
    bcs = {0: (pb.BC_SUPERSONIC_INFLOW, fs), 1: (pb.BC_SUPERSONIC_OUTFLOW, None), 2: (pb.BC_SLIP_WALL, None)}
    if dim == 3:
        bcs[3] = (pb.BC_SYMMETRY, None)
    n = (4, 3, 2)[:dim]
    return box(dim, order, n, 0.0, 1.0, bdr=bdr, boundaries=bcs)


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 2)])
@pytest.mark.parametrize("compat", [0, 1])
def test_freestream_is_preserved(dim, order, compat):
    mesh = freestream_box(dim, order)
    u = uniform(mesh)
    orc = oracle.Oracle(mesh, compat=compat)
    r = orc.rhs(u)
    assert np.abs(r).max() < 1e-12 * np.abs(u).max()


@pytest.mark.parametrize("order", [2, 3])
def test_symmetry_equals_mirrored_periodic_domain(order):
    """A symmetry plane at y = 0 of [0,1]^2 gives the RHS of the periodic
    [-1,1] x [0,1]... mirrored: the domain y in [-1, 1], periodic, holding the
    state mirrored about y = 0 (v -> -v) has no flux through y = 0 beyond the
    symmetric one, so its upper half's RHS equals the symmetry-bounded one."""
    nx, ny = 3, 2
    half = box(2, order, (nx, ny), (0.0, 0.0), (1.0, 1.0), bdr=[None, (0, 0)],
               boundaries={0: (pb.BC_SYMMETRY, None)})
    full = periodic_box(2, order, (nx, 2 * ny), (0.0, -1.0), (1.0, 1.0))
    # a smooth positive state on the half mesh, mirrored to the full mesh
    u_half = rough(cases.kelvin_helmholtz(periodic_box(2, order, (nx, ny), -1.0, 1.0)), half, 3, 0.05, 0.01)
    Np = order + 1
    uh = u_half.reshape(4, ny, nx, Np, Np)          # v, ey, ex, j, i
    uf = np.empty((4, 2 * ny, nx, Np, Np))
    uf[:, ny:] = uh                                  # upper half: y in [0, 1]
    mir = uh[:, ::-1, :, ::-1, :].copy()             # reflected elements and nodes
    mir[2] = -mir[2]                                 # v -> -v
    uf[:, :ny] = mir
    r_half = oracle.Oracle(half, compat=0, blending=0).rhs(u_half).reshape(4, ny, nx, Np, Np)
    r_full = oracle.Oracle(full, compat=0, blending=0).rhs(uf.reshape(-1)).reshape(4, 2 * ny, nx, Np, Np)
    scale = np.abs(r_full).max()
    assert np.abs(r_half - r_full[:, ny:]).max() < 1e-12 * scale


def test_torch_reference_rejects_navier_stokes_boundaries():
    """The differentiable restatement (the adjoint's reference) has no
    Navier-Stokes boundary faces."""
    from oracle.torch_rhs import TorchDGSEM
    mesh = freestream_box(2, 2)
    with pytest.raises(ValueError):
        TorchDGSEM(mesh, parabolic=True, mu=0.01)


def _step_keep(n):
    keep = np.ones(n, dtype=bool)
    keep[2:, 0] = False
    return keep


def layouts():
    """Boundary layouts covering every condition type on every side."""
    fs2 = np.array([1.2, 0.3, -0.2, 2.6])
    fs3 = np.array([1.1, 0.2, -0.1, 0.15, 2.8])
    return {
        "2d_in_out_walls": (2, dict(bdr=[(0, 1), (2, 2)], boundaries={
            0: (pb.BC_SUPERSONIC_INFLOW, fs2), 1: (pb.BC_SUPERSONIC_OUTFLOW, None), 2: (pb.BC_SLIP_WALL, None)})),
        "2d_symmetry_state": (2, dict(bdr=[None, (0, 1)], boundaries={
            0: (pb.BC_SYMMETRY, None), 1: (pb.BC_SPECIFIED_STATE, fs2)})),
        "3d_all": (3, dict(bdr=[(0, 0), (1, 2), (3, 4)], boundaries={
            0: (pb.BC_SLIP_WALL, None), 1: (pb.BC_SYMMETRY, None), 2: (pb.BC_SUPERSONIC_OUTFLOW, None),
            3: (pb.BC_SPECIFIED_STATE, fs3), 4: (pb.BC_SUPERSONIC_INFLOW, fs3)})),
        # subsonic inflow from total pressure / temperature and flow angle,
        # subsonic outflow at a pressure, Riemann invariants, inflow from rho, V
        "2d_subsonic": (2, dict(bdr=[(0, 1), (2, 3)], boundaries={
            0: (pb.BC_SUBSONIC_INFLOW_PTTT, [3.5, 3.0, 2.0, 10.0, 0.0]), 1: (pb.BC_SUBSONIC_OUTFLOW_P, [2.2]),
            2: (pb.BC_RIEMANN_INVARIANT, [1.0, 0.3, -0.1, 2.0]), 3: (pb.BC_SUBSONIC_INFLOW_RV, [1.3, 0.2, 0.05])})),
        # no-slip walls in an Euler run act as slip walls (their viscous parts
        # are not evaluated)
        "2d_noslip_euler": (2, dict(bdr=[None, (0, 1)], boundaries={
            0: (pb.BC_NOSLIP_ADIABATIC, [0.0, 0.0]), 1: (pb.BC_NOSLIP_ISOTHERMAL, [0.009, 0.2, 0.0])})),
        # forward-facing step: the bottom row is removed from x = -1 + 2/5 * 2 on
        "2d_step": (2, dict(bdr=[(0, 1), (2, 2)], keep=_step_keep((5, 4)), cut=2, boundaries={
            0: (pb.BC_SUPERSONIC_INFLOW, np.array([1.4, 4.2, 0.0, 8.8])), 1: (pb.BC_SUPERSONIC_OUTFLOW, None),
            2: (pb.BC_SLIP_WALL, None)})),
        "3d_subsonic": (3, dict(bdr=[(0, 1), (2, 2), None], boundaries={
            0: (pb.BC_SUBSONIC_INFLOW_RV, [1.2, 0.1, 0.05, -0.02]), 1: (pb.BC_SUBSONIC_OUTFLOW_P, [2.0]),
            2: (pb.BC_RIEMANN_INVARIANT, [1.0, 0.2, 0.1, -0.1, 2.0])})),
    }


def layout_case(name, order):
    dim, kw = layouts()[name]
    if "keep" in kw:
        mesh = box(2, order, kw["keep"].shape, (-1.0, -1.0), (1.0, 1.0), **kw)
        return mesh, rough(cases.kelvin_helmholtz(mesh), mesh, 11, 0.05, 0.02)
    if dim == 2:
        mesh = box(2, order, (4, 3), (-1.0, -1.0), (1.0, 1.0), **kw)
        u = cases.kelvin_helmholtz(periodic_box(2, order, (4, 3), -1.0, 1.0))
    else:
        mesh = box(3, order, (3, 2, 3), 0.0, 2 * np.pi, **kw)
        u = cases.taylor_green(periodic_box(3, order, (3, 2, 3), 0.0, 2 * np.pi), Ma=0.4)
    return mesh, rough(u, mesh, 11, 0.05, 0.02)


@pytest.mark.skipif(not oracle.ref_available(False), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("name", sorted(layouts()))
def test_oracle_boundaries_match_live_reference(name, order):
    """The reference's own boundary integrators (BdrFaceIntegrator.cpp and the
    five condition files, compiled here against the stand-in MFEM header)."""
    mesh, u = layout_case(name, order)
    o = oracle.Oracle(mesh, compat=1)
    r = oracle.Reference(mesh, parabolic=False)
    ro, rr = o.rhs(u), r.rhs(u)
    assert np.abs(ro - rr).max() <= 1e-12 * np.abs(rr).max()
    assert abs(o.max_char_speed() - r.lam) <= 1e-13 * r.lam


@pytest.mark.parametrize("name", ["2d_subsonic", "3d_subsonic"])
def test_subsonic_conditions_differ_between_operators(name):
    """The reference's subsonic conditions divide the interior momenta in
    place before the face flux reads them (compat keeps that, fixed does
    not), so the two operators differ on these boundaries."""
    mesh, u = layout_case(name, 2)
    a = oracle.Oracle(mesh, compat=1).rhs(u)
    b = oracle.Oracle(mesh, compat=0).rhs(u)
    assert np.abs(a - b).max() > 1e-6 * np.abs(a).max()


@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("name", sorted(layouts()))
def test_torch_reference_boundaries_match_oracle(name, order):
    """The differentiable restatement (the adjoint's reference gradient) on
    boundary layouts of conditions 1-5, fixed operator."""
    import torch
    from oracle.torch_rhs import TorchDGSEM
    mesh, u = layout_case(name, order)
    got = TorchDGSEM(mesh).rhs(torch.tensor(u)).numpy()
    ref = oracle.Oracle(mesh, compat=0).rhs(u)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


NOSLIP = 10  # no-slip adiabatic wall (data: wall velocity)


def ns_layouts():
    """Navier-Stokes boundary layouts: inflow/outflow channels with no-slip
    walls and a lid-driven cavity."""
    fs2 = np.array([1.2, 0.3, -0.2, 2.6])
    fs3 = np.array([1.1, 0.2, -0.1, 0.15, 2.8])
    return {
        "ns_2d_channel": (2, dict(bdr=[(0, 1), (2, 2)], boundaries={
            0: (pb.BC_SUPERSONIC_INFLOW, fs2), 1: (pb.BC_SUPERSONIC_OUTFLOW, None), 2: (NOSLIP, [0.0, 0.0])})),
        "ns_2d_cavity": (2, dict(bdr=[(0, 0), (0, 1)], boundaries={
            0: (NOSLIP, [0.0, 0.0]), 1: (NOSLIP, [1.0, 0.0])})),
        "ns_2d_isothermal": (2, dict(bdr=[(0, 1), (2, 3)], boundaries={
            0: (pb.BC_SPECIFIED_STATE, fs2), 1: (pb.BC_SUPERSONIC_OUTFLOW, None),
            2: (pb.BC_NOSLIP_ISOTHERMAL, [0.009, 0.0, 0.0]), 3: (pb.BC_NOSLIP_ISOTHERMAL, [0.007, 0.3, 0.0])})),
        "ns_3d_channel": (3, dict(bdr=[(0, 1), (2, 2), None], boundaries={
            0: (pb.BC_SPECIFIED_STATE, fs3), 1: (pb.BC_SUPERSONIC_OUTFLOW, None), 2: (NOSLIP, [0.1, 0.0, 0.0])})),
        # subsonic inflow (rho, V) and outflow at a pressure between walls:
        # the default lifting flux through each condition's outer state
        "ns_2d_subsonic": (2, dict(bdr=[(0, 1), (2, 2)], boundaries={
            0: (pb.BC_SUBSONIC_INFLOW_RV, [1.3, 0.2, 0.05]), 1: (pb.BC_SUBSONIC_OUTFLOW_P, [2.2]),
            2: (NOSLIP, [0.0, 0.0])})),
        "ns_3d_subsonic": (3, dict(bdr=[(0, 1), (2, 2), None], boundaries={
            0: (pb.BC_SUBSONIC_INFLOW_RV, [1.2, 0.1, 0.05, -0.02]), 1: (pb.BC_SUBSONIC_OUTFLOW_P, [2.0]),
            2: (NOSLIP, [0.0, 0.0, 0.0])})),
        # total-pressure inflow: the outer state's viscous flux with the
        # interior gradients (2D)
        "ns_2d_pttt": (2, dict(bdr=[(0, 1), (2, 2)], boundaries={
            0: (pb.BC_SUBSONIC_INFLOW_PTTT, [3.5, 3.0, 2.0, 10.0, 0.0]), 1: (pb.BC_SUBSONIC_OUTFLOW_P, [2.2]),
            2: (NOSLIP, [0.0, 0.0])})),
        # Riemann invariants: fixed operator only (the reference's lifting
        # flux reads the normal left by the last face evaluation)
        "ns_2d_riemann": (2, dict(bdr=[(0, 0), (1, 1)], boundaries={
            0: (pb.BC_RIEMANN_INVARIANT, [1.0, 0.3, -0.1, 2.0]), 1: (NOSLIP, [0.2, 0.0])})),
    }


NS_PINNED = ["ns_2d_channel", "ns_2d_cavity", "ns_2d_isothermal", "ns_3d_channel", "ns_2d_subsonic",
             "ns_3d_subsonic", "ns_2d_pttt"]


def ns_layout_case(name, order):
    dim, kw = ns_layouts()[name]
    if dim == 2:
        mesh = box(2, order, (4, 3), (-1.0, -1.0), (1.0, 1.0), **kw)
        u = cases.kelvin_helmholtz(periodic_box(2, order, (4, 3), -1.0, 1.0))
    else:
        mesh = box(3, order, (3, 2, 3), 0.0, 2 * np.pi, **kw)
        u = cases.taylor_green(periodic_box(3, order, (3, 2, 3), 0.0, 2 * np.pi), Ma=0.4)
    return mesh, rough(u, mesh, 21, 0.05, 0.02)


NS_KW = dict(parabolic=1, mu=0.02, Pr=0.71)


@pytest.mark.skipif(not oracle.ref_available(True), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("name", NS_PINNED)
def test_oracle_ns_boundaries_match_live_reference(name, order):
    """BR1 boundary lifting and viscous boundary fluxes against the
    reference's own boundary integrators and LiftingBR1."""
    mesh, u = ns_layout_case(name, order)
    o = oracle.Oracle(mesh, compat=1, **NS_KW)
    r = oracle.Reference(mesh, parabolic=True, mu=NS_KW["mu"], Pr=NS_KW["Pr"])
    ro, rr = o.rhs(u), r.rhs(u)
    assert np.abs(ro - rr).max() <= 1e-12 * np.abs(rr).max()
    go, gr = o.gradients(), r.gradients()
    assert np.abs(go - gr).max() <= 1e-11 * np.abs(gr).max()


def test_case_builders():
    """The forward-facing step and lid-driven cavity builders: cell masks and
    conditions as documented; the step's walls get the slip condition."""
    m, u = cases.forward_facing_step(2, 5)
    assert m.num_elements == 15 * 5 - 12 * 1 and u.size == m.size
    assert set(m.boundaries) == {0, 1, 2} and m.boundaries[2][0] == pb.BC_SLIP_WALL
    assert (m.nbr == -3).sum() == 12 + 15 + 3 + 1   # top, bottom before the step, step front and top
    mc, uc = cases.lid_driven_cavity(4, 2)
    assert mc.boundaries[1] == (pb.BC_NOSLIP_ADIABATIC, [1.0, 0.0]) and uc.size == mc.size
