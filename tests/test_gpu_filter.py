"""Entropy filter after RK stages on the GPU against the oracle's filter.

The filter (EntropyFilter.cpp intent: element bound = min entropy over the
element and its face neighbours at the stage input; modal damping exp(-zeta
j^2) with zeta from 20-step bisections in node order) is exercised on states
where it fires: the Kelvin-Helmholtz shear layer and roughened states at CFL
0.5-2.  Tolerance 1e-12 relative in max norm, as for the right-hand side, and
the same number of filtered elements.
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import rel_maxnorm, rough

TOL = 1e-12
pytestmark = pytest.mark.gpu


def _case(kind, order):
    if kind == "kh":
        m = periodic_box(2, order, (8, 9), -1.0, 1.0)
        return m, cases.kelvin_helmholtz(m), dict(parabolic=0)
    if kind == "rough2d":
        m = periodic_box(2, order, (8, 9), -1.0, 1.0)
        return m, rough(cases.kelvin_helmholtz(m), m, 3), dict(parabolic=0)
    m = periodic_box(3, order, (4, 3, 5), 0.0, 2 * np.pi)
    par = dict(parabolic=1, mu=0.01, Pr=0.71) if kind == "rough3dns" else dict(parabolic=0)
    return m, rough(cases.taylor_green(m), m, 5), par


def _dt(mesh, u, order, cfl, par):
    o = oracle.Oracle(mesh, **par)
    o.rhs(u)
    return cfl * min(mesh.h) / (o.max_char_speed() * (order + 1) ** 2)


@pytest.mark.parametrize("compat", [1, 0])
@pytest.mark.parametrize("kind,order,cfl", [("kh", 3, 0.5), ("kh", 4, 0.5), ("kh", 4, 2.0), ("rough2d", 3, 2.0),
                                            ("rough2d", 5, 2.0), ("rough3d", 3, 2.0), ("rough3d", 2, 5.0),
                                            ("rough3dns", 3, 2.0)])
def test_filtered_stage_matches_oracle(kind, order, cfl, compat, cuda_device):
    import torch
    mesh, u, par = _case(kind, order)
    dt = _dt(mesh, u, order, cfl, par)
    orc = oracle.Oracle(mesh, filter=1, compat=compat, **par)
    op = pb.DGSEMOperator(mesh, filter=1, compat=compat, **par)
    ud_n = torch.from_numpy(u).to(cuda_device)
    us = u
    for stage in (0, 1, 2):  # the stages of one step, each from the oracle's previous stage
        want = orc.rk_stage(stage, dt, u, us)
        out = torch.empty_like(ud_n)
        op.rk_stage(stage, dt, ud_n, torch.from_numpy(us).to(cuda_device), out)
        got = out.cpu().numpy()
        assert rel_maxnorm(got, want) < TOL, f"stage {stage}"
        assert op.filter_count() == orc.filtered_elements()
        us = want
    assert orc.filtered_elements() > 0, "the case must exercise the filter"
    assert op.check() == 0


def test_filtered_trajectory_matches_oracle(cuda_device):
    """Kelvin-Helmholtz, N=4, ten filtered SSP-RK3 steps."""
    import torch
    mesh, u, par = _case("kh", 4)
    dt = _dt(mesh, u, 4, 0.5, par)
    orc = oracle.Oracle(mesh, filter=1, **par)
    op = pb.DGSEMOperator(mesh, filter=1, **par)
    x = torch.from_numpy(u).to(cuda_device)
    y = u.copy()
    for step in range(10):
        op.rk3_step(x, dt)
        y = orc.rk3_step(y, dt)
        assert rel_maxnorm(x.cpu().numpy(), y) < 1e-11, f"step {step}"
    assert op.filter_count() == orc.filtered_elements() > 0
    assert op.check() == 0


def test_filter_off_is_plain_stage(cuda_device):
    """filter=0 leaves the stage untouched even where the filter would fire."""
    import torch
    mesh, u, par = _case("kh", 3)
    dt = _dt(mesh, u, 3, 0.5, par)
    op0 = pb.DGSEMOperator(mesh, filter=0, **par)
    orc = oracle.Oracle(mesh, filter=0, **par)
    ud = torch.from_numpy(u).to(cuda_device)
    out = torch.empty_like(ud)
    op0.rk_stage(0, dt, ud, ud, out)
    assert rel_maxnorm(out.cpu().numpy(), orc.rk_stage(0, dt, u, u)) < TOL
    assert op0.filter_count() == 0
