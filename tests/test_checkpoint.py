"""Checkpoint / restart in the reference's layout (Simulation.cpp:350-388,
1084-1116): file names, MFEM grid-function text, meta JSON, and that a run
restarted from a checkpoint continues bit for bit."""
import io
import json
import os

import numpy as np
import pytest

import oracle
from prandtl_b200 import cases, checkpoint
from prandtl_b200.mesh import periodic_box


def test_paths_follow_reference_names(tmp_path):
    chk, meta = checkpoint.paths(str(tmp_path), 200, rank=3)
    assert chk == os.path.join(str(tmp_path), "Cycle200", "checkpoint_cycle_200.00000003.chk")
    assert meta == os.path.join(str(tmp_path), "Cycle200", "checkpoint_cycle_200.json")


def test_round_trip_is_exact(tmp_path):
    mesh = periodic_box(3, 3, (2, 3, 2), 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh)
    chk = checkpoint.save(str(tmp_path), 7, 0.123456789012345, u, 3, 3)
    with open(chk) as f:
        head = [f.readline() for _ in range(5)]
    assert head == ["FiniteElementSpace\n", "FiniteElementCollection: L2_T1_3D_P3\n", "VDim: 5\n",
                    "Ordering: 0\n", "\n"]
    meta = json.load(open(checkpoint.paths(str(tmp_path), 7)[1]))
    assert meta == {"time": 0.123456789012345, "cycle": 7}
    ck = checkpoint.load(str(tmp_path), 7)
    assert (ck.dim, ck.order, ck.cycle, ck.time) == (3, 3, 7, 0.123456789012345)
    assert np.array_equal(ck.u, u)


def test_reads_reference_written_text():
    """A file as the reference writes it: default stream precision (six
    significant digits), one value per line."""
    mesh = periodic_box(2, 1, (2, 1), -1.0, 1.0)
    u = cases.isentropic_vortex(mesh)
    text = ("FiniteElementSpace\nFiniteElementCollection: L2_T1_2D_P1\nVDim: 4\nOrdering: 0\n\n"
            + "".join("%g\n" % x for x in u))
    dim, order, got = checkpoint.read_gridfunction(io.StringIO(text))
    assert (dim, order) == (2, 1)
    np.testing.assert_allclose(got, u, rtol=5e-6, atol=0)


def test_byvdim_file_is_reordered():
    u = cases.kelvin_helmholtz(periodic_box(2, 2, (2, 2), -1.0, 1.0))
    inter = u.reshape(4, -1).T.reshape(-1)   # variables interleaved per node
    text = ("FiniteElementSpace\nFiniteElementCollection: L2_T1_2D_P2\nVDim: 4\nOrdering: 1\n\n"
            + "\n".join(repr(float(x)) for x in inter) + "\n")
    _, _, got = checkpoint.read_gridfunction(io.StringIO(text))
    assert np.array_equal(got, u)


@pytest.mark.parametrize("head,why", [
    ("FiniteElementCollection: L2_3D_P3\nVDim: 5\nOrdering: 0\n", "Gauss-Lobatto"),
    ("FiniteElementCollection: L2_T1_3D_P3\nVDim: 4\nOrdering: 0\n", "VDim"),
    ("FiniteElementCollection: H1_3D_P3\nVDim: 5\nOrdering: 0\n", "element collection"),
])
def test_rejects_other_spaces(head, why):
    text = "FiniteElementSpace\n" + head + "\n" + "1.0\n" * (5 * 64)
    with pytest.raises(ValueError, match=why):
        checkpoint.read_gridfunction(io.StringIO(text))


def test_rejects_partial_elements_and_cycle_mismatch(tmp_path):
    text = "FiniteElementSpace\nFiniteElementCollection: L2_T1_2D_P1\nVDim: 4\nOrdering: 0\n\n" + "1.0\n" * 15
    with pytest.raises(ValueError, match="whole elements"):
        checkpoint.read_gridfunction(io.StringIO(text))
    mesh = periodic_box(2, 1, (2, 2), 0.0, 1.0)
    checkpoint.save(str(tmp_path), 3, 0.5, cases.isentropic_vortex(mesh), 2, 1)
    meta = checkpoint.paths(str(tmp_path), 3)[1]
    with open(meta, "w") as f:
        f.write('{"time": 0.5, "cycle": 4}\n')
    with pytest.raises(ValueError, match="cycle 4"):
        checkpoint.load(str(tmp_path), 3)
    with pytest.raises(ValueError, match="cycle > 0"):
        checkpoint.load(str(tmp_path), 0)


def test_restart_continues_bit_for_bit(tmp_path):
    """Two SSP-RK3 steps equal one step, a checkpoint, a restart and one step
    (the oracle as the stepper)."""
    mesh = cases.vortex_mesh(4, 3)
    u0 = cases.isentropic_vortex(mesh)
    orc = oracle.Oracle(mesh, compat=0)
    orc.rhs(u0)
    dt = 0.5 * min(mesh.h) / (orc.max_char_speed() * 16)
    u2 = orc.rk3_step(orc.rk3_step(u0, dt), dt)
    u1 = orc.rk3_step(u0, dt)
    checkpoint.save(str(tmp_path), 1, dt, u1, mesh.dim, mesh.order)
    ck = checkpoint.load(str(tmp_path), 1)
    assert ck.time == dt
    assert np.array_equal(orc.rk3_step(ck.u, dt), u2)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["vortex_euler", "tgv_ns"])
def test_gpu_restart_continues_bit_for_bit(case, tmp_path, cuda_device):
    """On the CUDA operator: three steps, a checkpoint, a restart in a fresh
    operator and three more steps equal six uninterrupted steps bit for bit
    (the checkpoint writes 17 significant digits, an exact round trip).  Both
    runs use the same fixed dt, taken from the initial state."""
    import torch

    import prandtl_b200 as pb
    if case == "vortex_euler":
        mesh = cases.vortex_mesh(16, 3)
        u0 = cases.isentropic_vortex(mesh)
        par = dict(parabolic=0, compat=0)
    else:
        mesh = cases.tgv_mesh(8, 3)
        u0 = cases.taylor_green(mesh)
        par = dict(parabolic=1, mu=1.0 / 1600.0, Pr=0.71, compat=0)
    op = pb.DGSEMOperator(mesh, **par)
    x = torch.from_numpy(u0).to(cuda_device)
    op.Mult(x, torch.empty_like(x))
    dt = op.cfl_dt(0.5)
    ref = x.clone()
    op.rk3_step(ref, dt, nsteps=6)
    op.rk3_step(x, dt, nsteps=3)
    checkpoint.save(str(tmp_path), 3, 3 * dt, x, mesh.dim, mesh.order)
    op.close()
    ck = checkpoint.load(str(tmp_path), 3)
    assert ck.cycle == 3 and ck.time == 3 * dt and (ck.dim, ck.order) == (mesh.dim, mesh.order)
    op2 = pb.DGSEMOperator(mesh, **par)
    y = torch.from_numpy(ck.u).to(cuda_device)
    op2.rk3_step(y, dt, nsteps=3)
    assert torch.equal(y, ref)
    assert op2.check() == 0


def test_restart_on_a_general_mesh_in_reference_order(tmp_path):
    """The 15-degree ramp as read from the reference's file (general
    geometry; its fixture), saved in the reference's per-element node order
    and restarted: two steps equal one step, save, load, one step."""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from test_meshio import fixture_mesh
    from prandtl_b200 import meshio
    m = fixture_mesh("ramp", 2)
    free = [1.4, 4.2, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 9.0]
    kinds = {"inlet": 1, "outlet": 2}
    m.boundaries = {b: ((1, free) if kinds.get(nm) == 1 else (kinds.get(nm, 4), None))
                    for nm, b in m.boundary_names.items()}
    u0 = np.repeat(np.array(free), m.num_nodes)
    x = m.node_coords()
    u0[:m.num_nodes] *= 1 + 0.05 * np.sin(3 * x[0]) * np.cos(2 * x[1])
    orc = oracle.Oracle(m, compat=0, parabolic=0)
    orc.rhs(u0)
    dt = 0.3 * min(m.h) / (orc.max_char_speed() * 9)
    u1 = orc.rk3_step(u0, dt)
    u2 = orc.rk3_step(u1, dt)
    checkpoint.save(str(tmp_path), 1, dt, meshio.to_reference_order(m, u1), m.dim, m.order)
    ck = checkpoint.load(str(tmp_path), 1)
    assert np.array_equal(orc.rk3_step(meshio.from_reference_order(m, ck.u), dt), u2)
