"""The face-trace halo driver (TraceHaloRK3) on the GPU, with its ranks
emulated in one process on one GPU.

Each emulated rank has its slab's operator and local state.  The driver's
stage generator yields at every exchange point; the emulation advances all
ranks to the same point, then delivers each message by a device copy from
the sending rank's buffer to the receiving rank's (what the point-to-point
messages do between GPUs), and resumes them.  No kernel waits on another
rank's kernel: the ranks' launches simply follow one another on one stream.
Owned elements must equal the undivided mesh's SSP-RK3 steps bit for bit:
per element the arithmetic is the single-GPU kernels', and every value an
owned element reads — ghost face traces, ghost face columns — is the owner's.
"""
import numpy as np
import pytest

import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.distributed import SlabDecomposition, TraceHaloRK3

from helpers import rough

pytestmark = pytest.mark.gpu


def _emulated_stage(drivers, stage, dt, uns, uss, outs):
    world = len(drivers)
    gens = [d.stage_parts(stage, dt, un, us, out) for d, un, us, out in zip(drivers, uns, uss, outs)]
    while True:
        msgs = [next(g, None) for g in gens]
        if all(m is None for m in msgs):
            return
        assert all(m is not None and m[0] == msgs[0][0] for m in msgs)
        if msgs[0][0] == "wait":
            continue
        for r in range(world):
            prev, nxt = (r - 1) % world, (r + 1) % world
            from_next, from_prev = msgs[r][2]
            from_next.copy_(msgs[nxt][1][0])   # the next rank's message to its prev
            from_prev.copy_(msgs[prev][1][1])  # the previous rank's message to its next


@pytest.mark.parametrize("world,kind,compat", [(2, "tgv_ns", 0), (3, "tgv_ns", 0), (4, "tgv_ns", 0), (2, "tgv_euler", 0),
                                               (3, "kh_euler", 0), (2, "kh_ns", 0)])
def test_trace_halo_matches_undivided(world, kind, compat, cuda_device):
    import torch
    if kind.startswith("tgv"):
        dim, order, n, lo, hi = 3, 3, (4, 3, 4 * world), 0.0, 2 * np.pi
    else:
        dim, order, n, lo, hi = 2, 4, (5, 3 * world + 1), -1.0, 1.0
    par = dict(parabolic=1, mu=0.01, Pr=0.71) if kind.endswith("ns") else dict(parabolic=0)
    decs = [SlabDecomposition(dim, order, n, lo, hi, world, r) for r in range(world)]
    g = decs[0].glob
    u0 = cases.taylor_green(g) if dim == 3 else cases.kelvin_helmholtz(g)
    u0 = rough(u0, g, 5, 0.05, 0.01)
    op_g = pb.DGSEMOperator(g, compat=compat, **par)
    xg = torch.from_numpy(u0).to(cuda_device)
    op_g.Mult(xg, torch.empty_like(xg))
    dt = op_g.cfl_dt(0.5)
    ops = [pb.DGSEMOperator(d.mesh, compat=compat, **par) for d in decs]
    drivers = [TraceHaloRK3(d, op) for d, op in zip(decs, ops)]
    xs = [torch.from_numpy(d.scatter(u0)).to(cuda_device) for d in decs]
    for x, d in zip(xs, decs):  # ghost layers: a fluid at rest, then only what the exchange brings
        X = x.view(g.nv, -1, g.ndof)
        for pos in (d.ghost_lo_pos, d.ghost_hi_pos):
            sl = slice(pos * d.layer_size, (pos + 1) * d.layer_size)
            X[:, sl] = 0.0
            X[0, sl] = 1.0
            X[-1, sl] = 2.5
    As = [x.clone() for x in xs]
    Bs = [x.clone() for x in xs]
    for _ in range(2):
        _emulated_stage(drivers, 0, dt, xs, xs, As)
        _emulated_stage(drivers, 1, dt, xs, As, Bs)
        _emulated_stage(drivers, 2, dt, xs, Bs, xs)
    op_g.rk3_step(xg, dt, nsteps=2)
    want = xg.cpu().numpy().reshape(g.nv, g.num_elements, g.ndof)
    for d, x in zip(decs, xs):
        got = d.owned(x.cpu().numpy())
        assert np.array_equal(got, want[:, d.owned_global_elements(), :]), f"rank {d.rank}"
    for op in ops:
        assert op.check() == 0


@pytest.mark.parametrize("world,name,ns", [(2, "rotated2d", False), (3, "perturbed3d", False), (3, "warped3d", True)])
def test_element_partition_matches_undivided(world, name, ns, cuda_device):
    """General meshes split by a scattered element partition (ElementPartition:
    one ghost layer for Euler, two for Navier-Stokes), ranks emulated in one
    process: before each stage every rank's ghost elements are filled from
    their owners' tensors by device copies, then each rank's operator runs
    its stage.  Owned elements equal the undivided mesh's graph-free steps
    bit for bit."""
    import torch
    from helpers import geometry_case, smooth_state
    from prandtl_b200.distributed import ElementPartition
    g = geometry_case(name)
    par = dict(parabolic=1, mu=0.01, Pr=0.71) if ns else dict(parabolic=0)
    u0 = smooth_state(g, 17)
    part = np.random.default_rng(4).integers(0, world, g.num_elements)
    decs = [ElementPartition(g, world, r, layers=2 if ns else 1, part=part) for r in range(world)]
    ops = [pb.DGSEMOperator(d.mesh, compat=0, **par) for d in decs]
    xs = [torch.from_numpy(d.scatter(u0)).to(cuda_device) for d in decs]
    op_g = pb.DGSEMOperator(g, compat=0, **par)
    xg = torch.from_numpy(u0).to(cuda_device)
    op_g.Mult(xg, torch.empty_like(xg))
    dt = op_g.cfl_dt(0.3)

    def exchange(us):
        views = [u.view(g.nv, d.local.size, g.ndof) for u, d in zip(us, decs)]
        for r, d in enumerate(decs):
            for q, ridx in d.recv_idx.items():
                sidx = decs[q].send_idx[r]
                views[r][:, torch.as_tensor(ridx, device=cuda_device)] = \
                    views[q][:, torch.as_tensor(sidx, device=cuda_device)]

    As = [x.clone() for x in xs]
    Bs = [x.clone() for x in xs]
    for _ in range(2):
        exchange(xs)
        for op, x, a in zip(ops, xs, As):
            op.rk_stage(0, dt, x, x, a)
        exchange(As)
        for op, x, a, b in zip(ops, xs, As, Bs):
            op.rk_stage(1, dt, x, a, b)
        exchange(Bs)
        for op, x, b in zip(ops, xs, Bs):
            op.rk_stage(2, dt, x, b, x)
    ya, yb = xg.clone(), xg.clone()
    for _ in range(2):
        op_g.rk_stage(0, dt, xg, xg, ya)
        op_g.rk_stage(1, dt, xg, ya, yb)
        op_g.rk_stage(2, dt, xg, yb, xg)
    want = xg.cpu().numpy().reshape(g.nv, g.num_elements, g.ndof)
    for d, x in zip(decs, xs):
        assert np.array_equal(d.owned(x.cpu().numpy()), want[:, d.owned_global_elements(), :]), f"rank {d.rank}"
