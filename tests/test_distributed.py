"""Slab decomposition with ghost-layer exchange, run as world-size 2 and 3
process groups on the CPU (gloo).  Each rank advances its slab with the
oracle standing in for the GPU stage kernel; its owned elements must equal
the undivided mesh's trajectory exactly (the local numbering keeps the global
face orientation)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from prandtl_b200 import cases
from prandtl_b200.distributed import DistributedRK3, SlabDecomposition

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


class OracleStages:
    """rk_stage(stage, dt, un, us, uout) of the oracle on CPU tensors."""

    def __init__(self, mesh, **params):
        import oracle
        self.o = oracle.Oracle(mesh, **params)

    def rk_stage(self, stage, dt, un, us, uout):
        uout.copy_(torch.from_numpy(self.o.rk_stage(stage, dt, un.numpy(), us.numpy())))


CASES = {
    "ns3d": dict(dim=3, order=2, n=(3, 2, 6), lo=0.0, hi=2 * np.pi, params=dict(parabolic=1, mu=0.02, Pr=0.71)),
    "euler2d": dict(dim=2, order=3, n=(4, 5), lo=-1.0, hi=1.0, params=dict(parabolic=0)),
    # two layers on two ranks: each rank's two ghost layers are the same layer
    "euler2d_thin": dict(dim=2, order=2, n=(4, 2), lo=-1.0, hi=1.0, params=dict(parabolic=0)),
    # boundary faces across the slab axis: a Navier-Stokes channel (specified
    # state in, outflow out) and Euler slip / symmetry walls
    "ns2d_channel": dict(dim=2, order=2, n=(4, 6), lo=-1.0, hi=1.0, params=dict(parabolic=1, mu=0.02, Pr=0.71),
                         bdr=[(0, 1), None], boundaries={0: (3, [1.2, 0.3, -0.2, 2.6]), 1: (2, None)}),
    "euler3d_walls": dict(dim=3, order=2, n=(3, 2, 6), lo=0.0, hi=2 * np.pi, params=dict(parabolic=0),
                          bdr=[(0, 0), (1, 1), None], boundaries={0: (4, None), 1: (5, None)}),
}


def initial(case):
    c = CASES[case]
    from prandtl_b200.mesh import box
    m = box(c["dim"], c["order"], c["n"], c["lo"], c["hi"], bdr=c.get("bdr"), boundaries=c.get("boundaries"))
    u = cases.taylor_green(m) if c["dim"] == 3 else cases.kelvin_helmholtz(m)
    rng = np.random.default_rng(7)
    u[: m.num_nodes] *= 1 + 0.05 * rng.standard_normal(m.num_nodes)
    return m, u


def _worker(rank, world, port, case, compat, q):
    import torch.distributed as dist
    os.environ["OMP_NUM_THREADS"] = "1"
    import sys
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        c = CASES[case]
        gm, u0 = initial(case)
        dec = SlabDecomposition(c["dim"], c["order"], c["n"], c["lo"], c["hi"], world, rank,
                                bdr=c.get("bdr"), boundaries=c.get("boundaries"))
        op = OracleStages(dec.mesh, compat=compat, **c["params"])
        drv = DistributedRK3(dec, op)
        x = torch.from_numpy(dec.scatter(u0))
        dt = 2e-3
        for _ in range(3):
            drv.step(x, dt)
        # the undivided mesh, same steps
        import oracle
        ref = oracle.Oracle(gm, compat=compat, **c["params"])
        y = u0.copy()
        for _ in range(3):
            y = ref.rk3_step(y, dt)
        want = y.reshape(gm.nv, gm.num_elements, gm.ndof)[:, dec.owned_global_elements(), :]
        got = dec.owned(x.numpy())
        err = float(np.abs(got - want).max() / np.abs(want).max())
        lam = drv.max_char_speed(float(rank + 1))
        q.put((rank, err, lam))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world,case,compat", [(2, "ns3d", 1), (2, "ns3d", 0), (2, "euler2d", 1), (3, "ns3d", 1),
                                               (3, "ns3d", 0), (3, "euler2d", 1), (2, "euler2d_thin", 1),
                                               (2, "ns2d_channel", 0), (3, "ns2d_channel", 1), (2, "euler3d_walls", 1),
                                               (3, "euler3d_walls", 0)])
def test_slab_decomposition_matches_undivided(world, case, compat):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, compat, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err, lam in res:
        assert err == 0.0, f"rank {rank}: {err}"
        assert lam == float(world)


def test_decomposition_layout():
    for world in (1, 2, 3, 6):
        owned = []
        for r in range(world):
            d = SlabDecomposition(3, 2, (3, 2, 6), 0.0, 1.0, world, r)
            owned.extend(d.owned_global_elements().tolist())
            # local order keeps the global order
            assert np.all(np.diff(d.global_elements) > 0)
            assert d.mesh.nbr.min() >= 0 and d.mesh.nbr.max() < d.mesh.num_elements
        assert sorted(owned) == list(range(3 * 2 * 6))


def _trace_worker(rank, world, port, dim, q):
    """Face-trace halo plumbing on CPU tensors: ghost face nodes and ghost
    face-column slots, zeroed first, must receive their owners' values."""
    import torch.distributed as dist
    os.environ["OMP_NUM_THREADS"] = "1"
    import sys
    sys.path.insert(0, ROOT)
    from prandtl_b200.distributed import FaceTraceHalo
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        n = (3, 2, 2 * world + 2) if dim == 3 else (4, 2 * world + 1)
        dec = SlabDecomposition(dim, 2, n, 0.0, 1.0, world, rank)
        g = dec.glob
        u0 = np.arange(g.size, dtype=np.float64) * 1e-3 + 1.0
        x = torch.from_numpy(dec.scatter(u0))
        h = FaceTraceHalo(dec)
        X = x.view(g.nv, -1, g.ndof)
        for pos in (dec.ghost_lo_pos, dec.ghost_hi_pos):
            a, b = h.layer(pos)
            X[:, a:b] = 0.0
        # face columns: owned slots hold a function of the global element
        ne, fn = dec.mesh.num_elements, g.Np ** (dim - 1)
        ge = torch.from_numpy(dec.global_elements.astype(np.float64))
        cols = torch.zeros((dim, 2, ne, fn, dim + 1), dtype=torch.float64)
        own = slice(*h.layer(h.bottom)[:1], h.layer(h.top)[1])
        val = (ge[:, None, None] * 1000 + torch.arange(fn, dtype=torch.float64)[None, :, None] * 10 +
               torch.arange(dim + 1, dtype=torch.float64)[None, None, :])
        for d in range(dim):
            for side in range(2):
                cols[d, side, own] = val[own] + 0.5 * side + 0.25 * d
        sends, recvs = h.trace_sends(x), h.trace_recv_buffers(x)
        for r in h.post(sends[0], sends[1], recvs[0], recvs[1]):
            r.wait()
        h.trace_unpack(x, *recvs)
        cs, cr = h.column_sends(cols), h.column_recvs(cols)
        for r in h.post(cs[0], cs[1], cr[0], cr[1]):
            r.wait()
        U = u0.reshape(g.nv, g.num_elements, g.ndof)
        err = 0.0
        for pos, high in ((dec.ghost_lo_pos, True), (dec.ghost_hi_pos, False)):
            a, b = h.layer(pos)
            gl = dec.global_elements[a:b]
            want = U[:, gl, g.ndof - fn:] if high else U[:, gl, :fn]
            got = X[:, a:b, g.ndof - fn:] if high else X[:, a:b, :fn]
            err = max(err, float(np.abs(got.numpy() - want).max()))
            side = 1 if high else 0
            wc = val[a:b] + 0.5 * side + 0.25 * (dim - 1)
            err = max(err, float((cols[dim - 1, side, a:b] - wc).abs().max()))
        q.put((rank, err))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dim", [(2, 3), (3, 3), (2, 2), (4, 2)])
def test_face_trace_halo_delivers_owner_values(world, dim):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_trace_worker, args=(r, world, port, dim, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err in res:
        assert err == 0.0, f"rank {rank}: {err}"


def test_face_trace_halo_bytes():
    """Per stage and rank: face traces + face columns against whole ghost layers."""
    from prandtl_b200.distributed import FaceTraceHalo
    dec = SlabDecomposition(3, 3, (32, 32, 64), 0.0, 1.0, 2, 0)
    h = FaceTraceHalo(dec)
    g = dec.glob
    trace = 2 * h.ls * h.fn * (g.nv + g.nv - 1) * 8
    layers = 2 * h.ls * g.ndof * g.nv * 8
    assert trace == 2 * 1024 * 16 * 9 * 8 and layers == 2 * 1024 * 64 * 5 * 8
    assert layers / trace > 2.2


# ---- element partitions of general meshes (ElementPartition) ----

def general_case(case):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import geometry_case, ns_geometry_case, smooth_state
    name, par = {"perturbed2d": ("perturbed2d", dict(parabolic=0)),
                 "rotated2d": ("rotated2d", dict(parabolic=0, filter=3)),
                 "boundary3d": ("boundary3d", dict(parabolic=0)),
                 "warped3d_ns": ("warped3d", dict(parabolic=1, mu=0.02, Pr=0.71)),
                 "walls2d_ns": ("walls2d_ns", dict(parabolic=1, mu=0.02, Pr=0.71))}[case]
    m = ns_geometry_case(name) if name.endswith("_ns") else geometry_case(name)
    return m, smooth_state(m, 13), par


def _pworker(rank, world, port, case, compat, q):
    import torch.distributed as dist
    os.environ["OMP_NUM_THREADS"] = "1"
    import sys
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        from prandtl_b200.distributed import ElementPartition
        gm, u0, par = general_case(case)
        rng = np.random.default_rng(3)
        part = rng.integers(0, world, gm.num_elements)   # scattered, not contiguous
        dec = ElementPartition(gm, world, rank, layers=2 if par.get("parabolic") else 1, part=part)
        op = OracleStages(dec.mesh, compat=compat, **par)
        drv = DistributedRK3(dec, op)
        x = torch.from_numpy(dec.scatter(u0))
        dt = 2e-3
        for _ in range(2):
            drv.step(x, dt)
        import oracle
        ref = oracle.Oracle(gm, compat=compat, **par)
        y = u0.copy()
        for _ in range(2):
            y = ref.rk3_step(y, dt)
        want = y.reshape(gm.nv, gm.num_elements, gm.ndof)[:, dec.owned_global_elements(), :]
        got = dec.owned(x.numpy())
        err = float(np.abs(got - want).max() / np.abs(want).max())
        q.put((rank, err, dec.owned_local.size))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,case,compat", [(2, "perturbed2d", 1), (3, "perturbed2d", 0), (3, "rotated2d", 0),
                                               (2, "boundary3d", 1), (2, "warped3d_ns", 0), (3, "walls2d_ns", 1)])
def test_element_partition_matches_undivided(world, case, compat):
    """A general mesh split over 2-3 gloo ranks by a scattered element
    partition (one ghost layer for Euler, two for Navier-Stokes), the oracle
    as each rank's stage: owned elements equal the undivided mesh's SSP-RK3
    steps bit for bit (filter and limiter included in one case)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_pworker, args=(r, world, port, case, compat, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sum(n for _, _, n in res) == general_case(case)[0].num_elements
    for rank, err, _ in res:
        assert err == 0.0, f"rank {rank}: {err}"
