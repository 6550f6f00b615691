"""Slab decomposition of a Cartesian mesh (periodic along its last axis,
optionally with boundary faces on the others) over ranks, with a ghost layer
exchange per RK stage; element partitions of meshes of general geometry
(``ElementPartition``, whole ghost elements exchanged per stage).

The reference partitions elements over MPI ranks and exchanges face-neighbour
data once per right-hand-side pass (``ExchangeFaceNbrData``,
src/Operators/NonlinearForm/DGSEMNonlinearForm.cpp:748; Navier-Stokes also
for the gradients, :533, :1426-1429), with an ``MPI_Allreduce`` of the wave
speed for dt (src/Simulation/Simulation.cpp:905, 1016).  Here each rank owns
a slab of element layers along the last axis and holds one ghost layer on
each side.  Before every stage the ghost layers' states are received from the
owning ranks (``torch.distributed`` point-to-point: NCCL over NVLink on GPUs,
gloo in the CPU tests); the stage then runs on owned + ghost elements with
the unchanged single-GPU kernels.  Owned results are exact: a face between an
owned and a ghost element sees both states, and for Navier-Stokes the ghost's
gradients on that face depend only on the ghost layer itself (its far face,
whose neighbour is not held, only touches nodes on that far face).  Ghost
outputs are discarded and refreshed by the next exchange.

Local element order keeps the global order (layers sorted by global index),
so the face rule "element 1 = the lower-numbered element" gives the same
orientation as on the undivided mesh, and owned values equal the single-rank
ones.
"""
from __future__ import annotations

import numpy as np

from .mesh import CartesianMesh, box


class SlabDecomposition:
    """Rank `rank`'s share of box(dim, order, n, lo, hi, bdr, boundaries)
    split into `world` slabs of element layers along the last axis, which
    stays periodic; boundary faces of the other axes keep their conditions."""

    def __init__(self, dim: int, order: int, n, lo, hi, world: int, rank: int, bdr=None, boundaries=None):
        if bdr is not None and bdr[-1] is not None:
            raise ValueError("the last axis (the slab axis) must stay periodic")
        self.glob = box(dim, order, n, lo, hi, bdr=bdr, boundaries=boundaries)
        self.dim, self.order, self.world, self.rank = dim, order, world, rank
        n = self.glob.n
        nz = n[-1]
        if world < 1 or not (0 <= rank < world) or nz < world:
            raise ValueError("need 1 <= world <= layers along the last axis and 0 <= rank < world")
        base, extra = divmod(nz, world)
        self.z0 = rank * base + min(rank, extra)
        self.z1 = self.z0 + base + (1 if rank < extra else 0)
        owned = list(range(self.z0, self.z1))
        self.lo_layer = (self.z0 - 1) % nz
        self.hi_layer = self.z1 % nz
        ghosts = [] if world == 1 else [self.lo_layer, self.hi_layer]
        self.layers = sorted(set(owned) | set(ghosts))  # global layer of each local layer
        self.layer_size = int(np.prod(n[:-1]))
        ls = self.layer_size
        pos = {g: i for i, g in enumerate(self.layers)}
        self.owned_first = pos[self.z0]
        self.owned_count = len(owned)
        self.ghost_lo_pos = pos[self.lo_layer] if world > 1 else None
        self.ghost_hi_pos = pos[self.hi_layer] if world > 1 else None
        # local neighbour table: global neighbours mapped to local indices, a
        # neighbour that is not held maps to the element itself, a boundary
        # face (negative entry) keeps its condition
        gl = np.array([g * ls + k for g in self.layers for k in range(ls)], dtype=np.int64)
        g2l = {int(g): i for i, g in enumerate(gl)}
        gn = self.glob.nbr[gl]
        ln = np.empty_like(gn)
        for i in range(gn.shape[0]):
            for f in range(gn.shape[1]):
                ln[i, f] = gn[i, f] if gn[i, f] < 0 else g2l.get(int(gn[i, f]), i)
        self.global_elements = gl
        h = self.glob.h
        nloc = tuple(n[:-1]) + (len(self.layers),)
        lo_l = tuple(self.glob.lo)
        hi_l = tuple(self.glob.lo[d] + nloc[d] * h[d] for d in range(dim))
        # the global element extents exactly (a slab's own (hi - lo) / n can
        # differ in the last bit, which would change every metric term)
        self.mesh = CartesianMesh(dim, order, nloc, lo_l, hi_l, ln.astype(np.int32), spacing=tuple(h),
                                  boundaries=dict(self.glob.boundaries or {}))

    # ---- state scatter / gather (host numpy, byNODES) ----
    def scatter(self, u_global: np.ndarray) -> np.ndarray:
        """Local state (owned + ghost elements) from a global state."""
        nv, nd = self.glob.nv, self.glob.ndof
        ug = u_global.reshape(nv, self.glob.num_elements, nd)
        return np.ascontiguousarray(ug[:, self.global_elements, :]).reshape(-1)

    def owned_slice(self) -> slice:
        ls = self.layer_size
        return slice(self.owned_first * ls, (self.owned_first + self.owned_count) * ls)

    def owned(self, u_local):
        """Owned part of a local state, as [nv, owned elements, ndof]."""
        nv, nd = self.glob.nv, self.glob.ndof
        return u_local.reshape(nv, self.mesh.num_elements, nd)[:, self.owned_slice(), :]

    def node_coords(self) -> np.ndarray:
        """Coordinates of the local nodes (ghosts at their true positions)."""
        return self.glob.node_coords(self.global_elements)

    def owned_global_elements(self) -> np.ndarray:
        return self.global_elements[self.owned_slice()]


class GhostExchange:
    """Point-to-point exchange of the ghost layers of a local state tensor.
    Ghost layers are received in place (they are contiguous per variable);
    only when a rank's two ghost layers are the same layer (two ranks, one
    layer each) does the second message land in a scratch buffer."""

    def __init__(self, dec: SlabDecomposition, group=None):
        self.dec = dec
        self.group = group
        self._scratch = None

    def _layer_views(self, u, pos):
        dec = self.dec
        nv, nd = dec.glob.nv, dec.glob.ndof
        v = u.view(nv, dec.mesh.num_elements * nd)
        a = pos * dec.layer_size * nd
        b = a + dec.layer_size * nd
        return [v[k, a:b] for k in range(nv)]

    def exchange(self, u):
        """Fills u's ghost layers from their owners (all ranks call it)."""
        import torch.distributed as dist
        dec = self.dec
        if dec.world == 1:
            return
        prev = (dec.rank - 1) % dec.world
        nxt = (dec.rank + 1) % dec.world
        first = self._layer_views(u, dec.owned_first)
        last = self._layer_views(u, dec.owned_first + dec.owned_count - 1)
        ghost_hi = self._layer_views(u, dec.ghost_hi_pos)
        if dec.ghost_lo_pos == dec.ghost_hi_pos:
            nd = dec.layer_size * dec.glob.ndof
            if self._scratch is None or self._scratch.device != u.device or self._scratch.dtype != u.dtype:
                self._scratch = u.new_empty((dec.glob.nv, nd))
            ghost_lo = [self._scratch[k] for k in range(dec.glob.nv)]
        else:
            ghost_lo = self._layer_views(u, dec.ghost_lo_pos)
        # the same order on every rank: to prev (first owned layer), to next
        # (last owned layer); from next (ghost_hi), from prev (ghost_lo)
        ops = [dist.P2POp(dist.isend, t, prev, self.group) for t in first]
        ops += [dist.P2POp(dist.isend, t, nxt, self.group) for t in last]
        ops += [dist.P2POp(dist.irecv, t, nxt, self.group) for t in ghost_hi]
        ops += [dist.P2POp(dist.irecv, t, prev, self.group) for t in ghost_lo]
        for r in dist.batch_isend_irecv(ops):
            r.wait()


class ElementPartition:
    """Rank `rank`'s share of a mesh of general geometry (or any mesh): the
    elements with part[e] == rank (default: `world` contiguous index ranges)
    plus `layers` layers of ghost elements, the owned elements' face
    neighbours (one layer for Euler; Navier-Stokes needs two, so that the
    first layer's BR1 gradients at the shared faces are exact, its own face
    neighbours being held).  The local mesh keeps the elements in global
    order (so element 1 of every face, the lower-numbered element, is the
    same as on the whole mesh), their node coordinates and face orientation
    codes; a ghost's face towards an element that is not held becomes a
    boundary face of a spare condition (supersonic outflow), whose values
    reach no owned element.  The reference partitions with METIS and
    exchanges face-neighbour data (DGSEMNonlinearForm.cpp:748); here the
    partition is given and whole ghost elements are exchanged."""

    SPARE = 15  # boundary condition index of the cut faces

    def __init__(self, mesh: CartesianMesh, world: int, rank: int, layers: int = 1, part=None):
        ne = mesh.num_elements
        if world < 1 or not (0 <= rank < world):
            raise ValueError("need 0 <= rank < world")
        self.glob, self.world, self.rank, self.layers = mesh, world, rank, int(layers)
        self.part = (np.arange(ne) * world) // ne if part is None else np.asarray(part, dtype=np.int64)
        if self.part.shape != (ne,) or self.part.min() < 0 or self.part.max() >= world:
            raise ValueError("part must give every element a rank in [0, world)")
        self.local_sets = [self._local(q) for q in range(world)]
        local = self.local_sets[rank]
        self.local = local
        g2l = np.full(ne, -1, dtype=np.int64)
        g2l[local] = np.arange(local.size)
        nbr = mesh.nbr[local].astype(np.int64)
        inner = nbr >= 0
        tgt = np.where(inner, g2l[np.where(inner, nbr, 0)], 0)
        cut = inner & (tgt < 0)
        new = np.where(inner, tgt, nbr)
        boundaries = dict(mesh.boundaries or {})
        if cut.any():
            if self.SPARE in boundaries or (mesh.nbr == -1 - self.SPARE).any():
                raise ValueError(f"boundary condition {self.SPARE} is in use; the partition needs it for cut faces")
            new[cut] = -1 - self.SPARE
            boundaries[self.SPARE] = (2, None)
        dim = mesh.dim
        fo = None
        if mesh.face_orient is not None:
            fo = np.where(cut, 0, np.asarray(mesh.face_orient)[local]).astype(np.int32)
        nl = int(local.size)
        m = CartesianMesh(dim, mesh.order, (nl,) + (1,) * (dim - 1), tuple(mesh.lo), tuple(mesh.hi),
                          new.astype(np.int32), spacing=tuple(mesh.h), boundaries=boundaries)
        if mesh.coords is not None:
            X = np.asarray(mesh.coords).reshape(dim, ne, mesh.ndof)
            m.coords = np.ascontiguousarray(X[:, local, :].reshape(dim, -1))
            m.face_orient = fo
        elif (local != np.arange(ne)).any():
            raise ValueError("a partition of a box mesh needs its node coordinates (use geometry.warped(mesh, 0.0))")
        self.mesh = m
        self.owned_local = np.nonzero(self.part[local] == rank)[0]
        # exchange lists: per peer, the local positions to send (my owned
        # elements it holds) and to receive (its owned elements I hold), both
        # in ascending global order
        self.send_idx, self.recv_idx = {}, {}
        mine = set(np.nonzero(self.part == rank)[0].tolist())
        for q in range(world):
            if q == rank:
                continue
            theirs = self.local_sets[q]
            s_glob = np.array([g for g in theirs.tolist() if g in mine], dtype=np.int64)
            r_pos = np.nonzero(self.part[local] == q)[0]
            if s_glob.size:
                self.send_idx[q] = g2l[s_glob]
            if r_pos.size:
                self.recv_idx[q] = r_pos

    def _local(self, q):
        owned = np.nonzero(self.part == q)[0]
        have = set(owned.tolist())
        frontier = owned.tolist()
        for _ in range(self.layers):
            nxt = []
            for e in frontier:
                for nb in self.glob.nbr[e]:
                    nb = int(nb)
                    if nb >= 0 and nb not in have:
                        have.add(nb)
                        nxt.append(nb)
            frontier = nxt
        return np.array(sorted(have), dtype=np.int64)

    def scatter(self, u_global: np.ndarray) -> np.ndarray:
        g = self.glob
        U = np.asarray(u_global).reshape(g.nv, g.num_elements, g.ndof)
        return np.ascontiguousarray(U[:, self.local, :].reshape(-1))

    def owned(self, u_local):
        g = self.glob
        U = np.asarray(u_local).reshape(g.nv, self.local.size, g.ndof)
        return U[:, self.owned_local, :]

    def owned_global_elements(self) -> np.ndarray:
        return self.local[self.owned_local]


class PartitionExchange:
    """Point-to-point exchange of whole ghost elements of an ElementPartition:
    per peer, the owned elements it holds are gathered into one buffer per
    message and its owned elements held here scattered from one (every rank
    posts its messages in ascending peer order)."""

    def __init__(self, part: ElementPartition, group=None):
        self.dec = part
        self.group = group

    def exchange(self, u):
        import torch.distributed as dist
        p = self.dec
        if p.world == 1:
            return
        g = p.glob
        U = u.view(g.nv, p.local.size, g.ndof)
        ops, recvs = [], []
        for q in sorted(set(p.send_idx) | set(p.recv_idx)):
            if q in p.send_idx:
                idx = _index(u, p.send_idx[q])
                ops.append(dist.P2POp(dist.isend, U[:, idx, :].contiguous(), q, self.group))
            if q in p.recv_idx:
                buf = u.new_empty((g.nv, p.recv_idx[q].size, g.ndof))
                recvs.append((q, buf))
                ops.append(dist.P2POp(dist.irecv, buf, q, self.group))
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        for q, buf in recvs:
            U[:, _index(u, p.recv_idx[q]), :] = buf


def _index(t, idx):
    import torch
    return torch.as_tensor(idx, dtype=torch.long, device=t.device)


class DistributedRK3:
    """SSP-RK3 on a slab decomposition (or an ElementPartition): exchange,
    then one fused stage of the rank's operator (``op.rk_stage(stage, dt, un,
    us, uout)``) per stage."""

    def __init__(self, dec, op, group=None):
        self.dec, self.op = dec, op
        self.xchg = PartitionExchange(dec, group) if isinstance(dec, ElementPartition) else GhostExchange(dec, group)
        self._a = self._b = None

    def step(self, x, dt: float):
        if self._a is None or self._a.shape != x.shape:
            self._a, self._b = x.clone(), x.clone()
        a, b = self._a, self._b
        self.xchg.exchange(x)
        self.op.rk_stage(0, dt, x, x, a)
        self.xchg.exchange(a)
        self.op.rk_stage(1, dt, x, a, b)
        self.xchg.exchange(b)
        self.op.rk_stage(2, dt, x, b, x)
        return x

    def max_char_speed(self, local_speed: float, device=None) -> float:
        """Global running maximum wave speed (MPI_Allreduce MAX in the reference)."""
        import torch
        import torch.distributed as dist
        t = torch.tensor([local_speed], dtype=torch.float64, device=device)
        if self.dec.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.xchg.group)
        return float(t.item())


class FaceTraceHalo:
    """Face-trace exchange of a slab decomposition for the stage-part
    driver (TraceHaloRK3).  Per stage a rank needs, of each ghost layer, only
    the face shared with its own slab: the state at the ghost's face nodes
    before the face-node kernel, and (Navier-Stokes) the ghost's viscous
    columns at those nodes after the lifting kernel.  It sends the same of
    its own first and last owned layers, the shared-face exchange of the
    reference (``ExchangeFaceNbrData``, src/Operators/NonlinearForm/
    DGSEMNonlinearForm.cpp:748; gradients :1426-1429) restricted to the face
    nodes that are read.  Face traces are gathered into contiguous buffers
    (per variable, per element, the Np^(d-1) nodes of the face are contiguous
    in the byNODES layout); face columns of a layer are contiguous already.

    Bytes per stage and rank: 2 faces x layer elements x Np^(d-1) x (nv
    traces + (nv - 1) columns) doubles, against 2 x layer elements x Np^d x nv
    for whole ghost layers (GhostExchange)."""

    def __init__(self, dec: SlabDecomposition, group=None):
        if dec.world < 2 or dec.ghost_lo_pos == dec.ghost_hi_pos or dec.owned_count < 2:
            raise ValueError("face-trace halo needs two distinct ghost layers and two owned layers per rank")
        self.dec = dec
        self.group = group
        g = dec.glob
        self.nv, self.nd, self.ls = g.nv, g.ndof, dec.layer_size
        self.fn = g.Np ** (g.dim - 1)  # nodes per face; the face of position 0 / N along the slab axis
        self.bottom = dec.owned_first
        self.top = dec.owned_first + dec.owned_count - 1
        self.prev = (dec.rank - 1) % dec.world
        self.next = (dec.rank + 1) % dec.world

    def layer(self, pos):
        """Element range of local layer position pos."""
        return pos * self.ls, (pos + 1) * self.ls

    def _face(self, u, pos, high):
        """View [nv, layer elements, face nodes] of layer pos's face at
        position N (high) or 0 along the slab axis."""
        a, b = self.layer(pos)
        v = u.view(self.nv, -1, self.nd)[:, a:b]
        return v[:, :, self.nd - self.fn:] if high else v[:, :, :self.fn]

    def trace_sends(self, us):
        """(to prev, to next): the first owned layer's low face and the last
        owned layer's high face, packed."""
        return self._face(us, self.bottom, False).contiguous(), self._face(us, self.top, True).contiguous()

    def trace_recv_buffers(self, us):
        shape = (self.nv, self.ls, self.fn)
        return us.new_empty(shape), us.new_empty(shape)  # (from next: ghost_hi's low face, from prev: ghost_lo's high face)

    def trace_unpack(self, us, from_next, from_prev):
        self._face(us, self.dec.ghost_hi_pos, False).copy_(from_next)
        self._face(us, self.dec.ghost_lo_pos, True).copy_(from_prev)

    def column_sends(self, cols):
        """(to prev, to next): the first owned layer's low-face columns and the
        last owned layer's high-face columns (cols = op.face_columns())."""
        d = self.dec.dim - 1
        a, b = self.layer(self.bottom)
        c, e = self.layer(self.top)
        return cols[d, 0, a:b], cols[d, 1, c:e]

    def column_recvs(self, cols):
        """(from next, from prev): the ghost layers' slots, received in place."""
        d = self.dec.dim - 1
        a, b = self.layer(self.dec.ghost_hi_pos)
        c, e = self.layer(self.dec.ghost_lo_pos)
        return cols[d, 0, a:b], cols[d, 1, c:e]

    def post(self, to_prev, to_next, from_next, from_prev):
        """Starts the four point-to-point messages, in the same order on every
        rank (to prev, to next; from next, from prev); returns the requests."""
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, to_prev, self.prev, self.group),
               dist.P2POp(dist.isend, to_next, self.next, self.group),
               dist.P2POp(dist.irecv, from_next, self.next, self.group),
               dist.P2POp(dist.irecv, from_prev, self.prev, self.group)]
        return dist.batch_isend_irecv(ops)


class TraceHaloRK3:
    """SSP-RK3 on a slab decomposition exchanging face traces only, with the
    elements that need no neighbour rank's data computed while the messages
    are in flight (pdg_rk_stage_part over element ranges of the local layers).

    Per stage, with b and t the first and last owned layers and gl, gh the
    ghost layers:
      post the face traces;
      face-node kernel over layers b..t-1, lifting kernel over b+1..t-1,
      volume kernel over b+2..t-2 (none of them reads a ghost);
      wait for the traces; face-node kernel over gl and t, lifting kernel over
      b and t; post the face columns (Navier-Stokes);
      volume kernel over b+1 and t-1;
      wait for the columns; volume kernel over b and t.
    The ghost layers hold state only at their shared face (their other nodes
    are never read for an owned result), so owned results equal the
    undivided mesh's bit for bit, as with whole ghost layers."""

    def __init__(self, dec: SlabDecomposition, op, group=None):
        self.dec, self.op = dec, op
        self.halo = FaceTraceHalo(dec, group)
        self.ns = bool(op.params.parabolic)
        self._a = self._b = None

    def stage_parts(self, stage: int, dt: float, un, us, out):
        """One stage as a generator: it yields ("traces", sends, recvs) and
        ("columns", sends, recvs) where the caller must deliver the messages
        (sends are (to prev, to next), recvs (from next, from prev)), and
        finishes the stage when resumed after the last one."""
        import prandtl_b200 as pb
        h, op = self.halo, self.op
        b, t = h.bottom, h.top
        ls = h.ls

        def run(part, first, last):  # layers first..last inclusive
            if last >= first:
                op.rk_stage_part(part, stage, dt, un, us, out, first * ls, (last + 1) * ls)

        op.rk_stage_part(pb.PART_START, stage, dt, un, us, out, 0, 0)
        sends = h.trace_sends(us)
        recvs = h.trace_recv_buffers(us)
        yield ("traces", sends, recvs)
        run(pb.PART_FACES, b, t - 1)
        if self.ns:
            run(pb.PART_LIFT, b + 1, t - 1)
        run(pb.PART_VOLUME, b + 2, t - 2)
        yield ("wait", None, None)
        h.trace_unpack(us, *recvs)
        run(pb.PART_FACES, self.dec.ghost_lo_pos, self.dec.ghost_lo_pos)
        run(pb.PART_FACES, t, t)
        if self.ns:
            run(pb.PART_LIFT, b, b)
            run(pb.PART_LIFT, t, t)
            cols = op.face_columns()
            yield ("columns", h.column_sends(cols), h.column_recvs(cols))
        edge = sorted({b + 1, t - 1} - {b, t})
        for layer in edge:
            if not (b + 2 <= layer <= t - 2):
                run(pb.PART_VOLUME, layer, layer)
        if self.ns:
            yield ("wait", None, None)
        run(pb.PART_VOLUME, b, b)
        if t != b:
            run(pb.PART_VOLUME, t, t)

    def _stage(self, stage, dt, un, us, out):
        pending = None
        for kind, sends, recvs in self.stage_parts(stage, dt, un, us, out):
            if kind == "wait":
                for r in pending:
                    r.wait()
                pending = None
            else:
                pending = self.halo.post(sends[0], sends[1], recvs[0], recvs[1])

    def step(self, x, dt: float):
        if self._a is None or self._a.shape != x.shape:
            self._a, self._b = x.clone(), x.clone()
        a, b = self._a, self._b
        self._stage(0, dt, x, x, a)
        self._stage(1, dt, x, a, b)
        self._stage(2, dt, x, b, x)
        return x

    def max_char_speed(self, local_speed: float, device=None) -> float:
        """Global running maximum wave speed (MPI_Allreduce MAX in the reference)."""
        import torch
        import torch.distributed as dist
        t = torch.tensor([local_speed], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.halo.group)
        return float(t.item())
