"""Slab decomposition of a Cartesian mesh (periodic along its last axis,
optionally with boundary faces on the others) over ranks, with a ghost layer
exchange per RK stage.

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


class DistributedRK3:
    """SSP-RK3 on a slab decomposition: exchange, then one fused stage of the
    rank's operator (``op.rk_stage(stage, dt, un, us, uout)``) per stage."""

    def __init__(self, dec: SlabDecomposition, op, group=None):
        self.dec, self.op = dec, op
        self.xchg = GhostExchange(dec, group)
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
