"""Cartesian meshes in the layout the C ABI expects (general geometry —
node coordinates and face orientation codes — is carried by the same class;
see ``prandtl_b200.geometry``).

The reference builds its meshes with MFEM (src/Simulation/Simulation.cpp:271-336)
and numbers DG nodes element by element, lexicographically inside an element
(x fastest), with every field stored byNODES (Simulation.hpp:64).  Here a mesh
is an axis-aligned box split into n^dim equal elements, numbered x fastest,
with a face-neighbour table nbr[e, f], f = (-x, +x, -y, +y, -z, +z), wrapping
periodically.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def gll_nodes(Np: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Lobatto nodes and weights on [0, 1] (Np points).

    Interior nodes are roots of P_N' found by Newton's method in extended
    precision; weights are 1/(N(N+1) P_N(x)^2); the rule is mirrored about 1/2.
    """
    N = Np - 1
    x = np.zeros(Np)
    w = np.zeros(Np)
    for i in range(N // 2 + 1):
        if i == 0:
            t = np.longdouble(-1.0)
        else:
            t = -np.cos(np.longdouble(np.pi) * i / N)
            for _ in range(100):
                P, dP = _legendre(N, t)
                d2P = (2 * t * dP - N * (N + 1) * P) / (1 - t * t)
                dt = dP / d2P
                t = t - dt
                if abs(dt) < 1e-30:
                    break
        P, _ = _legendre(N, t)
        x[i] = float(0.5 * (1 + t))
        w[i] = float(1 / (N * (N + 1) * P * P))
        x[N - i] = 1.0 - x[i]
        w[N - i] = w[i]
    if N % 2 == 0:
        x[N // 2] = 0.5
    return x, w


def _legendre(n, t):
    p0, p1 = np.longdouble(1), t
    if n == 0:
        return np.longdouble(1), np.longdouble(0)
    for k in range(1, n):
        p0, p1 = p1, ((2 * k + 1) * t * p1 - k * p0) / (k + 1)
    if abs(t) == 1:
        return p1, np.longdouble(0)  # derivative unused at the end points
    return p1, n * (t * p1 - p0) / (t * t - 1)


@dataclass
class CartesianMesh:
    dim: int
    order: int
    n: tuple[int, ...]          # elements per direction
    lo: tuple[float, ...]
    hi: tuple[float, ...]
    nbr: np.ndarray             # (ne, 2*dim) int32
    spacing: tuple[float, ...] | None = None  # element extents, when not (hi - lo) / n exactly
    # boundary conditions of negative neighbour entries -1 - b: {b: (type, state or None)}
    boundaries: dict | None = None
    # the grid cells (x-fastest index into the n grid) that are elements, when
    # the domain is a subset of the box (a step, a channel with an obstacle)
    cells: np.ndarray | None = None
    # meshes read from a file (prandtl_b200.meshio): boundary name -> condition
    # index, and the element attributes
    boundary_names: dict | None = None
    attributes: np.ndarray | None = None
    reoriented: np.ndarray | None = None   # elements whose corner order the reader relabelled
    frames: np.ndarray | None = None       # (ne, dim) file frame of each element, +-(axis + 1)
    # general geometry (skewed, graded, curved or unstructured elements): the
    # physical coordinates of every DG node, (dim, num_nodes) byNODES, and the
    # face orientation codes of the C ABI's pdg_set_geometry, (ne, 2*dim)
    # (None: every neighbour meets a face with its opposite face, axes aligned)
    coords: np.ndarray | None = None
    face_orient: np.ndarray | None = None
    corners: np.ndarray | None = None      # (ne, 2^dim) corner vertex ids, lexicographic corner order

    @property
    def general(self) -> bool:
        """True when the mesh carries its own node coordinates (the general-geometry path)."""
        return self.coords is not None

    @property
    def Np(self) -> int:
        return self.order + 1

    @property
    def ndof(self) -> int:
        return self.Np ** self.dim

    @property
    def num_elements(self) -> int:
        return int(np.prod(self.n)) if self.cells is None else int(len(self.cells))

    @property
    def num_nodes(self) -> int:
        return self.num_elements * self.ndof

    @property
    def nv(self) -> int:
        return self.dim + 2

    @property
    def size(self) -> int:
        return self.num_nodes * self.nv

    @property
    def h(self) -> tuple[float, ...]:
        if self.spacing is not None:
            return tuple(self.spacing)
        return tuple((self.hi[d] - self.lo[d]) / self.n[d] for d in range(self.dim))

    def node_coords(self, elements=None) -> np.ndarray:
        """Physical coordinates, shape (dim, num_nodes), in the byNODES order
        (of the listed elements only, when `elements` is given)."""
        if self.coords is not None:
            if elements is None:
                return np.array(self.coords, dtype=np.float64)
            e = np.asarray(elements, dtype=np.int64)
            X = np.asarray(self.coords).reshape(self.dim, self.num_elements, self.ndof)
            return X[:, e, :].reshape(self.dim, -1)
        x1, _ = gll_nodes(self.Np)
        Np, dim = self.Np, self.dim
        e = np.arange(self.num_elements) if elements is None else np.asarray(elements, dtype=np.int64)
        if self.cells is not None:
            e = np.asarray(self.cells, dtype=np.int64)[e]
        ne = e.size
        eidx = []
        r = e.copy()
        for d in range(dim):
            eidx.append(r % self.n[d])
            r //= self.n[d]
        loc = np.arange(self.ndof)
        lidx = []
        r = loc.copy()
        for d in range(dim):
            lidx.append(r % Np)
            r //= Np
        h = self.h
        out = np.empty((dim, ne * self.ndof))
        for d in range(dim):
            c = self.lo[d] + (eidx[d][:, None] + x1[lidx[d]][None, :]) * h[d]
            out[d] = c.reshape(-1)
        return out


def periodic_box(dim: int, order: int, n, lo, hi) -> CartesianMesh:
    """Periodic box [lo, hi] split into n[d] elements per direction."""
    if np.isscalar(n):
        n = (int(n),) * dim
    n = tuple(int(v) for v in n)
    if np.isscalar(lo):
        lo = (float(lo),) * dim
    if np.isscalar(hi):
        hi = (float(hi),) * dim
    ne = int(np.prod(n))
    e = np.arange(ne)
    idx = []
    r = e.copy()
    for d in range(dim):
        idx.append(r % n[d])
        r //= n[d]
    strides = [int(np.prod(n[:d])) for d in range(dim)]
    nbr = np.empty((ne, 2 * dim), dtype=np.int32)
    for d in range(dim):
        base = e - idx[d] * strides[d]
        nbr[:, 2 * d] = base + ((idx[d] - 1) % n[d]) * strides[d]
        nbr[:, 2 * d + 1] = base + ((idx[d] + 1) % n[d]) * strides[d]
    return CartesianMesh(dim, order, n, tuple(lo), tuple(hi), nbr)


def box(dim: int, order: int, n, lo, hi, bdr=None, boundaries=None, keep=None, cut=None) -> CartesianMesh:
    """Box [lo, hi] with n[d] elements per direction.  bdr[d] = None keeps
    direction d periodic; bdr[d] = (b_lo, b_hi) makes its -d and +d sides
    boundary faces with conditions b_lo and b_hi (neighbour entry -1 - b).
    ``boundaries`` maps each condition to (type, state), the arguments of
    DGSEMOperator.set_boundary (the reference's boundary attributes and
    BdrFaceIntegrators, src/Simulation/Simulation.cpp:490-798).  ``keep``, a
    boolean array of shape n (index [i_x, i_y(, i_z)]), keeps only those
    cells as elements (in the box's x-fastest order): a face towards a removed
    cell becomes a boundary face with condition ``cut`` (a forward or
    backward facing step, an obstacle)."""
    m = periodic_box(dim, order, n, lo, hi)
    if bdr is None:
        bdr = [None] * dim
    nbr = m.nbr.copy()
    e = np.arange(m.num_elements)
    r = e.copy()
    for d in range(dim):
        i = r % m.n[d]
        r //= m.n[d]
        if bdr[d] is None:
            continue
        b_lo, b_hi = bdr[d]
        nbr[i == 0, 2 * d] = -1 - int(b_lo)
        nbr[i == m.n[d] - 1, 2 * d + 1] = -1 - int(b_hi)
    m.nbr = nbr
    m.boundaries = dict(boundaries or {})
    if keep is not None:
        k = np.asarray(keep, dtype=bool)
        if k.shape != tuple(m.n):
            raise ValueError(f"keep has shape {k.shape}, the grid {tuple(m.n)}")
        flat = k.reshape(-1, order="F")            # x-fastest cell order
        cells = np.nonzero(flat)[0]
        if cells.size == 0 or cut is None:
            raise ValueError("keep needs at least one cell and a boundary condition `cut`")
        new = np.full(flat.size, -1, dtype=np.int64)
        new[cells] = np.arange(cells.size)
        sub = nbr[cells].astype(np.int64)
        inner = sub >= 0
        tgt = np.where(inner, sub, 0)
        sub = np.where(inner, np.where(flat[tgt], new[tgt], -1 - int(cut)), sub)
        m.nbr = sub.astype(np.int32)
        m.cells = cells
    return m
