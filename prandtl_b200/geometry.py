"""Meshes of general geometry: skewed, graded, curved or unstructured
quadrilaterals and hexahedra, described the way the reference's MFEM mesh
describes them (src/Simulation/Simulation.cpp:271-336): every element maps
the reference square or cube [0,1]^dim to physical space, and the DG nodes
sit at the images of the LGL nodes.

A general mesh carries
  * ``coords`` (dim, num_nodes): the physical coordinates of every DG node
    (byNODES, like a state field), from which the kernels' metric terms are
    formed (the reference evaluates the same Jacobians with MFEM's
    ElementTransformation at every integration point,
    DGSEMIntegrator.cpp:252-255);
  * ``nbr`` (ne, 2 dim): the face neighbour of every element face (faces
    f = 2 d + side in the element's own frame) or ``-1 - b`` for a boundary
    face with condition b;
  * ``face_orient`` (ne, 2 dim): for an interior face, ``f2 + 8 o``: the
    neighbour's face f2 that meets it and the map o of face-node indices.
    With (a, b) this element's node indices along the face's two tangential
    axes (ascending axis order; b = 0 in 2D), the neighbour's are
    (a', b') = (b, a) if o & 1 else (a, b), then a' -> N - a' if o & 2 and
    b' -> N - b' if o & 4;
  * ``corners`` (ne, 2^dim): the corner vertex ids in lexicographic corner
    order (corner c at reference position (c & 1, c >> 1 & 1, c >> 2 & 1)),
    from which ``connect`` derives both tables.

Generators: ``perturbed_box`` (bilinear / trilinear elements whose interior
vertices are moved at random: skewed, non-affine quads and hexes),
``warped`` (a box mesh with its nodes moved by a smooth periodic field:
curved elements of degree N), ``skewed`` (an affine shear) and
``rotate_frames`` (the same mesh with some elements' local frames rotated,
so that neighbouring elements meet with different faces and orientations,
as in an unstructured mesh).
"""
from __future__ import annotations

import itertools

import numpy as np

from .mesh import CartesianMesh, box, gll_nodes


def face_corner_slots(dim: int, f: int) -> list[int]:
    """Local corner indices of face f = 2 d + side, in (a, b) order (a, the
    lower tangential axis, fastest)."""
    d, side = divmod(f, 2)
    axes = [q for q in range(dim) if q != d]
    out = []
    for b in ((0, 1) if dim == 3 else (0,)):
        for a in (0, 1):
            bits = [0] * dim
            bits[d] = side
            bits[axes[0]] = a
            if dim == 3:
                bits[axes[1]] = b
            out.append(sum(bit << q for q, bit in enumerate(bits)))
    return out


def map_face_index(dim: int, N: int, a: int, b: int, o: int) -> tuple[int, int]:
    """The neighbour's face-node indices (a', b') of this element's (a, b)
    under orientation o."""
    if o & 1:
        a, b = b, a
    if o & 2:
        a = N - a
    if o & 4:
        b = N - b
    return a, b


def orientation_code(dim: int, own: list[int], other: list[int]) -> int:
    """The o with own[(a, b)] == other[map(a, b)] at the face's corners
    (vertex ids in (a, b) order), or -1."""
    codes = (0, 2) if dim == 2 else range(8)
    for o in codes:
        ok = True
        for b in ((0, 1) if dim == 3 else (0,)):
            for a in (0, 1):
                a2, b2 = map_face_index(dim, 1, a, b, o)
                if own[a + 2 * b] != other[a2 + 2 * b2]:
                    ok = False
        if ok:
            return o
    return -1


def connect(dim: int, corners: np.ndarray, boundary=None):
    """Neighbour table and face orientation codes of elements given by their
    corner vertex ids.  Faces pair by vertex sets; an unpaired face takes
    ``boundary[frozenset(vertex ids)]`` (a neighbour entry -1 - b), or raises.
    Returns (nbr, face_orient), int32."""
    corners = np.asarray(corners, dtype=np.int64)
    ne = corners.shape[0]
    slots = [face_corner_slots(dim, f) for f in range(2 * dim)]
    faces: dict = {}
    for e in range(ne):
        for f in range(2 * dim):
            vs = corners[e, slots[f]].tolist()
            faces.setdefault(frozenset(vs), []).append((e, f, vs))
    nbr = np.zeros((ne, 2 * dim), dtype=np.int64)
    orient = np.zeros((ne, 2 * dim), dtype=np.int64)
    for key, owners in faces.items():
        if len(owners) == 2:
            (e1, f1, v1), (e2, f2, v2) = owners
            o12 = orientation_code(dim, v1, v2)
            o21 = orientation_code(dim, v2, v1)
            if o12 < 0 or o21 < 0:
                raise ValueError(f"elements {e1} and {e2}: faces with the same vertices do not match")
            nbr[e1, f1], orient[e1, f1] = e2, f2 + 8 * o12
            nbr[e2, f2], orient[e2, f2] = e1, f1 + 8 * o21
        elif len(owners) == 1:
            e, f, _ = owners[0]
            if boundary is None or key not in boundary:
                raise ValueError(f"element {e}: face {f} has no neighbour and no boundary condition")
            nbr[e, f] = -1 - int(boundary[key])
            orient[e, f] = 0
        else:
            raise ValueError(f"a face shared by {len(owners)} elements")
    return nbr.astype(np.int32), orient.astype(np.int32)


def multilinear_nodes(dim: int, order: int, corner_xyz: np.ndarray) -> np.ndarray:
    """DG node coordinates (dim, ne * Np^dim) of bilinear / trilinear
    elements with corner coordinates corner_xyz (ne, 2^dim, dim)."""
    x1, _ = gll_nodes(order + 1)
    Np = order + 1
    loc = np.arange(Np ** dim)
    xi = [x1[(loc // Np ** q) % Np] for q in range(dim)]
    phi = np.ones((2 ** dim, loc.size))
    for c in range(2 ** dim):
        for q in range(dim):
            phi[c] *= xi[q] if (c >> q) & 1 else 1.0 - xi[q]
    X = np.einsum("ecd,cn->den", np.asarray(corner_xyz, dtype=np.float64), phi)
    return X.reshape(dim, -1)


def _lattice(dim, n, lo, hi, periodic):
    """Vertex ids (wrapped in periodic directions) and unwrapped corner
    positions of the structured box's elements (x fastest)."""
    n = tuple(int(v) for v in n)
    ne = int(np.prod(n))
    e = np.arange(ne)
    idx, r = [], e.copy()
    for d in range(dim):
        idx.append(r % n[d])
        r //= n[d]
    nvert = [n[d] if periodic[d] else n[d] + 1 for d in range(dim)]
    corners = np.zeros((ne, 2 ** dim), dtype=np.int64)
    lattice = np.zeros((ne, 2 ** dim, dim), dtype=np.int64)
    for c in range(2 ** dim):
        vid, stride = np.zeros(ne, dtype=np.int64), 1
        for d in range(dim):
            i = idx[d] + ((c >> d) & 1)
            lattice[:, c, d] = i
            vid += (i % nvert[d]) * stride
            stride *= nvert[d]
        corners[:, c] = vid
    h = np.array([(hi[d] - lo[d]) / n[d] for d in range(dim)])
    xyz = np.asarray(lo, dtype=np.float64)[None, None, :dim] + lattice * h[None, None, :]
    return corners, lattice, xyz, nvert


def _box_boundary(dim, mesh, corners):
    """Boundary condition of every boundary face of a box mesh, by vertex set."""
    out = {}
    for e, f in zip(*np.nonzero(mesh.nbr < 0)):
        vs = corners[e, face_corner_slots(dim, int(f))]
        out[frozenset(vs.tolist())] = int(-1 - mesh.nbr[e, f])
    return out


def perturbed_box(dim: int, order: int, n, lo, hi, amp: float, seed: int = 0, bdr=None,
                  boundaries=None) -> CartesianMesh:
    """A box [lo, hi] of n[d] elements per direction whose vertices are moved
    by amp h U(-1/2, 1/2) per component (periodic images together; on a
    boundary side only along it): bilinear / trilinear elements, skewed and
    non-affine.  ``bdr`` and ``boundaries`` as in ``mesh.box``."""
    m = box(dim, order, n, lo, hi, bdr=bdr, boundaries=boundaries)
    periodic = [bdr is None or bdr[d] is None for d in range(dim)]
    corners, lattice, xyz, nvert = _lattice(dim, m.n, m.lo, m.hi, periodic)
    rng = np.random.default_rng(seed)
    h = np.array(m.h)
    disp = (rng.random((int(np.prod(nvert)), dim)) - 0.5) * amp * h[None, :]
    # vertices on a non-periodic side stay on it
    vidx, r = [], np.arange(int(np.prod(nvert)))
    for d in range(dim):
        vidx.append(r % nvert[d])
        r //= nvert[d]
    for d in range(dim):
        if not periodic[d]:
            disp[(vidx[d] == 0) | (vidx[d] == nvert[d] - 1), d] = 0.0
    xyz = xyz + disp[corners]
    m.coords = multilinear_nodes(dim, order, xyz)
    m.corners = corners
    nbr, orient = connect(dim, corners, _box_boundary(dim, m, corners))
    if not np.array_equal(nbr, m.nbr):
        raise AssertionError("lattice connectivity differs from the box's")
    m.face_orient = orient
    return m


def warped(mesh: CartesianMesh, amp: float, waves: int = 1, twist: float = 0.0) -> CartesianMesh:
    """A box mesh (periodic or not, all cells present) with its DG nodes
    moved by the smooth field dx_d = amp L_d prod_q sin(2 pi k (x_q - lo_q) / L_q)
    (1 + twist cos(2 pi k (x_{d+1} - lo_{d+1}) / L_{d+1})), k = waves, which
    vanishes on the box's sides and is periodic: curved elements whose
    geometry is the degree-N interpolant of the field.  With twist = 0 every
    component moves by the same scalar field, so in 3D the quadratic terms of
    the Jacobian's column cross products cancel and the pointwise metric
    terms meet the discrete metric identities; a twist turns the
    displacement's direction from node to node, and they do not."""
    if mesh.cells is not None or mesh.coords is not None:
        raise ValueError("warped() takes a full box mesh")
    X = mesh.node_coords()
    L = np.array(mesh.hi, dtype=np.float64) - np.array(mesh.lo, dtype=np.float64)
    s = np.ones(X.shape[1])
    for q in range(mesh.dim):
        s = s * np.sin(2 * np.pi * waves * (X[q] - mesh.lo[q]) / L[q])
    out = _copy(mesh)
    disp = amp * L[:, None] * s[None, :]
    if twist:
        for d in range(mesh.dim):
            q = (d + 1) % mesh.dim
            disp[d] *= 1.0 + twist * np.cos(2 * np.pi * waves * (X[q] - mesh.lo[q]) / L[q])
    out.coords = X + disp
    periodic = [bool(np.all(mesh.nbr[:, 2 * d:2 * d + 2] >= 0)) for d in range(mesh.dim)]
    corners, _, _, _ = _lattice(mesh.dim, mesh.n, mesh.lo, mesh.hi, periodic)
    out.corners = corners
    out.face_orient = connect(mesh.dim, corners, _box_boundary(mesh.dim, mesh, corners))[1]
    return out


def skewed(mesh: CartesianMesh, shear: float) -> CartesianMesh:
    """An affine shear x -> x + shear (y - lo_y) of a box mesh: parallelogram
    elements (2D) or sheared hexahedra (3D)."""
    if mesh.coords is not None:
        raise ValueError("skewed() takes a box mesh")
    X = mesh.node_coords()
    out = _copy(mesh)
    X[0] = X[0] + shear * (X[1] - mesh.lo[1])
    out.coords = X
    return out


def _copy(mesh: CartesianMesh) -> CartesianMesh:
    return CartesianMesh(mesh.dim, mesh.order, tuple(mesh.n), tuple(mesh.lo), tuple(mesh.hi), mesh.nbr.copy(),
                         spacing=mesh.spacing, boundaries=dict(mesh.boundaries or {}), cells=mesh.cells,
                         boundary_names=mesh.boundary_names, attributes=mesh.attributes)


def proper_rotations(dim: int):
    """The frame maps of the reference square / cube with determinant +1, as
    (perm, flip): new axis a runs along old axis perm[a], reversed when flip[a]."""
    out = []
    for perm in itertools.permutations(range(dim)):
        sgn = np.linalg.det(np.eye(dim)[list(perm)])
        for flip in itertools.product((0, 1), repeat=dim):
            if sgn * (-1) ** sum(flip) > 0:
                out.append((tuple(perm), tuple(flip)))
    return out


def rotate_frames(mesh: CartesianMesh, elements, seed: int = 0) -> CartesianMesh:
    """The same mesh with the local frames of ``elements`` rotated (a random
    proper rotation of the reference element each): their nodes, corners
    and faces are renumbered, and ``connect`` derives the neighbour table
    and the face orientation codes anew.  Fields of the rotated mesh are
    the original fields with those elements' nodes permuted
    (``node_maps``)."""
    if mesh.corners is None or mesh.coords is None:
        raise ValueError("rotate_frames() takes a general mesh with corners (perturbed_box, warped)")
    dim, Np, N = mesh.dim, mesh.Np, mesh.order
    rng = np.random.default_rng(seed)
    rots = proper_rotations(dim)[1:]  # not the identity
    ne, nd = mesh.num_elements, mesh.ndof
    perm_nodes = np.tile(np.arange(nd), (ne, 1))
    corners = np.array(mesh.corners, dtype=np.int64)
    loc = np.arange(nd)
    new_idx = [(loc // Np ** a) % Np for a in range(dim)]
    cl = np.arange(2 ** dim)
    new_cb = [(cl >> a) & 1 for a in range(dim)]
    for e in np.asarray(elements, dtype=np.int64):
        perm, flip = rots[int(rng.integers(len(rots)))]
        old = np.zeros(nd, dtype=np.int64)
        oldc = np.zeros(2 ** dim, dtype=np.int64)
        for a in range(dim):
            i = N - new_idx[a] if flip[a] else new_idx[a]
            old += i * Np ** perm[a]
            cb = 1 - new_cb[a] if flip[a] else new_cb[a]
            oldc += cb << perm[a]
        perm_nodes[e] = old
        corners[e] = mesh.corners[e][oldc]
    boundary = _box_boundary(dim, mesh, np.asarray(mesh.corners))
    out = _copy(mesh)
    X = np.asarray(mesh.coords).reshape(dim, ne, nd)
    out.coords = np.take_along_axis(X, perm_nodes[None, :, :], axis=2).reshape(dim, -1)
    out.corners = corners
    out.nbr, out.face_orient = connect(dim, corners, boundary)
    out.node_maps = perm_nodes
    return out


def permute_nodes(mesh: CartesianMesh, u: np.ndarray) -> np.ndarray:
    """A field of the mesh ``rotate_frames`` started from, in the rotated
    mesh's node order (``mesh`` is the rotated mesh)."""
    P = mesh.node_maps
    X = np.asarray(u).reshape(-1, mesh.num_elements, mesh.ndof)
    return np.take_along_axis(X, P[None, :, :], axis=2).reshape(np.shape(u))
