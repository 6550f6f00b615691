"""Readers of the reference's mesh files into the neighbour-table layout.

The reference loads its mesh with ``mfem::Mesh(mesh_file)``
(src/Simulation/Simulation.cpp:271-272), refines it ``ser_ref_levels`` times
(:292-300) and attaches each boundary condition to the boundary attributes
named in its configuration (``bdr_attribute_sets``, :490-506; for a Gmsh
file the names are the ``$PhysicalNames`` of the boundary entities and the
attribute is the physical tag).  Two formats are read here:

* MFEM mesh v1.0 (``TestCases/Euler/2D/IsentropicVortex/IsentropicVortex.mesh``
  and ``KelvinHelmholtzInstability.mesh``): ``elements`` and ``boundary``
  list ``<attribute> <geometry> <vertex ...>``; coordinates come from
  ``vertices`` or, for a periodic mesh, from a discontinuous ``nodes``
  section (``L2_T1_<dim>D_P1``, ``Ordering: 1``: the element's corners in
  lexicographic order, x fastest, one coordinate tuple each);
* Gmsh 2.2 ASCII (the ``.msh`` files of the step, double Mach reflection and
  lid-driven cavity cases): quadrilaterals (type 3) or hexahedra (type 5) for
  the domain, lines (type 1) or quadrilaterals for the boundary, the first tag
  being the physical tag.

Both number a quadrilateral's corners counter-clockwise from its first
corner, and a hexahedron's bottom face that way and then its top face.

A mesh whose elements are all axis-aligned boxes of one size is read for
the box kernels (one element size per direction, element axes along the
coordinate axes); any other mesh — graded, skewed or unstructured, like the
forward-facing step, the ramp and the ramjet — is read as a general-geometry
mesh (``build_general_mesh``: each element in the file's frame, node
coordinates from its bilinear or trilinear map, face orientation codes from
its corner vertices) for the general-geometry kernel.  For the box form, an
element whose corners the file lists
in a rotated or mirrored order (Gmsh does this in the step meshes) is
relabelled so that its first corner is its lowest one and its second lies
along +x (fourth along +y, fifth along +z); its DG nodes are then numbered in
that frame, not the reference's, ``mesh.reoriented`` lists it and
``to_reference_order`` / ``from_reference_order`` move fields between the two
node orders.  Elements keep the file's order; faces are paired by their corner vertices, so periodic
identifications of an MFEM mesh carry over (a periodic direction needs three
elements or more, else two faces share their vertices).  A boundary face takes condition
``attribute - 1`` (neighbour entry ``-attribute``).

``refine`` splits every element into 2^dim children, numbered ``2^dim e + c``
with c lexicographic (x fastest).  MFEM's own refinement order is not restated
here (MFEM is an external dependency), so element numbers after refinement
differ from the reference's while the mesh is the same.
"""
from __future__ import annotations

import numpy as np

from .geometry import connect, multilinear_nodes
from .mesh import CartesianMesh

MAX_CONDITIONS = 16          # PDG_MAX_BOUNDARIES


class NotBoxError(ValueError):
    """The elements are not equal axis-aligned boxes on one grid (the box
    kernels' form); the mesh may still be read as a general-geometry mesh."""

# corner k of an MFEM/Gmsh quadrilateral or hexahedron -> its (x, y, z) bits
_CORNER_BITS = {
    2: [(0, 0), (1, 0), (1, 1), (0, 1)],
    3: [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)],
}


def read_mesh(path: str, order: int, refine: int = 0, tol: float = 1e-8, general=None) -> CartesianMesh:
    """The mesh in ``path`` (MFEM v1.0 or Gmsh 2.2 ASCII) with polynomial
    order ``order``, refined ``refine`` times.  ``tol`` is the relative
    tolerance of the box-shape and uniform-size checks.  ``general``: False
    reads equal axis-aligned boxes only (the box kernels), True every mesh
    as a general-geometry mesh (``build_general_mesh``: node coordinates
    and face orientation codes for the general-geometry kernel), None the
    box form when the elements allow it, else the general form."""
    with open(path) as f:
        text = f.read()
    head = text.lstrip()[:40]
    if head.startswith("MFEM mesh v1.0"):
        parsed = _parse_mfem(text)
    elif head.startswith("$MeshFormat"):
        parsed = _parse_gmsh(text)
    else:
        raise ValueError(f"{path}: neither an MFEM v1.0 nor a Gmsh 2.2 mesh")
    if general:
        mesh = build_general_mesh(order=order, **parsed)
    else:
        try:
            mesh = build_mesh(order=order, tol=tol, **parsed)
        except NotBoxError:
            if general is False:
                raise
            mesh = build_general_mesh(order=order, **parsed)
    for _ in range(int(refine)):
        mesh = refine_general(mesh) if mesh.coords is not None else refine_mesh(mesh)
    return mesh


def _parse_mfem(text: str) -> dict:
    lines = [ln.split("#", 1)[0].strip() for ln in text.splitlines()]
    lines = [ln for ln in lines if ln]
    pos = {}
    for i, ln in enumerate(lines):
        if ln in ("dimension", "elements", "boundary", "vertices", "nodes") and ln not in pos:
            pos[ln] = i
    for key in ("dimension", "elements", "boundary", "vertices"):
        if key not in pos:
            raise ValueError(f"MFEM mesh without a '{key}' section")
    dim = int(lines[pos["dimension"] + 1])
    if dim not in (2, 3):
        raise ValueError(f"MFEM mesh of dimension {dim}: only 2 and 3 are read")
    nc = 2 ** dim

    def cells(key, geom, what):
        i = pos[key] + 1
        n = int(lines[i])
        rows = [lines[i + 1 + k].split() for k in range(n)]
        out = []
        for r in rows:
            if int(r[1]) != geom:
                raise ValueError(f"MFEM {key} of geometry {r[1]}: only {what} are read")
            out.append((int(r[0]), [int(v) for v in r[2:]]))
        return out

    # MFEM geometries: 1 segment, 3 square, 5 cube
    elements = cells("elements", 3 if dim == 2 else 5, "squares and cubes")
    boundary = cells("boundary", 1 if dim == 2 else 3, "segments (2D) and squares (3D)")
    verts = np.array([e[1] for e in elements], dtype=np.int64).reshape(-1, nc)
    i = pos["vertices"] + 1
    nvert = int(lines[i])
    if "nodes" in pos:
        j = pos["nodes"] + 1
        if lines[j] != "FiniteElementSpace":
            raise ValueError("MFEM nodes section without a FiniteElementSpace")
        j += 1
        header = {}
        while ":" in lines[j]:
            k, v = lines[j].split(":", 1)
            header[k.strip()] = v.strip()
            j += 1
        fec = header.get("FiniteElementCollection", "")
        if fec != f"L2_T1_{dim}D_P1" or header.get("Ordering", "1") != "1":
            raise ValueError(f"MFEM nodes of collection {fec!r}: only {f'L2_T1_{dim}D_P1'} (Ordering 1) "
                             "is read (curved geometry is not supported)")
        vals = np.array(" ".join(lines[j:]).split(), dtype=np.float64)
        if vals.size != len(elements) * nc * dim:
            raise ValueError("MFEM nodes section does not hold one point per element corner")
        lex = vals.reshape(len(elements), nc, dim)
        # corner k sits at lexicographic position bx + 2 by + 4 bz
        perm = [sum(b << d for d, b in enumerate(bits)) for bits in _CORNER_BITS[dim]]
        coords = lex[:, perm, :]
    else:
        sdim = int(lines[i + 1])
        pts = np.array([lines[i + 2 + k].split() for k in range(nvert)], dtype=np.float64)
        if sdim < dim:
            raise ValueError("MFEM vertices of lower dimension than the mesh")
        coords = pts[verts][:, :, :dim]
    return dict(dim=dim, verts=verts, coords=coords,
                attrs=np.array([e[0] for e in elements], dtype=np.int64),
                bdr={frozenset(v): a for a, v in boundary},
                names={str(a): a for a in sorted({a for a, _ in boundary})})


def _section(lines, name):
    try:
        i = lines.index(f"${name}")
    except ValueError:
        return None
    j = lines.index(f"$End{name}", i)
    return lines[i + 1:j]


def _parse_gmsh(text: str) -> dict:
    lines = [ln.strip() for ln in text.splitlines()]
    fmt = _section(lines, "MeshFormat")
    if not fmt or not fmt[0].split()[0].startswith("2.") or fmt[0].split()[1] != "0":
        raise ValueError("Gmsh mesh: only the ASCII 2.x format is read")
    names = {}
    pn = _section(lines, "PhysicalNames") or []
    phys = [ln.split(None, 2) for ln in pn[1:] if ln]
    node_sec = _section(lines, "Nodes")
    elem_sec = _section(lines, "Elements")
    if node_sec is None or elem_sec is None:
        raise ValueError("Gmsh mesh without a $Nodes or $Elements section")
    ids, xyz = [], []
    for ln in node_sec[1:]:
        if not ln:
            continue
        r = ln.split()
        ids.append(int(r[0]))
        xyz.append([float(r[1]), float(r[2]), float(r[3])])
    index = {v: k for k, v in enumerate(ids)}
    xyz = np.array(xyz)
    quads, hexes, lines1 = [], [], []
    for ln in elem_sec[1:]:
        if not ln:
            continue
        r = [int(v) for v in ln.split()]
        typ, ntags = r[1], r[2]
        tag = r[3] if ntags > 0 else 0
        nodes = [index[v] for v in r[3 + ntags:]]
        if typ == 3:
            quads.append((tag, nodes))
        elif typ == 5:
            hexes.append((tag, nodes))
        elif typ == 1:
            lines1.append((tag, nodes))
        elif typ != 15:
            raise ValueError(f"Gmsh element type {typ}: only points, lines, quadrilaterals and hexahedra "
                             "(first order) are read")
    if hexes:
        dim, dom, bnd = 3, hexes, quads
    else:
        dim, dom, bnd = 2, quads, lines1
    if not dom:
        raise ValueError("Gmsh mesh without quadrilateral or hexahedral elements")
    for row in phys:
        if int(row[0]) == dim - 1:
            names[row[2].strip().strip('"')] = int(row[1])
    verts = np.array([n for _, n in dom], dtype=np.int64)
    return dict(dim=dim, verts=verts, coords=xyz[verts][:, :, :dim],
                attrs=np.array([t for t, _ in dom], dtype=np.int64),
                bdr={frozenset(n): t for t, n in bnd},
                names=names or {str(t): t for t in sorted({t for t, _ in bnd})})


def _canonical_corners(dim, verts, coords):
    """Corners of each element relabelled so that corner k sits at the box
    position of _CORNER_BITS[k] (first corner lowest, second along +x, ...).
    Gmsh writes some elements of a structured mesh with a rotated or mirrored
    corner order; the kernels need every element's axes along +x, +y (+z).
    Returns the relabelled arrays, the indices of the elements whose corners
    moved (their DG nodes are numbered in the relabelled frame, not in the
    file's) and each element's file frame: frames[e, a] = +-(d + 1) when the
    file's local axis a (corner 0 -> 1, 0 -> 3, 0 -> 4) runs along +-axis d."""
    ne, nc = verts.shape
    centre = coords.mean(axis=1, keepdims=True)
    hb = (coords > centre).astype(np.int64)                           # (ne, nc, dim) corner bits
    key = np.zeros((ne, nc), dtype=np.int64)
    for d in range(dim):
        key += hb[:, :, d] << d
    want = np.array([sum(b << d for d, b in enumerate(bits)) for bits in _CORNER_BITS[dim]])
    # pos[e, k]: the file corner at box position want[k]
    inv = np.full((ne, nc), -1, dtype=np.int64)
    rows = np.repeat(np.arange(ne), nc)
    inv[rows, key.reshape(-1)] = np.tile(np.arange(nc), ne)
    if np.any(inv < 0):
        bad = int(np.nonzero(np.any(inv < 0, axis=1))[0][0])
        raise NotBoxError(f"element {bad} is not a box (degenerate or non-convex corners)")
    pos = inv[:, want]
    moved = np.nonzero(np.any(pos != np.arange(nc), axis=1))[0]
    cbits = np.array(_CORNER_BITS[dim], dtype=np.int64)
    kpos = np.argsort(pos, axis=1)                   # file corner f sits at box position kpos[e, f]
    frames = np.zeros((ne, dim), dtype=np.int8)
    for a, f in enumerate((1, 3, 4)[:dim]):
        step = cbits[kpos[:, f]] - cbits[kpos[:, 0]]  # (ne, dim): +-e_d
        d = np.argmax(np.abs(step), axis=1)
        frames[:, a] = (d + 1) * step[np.arange(ne), d]
    return (np.take_along_axis(verts, pos, axis=1),
            np.take_along_axis(coords, pos[:, :, None], axis=1), moved, frames)


def build_mesh(dim, order, verts, coords, bdr, names, attrs=None, tol=1e-8) -> CartesianMesh:
    """Neighbour table, element size and grid cells of elements given by
    their corner vertices ``verts`` (ne, 2^dim) and corner coordinates
    ``coords`` (ne, 2^dim, dim), in MFEM/Gmsh corner order; ``bdr`` maps the
    vertex set of each boundary element to its attribute, ``names`` the
    boundary names to attributes."""
    ne, nc = verts.shape
    if nc != 2 ** dim:
        raise ValueError(f"elements with {nc} corners in {dim}D")
    bits = np.array(_CORNER_BITS[dim], dtype=np.float64)              # (nc, dim)
    verts, coords, reoriented, frames = _canonical_corners(dim, verts, coords)
    origin = coords[:, 0, :]
    # extents: corner 1 lies along +x, corner 3 along +y, corner 4 along +z
    ext = np.stack([coords[:, (1, 3, 4)[d], d] - origin[:, d] for d in range(dim)], axis=1)
    if np.any(ext <= 0):
        bad = int(np.nonzero(np.any(ext <= 0, axis=1))[0][0])
        raise NotBoxError(f"element {bad} is degenerate (an extent of zero)")
    h = ext.mean(axis=0)
    expect = origin[:, None, :] + bits[None, :, :] * ext[:, None, :]
    if np.any(np.abs(coords - expect) > tol * h):
        bad = int(np.nonzero(np.any(np.abs(coords - expect) > tol * h, axis=(1, 2)))[0][0])
        raise NotBoxError(f"element {bad} is not an axis-aligned box (curved or skewed geometry is not supported)")
    if np.any(np.abs(ext - h) > tol * h):
        raise NotBoxError("elements of different sizes (graded meshes are not supported)")
    lo = origin.min(axis=0)
    hi = (origin + ext).max(axis=0)
    g = (origin - lo) / h
    gi = np.rint(g).astype(np.int64)
    if np.any(np.abs(g - gi) > 1e-6):
        raise NotBoxError("element corners off the grid of the element size")
    n = tuple(int(v) for v in np.rint((hi - lo) / h))
    cells = np.zeros(ne, dtype=np.int64)
    stride = 1
    for d in range(dim):
        cells += gi[:, d] * stride
        stride *= n[d]
    if len(np.unique(cells)) != ne:
        raise NotBoxError("overlapping elements")

    nbr = np.full((ne, 2 * dim), np.iinfo(np.int32).min, dtype=np.int64)
    faces: dict = {}
    for d in range(dim):
        for side in (0, 1):
            sel = [k for k in range(nc) if _CORNER_BITS[dim][k][d] == side]
            fv = verts[:, sel]
            for e in range(ne):
                faces.setdefault(frozenset(fv[e].tolist()), []).append((e, d, side))
    used = set()
    for key, owners in faces.items():
        if len(owners) == 2:
            (e1, d1, s1), (e2, d2, s2) = owners
            if d1 != d2 or s1 == s2:
                raise NotBoxError(f"elements {e1} and {e2} meet with differently oriented axes")
            nbr[e1, 2 * d1 + s1] = e2
            nbr[e2, 2 * d2 + s2] = e1
        elif len(owners) == 1:
            e, d, side = owners[0]
            if key not in bdr:
                raise ValueError(f"element {e}: boundary face ({'-+'[side]}{'xyz'[d]}) without a boundary element")
            a = int(bdr[key])
            if not 1 <= a <= MAX_CONDITIONS:
                raise ValueError(f"boundary attribute {a}: attributes 1..{MAX_CONDITIONS} are supported")
            nbr[e, 2 * d + side] = -a
            used.add(a)
        else:
            raise ValueError(f"a face shared by {len(owners)} elements (a non-conforming mesh, or a periodic "
                             "direction of fewer than three elements)")
    return CartesianMesh(dim, int(order), n, tuple(float(v) for v in lo), tuple(float(v) for v in hi),
                         nbr.astype(np.int32), spacing=tuple(float(v) for v in h), boundaries={}, cells=cells,
                         boundary_names={k: int(v) - 1 for k, v in names.items() if int(v) in used},
                         attributes=None if attrs is None else np.asarray(attrs), reoriented=reoriented,
                         frames=frames)


def refine_mesh(mesh: CartesianMesh) -> CartesianMesh:
    """Every element split into 2^dim children (``2^dim e + c``, c
    lexicographic, x fastest); boundary faces keep their conditions."""
    dim, K = mesh.dim, 2 ** mesh.dim
    nbr = mesh.nbr.astype(np.int64)
    ne = nbr.shape[0]
    parent = np.arange(ne, dtype=np.int64)
    new = np.empty((ne * K, 2 * dim), dtype=np.int64)
    cells = mesh.cells if mesh.cells is not None else np.arange(ne, dtype=np.int64)
    pidx = []
    r = np.asarray(cells, dtype=np.int64).copy()
    for d in range(dim):
        pidx.append(r % mesh.n[d])
        r //= mesh.n[d]
    n2 = tuple(2 * v for v in mesh.n)
    new_cells = np.empty(ne * K, dtype=np.int64)
    for c in range(K):
        child = parent * K + c
        cell = np.zeros(ne, dtype=np.int64)
        stride = 1
        for d in range(dim):
            b = (c >> d) & 1
            cell += (2 * pidx[d] + b) * stride
            stride *= n2[d]
            sib = c ^ (1 << d)
            for side in (0, 1):
                if b != side:
                    new[child, 2 * d + side] = parent * K + sib
                else:
                    nb = nbr[:, 2 * d + side]
                    new[child, 2 * d + side] = np.where(nb >= 0, nb * K + sib, nb)
        new_cells[child] = cell
    h = tuple(v / 2 for v in mesh.h)
    # no file frames: the children are numbered here, not by the reference
    return CartesianMesh(dim, mesh.order, n2, mesh.lo, mesh.hi, new.astype(np.int32), spacing=h,
                         boundaries=dict(mesh.boundaries or {}), cells=new_cells,
                         boundary_names=dict(mesh.boundary_names or {}),
                         attributes=None if mesh.attributes is None else np.repeat(mesh.attributes, K))


def node_permutation(mesh: CartesianMesh) -> np.ndarray:
    """perm[e, i]: this mesh's node of element e at the reference's node i.

    The reference numbers an element's DG nodes lexicographically in the
    element's own frame (its corner 0 -> 1 axis fastest); an element the
    reader relabelled has another frame here (``mesh.frames``).  Only for
    meshes as read (refinement renumbers the elements)."""
    if mesh.frames is None:
        raise ValueError("the mesh has no file frames (not read from a file, or refined)")
    Np, dim, ne = mesh.Np, mesh.dim, mesh.num_elements
    i = np.arange(Np ** dim)
    idx = [(i // Np ** a) % Np for a in range(dim)]            # file-frame multi-index, axis 0 fastest
    fr = np.asarray(mesh.frames, dtype=np.int64)
    out = np.zeros((ne, Np ** dim), dtype=np.int64)
    for a in range(dim):
        d = np.abs(fr[:, a]) - 1
        j = np.where(fr[:, a][:, None] > 0, idx[a][None, :], mesh.order - idx[a][None, :])
        out += j * (Np ** d)[:, None]
    return out


def from_reference_order(mesh: CartesianMesh, u: np.ndarray) -> np.ndarray:
    """A byNODES field (components x elements x nodes) in the reference's
    per-element node order, in this mesh's order."""
    perm = node_permutation(mesh)
    x = np.asarray(u).reshape(-1, mesh.num_elements, mesh.ndof)
    out = np.empty_like(x)
    rows = np.arange(mesh.num_elements)[:, None]
    out[:, rows, perm] = x
    return out.reshape(np.shape(u))


def to_reference_order(mesh: CartesianMesh, u: np.ndarray) -> np.ndarray:
    """This mesh's byNODES field in the reference's per-element node order."""
    perm = node_permutation(mesh)
    x = np.asarray(u).reshape(-1, mesh.num_elements, mesh.ndof)
    rows = np.arange(mesh.num_elements)[:, None]
    return x[:, rows, perm].reshape(np.shape(u))


def _lex_positions(dim):
    """Lexicographic corner index (x fastest) of each MFEM/Gmsh corner k."""
    return [sum(b << d for d, b in enumerate(bits)) for bits in _CORNER_BITS[dim]]


def _corner_jacobians(dim, xyz):
    """Determinant of the multilinear map's Jacobian at every corner of
    every element (corners in lexicographic order), (ne, 2^dim)."""
    ne, nc = xyz.shape[0], xyz.shape[1]
    out = np.empty((ne, nc))
    for c in range(nc):
        cols = []
        for a in range(dim):
            lo_c, hi_c = c & ~(1 << a), c | (1 << a)
            cols.append(xyz[:, hi_c, :] - xyz[:, lo_c, :])
        out[:, c] = np.linalg.det(np.stack(cols, axis=2))
    return out


def _general_mesh(dim, order, corners, xyz, boundary, names, attrs, frames, reoriented):
    nbr, orient = connect(dim, corners, boundary)
    ne = corners.shape[0]
    lo = xyz.reshape(-1, dim).min(axis=0)
    hi = xyz.reshape(-1, dim).max(axis=0)
    size = np.sqrt(np.abs(_corner_jacobians(dim, xyz)).min()) if dim == 2 else np.cbrt(
        np.abs(_corner_jacobians(dim, xyz)).min())
    used = {int(-1 - b) + 1 for b in nbr[nbr < 0]}
    m = CartesianMesh(dim, int(order), (ne,) + (1,) * (dim - 1), tuple(float(v) for v in lo),
                      tuple(float(v) for v in hi), nbr, spacing=(float(size),) * dim, boundaries={},
                      boundary_names={k: int(v) - 1 for k, v in names.items() if int(v) in used},
                      attributes=None if attrs is None else np.asarray(attrs), reoriented=reoriented, frames=frames)
    m.coords = multilinear_nodes(dim, order, xyz)
    m.face_orient = orient
    m.corners = corners
    m.corner_xyz = xyz
    return m


def build_general_mesh(dim, order, verts, coords, bdr, names, attrs=None) -> CartesianMesh:
    """A general-geometry mesh (skewed, graded or unstructured quadrilaterals
    or hexahedra with straight edges): each element keeps the file's frame
    (its corners in MFEM/Gmsh order map to the reference element's corners),
    its DG nodes sit at the images of the LGL nodes under the element's
    bilinear / trilinear map, and ``connect`` pairs faces by their vertices
    and derives the orientation codes.  An element whose corners the file
    lists clockwise (a negative Jacobian) is mirrored by exchanging its first
    two local axes (corners 1 and 3 of the listing exchanged); MFEM fixes
    inverted elements when it reads a mesh, and for a quadrilateral that fix
    is taken here to be the same exchange, so the element's DG nodes keep
    the reference's order (``mesh.frames`` is the identity) while
    ``mesh.reoriented`` lists it.  None of the reference's meshes has such an
    element, so this choice has not been compared with the reference."""
    ne, nc = verts.shape
    if nc != 2 ** dim:
        raise ValueError(f"elements with {nc} corners in {dim}D")
    lex = _lex_positions(dim)
    corners = np.empty((ne, nc), dtype=np.int64)
    xyz = np.empty((ne, nc, dim))
    corners[:, lex] = verts
    xyz[:, lex, :] = coords
    det = _corner_jacobians(dim, xyz)
    neg = np.all(det < 0, axis=1)
    bad = ~(np.all(det > 0, axis=1) | neg)
    if bad.any():
        raise ValueError(f"element {int(np.nonzero(bad)[0][0])} is degenerate or not convex")
    frames = np.tile(np.arange(1, dim + 1, dtype=np.int8), (ne, 1))
    reoriented = np.nonzero(neg)[0]
    if reoriented.size:
        swap = np.array([(c & ~3) | ((c & 1) << 1) | ((c >> 1) & 1) for c in range(nc)])
        corners[reoriented] = corners[reoriented][:, swap]
        xyz[reoriented] = xyz[reoriented][:, swap, :]
    boundary = {}
    for key, a in bdr.items():
        if not 1 <= int(a) <= MAX_CONDITIONS:
            raise ValueError(f"boundary attribute {a}: attributes 1..{MAX_CONDITIONS} are supported")
        boundary[frozenset(int(v) for v in key)] = int(a) - 1
    return _general_mesh(dim, order, corners, xyz, boundary, names, attrs, frames, reoriented)


def refine_general(mesh: CartesianMesh) -> CartesianMesh:
    """Every element of a general mesh split into 2^dim children (``2^dim e
    + c``, c lexicographic in the element's frame) at the midpoints of its
    multilinear map; new vertices are shared through the parent vertices
    they lie between, boundary faces keep their conditions."""
    if getattr(mesh, "corner_xyz", None) is None:
        raise ValueError("refine_general() takes a mesh from build_general_mesh")
    dim, nc = mesh.dim, 2 ** mesh.dim
    ne = mesh.num_elements
    P, X = np.asarray(mesh.corners), np.asarray(mesh.corner_xyz)
    keys: dict = {}
    corners = np.empty((ne * nc, nc), dtype=np.int64)
    xyz = np.empty((ne * nc, nc, dim))
    for e in range(ne):
        for c in range(nc):
            for k in range(nc):
                half = [((c >> q) & 1) + ((k >> q) & 1) for q in range(dim)]   # 0, 1, 2 in half steps
                touched = [pc for pc in range(nc)
                           if all((half[q] == 1) or (((pc >> q) & 1) == half[q] // 2) for q in range(dim))]
                key = frozenset(int(P[e, pc]) for pc in touched)
                if len(touched) == nc:
                    key = ("cell", e)
                if key not in keys:
                    keys[key] = len(keys)
                corners[e * nc + c, k] = keys[key]
                w = np.ones(nc)
                for pc in range(nc):
                    for q in range(dim):
                        t = half[q] / 2.0
                        w[pc] *= t if (pc >> q) & 1 else 1.0 - t
                xyz[e * nc + c, k] = w @ X[e]
    # boundary faces: a child face on a parent boundary face keeps its condition
    boundary = {}
    from .geometry import face_corner_slots
    for e, f in zip(*np.nonzero(mesh.nbr < 0)):
        b = int(-1 - mesh.nbr[e, f])
        d, side = divmod(int(f), 2)
        for c in range(nc):
            if ((c >> d) & 1) != side:
                continue
            vs = corners[e * nc + c, face_corner_slots(dim, int(f))]
            boundary[frozenset(int(v) for v in vs)] = b
    names = {k: v + 1 for k, v in (mesh.boundary_names or {}).items()}
    attrs = None if mesh.attributes is None else np.repeat(mesh.attributes, nc)
    m = _general_mesh(dim, mesh.order, corners, xyz, boundary, names, attrs, None, None)
    m.boundaries = dict(mesh.boundaries or {})
    return m
