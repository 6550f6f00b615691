"""Mesh files of the reference's formats (MFEM v1.0, Gmsh 2.2 ASCII) read into
the neighbour table (prandtl_b200.meshio).

Files written here from box meshes, with shuffled element and vertex
numbers and rotated or mirrored corner orders, must read back as the same
mesh; the reference's own mesh files are read when its source tree is
present (they do not travel with the repository)."""
import os

import numpy as np
import pytest

import prandtl_b200 as pb
from prandtl_b200 import meshio
from prandtl_b200.mesh import box, gll_nodes, periodic_box

CORNERS = meshio._CORNER_BITS


def _reference_tree():
    """The reference tree: PRANDTL_REFERENCE, else where oracle/build_ref.sh
    found it (it records that in oracle/_ref/REFERENCE_TREE); '' when unknown."""
    if os.environ.get("PRANDTL_REFERENCE"):
        return os.environ["PRANDTL_REFERENCE"]
    rec = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "REFERENCE_TREE")
    return open(rec).read().strip() if os.path.exists(rec) else ""


REF_CASES = os.path.join(_reference_tree(), "TestCases")


def grid_points(mesh):
    """Vertex grid of a box mesh: index of grid point (i, j, k) and its
    coordinates; element corners by _CORNER_BITS."""
    n = [v + 1 for v in mesh.n]

    def pid(idx):
        out, stride = 0, 1
        for d in range(mesh.dim):
            out = out + idx[d] * stride
            stride *= n[d]
        return out
    coords = np.empty((int(np.prod(n)), mesh.dim))
    for flat in range(coords.shape[0]):
        r, idx = flat, []
        for d in range(mesh.dim):
            idx.append(r % n[d])
            r //= n[d]
        coords[flat] = [mesh.lo[d] + idx[d] * mesh.h[d] for d in range(mesh.dim)]
    return pid, coords


def element_corners(mesh, pid):
    cells = mesh.cells if mesh.cells is not None else np.arange(mesh.num_elements)
    out = []
    for c in cells:
        r, idx = int(c), []
        for d in range(mesh.dim):
            idx.append(r % mesh.n[d])
            r //= mesh.n[d]
        out.append([pid([idx[d] + bits[d] for d in range(mesh.dim)]) for bits in CORNERS[mesh.dim]])
    return np.array(out)


def boundary_faces(mesh, corners):
    """(attribute, corner vertex list) of every boundary face."""
    faces = []
    for e in range(mesh.num_elements):
        for d in range(mesh.dim):
            for side in (0, 1):
                nb = mesh.nbr[e, 2 * d + side]
                if nb < 0:
                    sel = [k for k in range(2 ** mesh.dim) if CORNERS[mesh.dim][k][d] == side]
                    faces.append((int(-nb), [int(corners[e, k]) for k in sel]))
    return faces


def rotate(corners, dim, rng):
    """A rotated or mirrored listing of each element's corners."""
    out = corners.copy()
    for e in range(len(corners)):
        if dim == 2:
            cyc = [0, 1, 2, 3]
            r = rng.integers(4)
            seq = cyc[r:] + cyc[:r]
            if rng.integers(2):
                seq = seq[::-1]
            out[e] = corners[e, seq]
        else:                       # quarter turns about z keep bottom then top
            r = rng.integers(4)
            bot = [0, 1, 2, 3][r:] + [0, 1, 2, 3][:r]
            out[e] = corners[e, bot + [k + 4 for k in bot]]
    return out


def write_gmsh(path, mesh, rng, names=None, info=None):
    pid, coords = grid_points(mesh)
    corners = element_corners(mesh, pid)
    bfaces = boundary_faces(mesh, corners)
    perm = rng.permutation(mesh.num_elements)             # file element i = mesh element perm[i]
    node_ids = rng.permutation(np.arange(7, 7 + 3 * len(coords)))[:len(coords)]   # sparse 1-based ids
    listed = rotate(corners[perm], mesh.dim, rng)
    if info is not None:
        info.update(listed=listed, coords=coords)
    dom, bnd = (3, 1) if mesh.dim == 2 else (5, 3)
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat"]
    if names:
        lines += ["$PhysicalNames", str(len(names))]
        lines += [f'{mesh.dim - 1} {a} "{nm}"' for nm, a in names.items()]
        lines += ["$EndPhysicalNames"]
    lines += ["$Nodes", str(len(coords))]
    for k in rng.permutation(len(coords)):
        xyz = list(coords[k]) + [0.0] * (3 - mesh.dim)
        lines.append(f"{node_ids[k]} " + " ".join(f"{v:.17g}" for v in xyz))
    lines += ["$EndNodes", "$Elements", str(1 + len(bfaces) + len(listed))]
    eid = 1
    lines.append(f"{eid} 15 2 0 1 {node_ids[0]}")     # a point entity, ignored
    for a, fv in bfaces:
        eid += 1
        lines.append(f"{eid} {bnd} 2 {a} {a} " + " ".join(str(node_ids[v]) for v in fv))
    for c in listed:
        eid += 1
        lines.append(f"{eid} {dom} 2 99 1 " + " ".join(str(node_ids[v]) for v in c))
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return perm


def same_mesh(read, orig, perm):
    """read element i is orig element perm[i]: same cells, neighbours and
    boundary entries."""
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    assert read.dim == orig.dim and tuple(read.n) == tuple(orig.n)
    np.testing.assert_allclose(read.h, orig.h, rtol=1e-13)
    np.testing.assert_allclose(read.lo, orig.lo, atol=1e-13)
    oc = orig.cells if orig.cells is not None else np.arange(orig.num_elements)
    assert np.array_equal(read.cells, oc[perm])
    on = orig.nbr[perm].astype(np.int64)
    expect = np.where(on >= 0, inv[np.maximum(on, 0)], on)
    assert np.array_equal(read.nbr, expect)
    np.testing.assert_allclose(read.node_coords(), orig.node_coords(perm), atol=1e-12)


@pytest.mark.parametrize("dim", [2, 3])
def test_gmsh_round_trip(tmp_path, dim):
    rng = np.random.default_rng(dim)
    n = (6, 4) if dim == 2 else (4, 3, 3)
    keep = np.ones(n, dtype=bool)
    keep[:2, :2] = False                                   # a step
    bdr = [(0, 1), (2, 3), (2, 3)][:dim]                   # a Gmsh file has no periodic sides here
    orig = box(dim, 2, n, 0.0, [3.0, 2.0, 1.5][:dim], bdr=bdr, keep=keep, cut=4)
    names = {"inflow": 1, "outflow": 2, "bottom": 3, "top": 4, "step": 5}
    path = str(tmp_path / "m.msh")
    perm = write_gmsh(path, orig, rng, names)
    m = meshio.read_mesh(path, 2)
    same_mesh(m, orig, perm)
    assert m.boundary_names == {k: v - 1 for k, v in names.items()}
    assert len(m.reoriented) > 0 and np.all(m.attributes == 99)


def write_mfem_periodic(path, mesh):
    """A periodic MFEM v1.0 mesh: topological vertices identified across the
    periodic sides, coordinates in a discontinuous L2_T1 P1 nodes section."""
    n = mesh.n
    def vid(idx):
        out, stride = 0, 1
        for d in range(mesh.dim):
            out += (idx[d] % n[d]) * stride
            stride *= n[d]
        return out
    rows, nodes = [], []
    for e in range(mesh.num_elements):
        r, idx = e, []
        for d in range(mesh.dim):
            idx.append(r % n[d])
            r //= n[d]
        cs = [vid([idx[d] + b[d] for d in range(mesh.dim)]) for b in CORNERS[mesh.dim]]
        rows.append(f"1 {3 if mesh.dim == 2 else 5} " + " ".join(map(str, cs)))
        for lex in range(2 ** mesh.dim):                   # corners in lexicographic order
            nodes.append(" ".join(f"{mesh.lo[d] + (idx[d] + ((lex >> d) & 1)) * mesh.h[d]:.17g}"
                                  for d in range(mesh.dim)))
    text = ["MFEM mesh v1.0", "", "# a comment", "dimension", str(mesh.dim), "", "elements", str(len(rows))]
    text += rows + ["", "boundary", "0", "", "vertices", str(int(np.prod(n))), "", "nodes",
                    "FiniteElementSpace", f"FiniteElementCollection: L2_T1_{mesh.dim}D_P1",
                    f"VDim: {mesh.dim}", "Ordering: 1", ""] + nodes
    with open(path, "w") as f:
        f.write("\n".join(text) + "\n")


@pytest.mark.parametrize("dim,n", [(2, (3, 4)), (3, (3, 4, 3))])
def test_mfem_periodic(tmp_path, dim, n):
    orig = periodic_box(dim, 3, n, -1.0, 1.0)
    path = str(tmp_path / "p.mesh")
    write_mfem_periodic(path, orig)
    m = meshio.read_mesh(path, 3)
    same_mesh(m, orig, np.arange(orig.num_elements))
    assert len(m.reoriented) == 0 and m.boundary_names == {}


def write_mfem_bounded(path, mesh, rng):
    """An MFEM v1.0 mesh with vertex coordinates and boundary elements,
    elements shuffled; returns the permutation (file element i = perm[i])."""
    pid, coords = grid_points(mesh)
    corners = element_corners(mesh, pid)
    bfaces = boundary_faces(mesh, corners)
    perm = rng.permutation(mesh.num_elements)
    geom = 3 if mesh.dim == 2 else 5
    text = ["MFEM mesh v1.0", "", "dimension", str(mesh.dim), "", "elements", str(len(perm))]
    text += [f"7 {geom} " + " ".join(map(str, corners[e])) for e in perm]
    text += ["", "boundary", str(len(bfaces))]
    text += [f"{a} {geom - 2} " + " ".join(map(str, fv)) for a, fv in bfaces]
    text += ["", "vertices", str(len(coords)), str(mesh.dim)]
    text += [" ".join(f"{v:.17g}" for v in x) for x in coords]
    with open(path, "w") as f:
        f.write("\n".join(text) + "\n")
    return perm


@pytest.mark.parametrize("dim", [2, 3])
def test_mfem_bounded(tmp_path, dim):
    rng = np.random.default_rng(20 + dim)
    n = (5, 3) if dim == 2 else (3, 3, 2)
    keep = np.ones(n, dtype=bool)
    keep[-1, -1] = False
    orig = box(dim, 2, n, -1.0, 1.0, bdr=[(0, 1), (2, 3), (0, 1)][:dim], keep=keep, cut=4)
    path = str(tmp_path / "b.mesh")
    perm = write_mfem_bounded(path, orig, rng)
    m = meshio.read_mesh(path, 2)
    same_mesh(m, orig, perm)
    assert m.boundary_names == {str(a): a - 1 for a in range(1, 6)}
    assert np.all(m.attributes == 7) and len(m.reoriented) == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_refinement(dim):
    """Two refinements of a 3 x 2 (x 2) box with boundaries equal the 12 x 8
    (x 8) box under the children's numbering."""
    n = (3, 2, 2)[:dim]
    bdr = [(0, 1), None, (2, 3)][:dim]
    coarse = box(dim, 1, n, 0.0, 1.0, bdr=bdr)
    coarse.cells = np.arange(coarse.num_elements)
    fine = box(dim, 1, tuple(4 * v for v in n), 0.0, 1.0, bdr=bdr)
    m = meshio.refine_mesh(meshio.refine_mesh(coarse))
    perm = np.asarray(m.cells)                             # refined element i = fine element cells[i]
    assert sorted(perm.tolist()) == list(range(fine.num_elements))
    same_mesh(m, fine, perm)


def test_rejections(tmp_path):
    rng = np.random.default_rng(1)
    orig = box(2, 1, (3, 2), 0.0, 1.0, bdr=[(0, 1), (2, 3)])
    path = str(tmp_path / "m.msh")
    write_gmsh(path, orig, rng)
    text = open(path).read()
    lines = text.splitlines()
    i = lines.index("$Nodes") + 2
    r = lines[i].split()
    lines[i] = " ".join([r[0], str(float(r[1]) + 0.01)] + r[2:])      # skew one vertex
    open(path, "w").write("\n".join(lines))
    with pytest.raises(ValueError, match="box|sizes|grid"):
        meshio.read_mesh(path, 1, general=False)
    assert meshio.read_mesh(path, 1).coords is not None  # read as a general-geometry mesh
    open(path, "w").write(text.replace("$MeshFormat\n2.2 0 8", "$MeshFormat\n2.2 1 8"))
    with pytest.raises(ValueError, match="ASCII"):
        meshio.read_mesh(path, 1)
    open(path, "w").write(text.replace("$Nodes", "$Knots").replace("$EndNodes", "$EndKnots"))
    with pytest.raises(ValueError, match="Nodes"):
        meshio.read_mesh(path, 1)
    open(path, "w").write(text.replace(" 15 2 0 1 ", " 9 2 0 1 "))   # a second-order triangle
    with pytest.raises(ValueError, match="element type 9"):
        meshio.read_mesh(path, 1)
    # a boundary face with no boundary element
    keep = [ln for ln in text.splitlines() if not (len(ln.split()) == 7 and ln.split()[1] == "1")]
    open(path, "w").write("\n".join(keep))
    with pytest.raises(ValueError, match="without a boundary element"):
        meshio.read_mesh(path, 1)
    pmesh = periodic_box(2, 1, (3, 3), 0.0, 1.0)
    p2 = str(tmp_path / "p.mesh")
    write_mfem_periodic(p2, pmesh)
    ptext = open(p2).read()
    open(p2, "w").write(ptext.replace("L2_T1_2D_P1", "H1_2D_P2"))
    with pytest.raises(ValueError, match="curved"):
        meshio.read_mesh(p2, 1)


def ref_file(rel):
    path = os.path.join(REF_CASES, rel)
    if not os.path.exists(path):
        pytest.skip("the reference's test cases are not present")
    return path


def test_reference_periodic_meshes():
    """IsentropicVortex.mesh with ser_ref_levels = 3 (its configuration) is
    the periodic 24 x 24 box on [-1, 1]^2."""
    for rel in ("Euler/2D/IsentropicVortex/IsentropicVortex.mesh",
                "Euler/2D/KelvinHelmholtzInstability/KelvinHelmholtzInstability.mesh"):
        m = meshio.read_mesh(ref_file(rel), 3, refine=3)
        fine = periodic_box(2, 3, 24, -1.0, 1.0)
        same_mesh(m, fine, np.asarray(m.cells))


def test_reference_gmsh_meshes():
    m = meshio.read_mesh(ref_file("NavierStokes/2D/LidDrivenCavity/LidDrivenCavity.msh"), 3)
    assert tuple(m.n) == (16, 16) and m.boundary_names == {"bottom": 0, "right": 1, "lid": 2, "left": 3}
    full = box(2, 3, 16, 0.0, 2.0, bdr=[(3, 1), (0, 2)])
    same_mesh(m, full, np.asarray(m.cells))
    m = meshio.read_mesh(ref_file("Euler/2D/DoubleMachReflection/DoubleMachReflection.msh"), 3)
    assert tuple(m.n) == (384, 96)
    nb = m.boundary_names
    x0 = m.node_coords(np.arange(m.num_elements))[0].reshape(m.num_elements, -1).min(axis=1)
    bottom = m.nbr[:, 2]
    on = bottom < 0
    assert np.all(bottom[on & (x0 < 1 / 6 - 1e-9)] == -1 - nb["bottom1"])
    assert np.all(bottom[on & (x0 > 1 / 6 - 1e-9)] == -1 - nb["bottom2"])
    m = meshio.read_mesh(ref_file("Euler/2D/BackwardFacingStep/BackwardFacingStep.msh"), 2)
    assert m.num_elements == 35000 and len(m.reoriented) > 0
    for rel, why in (("Euler/2D/ForwardFacingStep/ForwardFacingStep.msh", "sizes"),
                     ("Euler/2D/Ramp/Ramp15deg_v2.msh", "axis-aligned"),
                     ("Euler/2D/Nagashima_Ramjet/TR0/Nagashima_TR0_11kQuad_v2.msh", "box")):
        with pytest.raises(ValueError, match=why):
            meshio.read_mesh(ref_file(rel), 2, general=False)


def test_read_mesh_runs_in_the_oracle(tmp_path):
    """A shuffled, rotated Gmsh copy of a channel with a step gives the same
    right-hand side as the box it came from (permuted), in the oracle."""
    import oracle
    from test_boundaries import uniform
    rng = np.random.default_rng(5)
    keep = np.ones((6, 4), dtype=bool)
    keep[:2, :1] = False
    orig = box(2, 2, (6, 4), 0.0, [3.0, 2.0], bdr=[(0, 1), (2, 3)], keep=keep, cut=2)
    path = str(tmp_path / "c.msh")
    perm = write_gmsh(path, orig, rng, {"in": 1, "out": 2, "wall": 3, "top": 4})
    m = meshio.read_mesh(path, 2)
    fs = [1.0, 2.0, 0.0, 1.0 / 0.4 + 0.5 * 4.0]
    conds = {"in": (pb.BC_SUPERSONIC_INFLOW, fs), "out": (pb.BC_SUPERSONIC_OUTFLOW, None),
             "wall": (pb.BC_SLIP_WALL, None), "top": (pb.BC_SLIP_WALL, None)}
    m.boundaries = {m.boundary_names[k]: v for k, v in conds.items()}
    orig.boundaries = {i: conds[k] for k, i in {"in": 0, "out": 1, "wall": 2, "top": 3}.items()}
    u0 = uniform(orig, vel=(2.0, 0.0))
    x = orig.node_coords()
    u0 = u0.reshape(4, -1)
    u0[0] *= 1.0 + 0.05 * np.sin(2.0 * x[0]) * np.cos(3.0 * x[1])
    u0 = u0.reshape(-1)
    nd = orig.ndof
    um = u0.reshape(4, orig.num_elements, nd)[:, perm].reshape(-1)
    reo = np.zeros(m.num_elements, dtype=bool)
    reo[m.reoriented] = True
    assert reo.any()
    # reoriented elements keep the box frame here, so node orders agree
    r0 = oracle.Oracle(orig, compat=0).rhs(u0).reshape(4, orig.num_elements, nd)[:, perm]
    r1 = oracle.Oracle(m, compat=0).rhs(um).reshape(4, m.num_elements, nd)
    assert np.max(np.abs(r1 - r0)) <= 1e-12 * np.max(np.abs(r0))



@pytest.mark.parametrize("dim", [2, 3])
def test_reference_node_order(tmp_path, dim):
    """Fields move between the reference's per-element node order (each
    element's own frame from its listed corners, LGL nodes lexicographic)
    and this mesh's: node coordinates computed in the file frames match."""
    from prandtl_b200.mesh import gll_nodes
    rng = np.random.default_rng(7 + dim)
    n = (4, 3) if dim == 2 else (3, 2, 2)
    orig = box(dim, 3, n, 0.0, [2.0, 1.5, 1.0][:dim], bdr=[(0, 1), (2, 3), (2, 3)][:dim])
    info = {}
    write_gmsh(str(tmp_path / "f.msh"), orig, rng, info=info)
    m = meshio.read_mesh(str(tmp_path / "f.msh"), 3)
    assert len(m.reoriented) > 0
    x1, _ = gll_nodes(m.Np)
    Np = m.Np
    want = np.empty((dim, m.num_elements, Np ** dim))
    for e in range(m.num_elements):
        c = info["coords"][info["listed"][e]]                  # listed corners, file order
        axes = [c[1] - c[0], c[3] - c[0]] + ([c[4] - c[0]] if dim == 3 else [])
        for i in range(Np ** dim):
            p = c[0].copy()
            for a in range(dim):
                p = p + x1[(i // Np ** a) % Np] * axes[a]
            want[:, e, i] = p
    ours = m.node_coords().reshape(dim, m.num_elements, -1)
    got = meshio.to_reference_order(m, ours)
    np.testing.assert_allclose(got, want, atol=1e-12)
    np.testing.assert_allclose(meshio.from_reference_order(m, want), ours, atol=1e-12)
    with pytest.raises(ValueError, match="frames"):
        meshio.node_permutation(meshio.refine_mesh(m))


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("parabolic", [0, 1])
def test_gpu_read_mesh_matches_oracle(tmp_path, compat, parabolic, dim, cuda_device):
    """The operator on a mesh read from a shuffled, rotated Gmsh file
    (elements in file order, a step cut out, named boundaries) against the
    oracle on the same mesh, Euler with a slip wall and Navier-Stokes with
    no-slip walls, for both operators and graph-replayed steps."""
    import torch
    import oracle
    from helpers import rel_maxnorm, rough
    from test_boundaries import uniform
    rng = np.random.default_rng(11 + parabolic + 2 * dim)
    if dim == 2:
        keep = np.ones((8, 5), dtype=bool)
        keep[:3, :2] = False
        orig = box(2, 3, (8, 5), 0.0, [4.0, 2.5], bdr=[(0, 1), (2, 3)], keep=keep, cut=2)
        order = 3
    else:                       # hexahedra, every side bounded, a step cut out
        keep = np.ones((5, 3, 3), dtype=bool)
        keep[:2, :1, :] = False
        orig = box(3, 2, (5, 3, 3), 0.0, [2.5, 1.5, 1.5], bdr=[(0, 1), (2, 3), (3, 3)], keep=keep, cut=2)
        order = 2
    path = str(tmp_path / "g.msh")
    write_gmsh(path, orig, rng, {"in": 1, "out": 2, "wall": 3, "top": 4})
    m = meshio.read_mesh(path, order)
    fs = [1.0, 2.0, 0.0, 1.0 / 0.4 + 0.5 * 4.0] if dim == 2 else [1.0, 2.0, 0.0, 0.0, 1.0 / 0.4 + 0.5 * 4.0]
    wall = (pb.BC_NOSLIP_ADIABATIC, [0.0] * dim) if parabolic else (pb.BC_SLIP_WALL, None)
    conds = {"in": (pb.BC_SUPERSONIC_INFLOW, fs), "out": (pb.BC_SUPERSONIC_OUTFLOW, None),
             "wall": wall, "top": wall}
    m.boundaries = {m.boundary_names[k]: v for k, v in conds.items()}
    kw = dict(compat=compat, parabolic=parabolic, mu=0.02 if parabolic else 0.0, Pr=0.71)
    u = rough(uniform(m, vel=(2.0, 0.0, 0.0)[:dim]), m, 4, 0.02, 0.002)
    orc = oracle.Oracle(m, **kw)
    ref = orc.rhs(u)
    op = pb.DGSEMOperator(m, **kw)
    x = torch.from_numpy(u).to(cuda_device)
    out = torch.empty_like(x)
    op.Mult(x, out)
    torch.cuda.synchronize()
    assert rel_maxnorm(out.cpu().numpy(), ref) < 1e-12
    dt = 0.2 * min(m.h) / (orc.max_char_speed() * 16)
    y = orc.rk3_step(u, dt)
    op.rk3_step(x, dt, nsteps=1, graph=True)
    torch.cuda.synchronize()
    assert rel_maxnorm(x.cpu().numpy(), y) < 1e-11
    assert op.check() == 0


# ---- general-geometry meshes (graded, skewed, unstructured) ----

def face_tables_consistent(m, period=None):
    """Every interior face node meets its neighbour's matching node (up to one
    periodic shift per face) and every neighbour points back."""
    from prandtl_b200.geometry import map_face_index
    dim, Np, N = m.dim, m.Np, m.order
    X = np.asarray(m.coords).reshape(dim, m.num_elements, m.ndof)
    fo = m.face_orient
    nfn = Np ** (dim - 1)
    for e in range(m.num_elements):
        for f in range(2 * dim):
            nb = int(m.nbr[e, f])
            if nb < 0:
                continue
            f2, o = int(fo[e, f]) & 7, int(fo[e, f]) >> 3
            assert int(m.nbr[nb, f2]) == e
            shift = None
            for t in range(nfn):
                a, b = t % Np, t // Np
                a2, b2 = map_face_index(dim, N, a, b, o)
                d = X[:, e, _fnode(dim, Np, f, a + Np * b)] - X[:, nb, _fnode(dim, Np, f2, a2 + Np * b2)]
                shift = d if shift is None else shift
                assert np.abs(d - shift).max() < 1e-9


def _fnode(dim, Np, f, t):
    d, side = divmod(f, 2)
    pos = Np - 1 if side else 0
    if dim == 2:
        return t * Np + pos if d == 0 else pos * Np + t
    if d == 0:
        return t * Np + pos
    if d == 1:
        return (t // Np) * Np * Np + pos * Np + (t % Np)
    return pos * Np * Np + t


def write_gmsh_general(path, m, rng):
    """A Gmsh file of a general mesh with straight edges: vertices from its
    corner nodes, elements listed with rotated or mirrored corners in a
    shuffled order, boundary lines with attribute b + 1."""
    dim, Np = m.dim, m.Np
    X = np.asarray(m.coords).reshape(dim, m.num_elements, m.ndof)
    lexc = [sum(((c >> q) & 1) * (Np - 1) * Np ** q for q in range(dim)) for c in range(2 ** dim)]
    nv = int(m.corners.max()) + 1
    vxyz = np.zeros((nv, 3))
    for e in range(m.num_elements):
        for c in range(2 ** dim):
            vxyz[m.corners[e, c], :dim] = X[:, e, lexc[c]]
    gorder = [sum(b << d for d, b in enumerate(bits)) for bits in meshio._CORNER_BITS[dim]]
    file_corners = m.corners[:, gorder]                # MFEM/Gmsh order
    perm = rng.permutation(m.num_elements)
    listed = rotate(file_corners[perm], dim, rng)
    from prandtl_b200.geometry import face_corner_slots
    bl = []
    for e, f in zip(*np.nonzero(m.nbr < 0)):
        bl.append((int(-m.nbr[e, f]), m.corners[e, face_corner_slots(dim, int(f))]))
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(nv)]
    lines += [f"{k + 1} " + " ".join(f"{v:.17g}" for v in vxyz[k]) for k in range(nv)]
    lines += ["$EndNodes", "$Elements", str(len(bl) + len(listed))]
    eid = 0
    for a, vs in bl:
        eid += 1
        lines.append(f"{eid} 1 2 {a} {a} " + " ".join(str(v + 1) for v in vs))
    for c in listed:
        eid += 1
        lines.append(f"{eid} 3 2 99 1 " + " ".join(str(v + 1) for v in c))
    lines.append("$EndElements")
    open(path, "w").write("\n".join(lines) + "\n")
    return perm


def test_general_gmsh_round_trip(tmp_path):
    """A perturbed (skewed, non-affine) channel written with shuffled elements
    and rotated or mirrored corner listings reads back as the same mesh: the
    oracle's right-hand side agrees node by node (matched by position)."""
    import oracle
    from prandtl_b200 import geometry as G
    bcs = {0: (1, [1.4, 4.2, 0.3, 8.8]), 1: (2, None), 2: (4, None), 3: (4, None)}
    orig = G.perturbed_box(2, 3, (6, 4), 0.0, 1.0, 0.3, seed=3, bdr=[(0, 1), (2, 3)], boundaries=bcs)
    rng = np.random.default_rng(5)
    path = str(tmp_path / "g.msh")
    perm = write_gmsh_general(path, orig, rng)
    m = meshio.read_mesh(path, 3)
    assert m.coords is not None and m.num_elements == orig.num_elements and len(m.reoriented) > 0
    face_tables_consistent(m)
    m.boundaries = {b: bcs[b] for b in bcs}
    x = m.node_coords()
    u = np.concatenate([1 + 0.2 * np.sin(3 * x[0]) * np.cos(2 * x[1]), 0.3 + 0.1 * x[1], 0.1 * x[0] - 0.05,
                        2.5 + 0.1 * np.cos(x[0] + x[1])])
    xo = orig.node_coords()
    uo = np.concatenate([1 + 0.2 * np.sin(3 * xo[0]) * np.cos(2 * xo[1]), 0.3 + 0.1 * xo[1], 0.1 * xo[0] - 0.05,
                         2.5 + 0.1 * np.cos(xo[0] + xo[1])])
    r = oracle.Oracle(m, compat=0, parabolic=0).rhs(u).reshape(4, m.num_elements, m.ndof)
    ro = oracle.Oracle(orig, compat=0, parabolic=0).rhs(uo).reshape(4, orig.num_elements, orig.ndof)
    X = x.reshape(2, m.num_elements, m.ndof)
    XO = xo.reshape(2, orig.num_elements, orig.ndof)
    for i in range(m.num_elements):
        eo = perm[i]
        for n in range(m.ndof):
            k = int(np.argmin(np.abs(XO[0, eo] - X[0, i, n]) + np.abs(XO[1, eo] - X[1, i, n])))
            assert abs(XO[0, eo, k] - X[0, i, n]) + abs(XO[1, eo, k] - X[1, i, n]) < 1e-12
            np.testing.assert_allclose(r[:, i, n], ro[:, eo, k], rtol=1e-11, atol=1e-11 * np.abs(ro).max())


def test_general_refinement():
    """Two refinements of a general mesh: 16x the elements, conforming faces,
    the same area, and the oracle runs on it."""
    import oracle
    from prandtl_b200 import geometry as G
    orig = G.perturbed_box(2, 2, (3, 4), 0.0, 1.0, 0.3, seed=2, bdr=[(0, 0), (0, 0)], boundaries={0: (2, None)})
    gm = meshio.build_general_mesh(2, 2, _file_corners(orig), _corner_xyz(orig), _bdr(orig), {"wall": 1})
    fine = meshio.refine_general(meshio.refine_general(gm))
    assert fine.num_elements == 16 * orig.num_elements
    face_tables_consistent(fine)
    _, w = gll_nodes(3)
    area = lambda mm: float(np.sum(oracle_J(mm) * np.tile(np.outer(w, w).reshape(-1), mm.num_elements)))
    assert abs(area(fine) - area(gm)) < 1e-12
    oracle.Oracle(fine, compat=0, parabolic=0)


def _file_corners(m):
    gorder = [sum(b << d for d, b in enumerate(bits)) for bits in meshio._CORNER_BITS[m.dim]]
    return np.asarray(m.corners)[:, gorder]


def _corner_xyz(m):
    dim, Np = m.dim, m.Np
    X = np.asarray(m.coords).reshape(dim, m.num_elements, m.ndof)
    gorder = [sum(b << d for d, b in enumerate(bits)) for bits in meshio._CORNER_BITS[dim]]
    lexc = [sum(((c >> q) & 1) * (Np - 1) * Np ** q for q in range(dim)) for c in gorder]
    return np.transpose(X[:, :, lexc], (1, 2, 0))


def _bdr(m):
    from prandtl_b200.geometry import face_corner_slots
    return {frozenset(int(v) for v in m.corners[e, face_corner_slots(m.dim, int(f))]): int(-m.nbr[e, f])
            for e, f in zip(*np.nonzero(m.nbr < 0))}


def oracle_J(m):
    """det of the Jacobian at every node (order-2 LGL derivative of the coordinates)."""
    from prandtl_b200.mesh import gll_nodes as g
    Np = m.Np
    x1, _ = g(Np)
    D = np.array([[_lagrange_deriv(x1, l, x1[i]) for l in range(Np)] for i in range(Np)])
    X = np.asarray(m.coords).reshape(2, m.num_elements, Np, Np)      # [k, e, j, i]
    dxi = np.einsum("il,kejl->keji", D, X)
    deta = np.einsum("jl,keli->keji", D, X)
    return (dxi[0] * deta[1] - dxi[1] * deta[0]).reshape(-1)


def _lagrange_deriv(x, l, t):
    s = 0.0
    for m_ in range(len(x)):
        if m_ == l:
            continue
        p = 1.0 / (x[l] - x[m_])
        for q in range(len(x)):
            if q != l and q != m_:
                p *= (t - x[q]) / (x[l] - x[q])
        s += p
    return s


def test_reference_general_meshes():
    """The graded forward-facing step (ser_ref_levels = 1), the 15-degree ramp
    and the unstructured ramjet read as general-geometry meshes: conforming
    face tables and, with every boundary given the free stream, a uniform
    state has a right-hand side of rounding size (free-stream preservation)."""
    import oracle
    for rel, refine, ne, names in (
            ("Euler/2D/ForwardFacingStep/ForwardFacingStep.msh", 1, 13600, {"left", "right", "top", "bottom"}),
            ("Euler/2D/Ramp/Ramp15deg_v2.msh", 0, 4802, {"inlet", "outlet", "axis", "ramp", "top"}),
            ("Euler/2D/Nagashima_Ramjet/TR0/Nagashima_TR0_11kQuad_v2.msh", 0, 10856,
             {"inlet", "outlet", "axis", "center-body", "cowl-inner", "cowl-outer", "valve"})):
        m = meshio.read_mesh(ref_file(rel), 1, refine=refine)
        assert m.coords is not None and m.num_elements == ne and set(m.boundary_names) == names
        face_tables_consistent(m)
        state = [1.4, 4.2, 0.3, 8.8]
        m.boundaries = {b: (3, state) for b in m.boundary_names.values()}
        nn = m.num_nodes
        u = np.repeat(np.array(state), nn)
        r = oracle.Oracle(m, compat=0, parabolic=0).rhs(u)
        assert np.abs(r).max() < 1e-9 * np.abs(u).max() / min(m.h)


def fixture_mesh(case, order):
    """A reference mesh from its fixture (tests/golden/make_mesh_fixtures.py),
    refined as its configuration says (the step: ser_ref_levels = 1)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", f"mesh_{case}.npz"))
    bdr = {frozenset(int(v) for v in row): int(a) for row, a in zip(z["bverts"], z["battr"])}
    names = {str(k): int(v) for k, v in zip(z["name_keys"], z["name_vals"])}
    m = meshio.build_general_mesh(int(z["dim"]), order, z["verts"].astype(np.int64), z["coords"], bdr, names,
                                  z["attrs"])
    return meshio.refine_general(m) if case == "ffs" else m


def test_mesh_fixtures_match_files():
    """The fixtures hold what the reader parses from the reference's files."""
    for case, rel, refine in (("ffs", "Euler/2D/ForwardFacingStep/ForwardFacingStep.msh", 1),
                              ("ramp", "Euler/2D/Ramp/Ramp15deg_v2.msh", 0),
                              ("ramjet", "Euler/2D/Nagashima_Ramjet/TR0/Nagashima_TR0_11kQuad_v2.msh", 0)):
        a = meshio.read_mesh(ref_file(rel), 2, refine=refine)
        b = fixture_mesh(case, 2)
        assert np.array_equal(a.coords, b.coords) and np.array_equal(a.nbr, b.nbr)
        assert np.array_equal(a.face_orient, b.face_orient) and a.boundary_names == b.boundary_names


@pytest.mark.gpu
@pytest.mark.parametrize("compat", [0, 1])
@pytest.mark.parametrize("case", ["ffs", "ramp", "ramjet"])
def test_gpu_reference_general_meshes_match_oracle(case, compat, cuda_device):
    """The graded forward-facing step, the ramp and the unstructured ramjet at
    N = 3 with Mach-3 inflow, outflow, slip walls (and the ramp's and
    ramjet's axis as a symmetry plane): right-hand side and the three stages
    of an SSP-RK3 step, GPU against the oracle."""
    import oracle
    import torch
    m = fixture_mesh(case, 3)
    free = [1.4, 4.2, 0.0, 1.0 / 0.4 + 0.5 * 1.4 * 9.0]
    kinds = {"left": 1, "inlet": 1, "right": 2, "outlet": 2, "axis": 5}
    m.boundaries = {b: ((kinds[nm], free) if kinds.get(nm) == 1 else (kinds.get(nm, 4), None))
                    for nm, b in m.boundary_names.items()}
    x = m.node_coords()
    L = max(m.hi[0] - m.lo[0], m.hi[1] - m.lo[1])
    s = np.sin(7 * x[0] / L) * np.cos(5 * x[1] / L)
    u = np.concatenate([1.4 * (1 + 0.1 * s), 4.2 * (1 + 0.05 * s), 0.3 * s, free[3] * (1 + 0.02 * s)])
    kw = dict(compat=compat, parabolic=0)
    orc = oracle.Oracle(m, **kw)
    want = orc.rhs(u)
    op = pb.DGSEMOperator(m, **kw)
    xd = torch.from_numpy(u).to(cuda_device)
    out = torch.empty_like(xd)
    op.Mult(xd, out)
    fma = oracle.Oracle(m, fma=True, **kw).rhs(u)
    rel_err = np.abs(out.cpu().numpy() - want).max() / np.abs(want).max()
    floor = np.abs(fma - want).max() / np.abs(want).max()
    assert rel_err < max(1e-12, 4 * floor)
    dt = op.cfl_dt(0.3)
    us = u
    for stage in range(3):
        w = orc.rk_stage(stage, dt, u, us)
        o = torch.empty_like(xd)
        op.rk_stage(stage, dt, xd, torch.from_numpy(us).to(cuda_device), o)
        assert np.abs(o.cpu().numpy() - w).max() / np.abs(w).max() < 1e-12
        us = w
    assert op.check() == 0
