"""Shared helpers for the parity tests."""
from __future__ import annotations

import glob
import os

import numpy as np

from prandtl_b200.mesh import periodic_box

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden_cases():
    # (mesh_*.npz are mesh fixtures, not right-hand-side cases)
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("mesh_"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    mesh = periodic_box(int(z["dim"]), int(z["order"]), tuple(int(v) for v in z["n"]),
                        tuple(float(v) for v in z["lo"]), tuple(float(v) for v in z["hi"]))
    params = dict(parabolic=int(z["parabolic"]), mu=float(z["mu"]), Pr=float(z["Pr"]))
    if "nbr" in z.files:  # boundary faces and their conditions
        mesh.nbr = z["nbr"].reshape(mesh.num_elements, 2 * mesh.dim)
        mesh.boundaries = {int(b): (int(t), (z["bc_data"][r, :int(n)] if int(n) else None))
                           for r, (b, t, n) in enumerate(zip(z["bc_index"], z["bc_type"], z["bc_n"]))}
    return mesh, params, {k: z[k] for k in z.files}


def rel_maxnorm(a, b):
    """max|a - b| / max|b| (the parity measure: relative error in max norm)."""
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def rough(u, mesh, seed, amp_rho=0.15, amp_e=0.03):
    rng = np.random.default_rng(seed)
    nn = mesh.num_nodes
    u = u.copy()
    u[:nn] *= 1 + amp_rho * rng.standard_normal(nn)
    u[(mesh.nv - 1) * nn:] *= 1 + amp_e * rng.standard_normal(nn)
    return u


def smooth_state(mesh, seed=0):
    """A positive state with random smooth-free node values (every element
    rough enough that the blending switches on)."""
    rng = np.random.default_rng(seed)
    nn, dim = mesh.num_nodes, mesh.dim
    u = np.empty(mesh.size)
    u[:nn] = 1 + 0.1 * rng.random(nn)
    for d in range(dim):
        u[(1 + d) * nn:(2 + d) * nn] = 0.2 * rng.standard_normal(nn)
    u[(dim + 1) * nn:] = 2.5 + 0.1 * rng.random(nn)
    return u


# Boundary conditions of the general-geometry layouts with boundary faces:
# Mach-3-like inflow, outflow, slip wall, symmetry (2D); plus Riemann
# invariants and a subsonic pressure outflow (3D).
GEO_BCS_2D = {0: (1, [1.4, 4.2, 0.3, 8.8]), 1: (2, None), 2: (4, None), 3: (5, None)}
GEO_BCS_3D = {0: (1, [1.4, 4.2, 0.3, 0.1, 8.8]), 1: (2, None), 2: (4, None), 3: (5, None),
              4: (9, [1.0, 0.5, 0.1, 0.0, 1.0]), 5: (6, [0.9])}


def geometry_case(name):
    """General-geometry meshes: curved (a warped box, degree-N elements;
    twisted: the displacement's direction varies),
    skewed (an affine shear), perturbed (bilinear / trilinear elements with
    randomly moved vertices), rotated (element frames rotated, so that faces
    meet in other orientations, as in an unstructured mesh), and boundary
    layouts of perturbed boxes."""
    from prandtl_b200 import geometry as G
    from prandtl_b200.mesh import periodic_box
    if name == "warped2d":
        return G.warped(periodic_box(2, 3, (4, 5), 0.0, 1.0), 0.04)
    if name == "skewed2d":
        return G.skewed(periodic_box(2, 4, (5, 4), 0.0, 1.0), 0.4)
    if name == "perturbed2d":
        return G.perturbed_box(2, 3, (4, 5), 0.0, 1.0, 0.3, seed=1)
    if name == "rotated2d":
        return G.rotate_frames(G.perturbed_box(2, 3, (4, 5), 0.0, 1.0, 0.3, seed=1), [0, 3, 5, 7, 8, 12], seed=2)
    if name == "boundary2d":
        return G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=5, bdr=[(0, 1), (2, 3)], boundaries=GEO_BCS_2D)
    if name == "warped3d":
        return G.warped(periodic_box(3, 2, (3, 4, 3), 0.0, 1.0), 0.03)
    if name == "twisted3d":
        # the displacement turns from node to node: the pointwise metric terms
        # miss the discrete metric identities (no free-stream preservation)
        return G.warped(periodic_box(3, 3, (3, 4, 3), 0.0, 1.0), 0.03, twist=0.8)
    if name == "perturbed3d":
        return G.perturbed_box(3, 3, (3, 3, 3), 0.0, 1.0, 0.25, seed=3)
    if name == "rotated3d":
        return G.rotate_frames(G.perturbed_box(3, 2, (3, 3, 3), 0.0, 1.0, 0.25, seed=3), [0, 4, 9, 13, 20], seed=4)
    if name == "boundary3d":
        return G.perturbed_box(3, 2, (3, 3, 4), 0.0, 1.0, 0.25, seed=6, bdr=[(0, 1), (2, 3), (4, 5)],
                               boundaries=GEO_BCS_3D)
    raise KeyError(name)


GEO_CASES = ["warped2d", "skewed2d", "perturbed2d", "rotated2d", "boundary2d", "warped3d", "twisted3d",
             "perturbed3d", "rotated3d", "boundary3d"]


GEO_BCS_NS_2D = {0: (1, [1.4, 0.42, 0.03, 2.6]), 1: (2, None), 2: (3, [1.3, 0.2, 0.0, 2.4]), 3: (2, None)}


def ns_geometry_case(name):
    """Navier-Stokes layouts: the periodic general meshes and a perturbed
    channel with inflow, outflow and a prescribed state."""
    if name == "boundary2d_ns":
        from prandtl_b200 import geometry as G
        return G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=5, bdr=[(0, 1), (2, 3)], boundaries=GEO_BCS_NS_2D)
    if name in ("walls2d_ns", "subsonic2d_ns", "riemann2d_ns", "walls3d_ns"):
        return _ns_channel(name)
    return geometry_case(name)


GEO_BCS_NS_WALLS_2D = {0: (1, [1.4, 0.42, 0.03, 2.6]), 1: (2, None), 2: (10, [0.0, 0.0]),
                       3: (11, [0.0035, 0.1, 0.0])}
GEO_BCS_NS_SUBSONIC_2D = {0: (8, [3.5, 1.3, 2.0, 10.0, 0.0]), 1: (6, [0.95]), 2: (7, [1.2, 0.3, 0.0]),
                          3: (10, [0.0, 0.0])}
# the Riemann invariants (fixed operator only: the reference's NS lifting
# flux for them reads a normal left by an earlier face)
GEO_BCS_NS_RIEMANN_2D = {0: (9, [1.0, 0.3, 0.0, 1.0]), 1: (9, [1.0, 0.3, 0.0, 1.0]), 2: (10, [0.0, 0.0]),
                         3: (10, [0.0, 0.0])}
GEO_BCS_NS_WALLS_3D = {0: (1, [1.4, 0.42, 0.03, 0.0, 2.6]), 1: (2, None), 2: (10, [0.0, 0.0, 0.0]),
                       3: (11, [0.0035, 0.1, 0.0, 0.0]), 4: (6, [0.95]), 5: (7, [1.2, 0.3, 0.0, 0.0])}


def _ns_channel(name):
    from prandtl_b200 import geometry as G
    if name == "walls2d_ns":
        return G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=7, bdr=[(0, 1), (2, 3)], boundaries=GEO_BCS_NS_WALLS_2D)
    if name == "subsonic2d_ns":
        return G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=8, bdr=[(0, 1), (2, 3)],
                               boundaries=GEO_BCS_NS_SUBSONIC_2D)
    if name == "riemann2d_ns":
        return G.perturbed_box(2, 3, (5, 4), 0.0, 1.0, 0.3, seed=10, bdr=[(0, 1), (2, 3)],
                               boundaries=GEO_BCS_NS_RIEMANN_2D)
    return G.perturbed_box(3, 2, (3, 3, 4), 0.0, 1.0, 0.25, seed=9, bdr=[(0, 1), (2, 3), (4, 5)],
                           boundaries=GEO_BCS_NS_WALLS_3D)


NS_GEO_CASES = ["warped2d", "perturbed2d", "rotated2d", "warped3d", "twisted3d", "perturbed3d", "rotated3d",
                "boundary2d_ns", "walls2d_ns", "subsonic2d_ns", "walls3d_ns"]


def node_jacobian(mesh):
    """det of the Jacobian at every node of a general mesh: the LGL derivative
    matrix applied to each element's node coordinates (the element map is the
    degree-N interpolant of its nodes)."""
    from prandtl_b200.mesh import gll_nodes
    dim, Np, ne = mesh.dim, mesh.Np, mesh.num_elements
    x, _ = gll_nodes(Np)
    bw = np.array([1.0 / np.prod([x[l] - x[m] for m in range(Np) if m != l]) for l in range(Np)])
    D = np.zeros((Np, Np))
    for i in range(Np):
        for l in range(Np):
            if l != i:
                D[i, l] = bw[l] / bw[i] / (x[i] - x[l])
        D[i, i] = -D[i].sum()
    X = np.asarray(mesh.coords).reshape((dim, ne) + (Np,) * dim)   # [k, e, (z,) y, x]
    # A[k][d] = dX_k / dxi_d; xi_0 runs along the last axis
    A = [[np.moveaxis(np.tensordot(D, X[k], axes=([1], [dim - d])), 0, dim - d) for d in range(dim)]
         for k in range(dim)]
    if dim == 2:
        J = A[0][0] * A[1][1] - A[0][1] * A[1][0]
    else:
        J = (A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1])
             - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0])
             + A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]))
    return J.reshape(-1)


def entropy_vars(u, dim, nn, gamma=1.4):
    """Entropy variables (rows: nv) of conservative node values u (byNODES)."""
    U = u.reshape(dim + 2, nn)
    rho = U[0]
    vel = U[1:1 + dim] / rho
    vsq = np.sum(vel * vel, axis=0)
    p = (gamma - 1.0) * (U[-1] - 0.5 * rho * vsq)
    beta = rho / p
    s = np.log(p * rho ** (-gamma))
    return np.vstack([(gamma - s) / (gamma - 1.0) - 0.5 * beta * vsq, beta * vel, -beta])


def entropy_production(mesh, u, dudt):
    """(sum_i J_i w_i w(u_i) . du_i/dt, sum_i J_i w_i |w(u_i) . du_i/dt|) over
    every node, J_i the node's Jacobian determinant and w_i its LGL weight."""
    from prandtl_b200.mesh import gll_nodes
    dim, nn = mesh.dim, mesh.num_nodes
    _, w1 = gll_nodes(mesh.Np)
    wq = w1
    for _ in range(dim - 1):
        wq = np.kron(w1, wq)
    W = np.tile(wq, mesh.num_elements) * node_jacobian(mesh)
    local = np.sum(entropy_vars(u, dim, nn) * np.asarray(dudt).reshape(dim + 2, nn), axis=0)
    return float(np.sum(W * local)), float(np.sum(W * np.abs(local)))
