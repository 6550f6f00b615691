"""General geometry (skewed, curved, unstructured elements) on the CPU.

The oracle's general-geometry path (``orc_set_geometry``: J and the
adjugate at every node, the subcell metrics of ComputeSubcellMetrics,
DGSEMIntegrator.cpp:1199-1304, and each face's normal out of its element 1)
is checked against
  * the reference's own DGSEMIntegrator, ChandrashekarFlux, indicator and
    boundary integrators compiled here against the stand-in MFEM header,
    whose element transformation evaluates the Jacobian of each element's
    nodal map at every integration point and whose face transformations
    carry the neighbour's face and orientation (reference-value operator,
    1e-12 relative in max norm);
  * its own box path, on box meshes given as node coordinates (1e-13);
  * itself on the same mesh with element frames rotated (the right-hand
    side is the same field with nodes renumbered, 1e-12);
  * free-stream preservation on curved 2D meshes (a uniform state has a
    right-hand side of rounding size).
The mesh tables (``connect``: neighbours and orientation codes from corner
vertices) are checked against the structured box's.
"""
import numpy as np
import pytest

import oracle
from prandtl_b200 import geometry as G
from prandtl_b200.mesh import box, periodic_box

from helpers import GEO_CASES, NS_GEO_CASES, geometry_case, ns_geometry_case, rel_maxnorm, smooth_state

REF_TOL = 1e-12


@pytest.mark.parametrize("dim,n,bdr", [(2, (4, 5), None), (3, (3, 4, 3), None), (2, (4, 3), [(0, 1), None]),
                                       (3, (3, 3, 4), [None, (0, 1), (2, 3)])])
def test_connect_reproduces_box_tables(dim, n, bdr):
    m = box(dim, 2, n, 0.0, 1.0, bdr=bdr, boundaries={b: (2, None) for b in range(4)})
    periodic = [bdr is None or bdr[d] is None for d in range(dim)]
    corners, _, _, _ = G._lattice(dim, m.n, m.lo, m.hi, periodic)
    nbr, orient = G.connect(dim, corners, G._box_boundary(dim, m, corners))
    assert np.array_equal(nbr, m.nbr)
    want = np.where(m.nbr >= 0, np.arange(2 * dim)[None, :] ^ 1, 0)
    assert np.array_equal(orient, want)


@pytest.mark.parametrize("dim", [2, 3])
def test_rotated_frames_tables_are_consistent(dim):
    base = geometry_case("perturbed2d" if dim == 2 else "perturbed3d")
    rt = G.rotate_frames(base, range(0, base.num_elements, 2), seed=7)
    N, Np = rt.order, rt.Np
    nfn = Np ** (dim - 1)
    X = rt.coords.reshape(dim, rt.num_elements, rt.ndof)
    L = np.array([1.0] * dim)
    some_non_default = False
    for e in range(rt.num_elements):
        for f in range(2 * dim):
            nb = int(rt.nbr[e, f])
            code = int(rt.face_orient[e, f])
            f2, o = code & 7, code >> 3
            assert int(rt.nbr[nb, f2]) == e
            some_non_default |= (f2 != f ^ 1) or o != 0
            d, side = divmod(f, 2)
            d2, s2 = divmod(f2, 2)
            for t in range(nfn):
                a, b = t % Np, t // Np
                a2, b2 = G.map_face_index(dim, N, a, b, o)
                n1 = _face_node(dim, Np, d, side, a + Np * b)
                n2 = _face_node(dim, Np, d2, s2, a2 + Np * b2)
                dx = X[:, e, n1] - X[:, nb, n2]
                dx -= np.round(dx / L) * L  # periodic images
                assert np.abs(dx).max() < 1e-12
    assert some_non_default


def _face_node(dim, Np, d, side, t):
    line, pos = t, (Np - 1 if side else 0)
    if dim == 2:
        return line * Np + pos if d == 0 else pos * Np + line
    if d == 0:
        return line * Np + pos
    if d == 1:
        return (line // Np) * Np * Np + pos * Np + (line % Np)
    return pos * Np * Np + line


@pytest.mark.parametrize("dim,order,n", [(2, 3, (4, 5)), (3, 2, (3, 4, 3))])
@pytest.mark.parametrize("compat", [0, 1])
def test_oracle_geometry_path_equals_box_path_on_boxes(dim, order, n, compat):
    m = periodic_box(dim, order, n, 0.0, 1.0)
    g = G.warped(m, 0.0)
    u = smooth_state(m, 3)
    a = oracle.Oracle(m, compat=compat, parabolic=0).rhs(u)
    b = oracle.Oracle(g, compat=compat, parabolic=0).rhs(u)
    assert rel_maxnorm(b, a) < 1e-13


@pytest.mark.skipif(not oracle.ref_available(False), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("name", GEO_CASES)
def test_oracle_matches_reference_on_general_geometry(name):
    g = geometry_case(name)
    u = smooth_state(g, 11)
    ref = oracle.Reference(g)
    want = ref.rhs(u)
    orc = oracle.Oracle(g, compat=1, parabolic=0)
    got = orc.rhs(u)
    assert rel_maxnorm(got, want) < REF_TOL
    eta_r, alpha_r = ref.blending()
    eta_o, alpha_o = orc.blending()
    np.testing.assert_allclose(eta_o, eta_r, rtol=1e-12, atol=1e-14)
    assert np.array_equal(alpha_o > 0, alpha_r > 0) and (alpha_o > 0).any()
    assert abs(orc.max_char_speed() - ref.lam) <= 1e-12 * ref.lam


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_rotation_invariance(dim):
    base = geometry_case("perturbed2d" if dim == 2 else "perturbed3d")
    rt = G.rotate_frames(base, range(1, base.num_elements, 3), seed=9)
    u = smooth_state(base, 5)
    # the reference-value operator's 3D face dissipation term (rho_mean dw +
    # w_mean, ChandrashekarFlux.cpp:131) is not antisymmetric under exchange
    # of the two states, so reversing a line's direction changes the subcell
    # fluxes: the invariance holds for the fixed operator in 3D
    for compat in ((0, 1) if dim == 2 else (0,)):
        a = G.permute_nodes(rt, oracle.Oracle(base, compat=compat, parabolic=0).rhs(u))
        b = oracle.Oracle(rt, compat=compat, parabolic=0).rhs(G.permute_nodes(rt, u))
        assert rel_maxnorm(b, a) < 1e-12


@pytest.mark.parametrize("name", ["warped2d", "skewed2d", "perturbed2d", "rotated2d"])
def test_oracle_free_stream_preservation_2d(name):
    g = geometry_case(name)
    nn = g.num_nodes
    u = np.empty(g.size)
    u[:nn], u[nn:2 * nn], u[2 * nn:3 * nn], u[3 * nn:] = 1.2, 0.6, -0.3, 3.0
    r = oracle.Oracle(g, compat=0, parabolic=0).rhs(u)
    assert np.abs(r).max() < 1e-11


def test_oracle_rejects_inverted_elements():
    g = geometry_case("warped2d")
    Np = g.Np
    X = g.coords.reshape(2, g.num_elements, Np, Np).copy()
    X[:, 3] = X[:, 3, :, ::-1].copy()  # element 3's nodes mirrored along its x axis
    g.coords = X.reshape(2, -1)
    with pytest.raises(ValueError):
        oracle.Oracle(g, compat=0, parabolic=0)


NS = dict(mu=0.01, Pr=0.71)


@pytest.mark.skipif(not oracle.ref_available(True), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("name", NS_GEO_CASES)
def test_oracle_navier_stokes_matches_reference_on_general_geometry(name):
    """The BR1 lifting with the adjugate at every node (LiftingBR1.cpp), the
    contravariant viscous fluxes and the central viscous face fluxes, against
    the reference's own NS build (reference-value operator: stale viscous
    state, z-direction fill)."""
    g = ns_geometry_case(name)
    u = smooth_state(g, 11)
    ref = oracle.Reference(g, parabolic=True, **NS)
    want = ref.rhs(u)
    orc = oracle.Oracle(g, compat=1, parabolic=1, **NS)
    assert rel_maxnorm(orc.rhs(u), want) < REF_TOL
    assert rel_maxnorm(orc.gradients(), ref.gradients()) < REF_TOL


@pytest.mark.parametrize("dim,order,n", [(2, 3, (4, 5)), (3, 2, (3, 4, 3))])
@pytest.mark.parametrize("compat", [0, 1])
def test_oracle_navier_stokes_geometry_path_equals_box_path(dim, order, n, compat):
    m = periodic_box(dim, order, n, 0.0, 1.0)
    u = smooth_state(m, 3)
    a = oracle.Oracle(m, compat=compat, parabolic=1, **NS)
    b = oracle.Oracle(G.warped(m, 0.0), compat=compat, parabolic=1, **NS)
    assert rel_maxnorm(b.rhs(u), a.rhs(u)) < 1e-13
    assert rel_maxnorm(b.gradients(), a.gradients()) < 1e-13


@pytest.mark.parametrize("name", ["warped2d", "skewed2d", "perturbed2d", "rotated2d", "warped3d", "perturbed3d",
                                  "rotated3d"])
def test_oracle_entropy_conservation_on_general_geometry(name):
    """With the LLF term off and no blending, the flux-differencing operator
    with mean metrics conserves entropy on a periodic mesh whose metric terms
    meet the discrete metric identities: sum_i J_i w_i w(u_i) . du_i/dt = 0;
    with the LLF term on the sum is negative.  The identities hold on every
    2D mesh, on multilinear 3D elements (the cross products of the columns
    of the Jacobian have degree 2 per direction) and on the warped meshes,
    whose displacement is one scalar field times (L_x, L_y, L_z): the
    quadratic terms of the cross products cancel, so the metric terms have
    degree N and the LGL derivative differentiates them exactly."""
    from helpers import entropy_production
    g = geometry_case(name)
    assert (g.nbr >= 0).all()
    u = smooth_state(g, 4)
    prod, scale = entropy_production(g, u, oracle.Oracle(g, parabolic=0, blending=0, compat=0,
                                                         face_dissipation=0.0).rhs(u))
    assert abs(prod) < 1e-13 * scale
    prod_d, _ = entropy_production(g, u, oracle.Oracle(g, parabolic=0, blending=0, compat=0).rhs(u))
    assert prod_d < -1e-3 * scale


def test_oracle_twisted_mesh_misses_the_metric_identities():
    """On a 3D mesh whose displacement turns from node to node the pointwise
    metric terms miss the discrete metric identities, as in the reference
    (the right-hand side still matches the reference's, GEO_CASES): a free
    stream is not kept and entropy is not conserved without dissipation."""
    from helpers import entropy_production
    g = geometry_case("twisted3d")
    nn = g.num_nodes
    u = np.empty(g.size)
    u[:nn], u[nn:2 * nn], u[2 * nn:3 * nn], u[3 * nn:4 * nn], u[4 * nn:] = 1.2, 0.6, 0.3, 0.0, 3.0
    assert np.abs(oracle.Oracle(g, compat=0, parabolic=0, blending=0).rhs(u)).max() > 1e-3
    v = smooth_state(g, 4)
    prod, scale = entropy_production(g, v, oracle.Oracle(g, parabolic=0, blending=0, compat=0,
                                                         face_dissipation=0.0).rhs(v))
    assert abs(prod) > 1e-6 * scale
