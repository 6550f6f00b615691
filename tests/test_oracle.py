"""The CPU oracle against the reference's own sources and analytic properties.

The reference ships no tests or golden data; its hot-path sources are compiled
here against a stand-in MFEM header (oracle/build_ref.sh) and their outputs are
committed as fixtures (tests/golden, make_golden.py).  These tests pin the
oracle to those fixtures, to the live reference build when it is present, and
to properties the scheme must have (freestream preservation, entropy
conservation of the flux-differencing volume term, Tadmor's shuffle condition,
log-mean accuracy).
"""
import numpy as np
import pytest

import oracle
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import golden_cases, load_golden, rel_maxnorm, rough

TOL = 1e-12  # per-RHS agreement, relative max norm


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_reference_fixture(name):
    mesh, params, z = load_golden(name)
    o = oracle.Oracle(mesh, compat=1, **params)
    dudt = o.rhs(z["u"])
    assert rel_maxnorm(dudt, z["dudt"]) < TOL
    eta, alpha = o.blending()
    np.testing.assert_allclose(eta, z["eta"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(alpha, z["alpha"], rtol=0, atol=1e-12)
    assert abs(o.max_char_speed() - float(z["lam"])) <= 1e-13 * float(z["lam"])
    if params["parabolic"]:
        assert rel_maxnorm(o.gradients(), z["grads"]) < TOL


@pytest.mark.skipif(not (oracle.ref_available(False) and oracle.ref_available(True)),
                    reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("dim,order,par", [(2, 1, 0), (2, 5, 0), (3, 1, 1), (3, 4, 1), (2, 4, 1), (3, 2, 0)])
def test_oracle_matches_live_reference(dim, order, par):
    mesh = periodic_box(dim, order, 3, 0.0, 2 * np.pi)
    u = cases.taylor_green(mesh) if dim == 3 else cases.kelvin_helmholtz(periodic_box(2, order, 3, -1, 1))
    u = rough(u, mesh, 7)
    kw = dict(parabolic=par, mu=0.01, Pr=0.71)
    o = oracle.Oracle(mesh, compat=1, **kw)
    r = oracle.Reference(mesh, parabolic=bool(par), mu=0.01, Pr=0.71)
    assert rel_maxnorm(o.rhs(u), r.rhs(u)) < TOL
    assert abs(o.max_char_speed() - r.lam) <= 1e-13 * r.lam


@pytest.mark.skipif(not oracle.ref_available(True), reason="reference build (oracle/_ref) not present")
def test_pointwise_functions_match_reference_bitwise():
    rng = np.random.default_rng(5)
    L = oracle.lib()
    R = oracle.ref_lib(True)
    mesh = periodic_box(3, 2, 2, 0, 1)
    ref = oracle.Reference(mesh, parabolic=True, mu=0.01, Pr=0.71)
    dp = oracle._dp
    for _ in range(200):
        x, y = rng.uniform(0.1, 3.0, 2)
        y = x * np.exp(rng.choice([1e-6, 1e-3, 0.05, 1.0]) * rng.standard_normal())
        assert L.orc_logmean(x, y) == R.ref_logmean(x, y)
        s1 = np.array([rng.uniform(0.5, 2), *rng.normal(0, 1, 3), 0.0])
        s2 = np.array([rng.uniform(0.5, 2), *rng.normal(0, 1, 3), 0.0])
        for s in (s1, s2):
            s[4] = rng.uniform(2, 5) / 0.4 + 0.5 * (s[1] ** 2 + s[2] ** 2 + s[3] ** 2) / s[0]
        m1 = rng.normal(0, 1, 3)
        m2 = rng.normal(0, 1, 3)
        Fo, Fr = np.zeros(5), np.zeros(5)
        lo = L.orc_volume_flux(3, 1.4, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), m1.ctypes.data_as(dp),
                               m2.ctypes.data_as(dp), Fo.ctypes.data_as(dp))
        lr = R.ref_volume_flux(ref.h, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), m1.ctypes.data_as(dp),
                               m2.ctypes.data_as(dp), Fr.ctypes.data_as(dp))
        assert lo == lr and np.array_equal(Fo, Fr)
        lo = L.orc_face_flux(3, 1.4, 1, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), m1.ctypes.data_as(dp),
                             Fo.ctypes.data_as(dp))
        lr = R.ref_face_flux(ref.h, s1.ctypes.data_as(dp), s2.ctypes.data_as(dp), m1.ctypes.data_as(dp),
                             Fr.ctypes.data_as(dp))
        assert lo == lr and rel_maxnorm(Fo, Fr) < 1e-15
        dq = rng.normal(0, 1, 15)
        fo, fr = np.zeros(15), np.zeros(15)
        L.orc_viscous_flux(3, 1.4, 0.71, 0.01, s1.ctypes.data_as(dp), dq.ctypes.data_as(dp), fo.ctypes.data_as(dp))
        R.ref_viscous_flux(ref.h, s1.ctypes.data_as(dp), dq.ctypes.data_as(dp), fr.ctypes.data_as(dp))
        assert rel_maxnorm(fo, fr) < 1e-15
        wo, wr = np.zeros(5), np.zeros(5)
        L.orc_conserv2entropy(3, 1.4, s1.ctypes.data_as(dp), wo.ctypes.data_as(dp))
        R.ref_conserv2entropy(ref.h, s1.ctypes.data_as(dp), wr.ctypes.data_as(dp))
        assert rel_maxnorm(wo, wr) < 1e-15
        go, gr = dq[:5].copy(), dq[:5].copy()
        L.orc_entgrad2primgrad(3, 1.4, 1, s1.ctypes.data_as(dp), go.ctypes.data_as(dp))
        R.ref_entgrad2primgrad(ref.h, s1.ctypes.data_as(dp), gr.ctypes.data_as(dp))
        assert rel_maxnorm(go, gr) < 1e-14


def _logmean_exact(x, y):
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    X, Y = Decimal(x), Decimal(y)
    if X == Y:
        return float(X)
    return float((Y - X) / (Y.ln() - X.ln()))


@pytest.mark.parametrize("ratio", [1 + 1e-9, 1 + 1e-5, 1 + 1e-3, 1.0199, 1.0201, 1.5, 10.0, 1e3])
def test_logmean_accuracy(ratio):
    L = oracle.lib()
    for x in (1e-3, 0.7, 1.0, 3.0, 71.4):
        y = x * ratio
        assert abs(L.orc_logmean(x, y) - _logmean_exact(x, y)) <= 4e-15 * _logmean_exact(x, y)
        assert abs(L.orc_logmean(y, x) - _logmean_exact(x, y)) <= 4e-15 * _logmean_exact(x, y)


def test_volume_flux_consistency_symmetry_and_shuffle():
    """F#(u,u) = f(u).n, F#(a,b) = F#(b,a), (w_b - w_a).F#(a,b) = psi_b - psi_a."""
    rng = np.random.default_rng(3)
    L = oracle.lib()
    dp = oracle._dp
    g = 1.4
    for dim in (2, 3):
        nv = dim + 2
        for _ in range(50):
            def state():
                rho = rng.uniform(0.5, 2.0)
                v = rng.normal(0, 1, dim)
                p = rng.uniform(0.5, 3.0)
                return np.array([rho, *(rho * v), p / (g - 1) + 0.5 * rho * v @ v])
            a, b = state(), state()
            m = rng.normal(0, 1, dim)
            Fab, Fba, Faa = np.zeros(nv), np.zeros(nv), np.zeros(nv)
            L.orc_volume_flux(dim, g, a.ctypes.data_as(dp), b.ctypes.data_as(dp), m.ctypes.data_as(dp),
                              m.ctypes.data_as(dp), Fab.ctypes.data_as(dp))
            L.orc_volume_flux(dim, g, b.ctypes.data_as(dp), a.ctypes.data_as(dp), m.ctypes.data_as(dp),
                              m.ctypes.data_as(dp), Fba.ctypes.data_as(dp))
            L.orc_volume_flux(dim, g, a.ctypes.data_as(dp), a.ctypes.data_as(dp), m.ctypes.data_as(dp),
                              m.ctypes.data_as(dp), Faa.ctypes.data_as(dp))
            np.testing.assert_allclose(Fab, Fba, rtol=1e-14, atol=1e-14)
            rho, v = a[0], a[1:1 + dim] / a[0]
            p = (g - 1) * (a[-1] - 0.5 * rho * v @ v)
            vn = v @ m
            f = np.array([rho * vn, *(rho * v * vn + p * m), (a[-1] + p) * vn])
            np.testing.assert_allclose(Faa, f, rtol=1e-13, atol=1e-13)
            wa, wb = np.zeros(nv), np.zeros(nv)
            L.orc_conserv2entropy(dim, g, a.ctypes.data_as(dp), wa.ctypes.data_as(dp))
            L.orc_conserv2entropy(dim, g, b.ctypes.data_as(dp), wb.ctypes.data_as(dp))
            # the transform uses beta = rho/p, i.e. (g-1) times the entropy variables
            # for the entropy s*rho/(g-1); the potential is psi = rho v.n
            psi = lambda s: s[1:1 + dim] @ m  # noqa: E731
            lhs = (wb - wa) @ Fab
            assert abs(lhs - (psi(b) - psi(a))) < 1e-12 * (1 + abs(lhs))


@pytest.mark.parametrize("dim,order,par", [(2, 3, 0), (2, 4, 0), (3, 3, 1), (3, 2, 0)])
def test_freestream_preservation(dim, order, par):
    mesh = periodic_box(dim, order, 3, -1.0, 1.0)
    nn = mesh.num_nodes
    vel = [np.full(nn, 0.3 + 0.2 * d) for d in range(dim)]
    u = cases.prim_to_cons(dim, np.full(nn, 1.2), vel, np.full(nn, 0.9))
    o = oracle.Oracle(mesh, parabolic=par, mu=0.01, Pr=0.71, compat=0)
    assert np.abs(o.rhs(u)).max() < 1e-13


@pytest.mark.parametrize("dim,order", [(2, 3), (2, 4), (3, 3)])
def test_discrete_entropy_conservation(dim, order):
    """With the LLF term off and no blending, sum_i J w_i w(u_i) . du_i/dt = 0."""
    lo, hi = (0.0, 2 * np.pi)
    mesh = periodic_box(dim, order, 3, lo, hi)
    u = rough(cases.taylor_green(mesh) if dim == 3 else
              cases.isentropic_vortex(periodic_box(2, order, 3, -5, 5)), mesh, 21, 0.05, 0.01)
    if dim == 2:
        mesh = periodic_box(2, order, 3, -5, 5)
    o = oracle.Oracle(mesh, parabolic=0, blending=0, compat=0, face_dissipation=0.0)
    dudt = o.rhs(u)
    nv, nn = mesh.nv, mesh.num_nodes
    _, w1 = _gll(mesh.Np)
    wq = w1
    for _ in range(dim - 1):
        wq = np.multiply.outer(wq, w1).reshape(-1) if False else np.kron(w1, wq)
    J = np.prod(mesh.h)
    W = np.tile(wq, mesh.num_elements) * J
    L = oracle.lib()
    ent = np.zeros((nv, nn))
    s = np.zeros(nv)
    w = np.zeros(nv)
    U = u.reshape(nv, nn)
    for i in range(nn):
        s[:] = U[:, i]
        L.orc_conserv2entropy(dim, 1.4, s.ctypes.data_as(oracle._dp), w.ctypes.data_as(oracle._dp))
        ent[:, i] = w
    prod = np.sum(W * np.sum(ent * dudt.reshape(nv, nn), axis=0))
    scale = np.sum(W * np.sum(np.abs(ent * dudt.reshape(nv, nn)), axis=0))
    assert abs(prod) < 1e-12 * scale


def _gll(Np):
    from prandtl_b200.mesh import gll_nodes
    return gll_nodes(Np)


def test_compat_and_fixed_agree_on_euler_2d():
    mesh = cases.kh_mesh(4, 3)
    u = cases.kelvin_helmholtz(mesh)
    a = oracle.Oracle(mesh, compat=1).rhs(u)
    b = oracle.Oracle(mesh, compat=0).rhs(u)
    assert rel_maxnorm(a, b) < 1e-15


def test_compat_changes_navier_stokes_3d():
    mesh = cases.tgv_mesh(3, 3)
    u = rough(cases.taylor_green(mesh), mesh, 4)
    a = oracle.Oracle(mesh, parabolic=1, mu=0.01, Pr=0.71, compat=1).rhs(u)
    b = oracle.Oracle(mesh, parabolic=1, mu=0.01, Pr=0.71, compat=0).rhs(u)
    assert rel_maxnorm(a, b) > 1e-6
