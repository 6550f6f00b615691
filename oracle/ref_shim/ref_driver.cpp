// ref_driver.cpp — runs the reference's own hot-path classes (DGSEMIntegrator,
// ChandrashekarFlux, NavierStokesFlux, LiftingBR1, PerssonPeraireIndicator,
// ModalBasis and the BasicOperations free functions, compiled unmodified from
// the reference tree against the stand-in mfem.hpp) on a periodic Cartesian
// mesh, and exposes them through a small C interface for the parity tests.
//
// TEST INFRASTRUCTURE ONLY.  Built into oracle/_ref/ by oracle/build_ref.sh.
//
// The loops of DGSEMNonlinearForm::Mult / MultLifting
// (src/Operators/NonlinearForm/DGSEMNonlinearForm.cpp:424-849, 1302-1548) and
// the steps of DGSEMOperator::Mult (src/Operators/DGSEMOperator.cpp:60-159,
// 537-591) are restated here because those files need MFEM's parallel
// non-linear form machinery; everything they call is the reference's code.

#include "mfem.hpp"

#include "BasicOperations.hpp"
#include "ChandrashekarFlux.hpp"
#include "SlipWallBdrFaceIntegrator.hpp"
#include "SpecifiedStateBdrFaceIntegrator.hpp"
#include "SupersonicInflowBdrFaceIntegrator.hpp"
#include "SupersonicOutflowBdrFaceIntegrator.hpp"
#include "SymmetryBdrFaceIntegrator.hpp"
#include "SubsonicOutflowPBdrFaceIntegrator.hpp"
#include "SubsonicInflowRVBdrFaceIntegrator.hpp"
#include "SubsonicInflowPtTtAngBdrFaceIntegrator.hpp"
#include "RiemannInvariantBdrFaceIntegrator.hpp"
#include "NoSlipAdiabWallBdrFaceIntegrator.hpp"
#include "NoSlipIsothWallBdrFaceIntegrator.hpp"
#include "DGSEMIntegrator.hpp"
#include "ModalBasis.hpp"
#include "NavierStokesFlux.hpp"
#include "PerssonPeraireIndicator.hpp"
#ifdef PARABOLIC
#include "LiftingBR1.hpp"
#endif

#include <cstdint>

namespace mfem {

void StandInGaussLobatto(int Np, std::vector<real_t> &x, std::vector<real_t> &w)
{
    // Roots of P_N' by Newton in long double, weights 1/(N(N+1) P_N^2) on [0,1].
    const int N = Np - 1;
    x.assign(Np, 0.0);
    w.assign(Np, 0.0);
    auto leg = [&](long double t, long double &P, long double &dP) {
        long double p0 = 1.0L, p1 = t;
        if (N == 0) { P = 1.0L; dP = 0.0L; return; }
        for (int k = 1; k < N; k++) {
            long double p2 = ((2 * k + 1) * t * p1 - k * p0) / (k + 1);
            p0 = p1;
            p1 = p2;
        }
        P = p1;
        dP = N * (t * p1 - p0) / (t * t - 1.0L);
    };
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i <= N / 2; i++) {
        long double t = -1.0L;
        if (i > 0) {
            t = -std::cos(pi * i / N);
            for (int it = 0; it < 100; it++) {
                long double P, dP;
                leg(t, P, dP);
                long double d2P = (2.0L * t * dP - N * (N + 1) * P) / (1.0L - t * t);
                long double dt = dP / d2P;
                t -= dt;
                if (std::fabs(dt) < 1e-30L) break;
            }
        }
        long double P, dP;
        leg(t, P, dP);
        x[i] = (double)(0.5L * (1.0L + t));
        w[i] = (double)(1.0L / (N * (N + 1) * P * P));
        x[N - i] = 1.0 - x[i];
        w[N - i] = w[i];
    }
    if (N % 2 == 0) x[N / 2] = 0.5;
}

const IntegrationRule &IntegrationRules::Get(int geom, int order)
{
    auto *ir = new IntegrationRule();
    cache_.emplace_back(ir);
    if (geom == Geometry::POINT) {
        ir->SetSize(1);
        ir->IntPoint(0).weight = 1.0;
        return *ir;
    }
    const int n = order / 2 + 2;  // Gauss-Lobatto points exact for `order`
    std::vector<real_t> x, w;
    StandInGaussLobatto(n, x, w);
    const int d = geom == Geometry::SEGMENT ? 1 : geom == Geometry::SQUARE ? 2 : 3;
    int np = 1;
    for (int q = 0; q < d; q++) np *= n;
    ir->SetSize(np);
    for (int p = 0; p < np; p++) {
        int i = p % n, j = (p / n) % n, k = p / (n * n);
        IntegrationPoint &ip = ir->IntPoint(p);
        ip.x = x[i];
        ip.weight = w[i];
        if (d > 1) { ip.y = x[j]; ip.weight = w[i] * w[j]; }
        if (d > 2) { ip.z = x[k]; ip.weight = w[i] * w[j] * w[k]; }
        ip.index = p;
    }
    return *ir;
}

DG_FECollection::DG_FECollection(int order, int dim, int btype) : btype_(btype)
{
    fe_.dim = dim;
    fe_.order = order;
    fe_.geom = dim == 1 ? Geometry::SEGMENT : dim == 2 ? Geometry::SQUARE : Geometry::CUBE;
    std::vector<real_t> w;
    StandInGaussLobatto(order + 1, fe_.nodes1d, w);
    const int Np = order + 1;
    fe_.dof = 1;
    for (int d = 0; d < dim; d++) fe_.dof *= Np;
    fe_.nodes.SetSize(fe_.dof);
    for (int p = 0; p < fe_.dof; p++) {
        IntegrationPoint &ip = fe_.nodes.IntPoint(p);
        ip.x = fe_.nodes1d[p % Np];
        if (dim > 1) ip.y = fe_.nodes1d[(p / Np) % Np];
        if (dim > 2) ip.z = fe_.nodes1d[p / (Np * Np)];
    }
}

void Transpose(const Table &, Table &, int) {}

}  // namespace mfem

using namespace mfem;
using namespace Prandtl;

namespace {

struct RefCtx {
    int dim, N, Np, ndof, nv, ne;
    double gamma, alpha_max, alpha_min;
    std::vector<int> nbr;
    std::unique_ptr<DG_FECollection> fec, fec0;
    std::shared_ptr<Mesh> mesh;
    std::shared_ptr<ParFiniteElementSpace> vfes, fes0;
    std::shared_ptr<ParGridFunction> eta, alpha, dudx, dudy, dudz, went;
    FiniteElement fe0;
    std::unique_ptr<NavierStokesFlux> flux;
    std::unique_ptr<ChandrashekarFlux> rsolver;
    std::shared_ptr<LiftingScheme> lifting;
    std::unique_ptr<DGSEMIntegrator> integ;
    std::shared_ptr<ModalBasis> modal;
    std::unique_ptr<PerssonPeraireIndicator> indicator;
    double modalThreshold;
    double h[3];
    struct Face { int e1, e2, dir, side1, f2 = 0, orient = 0; };
    std::vector<Face> faces;
    bool general = false;  // nodal elements (ref_create_geo)
    // boundary faces (negative neighbour entries -1 - b) and the reference's
    // boundary integrator of each condition b
    struct BFace { int e, dir, side, b; };
    std::vector<BFace> bfaces;
    std::unique_ptr<BdrFaceIntegrator> bfi[16];
    double time = 0.0;
};

// Face between element a's +d face and its neighbour b's -d face; element 1
// is the lower-numbered element (MFEM's face generation order).
void build_faces(RefCtx &c)
{
    for (int e = 0; e < c.ne; e++)
        for (int d = 0; d < c.dim; d++) {
            for (int side = 0; side < 2; side++) {
                const int nb = c.nbr[e * 2 * c.dim + 2 * d + side];
                if (nb < 0) c.bfaces.push_back({e, d, side, -1 - nb});
            }
            int b = c.nbr[e * 2 * c.dim + 2 * d + 1];
            if (b < 0) continue;
            RefCtx::Face f;
            f.dir = d;
            if (e <= b) { f.e1 = e; f.e2 = b; f.side1 = 1; }
            else { f.e1 = b; f.e2 = e; f.side1 = 0; }
            c.faces.push_back(f);
        }
}

// General meshes: every face once, from its element 1 (the lower-numbered
// element), with the neighbour's face and orientation code.
void build_faces_general(RefCtx &c, const int32_t *fo)
{
    const int nf = 2 * c.dim;
    for (int e = 0; e < c.ne; e++)
        for (int f = 0; f < nf; f++) {
            const int nb = c.nbr[e * nf + f];
            if (nb < 0) {
                c.bfaces.push_back({e, f / 2, f % 2, -1 - nb});
                continue;
            }
            if (!(e < nb || (e == nb && (f & 1)))) continue;
            RefCtx::Face g;
            g.e1 = e;
            g.e2 = nb;
            g.dir = f / 2;
            g.side1 = f % 2;
            g.f2 = fo ? (fo[e * nf + f] & 7) : (f ^ 1);
            g.orient = fo ? (fo[e * nf + f] >> 3) : 0;
            c.faces.push_back(g);
        }
}

void setup_face(RefCtx &c, const RefCtx::Face &f, FaceElementTransformations &T)
{
    T.Elem1No = f.e1;
    T.Elem2No = f.e2;
    T.dim = c.dim;
    T.dir = f.dir;
    T.side1 = f.side1;
    T.T1 = c.mesh->T[f.e1];
    T.T2 = c.mesh->T[f.e2];
    if (c.general) {
        T.general = true;
        T.f2 = f.f2;
        T.orient = f.orient;
        return;
    }
    const double *h = c.h;
    const bool out_plus = f.side1 == 1;  // outward normal of element 1 along +dir
    if (c.dim == 2) {
        T.FJ.SetSize(2, 1);
        T.FJ = 0.0;
        if (f.dir == 0) T.FJ(1, 0) = out_plus ? h[1] : -h[1];
        else T.FJ(0, 0) = out_plus ? -h[0] : h[0];
    } else {
        T.FJ.SetSize(3, 2);
        T.FJ = 0.0;
        // tangents (a, b) with a x b along the outward normal
        int a = f.dir == 0 ? 1 : f.dir == 1 ? 2 : 0;
        int b = f.dir == 0 ? 2 : f.dir == 1 ? 0 : 1;
        if (!out_plus) std::swap(a, b);
        T.FJ(a, 0) = h[a];
        T.FJ(b, 1) = h[b];
    }
}

// Boundary face of element e on its +dir (side 1) or -dir (side 0) side: the
// element is element 1 and the face Jacobian points out of it.
void setup_bdr_face(RefCtx &c, const RefCtx::BFace &f, FaceElementTransformations &T)
{
    RefCtx::Face g{f.e, f.e, f.dir, f.side};
    setup_face(c, g, T);
    T.Elem2No = -1;
    T.ElementNo = f.e;
}

// DGSEMOperator::ComputeBlendingCoefficient (DGSEMOperator.cpp:60-80).
void blending(RefCtx &c, const Vector &u)
{
    c.indicator->CheckSmoothness(u);
    Array<int> ind;
    Vector d;
    for (int el = 0; el < c.ne; el++) {
        c.fes0->GetElementDofs(el, ind);
        c.eta->GetSubVector(ind, d);
        double a = 1.0 / (1.0 + std::exp(-9.21024 * (d(0) - c.modalThreshold) / c.modalThreshold));
        if (a < c.alpha_min) a = 0.0;
        else if (a > (1.0 - c.alpha_min)) a = 1.0;
        a = std::min(a, c.alpha_max);
        c.alpha->SetSubVector(ind, a);
    }
}

}  // namespace

extern "C" {

static void *create_impl(int dim, int order, int ne, const double *h, const int32_t *nbr, const double *x,
                         const int32_t *fo, double gamma, double Pr, double mu, double alpha_max, double alpha_min);

void *ref_create(int dim, int order, int ne, const double *h, const int32_t *nbr, double gamma, double Pr,
                 double mu, double alpha_max, double alpha_min)
{
    return create_impl(dim, order, ne, h, nbr, nullptr, nullptr, gamma, Pr, mu, alpha_max, alpha_min);
}

// A mesh of nodal elements: x[k * num_nodes + e * ndof + n] the DG nodes'
// coordinates, fo the face orientation codes (NULL: opposite faces, aligned).
void *ref_create_geo(int dim, int order, int ne, const int32_t *nbr, const double *x, const int32_t *fo,
                     double gamma, double Pr, double mu, double alpha_max, double alpha_min)
{
    const double h[3] = {1.0, 1.0, 1.0};
    return create_impl(dim, order, ne, h, nbr, x, fo, gamma, Pr, mu, alpha_max, alpha_min);
}

}  // extern "C"

static void *create_impl(int dim, int order, int ne, const double *h, const int32_t *nbr, const double *x,
                         const int32_t *fo, double gamma, double Pr, double mu, double alpha_max, double alpha_min)
{
    RefCtx *c = new RefCtx();
    c->dim = dim;
    c->N = order;
    c->Np = order + 1;
    c->ndof = 1;
    for (int d = 0; d < dim; d++) c->ndof *= c->Np;
    c->nv = dim + 2;
    c->ne = ne;
    c->gamma = gamma;
    c->alpha_max = alpha_max;
    c->alpha_min = alpha_min;
    for (int d = 0; d < 3; d++) c->h[d] = d < dim ? h[d] : 1.0;
    c->nbr.assign(nbr, nbr + (size_t)ne * 2 * dim);
    c->mesh = std::make_shared<Mesh>();
    c->mesh->dim = dim;
    c->mesh->ne = ne;
    c->mesh->T.resize(ne);
    c->fec.reset(new DG_FECollection(order, dim, BasisType::GaussLobatto));
    {
        std::vector<double> x1d, w1d;
        StandInGaussLobatto(order + 1, x1d, w1d);
        const size_t nn = (size_t)ne * c->ndof;
        std::vector<double> xe((size_t)dim * c->ndof);
        for (int e = 0; e < ne; e++) {
            if (!x) {
                double x0[3] = {0, 0, 0};
                c->mesh->T[e].Setup(dim, e, x0, c->h);
                continue;
            }
            for (int k = 0; k < dim; k++)
                for (int n = 0; n < c->ndof; n++) xe[(size_t)k * c->ndof + n] = x[k * nn + (size_t)e * c->ndof + n];
            c->mesh->T[e].SetupNodal(dim, e, x1d, xe.data(), c->ndof);
        }
    }
    c->vfes = std::make_shared<ParFiniteElementSpace>();
    c->vfes->mesh = c->mesh.get();
    c->vfes->fe = c->fec->FiniteElementForGeometry(Geometry::SQUARE);
    c->vfes->vdim = c->nv;
    c->vfes->ndof = c->ndof;
    c->fe0.dim = dim;
    c->fe0.order = 0;
    c->fe0.dof = 1;
    c->fes0 = std::make_shared<ParFiniteElementSpace>();
    c->fes0->mesh = c->mesh.get();
    c->fes0->fe = &c->fe0;
    c->fes0->vdim = 1;
    c->fes0->ndof = 1;
    c->eta = std::make_shared<ParGridFunction>(c->fes0.get());
    c->alpha = std::make_shared<ParGridFunction>(c->fes0.get());
    c->dudx = std::make_shared<ParGridFunction>(c->vfes.get());
    c->dudy = std::make_shared<ParGridFunction>(c->vfes.get());
    c->dudz = std::make_shared<ParGridFunction>(c->vfes.get());
    c->went = std::make_shared<ParGridFunction>(c->vfes.get());
    const double R_gas = 287.0, mu0 = 1.716e-5, mu_bulk = 2.0 / 3.0, Ts = 110.4, T0 = 273.15;
    c->flux.reset(new NavierStokesFlux(dim, gamma, Pr, mu, mu0, mu_bulk, R_gas, Ts, T0));
    c->rsolver.reset(new ChandrashekarFlux(*c->flux, gamma));
#ifdef PARABOLIC
    c->lifting = std::make_shared<LiftingBR1>();
#endif
    c->integ.reset(new DGSEMIntegrator(c->mesh, c->fes0, c->alpha, c->lifting, *c->rsolver, c->Np, gamma));
    Geometry::Type gtype = dim == 2 ? Geometry::SQUARE : Geometry::CUBE;
    c->modal = std::make_shared<ModalBasis>(*c->fec, gtype, order, dim);
    c->indicator.reset(new PerssonPeraireIndicator(c->vfes, c->fes0, c->eta, c->modal, gamma));
    c->modalThreshold = 0.5 * std::pow(10.0, -1.8 * std::pow(order, 0.25));
    c->general = x != nullptr;
    if (c->general) build_faces_general(*c, fo);
    else build_faces(*c);
    return c;
}

extern "C" {

void ref_destroy(void *h) { delete (RefCtx *)h; }

// Boundary condition `index` as the reference's integrator of `type` (1
// supersonic inflow, 2 supersonic outflow, 3 specified state, 4 slip wall,
// 5 symmetry, 6 subsonic outflow p, 7 subsonic inflow rho + V, 8 subsonic
// inflow pt, Tt, theta, phi, 9 Riemann invariant from a primitive state)
// with the constant data `state` where the type takes some.
int ref_set_boundary(void *h, int index, int type, const double *state)
{
    RefCtx &c = *(RefCtx *)h;
    if (index < 0 || index >= 16) return 1;
    const bool full = type == 1 || type == 3 || type == 9;  // a whole (conserved or primitive) state
    if (!state && (type == 10 || type == 11)) return 1;
    Vector st(c.nv);
    for (int v = 0; v < c.nv; v++) st(v) = (state && full) ? state[v] : 0.0;
    if (!state && type >= 6) return 1;
    BdrFaceIntegrator *b = nullptr;
    switch (type) {
    case 1: b = new SupersonicInflowBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, st); break;
    case 2: b = new SupersonicOutflowBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma); break;
    case 3: b = new SpecifiedStateBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, st); break;
    case 4: b = new SlipWallBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma); break;
    case 5: b = new SymmetryBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma); break;
    case 6: b = new SubsonicOutflowPBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, state[0]); break;
    case 7: {
        Vector V(c.dim);
        for (int d = 0; d < c.dim; d++) V(d) = state[1 + d];
        b = new SubsonicInflowRVBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, state[0], V);
        break;
    }
    case 8:
        b = new SubsonicInflowPtTtAngBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, state[0], state[1],
                                                       state[2], state[3], state[4]);
        break;
    case 9: b = new RiemannInvariantBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, st); break;
    case 10: {  // no-slip adiabatic wall, zero heat flux, wall velocity `state`
        Vector V(3);
        V = 0.0;
        for (int d = 0; d < c.dim; d++) V(d) = state[d];
        b = new NoSlipAdiabWallBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, 0.0, V);
        break;
    }
    case 11: {  // no-slip isothermal wall: state = {T, V}; R = 287 as in ref_create
        Vector V(3);
        V = 0.0;
        for (int d = 0; d < c.dim; d++) V(d) = state[1 + d];
        double T = state[0];
        b = new NoSlipIsothWallBdrFaceIntegrator(c.lifting, *c.rsolver, c.Np, c.time, c.gamma, 287.0, T, V);
        break;
    }
    default: return 1;
    }
    c.bfi[index].reset(b);
    return 0;
}

// DGSEMOperator::Mult.  u, dudt: byNODES vectors of the full size.
double ref_rhs(void *h, const double *u_in, double *dudt_out)
{
    RefCtx &c = *(RefCtx *)h;
    const int size = c.vfes->GetVSize();
    Vector u(size), dudt(size);
    for (int i = 0; i < size; i++) u(i) = u_in[i];
#ifdef SUBCELL_FV_BLENDING
    blending(c, u);
#endif
    const FiniteElement &fe = *c.vfes->GetFE(0);
    Array<int> vdofs, vdofs2;
    Vector el_u, el_dudt;
#ifdef PARABOLIC
    {
        // ComputeGlobalEntropyVector (DGSEMOperator.cpp:82-94)
        DenseMatrix ent_mat(c.ndof, c.nv);
        Vector el_vdofs;
        for (int el = 0; el < c.ne; el++) {
            c.vfes->GetElementVDofs(el, vdofs);
            u.GetSubVector(vdofs, el_vdofs);
            DenseMatrix vdof_mat(el_vdofs.GetData(), c.ndof, c.nv);
            Conserv2Entropy(vdof_mat, ent_mat, c.gamma, c.gamma - 1.0, 1.0 / (c.gamma - 1.0));
            c.went->SetSubVector(vdofs, ent_mat.GetData());
        }
        // MultLifting (DGSEMNonlinearForm.cpp:424-645 / 213-422)
        ParGridFunction *G[3] = {c.dudx.get(), c.dudy.get(), c.dudz.get()};
        for (int d = 0; d < 3; d++) *G[d] = 0.0;
        Vector gx, gy, gz;
        for (int el = 0; el < c.ne; el++) {
            c.vfes->GetElementVDofs(el, vdofs);
            c.went->GetSubVector(vdofs, el_u);
            if (c.dim == 3) {
                c.integ->AssembleLiftingElementVector(fe, c.mesh->T[el], el_u, gx, gy, gz);
                G[2]->AddElementVector(vdofs, gz);
            } else {
                c.integ->AssembleLiftingElementVector(fe, c.mesh->T[el], el_u, gx, gy);
            }
            G[0]->AddElementVector(vdofs, gx);
            G[1]->AddElementVector(vdofs, gy);
        }
        FaceElementTransformations T;
        for (auto &f : c.faces) {
            setup_face(c, f, T);
            c.vfes->GetElementVDofs(f.e1, vdofs);
            c.vfes->GetElementVDofs(f.e2, vdofs2);
            vdofs.Append(vdofs2);
            c.went->GetSubVector(vdofs, el_u);
            if (c.dim == 3) {
                c.integ->AssembleLiftingFaceVector(fe, fe, T, el_u, gx, gy, gz);
                G[2]->AddElementVector(vdofs, gz);
            } else {
                c.integ->AssembleLiftingFaceVector(fe, fe, T, el_u, gx, gy);
            }
            G[0]->AddElementVector(vdofs, gx);
            G[1]->AddElementVector(vdofs, gy);
        }
        // boundary faces (MultLifting's boundary-face loop)
        for (auto &f : c.bfaces) {
            setup_bdr_face(c, f, T);
            c.vfes->GetElementVDofs(f.e, vdofs);
            c.went->GetSubVector(vdofs, el_u);
            if (c.dim == 3) {
                c.bfi[f.b]->AssembleLiftingFaceVector(fe, fe, T, el_u, gx, gy, gz);
                G[2]->AddElementVector(vdofs, gz);
            } else {
                c.bfi[f.b]->AssembleLiftingFaceVector(fe, fe, T, el_u, gx, gy);
            }
            G[0]->AddElementVector(vdofs, gx);
            G[1]->AddElementVector(vdofs, gy);
        }
        // ComputeGlobalPrimitiveGradVector (DGSEMOperator.cpp:112-159)
        Vector grad_vdofs;
        for (int el = 0; el < c.ne; el++) {
            c.vfes->GetElementVDofs(el, vdofs);
            u.GetSubVector(vdofs, el_vdofs);
            DenseMatrix vdof_mat(el_vdofs.GetData(), c.ndof, c.nv);
            for (int d = 0; d < c.dim; d++) {
                G[d]->GetSubVector(vdofs, grad_vdofs);
                DenseMatrix grad_mat(grad_vdofs.GetData(), c.ndof, c.nv);
                EntropyGrad2PrimGrad(vdof_mat, grad_mat, c.gamma - 1.0, 1.0 / (c.gamma - 1.0));
                G[d]->SetSubVector(vdofs, grad_mat.GetData());
            }
        }
        // DGSEMNonlinearForm::Mult with gradients (:1302-1548 / :1070-1300)
        dudt = 0.0;
        Vector el_gx, el_gy, el_gz;
        for (int el = 0; el < c.ne; el++) {
            c.vfes->GetElementVDofs(el, vdofs);
            u.GetSubVector(vdofs, el_u);
            G[0]->GetSubVector(vdofs, el_gx);
            G[1]->GetSubVector(vdofs, el_gy);
            if (c.dim == 3) {
                G[2]->GetSubVector(vdofs, el_gz);
                c.integ->AssembleElementVector(fe, c.mesh->T[el], el_u, el_gx, el_gy, el_gz, el_dudt);
            } else {
                c.integ->AssembleElementVector(fe, c.mesh->T[el], el_u, el_gx, el_gy, el_dudt);
            }
            dudt.AddElementVector(vdofs, el_dudt);
        }
        for (auto &f : c.faces) {
            setup_face(c, f, T);
            c.vfes->GetElementVDofs(f.e1, vdofs);
            c.vfes->GetElementVDofs(f.e2, vdofs2);
            vdofs.Append(vdofs2);
            u.GetSubVector(vdofs, el_u);
            G[0]->GetSubVector(vdofs, el_gx);
            G[1]->GetSubVector(vdofs, el_gy);
            if (c.dim == 3) {
                G[2]->GetSubVector(vdofs, el_gz);
                c.integ->AssembleFaceVector(fe, fe, T, el_u, el_gx, el_gy, el_gz, el_dudt);
            } else {
                c.integ->AssembleFaceVector(fe, fe, T, el_u, el_gx, el_gy, el_dudt);
            }
            dudt.AddElementVector(vdofs, el_dudt);
        }
        for (auto &f : c.bfaces) {
            setup_bdr_face(c, f, T);
            c.vfes->GetElementVDofs(f.e, vdofs);
            u.GetSubVector(vdofs, el_u);
            G[0]->GetSubVector(vdofs, el_gx);
            G[1]->GetSubVector(vdofs, el_gy);
            if (c.dim == 3) {
                G[2]->GetSubVector(vdofs, el_gz);
                c.bfi[f.b]->AssembleFaceVector(fe, fe, T, el_u, el_gx, el_gy, el_gz, el_dudt);
            } else {
                c.bfi[f.b]->AssembleFaceVector(fe, fe, T, el_u, el_gx, el_gy, el_dudt);
            }
            dudt.AddElementVector(vdofs, el_dudt);
        }
    }
#else
    // DGSEMNonlinearForm::Mult (:647-849)
    dudt = 0.0;
    for (int el = 0; el < c.ne; el++) {
        c.vfes->GetElementVDofs(el, vdofs);
        u.GetSubVector(vdofs, el_u);
        c.integ->AssembleElementVector(fe, c.mesh->T[el], el_u, el_dudt);
        dudt.AddElementVector(vdofs, el_dudt);
    }
    {
        FaceElementTransformations T;
        for (auto &f : c.faces) {
            setup_face(c, f, T);
            c.vfes->GetElementVDofs(f.e1, vdofs);
            c.vfes->GetElementVDofs(f.e2, vdofs2);
            vdofs.Append(vdofs2);
            u.GetSubVector(vdofs, el_u);
            c.integ->AssembleFaceVector(fe, fe, T, el_u, el_dudt);
            dudt.AddElementVector(vdofs, el_dudt);
        }
        // boundary faces (DGSEMNonlinearForm::Mult's boundary-face loop)
        for (auto &f : c.bfaces) {
            setup_bdr_face(c, f, T);
            c.vfes->GetElementVDofs(f.e, vdofs);
            u.GetSubVector(vdofs, el_u);
            c.bfi[f.b]->AssembleFaceVector(fe, fe, T, el_u, el_dudt);
            dudt.AddElementVector(vdofs, el_dudt);
        }
    }
#endif
    for (int i = 0; i < size; i++) dudt_out[i] = dudt(i);
    // DGSEMOperator::Mult (DGSEMOperator.cpp:585-589)
    double lam = c.integ->GetMaxCharSpeed();
    for (auto &b : c.bfi)
        if (b) lam = std::max(lam, b->GetMaxCharSpeed());
    return lam;
}

void ref_get_blending(void *h, double *eta, double *alpha)
{
    RefCtx &c = *(RefCtx *)h;
    for (int e = 0; e < c.ne; e++) {
        if (eta) eta[e] = (*c.eta)(e);
        if (alpha) alpha[e] = (*c.alpha)(e);
    }
}

void ref_get_gradients(void *h, double *g)
{
    RefCtx &c = *(RefCtx *)h;
    const int size = c.vfes->GetVSize();
    ParGridFunction *G[3] = {c.dudx.get(), c.dudy.get(), c.dudz.get()};
    for (int d = 0; d < c.dim; d++)
        for (int i = 0; i < size; i++) g[(size_t)d * size + i] = (*G[d])(i);
}

// Pointwise reference functions.
double ref_logmean(double x, double y) { return ComputeLogMean(x, y); }

double ref_volume_flux(void *h, const double *s1, const double *s2, const double *m1, const double *m2, double *F)
{
    RefCtx &c = *(RefCtx *)h;
    Vector a(c.nv), b(c.nv), ma(c.dim), mb(c.dim), f(c.nv);
    for (int i = 0; i < c.nv; i++) { a(i) = s1[i]; b(i) = s2[i]; }
    for (int i = 0; i < c.dim; i++) { ma(i) = m1[i]; mb(i) = m2[i]; }
    double lam = c.rsolver->ComputeVolumeFlux(a, b, ma, mb, f);
    for (int i = 0; i < c.nv; i++) F[i] = f(i);
    return lam;
}

double ref_face_flux(void *h, const double *s1, const double *s2, const double *nor, double *F)
{
    RefCtx &c = *(RefCtx *)h;
    Vector a(c.nv), b(c.nv), n(c.dim), f(c.nv);
    for (int i = 0; i < c.nv; i++) { a(i) = s1[i]; b(i) = s2[i]; }
    for (int i = 0; i < c.dim; i++) n(i) = nor[i];
    double lam = c.rsolver->ComputeFaceFlux(a, b, n, f);
    for (int i = 0; i < c.nv; i++) F[i] = f(i);
    return lam;
}

// flux[v*dim + d]; dq[d*nv + v].  The state is passed by value so the
// in-place edit the reference makes to it stays local.
void ref_viscous_flux(void *h, const double *state, const double *dq, double *flux)
{
    RefCtx &c = *(RefCtx *)h;
    Vector s(c.nv), dx(c.nv), dy(c.nv), dz(c.nv);
    for (int i = 0; i < c.nv; i++) {
        s(i) = state[i];
        dx(i) = dq[i];
        dy(i) = c.dim > 1 ? dq[c.nv + i] : 0.0;
        dz(i) = c.dim > 2 ? dq[2 * c.nv + i] : 0.0;
    }
    DenseMatrix F(c.nv, c.dim);
    F = 0.0;
    if (c.dim == 3) c.flux->ComputeViscousFlux(s, dx, dy, dz, F);
    else c.flux->ComputeViscousFlux(s, dx, dy, F);
    for (int v = 0; v < c.nv; v++)
        for (int d = 0; d < c.dim; d++) flux[v * c.dim + d] = F(v, d);
}

void ref_conserv2entropy(void *h, const double *state, double *w)
{
    RefCtx &c = *(RefCtx *)h;
    Vector s(c.nv), e(c.nv);
    for (int i = 0; i < c.nv; i++) s(i) = state[i];
    Conserv2Entropy(s, e, c.gamma, c.gamma - 1.0, 1.0 / (c.gamma - 1.0));
    for (int i = 0; i < c.nv; i++) w[i] = e(i);
}

// One node, one direction, through the reference's matrix form.
void ref_entgrad2primgrad(void *h, const double *state, double *g)
{
    RefCtx &c = *(RefCtx *)h;
    DenseMatrix S(1, c.nv), G(1, c.nv);
    for (int i = 0; i < c.nv; i++) { S(0, i) = state[i]; G(0, i) = g[i]; }
    EntropyGrad2PrimGrad(S, G, c.gamma - 1.0, 1.0 / (c.gamma - 1.0));
    for (int i = 0; i < c.nv; i++) g[i] = G(0, i);
}

}  // extern "C"
