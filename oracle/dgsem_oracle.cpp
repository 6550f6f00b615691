// dgsem_oracle.cpp — CPU restatement of Prandtl's DGSEM right-hand side
// (DGSEMOperator::Mult) and SSP-RK3 step, used as the parity oracle and as the
// timed CPU baseline.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (prandtl_b200/) links or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline load it, always as the reference result.
//
// Parity status: the pointwise physics (log-mean, Chandrashekar volume and
// face fluxes, viscous flux, entropy-variable transforms) is pinned bit for
// bit against the reference's own sources compiled here with a stand-in MFEM
// header (oracle/ref_shim, built into oracle/_ref/).  The assembly loops are
// restated from the reference source cited at each function; the reference
// ships no tests, golden vectors or fixtures and cannot be linked against MFEM
// here, so those loops are not pinned against a run of the reference.
//
// Mesh model: affine, axis-aligned Cartesian elements, periodic via the
// neighbour table.  MFEM pieces the reference relies on are restated from
// their mathematics: the Gauss-Lobatto rule on [0,1], Lagrange shape values at
// the nodes (Kronecker delta), CalcOrtho face normals (|n| = face measure,
// outward from element 1), ElementTransformation::Weight / AdjugateJacobian
// of an affine map, shifted Legendre polynomials, RK3SSPSolver.
//
// Build: g++ -O3 -march=native -fopenmp -ffp-contract=off -shared -fPIC.
// -ffp-contract=off keeps every product and sum rounded as written, which is
// how the reference's pointwise functions are compiled for the pin.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/prandtl_b200.h"

namespace orc {

// ---------------------------------------------------------------------------
// Pointwise physics
// ---------------------------------------------------------------------------

// ComputeLogMean, src/BasicOperations/BasicOperations.cpp:6-12 (eps = 1e-4,
// BasicOperations.hpp:9).
static inline double logmean(double x, double y)
{
    const double eps = 1e-4;
    double xi = y / x;
    double u = (xi * (xi - 2.0) + 1.0) / (xi * (xi + 2.0) + 1);
    return (u < eps) ? (x + y) * 52.5 / (105.0 + u * (35.0 + u * (21.0 + 15.0 * u)))
                     : (y - x) / std::log(xi);
}

// ComputeSoundSpeed with b = 0, BasicOperations.cpp:52-55.
static inline double sound_speed(double p, double rho, double gamma)
{
    return std::sqrt(gamma * p / (1.0 - 0.0 * rho) / rho);
}

// ChandrashekarFlux::ComputeVolumeFlux, src/RiemannSolvers/ChandrashekarFlux.cpp:11-83.
// metric1/metric2 are the contravariant metric rows of the two nodes; their
// mean is used.  Returns lambda_max.
static double volume_flux(int dim, double gamma, const double *s1, const double *s2,
                          const double *metric1, const double *metric2, double *F)
{
    const int ne = dim + 2;
    const double gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1;
    double metric[3];
    for (int d = 0; d < dim; d++) {
        metric[d] = metric1[d];
        metric[d] += metric2[d];
        metric[d] *= 0.5;
    }
    double mom[3];
    double rho1 = s1[0], rho2 = s2[0];
    double rho_ln = logmean(rho1, rho2);
    double u1 = s1[1] / rho1, u2 = s2[1] / rho2;
    double u_mean = 0.5 * (u1 + u2);
    double V_sq1 = u1 * u1, V_sq2 = u2 * u2;
    double Vn = u_mean * metric[0];
    mom[0] = rho_ln * u_mean;
    double h_hat = -0.25 * (u1 * u1 + u2 * u2) + u_mean * u_mean;
    if (dim > 1) {
        double v1 = s1[2] / rho1, v2 = s2[2] / rho2;
        double v_mean = 0.5 * (v1 + v2);
        V_sq1 += v1 * v1;
        V_sq2 += v2 * v2;
        Vn += v_mean * metric[1];
        mom[1] = rho_ln * v_mean;
        h_hat += -0.25 * (v1 * v1 + v2 * v2) + v_mean * v_mean;
        if (dim > 2) {
            double w1 = s1[3] / rho1, w2 = s2[3] / rho2;
            double w_mean = 0.5 * (w1 + w2);
            V_sq1 += w1 * w1;
            V_sq2 += w2 * w2;
            Vn += w_mean * metric[2];
            mom[2] = rho_ln * w_mean;
            h_hat += -0.25 * (w1 * w1 + w2 * w2) + w_mean * w_mean;
        }
    }
    double p1 = gammaM1 * (s1[ne - 1] - 0.5 * rho1 * V_sq1);
    double p2 = gammaM1 * (s2[ne - 1] - 0.5 * rho2 * V_sq2);
    double lambda_max = std::sqrt(V_sq1) + sound_speed(p1, rho1, gamma);
    lambda_max = std::max(lambda_max, std::sqrt(V_sq2) + sound_speed(p2, rho2, gamma));
    double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
    double beta_ln = logmean(beta1, beta2);
    double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
    h_hat += 0.5 / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    F[0] = rho_ln * Vn;
    for (int d = 0; d < dim; d++) F[1 + d] = Vn * mom[d] + p_hat * metric[d];
    F[1 + dim] = rho_ln * Vn * h_hat;
    return lambda_max;
}

// ChandrashekarFlux::ComputeFaceFlux, ChandrashekarFlux.cpp:85-161.
// compat=1 keeps the 3D energy-dissipation term as the reference writes it
// (`rho_mean * dw + w_mean`, line 131); compat=0 uses rho_mean * dw * w_mean.
// diss_scale multiplies the local Lax-Friedrichs term (1 = reference).
static double face_flux(int dim, double gamma, int compat, double diss_scale,
                        const double *s1, const double *s2, const double *nor, double *flux)
{
    const int ne = dim + 2;
    const double gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1;
    double nn = 0.0;  // Vector::Norml2
    for (int d = 0; d < dim; d++) nn += nor[d] * nor[d];
    double nor_mag = std::sqrt(nn);
    double mom[3];
    double rho1 = s1[0], rho2 = s2[0];
    double rho_mean = 0.5 * (rho1 + rho2);
    double rho_ln = logmean(rho1, rho2);
    double drho = rho2 - rho1;
    double u1 = s1[1] / rho1, u2 = s2[1] / rho2;
    double u_mean = 0.5 * (u1 + u2);
    double du = u2 - u1;
    double V_sq1 = u1 * u1, V_sq2 = u2 * u2;
    double Vn = u_mean * nor[0];
    mom[0] = rho_ln * u_mean;
    double h_hat = -0.25 * (u1 * u1 + u2 * u2) + u_mean * u_mean;
    double diss = 0.5 * drho * u1 * u2 + rho_mean * du * u_mean;
    if (dim > 1) {
        double v1 = s1[2] / rho1, v2 = s2[2] / rho2;
        double v_mean = 0.5 * (v1 + v2);
        double dv = v2 - v1;
        V_sq1 += v1 * v1;
        V_sq2 += v2 * v2;
        Vn += v_mean * nor[1];
        mom[1] = rho_ln * v_mean;
        h_hat += -0.25 * (v1 * v1 + v2 * v2) + v_mean * v_mean;
        diss += 0.5 * drho * v1 * v2 + rho_mean * dv * v_mean;
        if (dim > 2) {
            double w1 = s1[3] / rho1, w2 = s2[3] / rho2;
            double w_mean = 0.5 * (w1 + w2);
            double dw = w2 - w1;
            V_sq1 += w1 * w1;
            V_sq2 += w2 * w2;
            Vn += w_mean * nor[2];
            mom[2] = rho_ln * w_mean;
            h_hat += -0.25 * (w1 * w1 + w2 * w2) + w_mean * w_mean;
            if (compat)
                diss += 0.5 * drho * w1 * w2 + rho_mean * dw + w_mean;
            else
                diss += 0.5 * drho * w1 * w2 + rho_mean * dw * w_mean;
        }
    }
    double p1 = gammaM1 * (s1[ne - 1] - 0.5 * rho1 * V_sq1);
    double p2 = gammaM1 * (s2[ne - 1] - 0.5 * rho2 * V_sq2);
    double lambda_max = std::sqrt(V_sq1) + sound_speed(p1, rho1, gamma);
    lambda_max = std::max(lambda_max, std::sqrt(V_sq2) + sound_speed(p2, rho2, gamma));
    double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
    double beta_ln = logmean(beta1, beta2);
    double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
    h_hat += 0.5 / beta_ln * gammaM1Inverse + p_hat / rho_ln;
    diss += 0.5 * drho * gammaM1Inverse / beta_ln + 0.5 * rho_mean * gammaM1Inverse * (1.0 / beta2 - 1.0 / beta1);
    const double lam = lambda_max * diss_scale;
    flux[0] = rho_ln * Vn - 0.5 * lam * (rho2 - rho1) * nor_mag;
    for (int d = 0; d < dim; d++)
        flux[1 + d] = Vn * mom[d] + p_hat * nor[d] - 0.5 * lam * (s2[1 + d] - s1[1 + d]) * nor_mag;
    flux[1 + dim] = rho_ln * Vn * h_hat - 0.5 * lam * diss * nor_mag;
    return lambda_max;
}

// NavierStokesFlux::ComputeViscousFlux, src/Fluxes/NavierStokesFlux.cpp:12-58
// (3D) and :60-90 (2D), constant mu, mu_bulk = 2/3 (src/Physics/Physics.hpp:34).
// dq[d*ne + v]: primitive gradient of variable v along x_d.  Output
// flux[v*dim + d]; row v = 0 (mass) is left at zero.
static void viscous_flux(int dim, double gamma, double Pr, double mu, const double *state,
                         const double *dq, double *flux)
{
    const int ne = dim + 2;
    const double gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1, PrInverse = 1.0 / Pr;
    const double mu_bulk = 2.0 / 3.0;
    // Conserv2Prim, BasicOperations.cpp:225-239 (pressure via ComputePressure).
    double prim[5];
    prim[0] = state[0];
    for (int d = 0; d < dim; d++) prim[1 + d] = state[1 + d] / state[0];
    {
        double V[3], VV = 0.0;
        for (int d = 0; d < dim; d++) V[d] = state[1 + d] / state[0];
        for (int d = 0; d < dim; d++) VV += V[d] * V[d];
        prim[ne - 1] = gammaM1 * (state[ne - 1] - 0.5 * state[0] * VV);
    }
    for (int i = 0; i < ne * dim; i++) flux[i] = 0.0;
    const double lambda = mu * gamma * PrInverse;
    const double *dqdx = dq, *dqdy = dq + ne, *dqdz = dq + 2 * ne;
    auto F = [&](int v, int d) -> double & { return flux[v * dim + d]; };
    if (dim == 3) {
        double dudx = dqdx[1], dvdx = dqdx[2], dwdx = dqdx[3];
        double dudy = dqdy[1], dvdy = dqdy[2], dwdy = dqdy[3];
        double dudz = dqdz[1], dvdz = dqdz[2], dwdz = dqdz[3];
        double div = dudx + dvdy + dwdz;
        double cv_dTdx = gammaM1Inverse / prim[0] * (dqdx[4] - prim[4] / prim[0] * dqdx[0]);
        double cv_dTdy = gammaM1Inverse / prim[0] * (dqdy[4] - prim[4] / prim[0] * dqdy[0]);
        double cv_dTdz = gammaM1Inverse / prim[0] * (dqdz[4] - prim[4] / prim[0] * dqdz[0]);
        F(1, 0) = mu * (2.0 * dudx - mu_bulk * div);
        F(2, 0) = mu * (dudy + dvdx);
        F(3, 0) = mu * (dudz + dwdx);
        F(4, 0) = prim[1] * F(1, 0) + prim[2] * F(2, 0) + prim[3] * F(3, 0) + lambda * cv_dTdx;
        F(1, 1) = mu * (dvdx + dudy);
        F(2, 1) = mu * (2.0 * dvdy - mu_bulk * div);
        F(3, 1) = mu * (dvdz + dwdy);
        F(4, 1) = prim[1] * F(1, 1) + prim[2] * F(2, 1) + prim[3] * F(3, 1) + lambda * cv_dTdy;
        F(1, 2) = mu * (dwdx + dudz);
        F(2, 2) = mu * (dwdy + dvdz);
        F(3, 2) = mu * (2.0 * dwdz - mu_bulk * div);
        F(4, 2) = prim[1] * F(1, 2) + prim[2] * F(2, 2) + prim[3] * F(3, 2) + lambda * cv_dTdz;
    } else {
        double dudx = dqdx[1], dvdx = dqdx[2];
        double dudy = dqdy[1], dvdy = dqdy[2];
        double div = dudx + dvdy;
        double cv_dTdx = gammaM1Inverse / prim[0] * (dqdx[3] - prim[3] / prim[0] * dqdx[0]);
        double cv_dTdy = gammaM1Inverse / prim[0] * (dqdy[3] - prim[3] / prim[0] * dqdy[0]);
        F(1, 0) = mu * (2.0 * dudx - mu_bulk * div);
        F(2, 0) = mu * (dudy + dvdx);
        F(3, 0) = prim[1] * F(1, 0) + prim[2] * F(2, 0) + lambda * cv_dTdx;
        F(1, 1) = mu * (dvdx + dudy);
        F(2, 1) = mu * (2.0 * dvdy - mu_bulk * div);
        F(3, 1) = prim[1] * F(1, 1) + prim[2] * F(2, 1) + lambda * cv_dTdy;
    }
}

// Conserv2Entropy, BasicOperations.cpp:134-157 (beta = rho/p here).
static void conserv2entropy(int dim, double gamma, const double *state, double *w)
{
    const int ne = dim + 2;
    const double gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1;
    double vel[3], vv = 0.0;
    for (int d = 0; d < dim; d++) vel[d] = state[1 + d] / state[0];
    for (int d = 0; d < dim; d++) vv += vel[d] * vel[d];
    double v_sq = 0.5 * vv;
    double p = gammaM1 * (state[ne - 1] - state[0] * v_sq);
    double beta = state[0] / p;
    double s = std::log(p * std::pow(state[0], -gamma));
    w[0] = (gamma - s) * gammaM1Inverse - beta * v_sq;
    for (int d = 0; d < dim; d++) w[1 + d] = beta * vel[d];
    w[ne - 1] = -beta;
}

// EntropyGrad2PrimGrad, BasicOperations.cpp:179-223, for one node and one
// direction: g holds the entropy-variable gradient on entry and the primitive
// gradient on exit.  The reference divides the momenta of its row copy in
// place (`Vector vel(state.GetData() + 1, dim); vel /= state(0);`, :190-191),
// so the density-gradient term reads velocities where it means momenta;
// compat=1 keeps that, compat=0 uses the momenta.
static void entgrad2primgrad(int dim, double gamma, int compat, const double *state_in, double *g)
{
    double state[5];
    for (int v = 0; v < dim + 2; v++) state[v] = state_in[v];
    if (compat)
        for (int d = 0; d < dim; d++) state[1 + d] = state_in[1 + d] / state_in[0];
    const int ne = dim + 2;
    const double gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1;
    double gs[5];
    for (int v = 0; v < ne; v++) gs[v] = g[v];
    double vel[3], vv = 0.0;
    for (int d = 0; d < dim; d++) vel[d] = state_in[1 + d] / state_in[0];
    for (int d = 0; d < dim; d++) vv += vel[d] * vel[d];
    double v_sq = 0.5 * vv;
    double p = gammaM1 * (state[ne - 1] - state[0] * v_sq);
    double KE = v_sq * state[0];
    if (dim == 2) {
        g[1] = p / state[0] * (gs[1] + vel[0] * gs[3]);
        g[2] = p / state[0] * (gs[2] + vel[1] * gs[3]);
        g[0] = state[0] * gs[0] - gs[3] * (KE - p * gammaM1Inverse)
             + state[0] / p * (state[1] * g[1] + state[2] * g[2]);
        g[3] = p / state[0] * (g[0] + p * gs[3]);
    } else {
        g[1] = p / state[0] * (gs[1] + vel[0] * gs[4]);
        g[2] = p / state[0] * (gs[2] + vel[1] * gs[4]);
        g[3] = p / state[0] * (gs[3] + vel[2] * gs[4]);
        g[0] = state[0] * gs[0] - gs[4] * (KE - p * gammaM1Inverse)
             + state[0] / p * (state[1] * g[1] + state[2] * g[2] + state[3] * g[3]);
        g[4] = p / state[0] * (g[0] + p * gs[4]);
    }
}

// ComputePressure, BasicOperations.cpp:31-37.
static inline double pressure(int dim, double gamma, const double *s)
{
    double V[3], VV = 0.0;
    for (int d = 0; d < dim; d++) V[d] = s[1 + d] / s[0];
    for (int d = 0; d < dim; d++) VV += V[d] * V[d];
    return (gamma - 1.0) * (s[dim + 1] - 0.5 * s[0] * VV);
}

// ComputeEntropy (Euler branch), BasicOperations.cpp:39-46.
static inline double entropy_fn(double rho, double p, double gamma)
{
    return rho > 0.0 && p > 0.0 ? rho * std::log(p * std::pow(rho, -gamma))
                                : std::numeric_limits<double>::infinity();
}

// ---------------------------------------------------------------------------
// One-dimensional operators
// ---------------------------------------------------------------------------

// Legendre P_n and P_n' on [-1,1] by the three-term recurrence.
static void legendre(int n, long double x, long double &P, long double &dP)
{
    long double p0 = 1.0L, p1 = x;
    if (n == 0) { P = 1.0L; dP = 0.0L; return; }
    for (int k = 1; k < n; k++) {
        long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
        p0 = p1;
        p1 = p2;
    }
    P = p1;
    dP = n * (x * p1 - p0) / (x * x - 1.0L);
}

// Gauss-Lobatto rule with Np points on [0,1] (what MFEM's
// IntegrationRules(0, GaussLobatto).Get(SEGMENT, 2Np-3) returns,
// DGSEMIntegrator.cpp:18-22): interior nodes are the roots of P_N', found by
// Newton in long double; weights 1/(N(N+1) P_N(x)^2) on [0,1]; the rule is
// mirrored so x[N-i] = 1 - x[i].
static void gll(int Np, std::vector<double> &x, std::vector<double> &w)
{
    const int N = Np - 1;
    x.assign(Np, 0.0);
    w.assign(Np, 0.0);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i <= N / 2; i++) {
        long double t;
        if (i == 0) {
            t = -1.0L;
        } else {
            t = -std::cos(pi * i / N);
            for (int it = 0; it < 100; it++) {
                long double P, dP;
                legendre(N, t, P, dP);
                long double d2P = (2.0L * t * dP - N * (N + 1) * P) / (1.0L - t * t);
                long double dt = dP / d2P;
                t -= dt;
                if (std::fabs(dt) < 1e-30L) break;
            }
        }
        long double P, dP;
        legendre(N, t, P, dP);
        long double wt = 1.0L / (N * (N + 1) * P * P);  // [0,1] weight
        x[i] = (double)(0.5L * (1.0L + t));
        w[i] = (double)wt;
        x[N - i] = 1.0 - x[i];
        w[N - i] = w[i];
    }
    if (N % 2 == 0) x[N / 2] = 0.5;
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------

struct Ctx {
    pdg_params p;
    int dim, N, Np, ndof, nv;
    int64_t ne, nnodes, size;
    double h[3];
    std::vector<int32_t> nbr;
    std::vector<double> x, w;           // GLL rule on [0,1]
    std::vector<double> D;              // D[i*Np + l] = l'_l(x_i)
    std::vector<double> Dhat, Dhat2;    // D + corr, 2D + corr (rows i)
    double J, adj[3], area[3];
    std::vector<double> snor[3];        // subcell normal component, interfaces 0..Np
    std::vector<double> Vinv;           // modal inverse Vandermonde, ndof x ndof
    std::vector<int> degs;              // ndof x dim 1D degrees of mode k
    std::vector<double> Vdm;            // modal Vandermonde
    std::vector<int> max_order;         // max 1D degree of mode k (filter)
    double modalThreshold;
    std::vector<double> eta, alpha;     // per element
    std::vector<double> grads;          // dim * size
    std::vector<double> went;           // entropy variables, size
    std::vector<double> facebuf;        // per (e, dir): contributions to both sides
    std::vector<double> emin;           // filter entropy bounds per element
    double max_char_speed;              // integrator running max
    double last_rhs_speed;              // max of the last RHS
    std::vector<double> k1, y1, z1;     // RK scratch
    int64_t filtered_elements;
    int64_t limited_elements;           // positivity limiter applications
    double bc[16][8] = {};              // boundary conditions: type, prescribed state
    // general geometry (orc_set_geometry): per node J and adjugate rows, the
    // subcell normals per element, direction, line and interface, and per
    // element face node the neighbour's face and matching node
    bool geo = false;
    std::vector<double> gJ, gadj;       // gJ[e*ndof + n], gadj[((e*ndof + n)*3 + r)*3 + k]
    std::vector<double> gsnor;          // [e][d][line][i = 0..Np][k]
    std::vector<int> gface;             // neighbour's face per element face
    std::vector<int> gnode;             // [e][f][t]: neighbour's node matching face node t
};

static inline int64_t idx(const Ctx &c, int v, int64_t e, int n)
{
    return (int64_t)v * c.nnodes + e * c.ndof + n;
}

// DGSEMIntegrator ctor: barycentric D, D-hat, D-hat2 (DGSEMIntegrator.cpp:41-82).
// Stored untransposed: Dhat2[i*Np+m] is what the reference reads as
// Dhat2_T(m, i) after its transpose.
static void build_derivative_matrices(Ctx &c)
{
    const int Np = c.Np;
    std::vector<double> wBary(Np, 1.0);
    for (int i = 1; i < Np; i++)
        for (int j = 0; j < i; j++) {
            wBary[j] *= (c.x[j] - c.x[i]);
            wBary[i] *= (c.x[i] - c.x[j]);
        }
    for (int i = 0; i < Np; i++) wBary[i] = 1.0 / wBary[i];
    c.D.assign(Np * Np, 0.0);
    for (int iL = 0; iL < Np; iL++)
        for (int i = 0; i < Np; i++)
            if (iL != i) {
                c.D[i * Np + iL] = wBary[iL] / wBary[i] / (c.x[i] - c.x[iL]);
                c.D[i * Np + i] -= c.D[i * Np + iL];
            }
    c.Dhat = c.D;
    c.Dhat[0] += 1.0 / c.w[0];
    c.Dhat[(Np - 1) * Np + Np - 1] -= 1.0 / c.w[Np - 1];
    c.Dhat2.assign(Np * Np, 0.0);
    for (int i = 0; i < Np * Np; i++) c.Dhat2[i] = c.D[i] * 2.0;
    c.Dhat2[0] += 1.0 / c.w[0];
    c.Dhat2[(Np - 1) * Np + Np - 1] -= 1.0 / c.w[Np - 1];
}

// ComputeSubcellMetrics on an affine element (DGSEMIntegrator.cpp:1199-1304):
// interface i normal = adj row + sum_{l<i} w_l * sum_m D(l,m) * adj row.  Only
// the diagonal component is non-zero.
static void build_subcell_normals(Ctx &c)
{
    for (int d = 0; d < c.dim; d++) {
        c.snor[d].assign(c.Np + 1, 0.0);
        const double a = c.adj[d];
        for (int i = 0; i < c.Np + 1; i++) {
            double nor = a;
            for (int l = 0; l < i; l++) {
                double tmp = 0.0;
                for (int m = 0; m < c.Np; m++) {
                    double metric2 = a;
                    metric2 *= c.D[l * c.Np + m];
                    tmp += metric2;
                }
                tmp *= c.w[l];
                nor += tmp;
            }
            c.snor[d][i] = nor;
        }
    }
}

// Shifted Legendre on [0,1] (what Poly_1D::CalcLegendre evaluates).
static void legendre01(int order, double x, double *L)
{
    double z;
    L[0] = 1.0;
    if (order == 0) return;
    L[1] = z = 2.0 * x - 1.0;
    for (int n = 1; n < order; n++) L[n + 1] = ((2 * n + 1) * z * L[n] - n * L[n - 1]) / (n + 1);
}

// Dense inverse by Gauss-Jordan with partial pivoting.
static bool invert(std::vector<double> &A, int n)
{
    std::vector<double> I(n * n, 0.0);
    for (int i = 0; i < n; i++) I[i * n + i] = 1.0;
    for (int col = 0; col < n; col++) {
        int piv = col;
        for (int r = col + 1; r < n; r++)
            if (std::fabs(A[r * n + col]) > std::fabs(A[piv * n + col])) piv = r;
        if (A[piv * n + col] == 0.0) return false;
        if (piv != col)
            for (int k = 0; k < n; k++) {
                std::swap(A[piv * n + k], A[col * n + k]);
                std::swap(I[piv * n + k], I[col * n + k]);
            }
        double inv = 1.0 / A[col * n + col];
        for (int k = 0; k < n; k++) {
            A[col * n + k] *= inv;
            I[col * n + k] *= inv;
        }
        for (int r = 0; r < n; r++)
            if (r != col) {
                double f = A[r * n + col];
                if (f != 0.0)
                    for (int k = 0; k < n; k++) {
                        A[r * n + k] -= f * A[col * n + k];
                        I[r * n + k] -= f * I[col * n + k];
                    }
            }
    }
    A = I;
    return true;
}

// ModalBasis::ComputeUBDegs / ComputeVDM (src/ModalBasis/ModalBasis.cpp:42-135):
// mode k has degrees with the x-degree slowest; V(i,k) = prod_d L_deg(x_i,d).
static void build_modal(Ctx &c)
{
    const int nd = c.ndof, Np = c.Np, dim = c.dim;
    c.degs.assign(nd * dim, 0);
    for (int k = 0; k < nd; k++) {
        int r = k;
        for (int d = dim - 1; d >= 0; d--) {
            c.degs[k * dim + d] = r % Np;
            r /= Np;
        }
    }
    c.max_order.assign(nd, 0);
    for (int k = 0; k < nd; k++) {
        int m = 0;
        for (int d = 0; d < dim; d++) m = std::max(m, c.degs[k * dim + d]);
        c.max_order[k] = m;
    }
    c.Vdm.assign(nd * nd, 0.0);
    std::vector<double> L(Np);
    for (int i = 0; i < nd; i++) {
        int ii[3] = {i % Np, (i / Np) % Np, i / (Np * Np)};
        for (int d = 0; d < dim; d++) {
            legendre01(c.N, c.x[ii[d]], L.data());
            for (int k = 0; k < nd; k++) {
                double v = L[c.degs[k * dim + d]];
                c.Vdm[i * nd + k] = (d == 0) ? v : c.Vdm[i * nd + k] * v;
            }
        }
    }
    c.Vinv = c.Vdm;
    invert(c.Vinv, nd);
}

// ---------------------------------------------------------------------------
// Blending coefficient: PerssonPeraireIndicator::CheckSmoothness
// (src/Indicators/PerssonPeraireIndicator.cpp:21-58) and
// DGSEMOperator::ComputeBlendingCoefficient (DGSEMOperator.cpp:60-80).
// ---------------------------------------------------------------------------
static void blending_coefficient(Ctx &c, const double *u)
{
    const int nd = c.ndof, nv = c.nv, dim = c.dim;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        std::vector<double> q(nd), m(nd), m1(nd), m2(nd);
        double s[5];
        for (int i = 0; i < nd; i++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, i)];
            q[i] = s[0] * pressure(dim, c.p.gamma, s);
        }
        for (int r = 0; r < nd; r++) {  // DenseMatrix::Mult
            double acc = 0.0;
            for (int k = 0; k < nd; k++) acc += c.Vinv[r * nd + k] * q[k];
            m[r] = acc;
        }
        m1 = m;
        m2 = m;
        for (int i = 0; i < nd; i++)
            for (int d = 0; d < dim; d++)
                if (c.degs[i * dim + d] > c.N - 2) {
                    m2[i] = 0.0;
                    if (c.degs[i * dim + d] > c.N - 1) m1[i] = 0.0;
                }
        double mm = 0, m1m1 = 0, m2m2 = 0;
        for (int i = 0; i < nd; i++) {
            mm += m[i] * m[i];
            m1m1 += m1[i] * m1[i];
            m2m2 += m2[i] * m2[i];
        }
        double eta = 1.0 - m1m1 / mm;
        eta = std::max(eta, 1.0 - m2m2 / m1m1);
        c.eta[e] = eta;
        const double sharpness_fac = 9.21024, T = c.modalThreshold;
        double a = 1.0 / (1.0 + std::exp(-sharpness_fac * (eta - T) / T));
        if (a < c.p.alpha_min)
            a = 0.0;
        else if (a > (1.0 - c.p.alpha_min))
            a = 1.0;
        a = std::min(a, c.p.alpha_max);
        c.alpha[e] = a;
    }
}

// ---------------------------------------------------------------------------
// Element-local helpers
// ---------------------------------------------------------------------------

// Node index along direction d through node (i,j,k) at position l.
static inline int line_node(const Ctx &c, int d, int i, int j, int k, int l)
{
    const int Np = c.Np;
    if (d == 0) return (k * Np + j) * Np + l;
    if (d == 1) return (k * Np + l) * Np + i;
    return (l * Np + j) * Np + i;
}

// ComputeFVFluxes (DGSEMIntegrator.cpp:972-1196): writes el_dudt (ndof x nv,
// row-major node) = alpha * subcell FV update.  Returns the max wave speed.
static double fv_fluxes(const Ctx &c, const double *el_u, double alpha_value, double *el_dudt)
{
    const int Np = c.Np, nv = c.nv, dim = c.dim;
    const int Npy = dim > 1 ? Np : 1, Npz = dim > 2 ? Np : 1;
    double lam = -1.0;
    double dU[5], flux[5], nor[3];
    for (int dd = 0; dd < dim; dd++) {
        // x lines iterate (k, j), y lines (k, i), z lines (j, i)
        int A = (dd == 2) ? Npy : Npz;  // outer count
        int B = (dd == 0) ? Npy : Np;   // inner count
        for (int a = 0; a < A; a++)
            for (int b = 0; b < B; b++) {
                int i = 0, j = 0, k = 0;
                if (dd == 0) { k = a; j = b; }
                else if (dd == 1) { k = a; i = b; }
                else { j = a; i = b; }
                for (int v = 0; v < nv; v++) dU[v] = 0.0;
                int id1 = line_node(c, dd, i, j, k, 0);
                for (int q = 0; q < dim; q++) nor[q] = 0.0;
                for (int l = 0; l < Np - 1; l++) {
                    int id2 = line_node(c, dd, i, j, k, l + 1);
                    nor[dd] = c.snor[dd][l + 1];
                    const double *s1 = el_u + id1 * nv, *s2 = el_u + id2 * nv;
                    lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux));
                    for (int v = 0; v < nv; v++) {
                        dU[v] -= flux[v];
                        dU[v] /= c.J * c.w[l];
                    }
                    for (int v = 0; v < nv; v++) {
                        if (dd == 0) el_dudt[id1 * nv + v] = dU[v];
                        else el_dudt[id1 * nv + v] += dU[v];
                    }
                    for (int v = 0; v < nv; v++) dU[v] = flux[v];
                    id1 = id2;
                }
                for (int v = 0; v < nv; v++) {
                    dU[v] /= c.J * c.w[Np - 1];
                    if (dd == 0) el_dudt[id1 * nv + v] = dU[v];
                    else el_dudt[id1 * nv + v] += dU[v];
                }
            }
    }
    for (int i = 0; i < c.ndof * nv; i++) el_dudt[i] *= alpha_value;
    return lam;
}

// AssembleElementVector, Euler (DGSEMIntegrator.cpp:224-433) and NS
// (:601-750 3D, :752-864 2D).  el_u / el_dudt are node-major (ndof x nv);
// el_g (NS) holds the primitive gradients [d][node][v].
static double element_vector(const Ctx &c, const double *el_u, const double *el_g,
                             double alpha, double *el_dudt)
{
    const int Np = c.Np, nv = c.nv, dim = c.dim, nd = c.ndof;
    const int Npy = dim > 1 ? Np : 1, Npz = dim > 2 ? Np : 1;
    double lam = -1.0;
    for (int i = 0; i < nd * nv; i++) el_dudt[i] = 0.0;
    if (c.p.blending) lam = std::max(lam, fv_fluxes(c, el_u, alpha, el_dudt));

    // Contravariant viscous fluxes per node, per direction (NS only).
    std::vector<double> Fv;  // [d][node][v]
    if (c.p.parabolic) {
        Fv.assign((size_t)dim * nd * nv, 0.0);
        double flux[15], dq[15];
        for (int n = 0; n < nd; n++) {
            // The reference reads the state of its member id1 here
            // (DGSEMIntegrator.cpp:620, :770), which ComputeFVFluxes (and the
            // previous element's loops) leave at the element's last node.
            int sn = c.p.compat ? nd - 1 : n;
            for (int d = 0; d < dim; d++)
                for (int v = 0; v < nv; v++) dq[d * nv + v] = el_g[((size_t)d * nd + n) * nv + v];
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, el_u + sn * nv, dq, flux);
            // MultABt(adj, flux): row a = sum_b adj(a,b) flux(:,b); adj diagonal.
            for (int a = 0; a < dim; a++)
                for (int v = 0; v < nv; v++) {
                    double acc = 0.0;
                    for (int b = 0; b < dim; b++) acc += (a == b ? c.adj[a] : 0.0) * flux[v * dim + b];
                    Fv[((size_t)a * nd + n) * nv + v] = acc;
                }
        }
    }

    // Two-point fluxes: Fs[d][node][m][v] with column pos(node,d) zero.
    std::vector<double> Fs((size_t)dim * nd * Np * nv, 0.0);
    auto FS = [&](int d, int n, int m) -> double * { return &Fs[(((size_t)d * nd + n) * Np + m) * nv]; };
    double f[5], g[5], h[5];
    double metric[3] = {0, 0, 0}, metric_y[3] = {0, 0, 0}, metric_z[3] = {0, 0, 0};
    metric[0] = c.adj[0];
    if (dim > 1) metric_y[1] = c.adj[1];
    if (dim > 2) metric_z[2] = c.adj[2];
    for (int k = 0; k < Npz; k++)
        for (int j = 0; j < Npy; j++)
            for (int i = 0; i < Np; i++) {
                int id1 = (k * Npy + j) * Np + i;
                const double *s1 = el_u + id1 * nv;
                for (int v = 0; v < nv; v++) f[v] = 0.0;
                std::memcpy(FS(0, id1, i), f, sizeof(double) * nv);
                for (int m = i + 1; m < Np; m++) {
                    int id2 = (k * Npy + j) * Np + m;
                    lam = std::max(lam, volume_flux(dim, c.p.gamma, s1, el_u + id2 * nv, metric, metric, f));
                    std::memcpy(FS(0, id1, m), f, sizeof(double) * nv);
                    std::memcpy(FS(0, id2, i), f, sizeof(double) * nv);
                }
                if (dim > 1) {
                    for (int v = 0; v < nv; v++) g[v] = 0.0;
                    std::memcpy(FS(1, id1, j), g, sizeof(double) * nv);
                    for (int m = j + 1; m < Npy; m++) {
                        int id2 = (k * Npy + m) * Np + i;
                        lam = std::max(lam, volume_flux(dim, c.p.gamma, s1, el_u + id2 * nv, metric_y, metric_y, g));
                        std::memcpy(FS(1, id1, m), g, sizeof(double) * nv);
                        std::memcpy(FS(1, id2, j), g, sizeof(double) * nv);
                    }
                    if (dim > 2) {
                        for (int v = 0; v < nv; v++) h[v] = 0.0;
                        std::memcpy(FS(2, id1, k), h, sizeof(double) * nv);
                        for (int m = k + 1; m < Npz; m++) {
                            int id2 = (m * Npy + j) * Np + i;
                            lam = std::max(lam, volume_flux(dim, c.p.gamma, s1, el_u + id2 * nv, metric_z, metric_z, h));
                            std::memcpy(FS(2, id1, m), h, sizeof(double) * nv);
                            // The NS 3D path fills the partner column with the
                            // last y-direction flux `g` (DGSEMIntegrator.cpp:702).
                            const double *fill = (c.p.parabolic && c.p.compat) ? g : h;
                            std::memcpy(FS(2, id2, k), fill, sizeof(double) * nv);
                        }
                    }
                }
                // Flux differencing: dU = sum_d sum_m Dhat2(pos_d, m) F_d(:, m).
                double dU[5], dUv[5];
                int pos[3] = {i, j, k};
                for (int v = 0; v < nv; v++) dU[v] = 0.0;
                for (int d = 0; d < dim; d++)
                    for (int m = 0; m < Np; m++) {
                        const double *col = FS(d, id1, m);
                        double a = c.Dhat2[pos[d] * Np + m];
                        if (d == 0 && m == 0)
                            for (int v = 0; v < nv; v++) dU[v] = a * col[v];
                        else
                            for (int v = 0; v < nv; v++) dU[v] += a * col[v];
                    }
                for (int v = 0; v < nv; v++) dUv[v] = 0.0;
                if (c.p.parabolic) {
                    for (int d = 0; d < dim; d++)
                        for (int l = 0; l < Np; l++) {
                            int nl = line_node(c, d, i, j, k, l);
                            double a = c.Dhat[pos[d] * Np + l];
                            for (int v = 0; v < nv; v++) {
                                double t = Fv[((size_t)d * nd + nl) * nv + v];
                                t *= a;
                                dUv[v] += t;
                            }
                        }
                }
                for (int v = 0; v < nv; v++) {
                    double t = -dU[v];
                    if (c.p.blending) t *= (1.0 - alpha);
                    if (c.p.parabolic) {
                        t = t + dUv[v];
                    }
                    t /= c.J;
                    el_dudt[id1 * nv + v] += t;
                }
            }
    return lam;
}

// Face node list of face (d, side) of an element: node index of face node t.
static inline int face_node(const Ctx &c, int d, int side, int t)
{
    const int Np = c.Np;
    const int l = side ? Np - 1 : 0;
    int a = t % Np, b = t / Np;  // tangential indices (fastest first)
    if (c.dim == 2) b = 0;
    if (d == 0) return (b * Np + a) * Np + l;
    if (d == 1) return (b * Np + l) * Np + a;
    return (l * Np + b) * Np + a;
}

static double bdr_face_vector(const Ctx &c, const double *u, int64_t e, int d, int side, int b, double *out);

// AssembleFaceVector, Euler (DGSEMIntegrator.cpp:151-222) and NS
// (:435-494 3D, :496-549 2D) for the face between element a's +d face and its
// neighbour b's -d face.  Writes contributions for both sides into buf:
// buf[0][t][v] for a's face nodes, buf[1][t][v] for b's.
static double face_vector(const Ctx &c, const double *u, const double *gr, int64_t a, int d,
                          double *buf)
{
    const int nv = c.nv, dim = c.dim, nfn = c.ndof / c.Np;
    const int64_t b = c.nbr[a * 2 * dim + 2 * d + 1];
    if (b < 0) return bdr_face_vector(c, u, a, d, 1, (int)(-1 - b), buf);  // a's side only
    const bool a_is_1 = a <= b;
    const int64_t e1 = a_is_1 ? a : b, e2 = a_is_1 ? b : a;
    const int side1 = a_is_1 ? 1 : 0, side2 = a_is_1 ? 0 : 1;
    double nor[3] = {0, 0, 0};
    nor[d] = a_is_1 ? c.area[d] : -c.area[d];
    const double scale = 1.0 / (c.w[0] * c.J);
    double lam = -1.0;
    double s1[5], s2[5], flux[5], dU1[5], dU2[5];
    double dq1[15], dq2[15], fm1[15], fm2[15];
    for (int t = 0; t < nfn; t++) {
        int n1 = face_node(c, d, side1, t), n2 = face_node(c, d, side2, t);
        for (int v = 0; v < nv; v++) {
            s1[v] = u[idx(c, v, e1, n1)];
            s2[v] = u[idx(c, v, e2, n2)];
        }
        if (c.p.parabolic && c.p.compat) {
            // The NS face integrators call ComputeViscousFlux(state1, ...)
            // before ComputeFaceFlux(state1, state2, ...); its Conserv2Prim ->
            // ComputePressure divides the momenta of state1/state2 in place
            // (BasicOperations.cpp:33-34), so the Riemann flux receives
            // velocities in the momentum slots (DGSEMIntegrator.cpp:467-481).
            double t1[5], t2[5];
            for (int v = 0; v < nv; v++) { t1[v] = s1[v]; t2[v] = s2[v]; }
            for (int q = 0; q < dim; q++) { t1[1 + q] = s1[1 + q] / s1[0]; t2[1 + q] = s2[1 + q] / s2[0]; }
            lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, t1, t2, nor, flux));
        } else {
            lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux));
        }
        for (int v = 0; v < nv; v++) {
            dU2[v] = flux[v];
            dU1[v] = -flux[v];
        }
        if (c.p.parabolic) {
            for (int q = 0; q < dim; q++)
                for (int v = 0; v < nv; v++) {
                    dq1[q * nv + v] = gr[(size_t)q * c.size + idx(c, v, e1, n1)];
                    dq2[q * nv + v] = gr[(size_t)q * c.size + idx(c, v, e2, n2)];
                }
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, s1, dq1, fm1);
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, s2, dq2, fm2);
            for (int v = 0; v < nv; v++) {
                double fn = 0.0;
                for (int q = 0; q < dim; q++) {
                    double avg = fm1[v * dim + q];
                    avg += fm2[v * dim + q];
                    avg *= 0.5;
                    fn += avg * nor[q];
                }
                dU1[v] += fn;
                dU2[v] -= fn;
            }
        }
        // AddMult_a_VWt(1/(w0 J), shape, dU): entry += (a * dU_v) * 1.
        double *ba = buf + (size_t)(a_is_1 ? 0 : 1) * nfn * nv;
        double *bb = buf + (size_t)(a_is_1 ? 1 : 0) * nfn * nv;
        for (int v = 0; v < nv; v++) {
            ba[t * nv + v] = scale * dU1[v];
            bb[t * nv + v] = scale * dU2[v];
        }
    }
    return lam;
}

// ---------------------------------------------------------------------------
// Boundary faces (src/Integrators/BoundaryConditions/), Euler.
// ---------------------------------------------------------------------------
// MFEM-style helpers as BasicOperations restates them: Normalize
// (BasicOperations.hpp:39-42), Normal and Cross (BasicOperations.cpp:211-235),
// RotateState (:238-258).
static void unit_normal(int dim, const double *nor, double *un)
{
    double nn = 0.0;
    for (int d = 0; d < dim; d++) nn += nor[d] * nor[d];
    const double inv = 1.0 / std::sqrt(nn);
    for (int d = 0; d < dim; d++) un[d] = nor[d] * inv;
}
static void rotate_state(int dim, double *state, const double *n)
{
    double t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
    if (dim == 2) {
        t1[0] = -n[1];
        t1[1] = n[0];
    } else {
        const bool gen = std::abs(n[0]) > 1e-10;
        const double q = gen ? n[1] / n[0] : 0.0;
        t1[0] = gen ? -q / std::sqrt(1.0 + std::pow(q, 2)) : -1.0;
        t1[1] = gen ? 1.0 / std::sqrt(1.0 + std::pow(q, 2)) : 0.0;
        t1[2] = 0.0;
        t2[0] = n[1] * t1[2] - n[2] * t1[1];
        t2[1] = n[2] * t1[0] - n[0] * t1[2];
        t2[2] = n[0] * t1[1] - n[1] * t1[0];
    }
    double *m = state + 1;
    double ru = 0.0, rv = 0.0, rw = 0.0;
    for (int d = 0; d < dim; d++) { ru += m[d] * n[d]; rv += m[d] * t1[d]; }
    if (dim == 3) {
        for (int d = 0; d < 3; d++) rw += m[d] * t2[d];
        m[2] = rw;
    }
    m[0] = ru;
    m[1] = rv;
}

// Normal flux of boundary condition b for interior state s1 and outward
// normal nor (ComputeBdrFaceInviscidFlux); returns the reported wave speed.
// outer (optional): receives the outer state the face flux is given (the
// conditions other than the walls), for the boundary lifting flux.
static double bdr_flux(const Ctx &c, int b, const double *s1, const double *nor, double *flux,
                       double *outer = nullptr)
{
    const int dim = c.dim, nv = c.nv;
    const double gamma = c.p.gamma, gammaM1 = gamma - 1.0, gammaM1Inverse = 1.0 / gammaM1;
    const int type = (int)c.bc[b][0];
    double s2[5], un[3];
    for (int v = 0; v < nv; v++) s2[v] = s1[v];
    if (type == 4 || type == 10 || type == 11) {
        // SlipWallBdrFaceIntegrator::ComputeBdrFaceInviscidFlux (:15-58); the
        // no-slip wall derives from it
        const double gammaP1 = 1.0 + gamma, gammaP1Inverse = 1.0 / gammaP1;
        unit_normal(dim, nor, un);
        rotate_state(dim, s2, un);
        const double rho = s2[0];
        double V[3], vv = 0.0;
        for (int d = 0; d < dim; d++) { V[d] = s2[1 + d] / rho; vv += V[d] * V[d]; }
        const double p = gammaM1 * (s2[nv - 1] - 0.5 * rho * vv);
        const double an = sound_speed(p, rho, gamma);
        const double u = V[0];
        double p_star;
        if (u > 0.0)
            p_star = p + 0.25 * u * gammaP1 * rho *
                             (u + std::sqrt(std::pow(u, 2) + 8.0 * gammaP1Inverse / rho * p * (gammaM1 * gammaP1Inverse + 1.0)));
        else
            p_star = p * std::pow(std::max(1.0 + 0.5 * gammaM1 * u / an, 0.0001), 2.0 * gamma * gammaM1Inverse);
        for (int v = 0; v < nv; v++) flux[v] = 0.0;
        for (int d = 0; d < dim; d++) flux[1 + d] = p_star * nor[d];
        return std::sqrt(vv) + an;
    }
    // s1 as the face flux sees it: the subsonic conditions of the reference
    // divide the interior state's momenta in place through Vector views
    // (ComputePressure, BasicOperations.cpp:31-37, and the views V_i / vel);
    // compat keeps that, fixed uses the interior state as it is.
    double s1c[5];
    for (int v = 0; v < nv; v++) s1c[v] = s1[v];
    const double *prm = c.bc[b] + 1;
    const bool compat = c.p.compat != 0;
    if (type == 6) {
        // SubsonicOutflowPBdrFaceIntegrator::ComputeOuterInviscidState (:17-31)
        double vel[3], vv = 0.0;
        const double r1 = 1.0 / s1[0];
        for (int d = 0; d < dim; d++) vel[d] = compat ? s1[1 + d] * r1 : s1[1 + d] / s1[0];
        for (int d = 0; d < dim; d++) vv += vel[d] * vel[d];
        if (compat)
            for (int d = 0; d < dim; d++) s1c[1 + d] = vel[d];
        for (int v = 0; v < nv; v++) s2[v] = s1c[v];
        s2[nv - 1] = prm[0] * gammaM1Inverse + 0.5 * s1[0] * vv;
        if (outer) for (int v = 0; v < nv; v++) outer[v] = s2[v];
        return face_flux(dim, gamma, c.p.compat, c.p.face_dissipation, s1c, s2, nor, flux);
    }
    if (type == 7) {
        // SubsonicInflowRVBdrFaceIntegrator::ComputeOuterInviscidState (:20-50)
        const double r = prm[0];
        s2[0] = r;
        double dke = -s1[1] * s1[1];
        double uu = 0.0;
        for (int d = 0; d < dim; d++) {
            s2[1 + d] = r * prm[1 + d];
            if (d > 0) dke -= s1[1 + d] * s1[1 + d];
            uu += prm[1 + d] * prm[1 + d];
        }
        dke *= 0.5 / s1[0];
        dke += 0.5 * uu * r;
        s2[nv - 1] = s1[nv - 1] + dke;
        if (outer) for (int v = 0; v < nv; v++) outer[v] = s2[v];
        return face_flux(dim, gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux);
    }
    if (type == 8) {
        // SubsonicInflowPtTtAngBdrFaceIntegrator::ComputeOuterInviscidState
        // (:52-80), 2D: prm = cp, p0, T0, cos(theta), sin(theta)
        const double cp = prm[0], p0 = prm[1], T0 = prm[2];
        double V[3], vv = 0.0;
        const double r1 = 1.0 / s1[0];
        for (int d = 0; d < dim; d++) V[d] = compat ? s1[1 + d] * r1 : s1[1 + d] / s1[0];
        for (int d = 0; d < dim; d++) vv += V[d] * V[d];
        if (compat)
            for (int d = 0; d < dim; d++) s1c[1 + d] = V[d];
        const double p = gammaM1 * (s1[nv - 1] - 0.5 * s1[0] * vv);
        double V_sq = 2.0 * cp * T0 * (1.0 - std::pow(p / p0, gammaM1 / gamma));
        V_sq = std::max(0.0, V_sq);
        s2[0] = gamma * gammaM1Inverse * p / (cp * T0 - 0.5 * V_sq);
        for (int d = 0; d < dim; d++) s2[1 + d] = s2[0] * std::sqrt(V_sq) * prm[3 + d];
        s2[nv - 1] = p * gammaM1Inverse + 0.5 * s2[0] * V_sq;
        if (outer) for (int v = 0; v < nv; v++) outer[v] = s2[v];
        return face_flux(dim, gamma, c.p.compat, c.p.face_dissipation, s1c, s2, nor, flux);
    }
    if (type == 9) {
        // RiemannInvariantBdrFaceIntegrator::ComputeOuterInviscidState
        // (:43-112): prm = primitive outer state (rho, v, p)
        const double gammaInverse = 1.0 / gamma;
        unit_normal(dim, nor, un);
        const double rho_o = prm[0], p_o = prm[nv - 1];
        const double *V_o = prm + 1;
        const double r1 = 1.0 / s1[0];
        double V_i[3], Vn_i = 0.0, Vn_o = 0.0;
        for (int d = 0; d < dim; d++) V_i[d] = compat ? s1[1 + d] * r1 : s1[1 + d] / s1[0];
        for (int d = 0; d < dim; d++) { Vn_i += V_i[d] * un[d]; Vn_o += V_o[d] * un[d]; }
        // ComputePressure(state1): in compat its view divides the (already
        // divided) momenta once more, and V_i, a view of them, follows
        double W[3], ww = 0.0;
        for (int d = 0; d < dim; d++) W[d] = compat ? V_i[d] * r1 : V_i[d];
        for (int d = 0; d < dim; d++) ww += W[d] * W[d];
        const double p_i = gammaM1 * (s1[nv - 1] - 0.5 * s1[0] * ww);
        if (compat)
            for (int d = 0; d < dim; d++) { V_i[d] = W[d]; s1c[1 + d] = W[d]; }
        const double a_o = sound_speed(p_o, rho_o, gamma), a_i = sound_speed(p_i, s1[0], gamma);
        const double R_minus = (std::abs(Vn_o) >= a_o && Vn_i >= 0.0) ? Vn_i - 2.0 * a_i * gammaM1Inverse
                                                                       : Vn_o - 2.0 * a_o * gammaM1Inverse;
        const double R_plus = (std::abs(Vn_o) >= a_o && Vn_i < 0.0) ? Vn_o + 2.0 * a_o * gammaM1Inverse
                                                                     : Vn_i + 2.0 * a_i * gammaM1Inverse;
        const double Vn_b = 0.5 * (R_plus + R_minus);
        const double a_b = 0.25 * gammaM1 * (R_plus - R_minus);
        const double dVn_i = Vn_b - Vn_i, dVn_o = Vn_b - Vn_o;
        s2[0] = (Vn_i < 0.0) ? std::pow(a_b * a_b * gammaInverse * rho_o / p_o, gammaM1Inverse) * rho_o
                             : std::pow(a_b * a_b * gammaInverse * s1[0] / p_i, gammaM1Inverse) * s1[0];
        double e2 = 0.0;
        for (int d = 0; d < dim; d++) {
            s2[1 + d] = (Vn_i >= 0.0) ? s2[0] * (V_i[d] + dVn_i * un[d]) : s2[0] * (V_o[d] + dVn_o * un[d]);
            e2 = d == 0 ? s2[1] * s2[1] : e2 + s2[1 + d] * s2[1 + d];
        }
        const double p_b = a_b * a_b * s2[0] * gammaInverse;
        e2 *= (0.5 / s2[0]);
        e2 += p_b * gammaM1Inverse;
        s2[nv - 1] = e2;
        if (outer) for (int v = 0; v < nv; v++) outer[v] = s2[v];
        return face_flux(dim, gamma, c.p.compat, c.p.face_dissipation, s1c, s2, nor, flux);
    }
    if (type == 1 || type == 3) {
        // SupersonicInflow / SpecifiedState: the prescribed state (:22-35, :21-35)
        for (int v = 0; v < nv; v++) s2[v] = c.bc[b][1 + v];
    } else if (type == 5) {
        // SymmetryBdrFaceIntegrator (:12-37): mirrored normal momentum
        unit_normal(dim, nor, un);
        double mn = 0.0;
        for (int d = 0; d < dim; d++) mn += s2[1 + d] * un[d];
        for (int d = 0; d < dim; d++) s2[1 + d] += -2.0 * mn * un[d];
    }  // type 2, SupersonicOutflow (:10-13): the interior state
    if (outer) for (int v = 0; v < nv; v++) outer[v] = s2[v];
    return face_flux(dim, gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux);
}

// BdrFaceIntegrator::AssembleFaceVector (BdrFaceIntegrator.cpp:64-130): the
// boundary face of element e on its +d (side 1) or -d (side 0) side, with
// the outward normal; out[t][v] = -flux / (w0 J1) at face node t.
static double bdr_face_vector(const Ctx &c, const double *u, int64_t e, int d, int side, int b, double *out)
{
    const int nv = c.nv, nfn = c.ndof / c.Np, dim = c.dim;
    double nor[3] = {0, 0, 0};
    nor[d] = side ? c.area[d] : -c.area[d];
    const double scale = 1.0 / (c.w[0] * c.J);
    const int type = (int)c.bc[b][0];
    double lam = -1.0, s1[5], flux[5], dq[15], fm[15];
    for (int t = 0; t < nfn; t++) {
        const int n = face_node(c, d, side, t);
        for (int v = 0; v < nv; v++) s1[v] = u[idx(c, v, e, n)];
        lam = std::max(lam, bdr_flux(c, b, s1, nor, flux));
        double dU[5];
        for (int v = 0; v < nv; v++) dU[v] = -flux[v];
        if (c.p.parabolic && (type == 2 || type == 10 || type == 11 || type == 8)) {
            // ComputeBdrFaceViscousFlux: the interior state's viscous flux
            // with its own gradients (SupersonicOutflowBdrFaceIntegrator.cpp:
            // 15-20); the no-slip wall replaces the energy row by the wall
            // velocity's work, its heat flux qn being zero
            // (NoSlipAdiabWallBdrFaceIntegrator.cpp:21-36)
            for (int q = 0; q < dim; q++)
                for (int v = 0; v < nv; v++) dq[q * nv + v] = c.grads[(size_t)q * c.size + idx(c, v, e, n)];
            if (type == 8) {
                // the total-pressure inflow: the outer state's viscous flux with
                // the interior gradients (SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:88-92)
                double so[5], fl[5];
                bdr_flux(c, b, s1, nor, fl, so);
                viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, so, dq, fm);
            } else {
                viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, s1, dq, fm);
            }
            double fn[5];
            for (int v = 0; v < nv; v++) {
                fn[v] = 0.0;
                for (int q = 0; q < dim; q++) fn[v] += fm[v * dim + q] * nor[q];
            }
            if (type == 10) {
                double en = 0.0;
                for (int q = 0; q < dim; q++) en += c.bc[b][1 + q] * fn[1 + q];
                fn[nv - 1] = en + 0.0;
            }
            for (int v = 0; v < nv; v++) dU[v] += fn[v];
        }  // types 1, 3: the viscous flux of the outer state with zero gradients, 0
        for (int v = 0; v < nv; v++) out[t * nv + v] = scale * dU[v];
    }
    return lam;
}

// ComputeBdrFaceLiftingFlux (BdrFaceIntegrator.cpp:275-282; the no-slip wall's
// NoSlipAdiabWallBdrFaceIntegrator.cpp:74-95): the BR1 boundary jump of the
// entropy variables w1 at a boundary node with interior state s1.  Default:
// 0.5 (w(s2) - w1) with s2 the outer state; the reference reaches s2 through
// Entropy2Conserv(w1) (BasicOperations.cpp:106-124), whose velocity view
// divides w1's momentum entries by beta in place before they are
// subtracted; compat keeps that.  No-slip: (w1_0, beta V, -beta) - w1.
static void bdr_lifting_flux(const Ctx &c, int b, const double *s1, const double *w1_in, const double *nor,
                             double *f)
{
    const int nv = c.nv, dim = c.dim;
    const double gamma = c.p.gamma, gm1 = gamma - 1.0, gm1inv = 1.0 / gm1;
    const int type = (int)c.bc[b][0];
    double w1[5];
    for (int v = 0; v < nv; v++) w1[v] = w1_in[v];
    if (type == 10 || type == 11) {
        // the isothermal wall (NoSlipIsothWallBdrFaceIntegrator.cpp:41-65)
        // takes 1/(R T_wall), stored after the wall velocity, for beta
        const double beta = type == 10 ? -w1[nv - 1] : c.bc[b][1 + dim];
        f[0] = w1[0];
        for (int q = 0; q < dim; q++) f[1 + q] = c.bc[b][1 + q] * beta;
        f[nv - 1] = -beta;
        for (int v = 0; v < nv; v++) f[v] -= w1[v];
        return;
    }
    double s2[5];
    if (c.p.compat) {
        // Entropy2Conserv(w1) with its in-place division of w1's momenta
        const double beta = -w1[nv - 1], ib = 1.0 / beta;
        double vv = 0.0;
        for (int q = 0; q < dim; q++) { w1[1 + q] *= ib; vv += w1[1 + q] * w1[1 + q]; }
        const double sent = gamma - (w1[0] + 0.5 * beta * vv) * gm1;
        double cons[5];
        cons[0] = std::pow(std::exp(-sent) / beta, gm1inv);
        for (int q = 0; q < dim; q++) cons[1 + q] = cons[0] * w1[1 + q];
        cons[nv - 1] = cons[0] * (1.0 / beta * gm1inv + 0.5 * vv);
        for (int v = 0; v < nv; v++) s2[v] = cons[v];
    } else {
        for (int v = 0; v < nv; v++) s2[v] = s1[v];
    }
    if (type == 1 || type == 3)
        for (int v = 0; v < nv; v++) s2[v] = c.bc[b][1 + v];
    if (type == 6 || type == 7 || type == 8 || type == 9) {
        // ComputeOuterInviscidState of the subsonic outflow, the subsonic
        // inflow (rho, V) and the Riemann invariants, from s2 (the interior
        // state, or in compat what Entropy2Conserv made of w1), with their
        // own in-place divisions in compat
        double so[5], fl[5];
        bdr_flux(c, b, s2, nor, fl, so);
        for (int v = 0; v < nv; v++) s2[v] = so[v];
    }
    double w2[5];
    conserv2entropy(dim, gamma, s2, w2);
    for (int v = 0; v < nv; v++) {
        f[v] = w2[v];
        f[v] -= w1[v];
        f[v] *= 0.5;
    }
}

// ---------------------------------------------------------------------------
// BR1 lifting (LiftingBR1.cpp:10-115, 156-272; DGSEMNonlinearForm.cpp:213-645)
// and ComputeGlobalPrimitiveGradVector (DGSEMOperator.cpp:96-159).
// ---------------------------------------------------------------------------
static void lifting(Ctx &c, const double *u)
{
    const int nv = c.nv, dim = c.dim, nd = c.ndof, Np = c.Np, nfn = nd / Np;
    const int Npy = dim > 1 ? Np : 1, Npz = dim > 2 ? Np : 1;
    // ComputeGlobalEntropyVector (DGSEMOperator.cpp:82-94).
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        double s[5], w[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, n)];
            conserv2entropy(dim, c.p.gamma, s, w);
            for (int v = 0; v < nv; v++) c.went[idx(c, v, e, n)] = w[v];
        }
    }
    const double *W = c.went.data();
    double *G = c.grads.data();
    const double invJ = 1.0 / c.J;
    const double scale = 1.0 / (c.w[0] * c.J);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        // Element part: strong-form derivative, * adj / J.
        for (int k = 0; k < Npz; k++)
            for (int j = 0; j < Npy; j++)
                for (int i = 0; i < Np; i++) {
                    int id = (k * Npy + j) * Np + i;
                    int pos[3] = {i, j, k};
                    for (int d = 0; d < dim; d++)
                        for (int v = 0; v < nv; v++) {
                            double acc = 0.0;
                            for (int l = 0; l < Np; l++) {
                                double t = W[idx(c, v, e, line_node(c, d, i, j, k, l))];
                                t *= c.D[pos[d] * Np + l];
                                acc += t;
                            }
                            // grad_mat1 * adj (diagonal), then * (1/J)
                            double g = acc * c.adj[d];
                            g *= invJ;
                            G[(size_t)d * c.size + idx(c, v, e, id)] = g;
                        }
                }
        // Face parts: each face adds 0.5*(w2 - w1)*n_d/(w0 J) to both sides.
        for (int d = 0; d < dim; d++)
            for (int side = 0; side < 2; side++) {
                int64_t nb = c.nbr[e * 2 * dim + 2 * d + side];
                if (nb < 0) {
                    // boundary face (LiftingBR1::AssembleLiftingBdrFaceVector,
                    // LiftingBR1.cpp:311-345): the element is element 1, the
                    // normal points out of it
                    const double ndb = side ? c.area[d] : -c.area[d];
                    double s1[5], w1[5], f[5], norb[3] = {0.0, 0.0, 0.0};
                    norb[d] = ndb;
                    for (int t = 0; t < nfn; t++) {
                        const int n = face_node(c, d, side, t);
                        for (int v = 0; v < nv; v++) {
                            s1[v] = u[idx(c, v, e, n)];
                            w1[v] = W[idx(c, v, e, n)];
                        }
                        bdr_lifting_flux(c, (int)(-1 - nb), s1, w1, norb, f);
                        for (int v = 0; v < nv; v++) {
                            double fval = f[v];
                            fval *= ndb;
                            G[(size_t)d * c.size + idx(c, v, e, n)] += scale * fval;
                        }
                    }
                    continue;
                }
                // The face between (e, side) and nb: element 1 rule.
                int64_t a = side ? e : nb;  // element on the -d side of the face
                int64_t bb = side ? nb : e;
                bool a_is_1 = a <= bb;
                int64_t e1 = a_is_1 ? a : bb, e2 = a_is_1 ? bb : a;
                int side1 = a_is_1 ? 1 : 0, side2 = a_is_1 ? 0 : 1;
                double nd_ = a_is_1 ? c.area[d] : -c.area[d];
                bool me_is_1 = (e == e1) && !(e1 == e2 && side != side1);
                for (int t = 0; t < nfn; t++) {
                    int n1 = face_node(c, d, side1, t), n2 = face_node(c, d, side2, t);
                    int nme = me_is_1 ? n1 : n2;
                    for (int v = 0; v < nv; v++) {
                        double fval = 0.5 * (W[idx(c, v, e2, n2)] - W[idx(c, v, e1, n1)]);
                        fval *= nd_;
                        G[(size_t)d * c.size + idx(c, v, e, nme)] += scale * fval;
                    }
                }
            }
        // EntropyGrad2PrimGrad per node, per direction.
        double s[5], g[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, n)];
            for (int d = 0; d < dim; d++) {
                for (int v = 0; v < nv; v++) g[v] = G[(size_t)d * c.size + idx(c, v, e, n)];
                entgrad2primgrad(dim, c.p.gamma, c.p.compat, s, g);
                for (int v = 0; v < nv; v++) G[(size_t)d * c.size + idx(c, v, e, n)] = g[v];
            }
        }
    }
}

// DGSEMOperator::Mult (DGSEMOperator.cpp:537-591) with the loops of
// DGSEMNonlinearForm::Mult (DGSEMNonlinearForm.cpp:647-849, 1302-1548).
// ---------------------------------------------------------------------------
// General geometry (Euler): the same steps with the metric terms of every
// node (DGSEMIntegrator.cpp:252-266: Tr.SetIntPoint, Weight, AdjugateJacobian
// at each integration point), the subcell metrics of ComputeSubcellMetrics
// (:1199-1304) and the faces' CalcOrtho normals out of element 1 (:186).
// ---------------------------------------------------------------------------
static inline const double *gadj_row(const Ctx &c, int64_t e, int n, int r)
{
    return &c.gadj[(((size_t)e * c.ndof + n) * 3 + r) * 3];
}
static inline double gJ(const Ctx &c, int64_t e, int n) { return c.gJ[(size_t)e * c.ndof + n]; }

// ComputeFVFluxes (DGSEMIntegrator.cpp:972-1196) on element e with its subcell
// metrics; dU is divided by the node's own J times w.
static double fv_fluxes_geo(const Ctx &c, int64_t e, const double *el_u, double alpha_value, double *el_dudt)
{
    const int Np = c.Np, nv = c.nv, dim = c.dim, nfn = c.ndof / Np;
    const int Npy = dim > 1 ? Np : 1, Npz = dim > 2 ? Np : 1;
    double lam = -1.0;
    double dU[5], flux[5];
    for (int dd = 0; dd < dim; dd++) {
        int A = (dd == 2) ? Npy : Npz;
        int B = (dd == 0) ? Npy : Np;
        for (int a = 0; a < A; a++)
            for (int b = 0; b < B; b++) {
                int i = 0, j = 0, k = 0;
                if (dd == 0) { k = a; j = b; }
                else if (dd == 1) { k = a; i = b; }
                else { j = a; i = b; }
                const int line = dd == 0 ? j + Np * k : dd == 1 ? i + Np * k : i + Np * j;
                const double *sn = &c.gsnor[((((size_t)e * dim + dd) * nfn + line) * (Np + 1)) * 3];
                for (int v = 0; v < nv; v++) dU[v] = 0.0;
                int id1 = line_node(c, dd, i, j, k, 0);
                for (int l = 0; l < Np - 1; l++) {
                    int id2 = line_node(c, dd, i, j, k, l + 1);
                    const double *nor = sn + (size_t)(l + 1) * 3;
                    const double *s1 = el_u + id1 * nv, *s2 = el_u + id2 * nv;
                    lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux));
                    for (int v = 0; v < nv; v++) {
                        dU[v] -= flux[v];
                        dU[v] /= gJ(c, e, id1) * c.w[l];
                    }
                    for (int v = 0; v < nv; v++) {
                        if (dd == 0) el_dudt[id1 * nv + v] = dU[v];
                        else el_dudt[id1 * nv + v] += dU[v];
                    }
                    for (int v = 0; v < nv; v++) dU[v] = flux[v];
                    id1 = id2;
                }
                for (int v = 0; v < nv; v++) {
                    dU[v] /= gJ(c, e, id1) * c.w[Np - 1];
                    if (dd == 0) el_dudt[id1 * nv + v] = dU[v];
                    else el_dudt[id1 * nv + v] += dU[v];
                }
            }
    }
    for (int i = 0; i < c.ndof * nv; i++) el_dudt[i] *= alpha_value;
    return lam;
}

// AssembleElementVector, Euler (DGSEMIntegrator.cpp:224-433): two-point
// fluxes with both nodes' metric rows, divided by the node's J.
static double element_vector_geo(const Ctx &c, int64_t e, const double *el_u, const double *el_g, double alpha,
                                 double *el_dudt)
{
    const int Np = c.Np, nv = c.nv, dim = c.dim, nd = c.ndof;
    const int Npy = dim > 1 ? Np : 1, Npz = dim > 2 ? Np : 1;
    double lam = -1.0;
    for (int i = 0; i < nd * nv; i++) el_dudt[i] = 0.0;
    if (c.p.blending) lam = std::max(lam, fv_fluxes_geo(c, e, el_u, alpha, el_dudt));
    // Navier-Stokes: contravariant viscous fluxes MultABt(adj, flux) per node
    // (DGSEMIntegrator.cpp:616-640, 764-786), with the state of the member
    // id1 in compat (the element's last node, Q1)
    std::vector<double> Fv;  // [d][node][v]
    if (c.p.parabolic) {
        Fv.assign((size_t)dim * nd * nv, 0.0);
        double flux[15], dq[15];
        for (int n = 0; n < nd; n++) {
            const int sn = c.p.compat ? nd - 1 : n;
            for (int d = 0; d < dim; d++)
                for (int v = 0; v < nv; v++) dq[d * nv + v] = el_g[((size_t)d * nd + n) * nv + v];
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, el_u + sn * nv, dq, flux);
            for (int a = 0; a < dim; a++) {
                const double *adj = gadj_row(c, e, n, a);
                for (int v = 0; v < nv; v++) {
                    double acc = 0.0;
                    for (int b = 0; b < dim; b++) acc += adj[b] * flux[v * dim + b];
                    Fv[((size_t)a * nd + n) * nv + v] = acc;
                }
            }
        }
    }
    std::vector<double> Fs((size_t)dim * nd * Np * nv, 0.0);
    auto FS = [&](int d, int n, int m) -> double * { return &Fs[(((size_t)d * nd + n) * Np + m) * nv]; };
    double f[5], g[5];
    for (int k = 0; k < Npz; k++)
        for (int j = 0; j < Npy; j++)
            for (int i = 0; i < Np; i++) {
                const int id1 = (k * Npy + j) * Np + i;
                const int pos[3] = {i, j, k};
                for (int v = 0; v < nv; v++) g[v] = 0.0;
                for (int d = 0; d < dim; d++) {
                    for (int v = 0; v < nv; v++) f[v] = 0.0;
                    std::memcpy(FS(d, id1, pos[d]), f, sizeof(double) * nv);
                    for (int m = pos[d] + 1; m < Np; m++) {
                        const int id2 = line_node(c, d, i, j, k, m);
                        lam = std::max(lam, volume_flux(dim, c.p.gamma, el_u + id1 * nv, el_u + id2 * nv,
                                                        gadj_row(c, e, id1, d), gadj_row(c, e, id2, d), f));
                        std::memcpy(FS(d, id1, m), f, sizeof(double) * nv);
                        // the NS 3D path fills the z partner column with the
                        // last y-direction flux g (DGSEMIntegrator.cpp:702, Q2)
                        const double *fill = (d == 2 && c.p.parabolic && c.p.compat) ? g : f;
                        std::memcpy(FS(d, id2, pos[d]), fill, sizeof(double) * nv);
                        if (d == 1) std::memcpy(g, f, sizeof(double) * nv);
                    }
                }
            }
    for (int k = 0; k < Npz; k++)
        for (int j = 0; j < Npy; j++)
            for (int i = 0; i < Np; i++) {
                const int id1 = (k * Npy + j) * Np + i;
                const int pos[3] = {i, j, k};
                double dU[5], dUv[5];
                for (int v = 0; v < nv; v++) dU[v] = dUv[v] = 0.0;
                for (int d = 0; d < dim; d++)
                    for (int m = 0; m < Np; m++) {
                        const double *col = FS(d, id1, m);
                        const double a = c.Dhat2[pos[d] * Np + m];
                        for (int v = 0; v < nv; v++) dU[v] += a * col[v];
                    }
                if (c.p.parabolic)
                    for (int d = 0; d < dim; d++)
                        for (int l = 0; l < Np; l++) {
                            const int nl = line_node(c, d, i, j, k, l);
                            const double a = c.Dhat[pos[d] * Np + l];
                            for (int v = 0; v < nv; v++) {
                                double t = Fv[((size_t)d * nd + nl) * nv + v];
                                t *= a;
                                dUv[v] += t;
                            }
                        }
                for (int v = 0; v < nv; v++) {
                    double t = -dU[v];
                    if (c.p.blending) t *= (1.0 - alpha);
                    if (c.p.parabolic) t = t + dUv[v];
                    t /= gJ(c, e, id1);
                    el_dudt[id1 * nv + v] += t;
                }
            }
    return lam;
}

static inline bool is_element1(const Ctx &c, int64_t e, int f)
{
    const int64_t nb = c.nbr[e * 2 * c.dim + f];
    return nb >= 0 && (e < nb || (e == nb && (f & 1)));
}

// AssembleFaceVector, Euler (DGSEMIntegrator.cpp:151-222) for face f of
// element a, a being the face's element 1: buf[0][t][v] for a's face nodes,
// buf[1][t][v] for the neighbour's matching nodes.
static double face_vector_geo(const Ctx &c, const double *u, int64_t a, int f, double *buf)
{
    const int nv = c.nv, dim = c.dim, Np = c.Np, nfn = c.ndof / Np, nf = 2 * dim;
    const int64_t b = c.nbr[a * nf + f];
    const int d = f / 2, side = f % 2;
    double lam = -1.0, s1[5], s2[5], flux[5], nor[3];
    for (int t = 0; t < nfn; t++) {
        const int n1 = face_node(c, d, side, t);
        const int n2 = c.gnode[((size_t)a * nf + f) * nfn + t];
        for (int v = 0; v < nv; v++) {
            s1[v] = u[idx(c, v, a, n1)];
            s2[v] = u[idx(c, v, b, n2)];
        }
        const double *row = gadj_row(c, a, n1, d);
        for (int k = 0; k < dim; k++) nor[k] = side ? row[k] : -row[k];
        if (c.p.parabolic && c.p.compat) {
            // velocities in the momentum slots, as the NS face integrator
            // leaves them (DGSEMIntegrator.cpp:467-481)
            double t1[5], t2[5];
            for (int v = 0; v < nv; v++) { t1[v] = s1[v]; t2[v] = s2[v]; }
            for (int q = 0; q < dim; q++) { t1[1 + q] = s1[1 + q] / s1[0]; t2[1 + q] = s2[1 + q] / s2[0]; }
            lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, t1, t2, nor, flux));
        } else {
            lam = std::max(lam, face_flux(dim, c.p.gamma, c.p.compat, c.p.face_dissipation, s1, s2, nor, flux));
        }
        double dU1[5], dU2[5];
        for (int v = 0; v < nv; v++) {
            dU2[v] = flux[v];
            dU1[v] = -flux[v];
        }
        if (c.p.parabolic) {
            // central viscous flux of both sides' states and gradients
            // (DGSEMIntegrator.cpp:435-549)
            double dq1[15], dq2[15], fm1[15], fm2[15];
            for (int q = 0; q < dim; q++)
                for (int v = 0; v < nv; v++) {
                    dq1[q * nv + v] = c.grads[(size_t)q * c.size + idx(c, v, a, n1)];
                    dq2[q * nv + v] = c.grads[(size_t)q * c.size + idx(c, v, b, n2)];
                }
            double u1[5], u2[5];
            for (int v = 0; v < nv; v++) {
                u1[v] = u[idx(c, v, a, n1)];
                u2[v] = u[idx(c, v, b, n2)];
            }
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, u1, dq1, fm1);
            viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, u2, dq2, fm2);
            for (int v = 0; v < nv; v++) {
                double fn = 0.0;
                for (int q = 0; q < dim; q++) {
                    double avg = fm1[v * dim + q];
                    avg += fm2[v * dim + q];
                    avg *= 0.5;
                    fn += avg * nor[q];
                }
                dU1[v] += fn;
                dU2[v] -= fn;
            }
        }
        const double sc1 = 1.0 / (c.w[0] * gJ(c, a, n1)), sc2 = 1.0 / (c.w[0] * gJ(c, b, n2));
        for (int v = 0; v < nv; v++) {
            buf[t * nv + v] = sc1 * dU1[v];
            buf[(size_t)nfn * nv + t * nv + v] = sc2 * dU2[v];
        }
    }
    return lam;
}

// Boundary face f of element e (BdrFaceIntegrator::AssembleFaceVector,
// BdrFaceIntegrator.cpp:64-130) with the outward normal of the node.
static double bdr_face_vector_geo(const Ctx &c, const double *u, int64_t e, int f, int b, double *out)
{
    const int nv = c.nv, dim = c.dim, nfn = c.ndof / c.Np;
    const int d = f / 2, side = f % 2;
    double lam = -1.0, s1[5], flux[5], nor[3];
    for (int t = 0; t < nfn; t++) {
        const int n = face_node(c, d, side, t);
        for (int v = 0; v < nv; v++) s1[v] = u[idx(c, v, e, n)];
        const double *row = gadj_row(c, e, n, d);
        for (int k = 0; k < dim; k++) nor[k] = side ? row[k] : -row[k];
        lam = std::max(lam, bdr_flux(c, b, s1, nor, flux));
        const double scale = 1.0 / (c.w[0] * gJ(c, e, n));
        double dU[5];
        for (int v = 0; v < nv; v++) dU[v] = -flux[v];
        const int type = (int)c.bc[b][0];
        if (c.p.parabolic && (type == 2 || type == 10 || type == 11 || type == 8)) {
            // ComputeBdrFaceViscousFlux with the node's own normal, as on box meshes
            double dq[15], fm[15], fn[5];
            for (int q = 0; q < dim; q++)
                for (int v = 0; v < nv; v++) dq[q * nv + v] = c.grads[(size_t)q * c.size + idx(c, v, e, n)];
            if (type == 8) {
                double so[5], fl[5];
                bdr_flux(c, b, s1, nor, fl, so);
                viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, so, dq, fm);
            } else {
                viscous_flux(dim, c.p.gamma, c.p.Pr, c.p.mu, s1, dq, fm);
            }
            for (int v = 0; v < nv; v++) {
                fn[v] = 0.0;
                for (int q = 0; q < dim; q++) fn[v] += fm[v * dim + q] * nor[q];
            }
            if (type == 10) {
                double en = 0.0;
                for (int q = 0; q < dim; q++) en += c.bc[b][1 + q] * fn[1 + q];
                fn[nv - 1] = en + 0.0;
            }
            for (int v = 0; v < nv; v++) dU[v] += fn[v];
        }
        for (int v = 0; v < nv; v++) out[t * nv + v] = scale * dU[v];
    }
    return lam;
}

static void lifting_geo(Ctx &c, const double *u);

static void rhs_geo(Ctx &c, const double *u, double *dudt)
{
    const int nv = c.nv, dim = c.dim, nd = c.ndof, Np = c.Np, nfn = nd / Np, nf = 2 * dim;
    if (c.p.blending) blending_coefficient(c, u);
    else {
        std::fill(c.alpha.begin(), c.alpha.end(), 0.0);
        std::fill(c.eta.begin(), c.eta.end(), 0.0);
    }
    if (c.p.parabolic) lifting_geo(c, u);
    const double *G = c.grads.data();
    double lam = -1.0;
    const size_t fstride = (size_t)2 * nfn * nv;
#pragma omp parallel for schedule(static) reduction(max : lam)
    for (int64_t e = 0; e < c.ne; e++)
        for (int f = 0; f < nf; f++)
            if (is_element1(c, e, f))
                lam = std::max(lam, face_vector_geo(c, u, e, f, &c.facebuf[((size_t)e * nf + f) * fstride]));
#pragma omp parallel for schedule(static) reduction(max : lam)
    for (int64_t e = 0; e < c.ne; e++) {
        std::vector<double> el_u(nd * nv), el_d(nd * nv), bface((size_t)nfn * nv), el_g;
        for (int n = 0; n < nd; n++)
            for (int v = 0; v < nv; v++) el_u[n * nv + v] = u[idx(c, v, e, n)];
        if (c.p.parabolic) {
            el_g.resize((size_t)dim * nd * nv);
            for (int d = 0; d < dim; d++)
                for (int n = 0; n < nd; n++)
                    for (int v = 0; v < nv; v++)
                        el_g[((size_t)d * nd + n) * nv + v] = G[(size_t)d * c.size + idx(c, v, e, n)];
        }
        lam = std::max(lam, element_vector_geo(c, e, el_u.data(), el_g.data(), c.alpha[e], el_d.data()));
        for (int n = 0; n < nd; n++)
            for (int v = 0; v < nv; v++) dudt[idx(c, v, e, n)] = 0.0 + el_d[n * nv + v];
        for (int f = 0; f < nf; f++) {
            const int64_t nb = c.nbr[e * nf + f];
            const double *mine;
            if (nb < 0) {
                lam = std::max(lam, bdr_face_vector_geo(c, u, e, f, (int)(-1 - nb), bface.data()));
                mine = bface.data();
            } else if (is_element1(c, e, f)) {
                mine = &c.facebuf[((size_t)e * nf + f) * fstride];
            } else {
                const int f2 = c.gface[e * nf + f];
                mine = &c.facebuf[((size_t)nb * nf + f2) * fstride] + (size_t)nfn * nv;
                // the neighbour's face-node order: its node n2 of face node t2 is ours at t
                std::vector<double> tmp((size_t)nfn * nv);
                for (int t2 = 0; t2 < nfn; t2++) {
                    const int n2 = c.gnode[((size_t)nb * nf + f2) * nfn + t2];  // our node
                    int t = -1;
                    for (int q = 0; q < nfn; q++)
                        if (face_node(c, f / 2, f % 2, q) == n2) t = q;
                    for (int v = 0; v < nv; v++) tmp[(size_t)t * nv + v] = mine[t2 * nv + v];
                }
                for (int n = 0; n < nfn * nv; n++) bface[n] = tmp[n];
                mine = bface.data();
            }
            for (int t = 0; t < nfn; t++) {
                const int n = face_node(c, f / 2, f % 2, t);
                for (int v = 0; v < nv; v++) dudt[idx(c, v, e, n)] += mine[t * nv + v];
            }
        }
    }
    c.last_rhs_speed = lam;
    c.max_char_speed = std::max(c.max_char_speed, lam);
}

// BR1 lifting on a general mesh (LiftingBR1.cpp:10-115 faces, :156-272
// elements, :311-407 boundary faces): per node the reference-direction
// derivatives of the entropy variables times the adjugate (mfem::Mult) times
// 1/J, each face adding 0.5 (w2 - w1) n_k / (w0 J) to both sides' gradient k
// with element 1's normal, then EntropyGrad2PrimGrad per direction.
static void lifting_geo(Ctx &c, const double *u)
{
    const int nv = c.nv, dim = c.dim, nd = c.ndof, Np = c.Np, nfn = nd / Np, nf = 2 * dim;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        double s[5], w[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, n)];
            conserv2entropy(dim, c.p.gamma, s, w);
            for (int v = 0; v < nv; v++) c.went[idx(c, v, e, n)] = w[v];
        }
    }
    const double *W = c.went.data();
    double *G = c.grads.data();
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        for (int n = 0; n < nd; n++) {
            const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            double gr[5][3] = {};
            for (int r = 0; r < dim; r++)
                for (int v = 0; v < nv; v++) {
                    double acc = 0.0;
                    for (int l = 0; l < Np; l++) {
                        double t = W[idx(c, v, e, line_node(c, r, pos[0], pos[1], pos[2], l))];
                        t *= c.D[pos[r] * Np + l];
                        acc += t;
                    }
                    gr[v][r] = acc;
                }
            const double ij = 1.0 / gJ(c, e, n);
            for (int k = 0; k < dim; k++)
                for (int v = 0; v < nv; v++) {
                    double g = 0.0;
                    for (int r = 0; r < dim; r++) g += gr[v][r] * gadj_row(c, e, n, r)[k];
                    g *= ij;
                    G[(size_t)k * c.size + idx(c, v, e, n)] = g;
                }
        }
        for (int f = 0; f < nf; f++) {
            const int d = f / 2, side = f % 2;
            const int64_t nb = c.nbr[e * nf + f];
            for (int t = 0; t < nfn; t++) {
                const int n = face_node(c, d, side, t);
                const double scale = 1.0 / (c.w[0] * gJ(c, e, n));
                double fl[5], nor[3];
                if (nb < 0) {
                    double s1[5], w1[5];
                    const double *row = gadj_row(c, e, n, d);
                    for (int k = 0; k < dim; k++) nor[k] = side ? row[k] : -row[k];
                    for (int v = 0; v < nv; v++) {
                        s1[v] = u[idx(c, v, e, n)];
                        w1[v] = W[idx(c, v, e, n)];
                    }
                    bdr_lifting_flux(c, (int)(-1 - nb), s1, w1, nor, fl);
                } else {
                    const int n2 = c.gnode[((size_t)e * nf + f) * nfn + t];
                    const bool is1 = is_element1(c, e, f);
                    const int f2 = c.gface[e * nf + f];
                    const double *row = is1 ? gadj_row(c, e, n, d) : gadj_row(c, nb, n2, f2 / 2);
                    const int sd = is1 ? side : f2 % 2;
                    for (int k = 0; k < dim; k++) nor[k] = sd ? row[k] : -row[k];
                    for (int v = 0; v < nv; v++) {
                        const double w1 = is1 ? W[idx(c, v, e, n)] : W[idx(c, v, nb, n2)];
                        const double w2 = is1 ? W[idx(c, v, nb, n2)] : W[idx(c, v, e, n)];
                        fl[v] = 0.5 * (w2 - w1);
                    }
                }
                for (int k = 0; k < dim; k++)
                    for (int v = 0; v < nv; v++) {
                        double fv = fl[v];
                        fv *= nor[k];
                        G[(size_t)k * c.size + idx(c, v, e, n)] += scale * fv;
                    }
            }
        }
        double s[5], g[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, n)];
            for (int d = 0; d < dim; d++) {
                for (int v = 0; v < nv; v++) g[v] = G[(size_t)d * c.size + idx(c, v, e, n)];
                entgrad2primgrad(dim, c.p.gamma, c.p.compat, s, g);
                for (int v = 0; v < nv; v++) G[(size_t)d * c.size + idx(c, v, e, n)] = g[v];
            }
        }
    }
}

static void rhs(Ctx &c, const double *u, double *dudt)
{
    if (c.geo) return rhs_geo(c, u, dudt);
    const int nv = c.nv, dim = c.dim, nd = c.ndof, Np = c.Np, nfn = nd / Np;
    if (c.p.blending) blending_coefficient(c, u);
    else {
        std::fill(c.alpha.begin(), c.alpha.end(), 0.0);
        std::fill(c.eta.begin(), c.eta.end(), 0.0);
    }
    if (c.p.parabolic) lifting(c, u);
    const double *G = c.grads.data();
    double lam = -1.0;
    // Face contributions first into a per-face buffer (both sides).
    const size_t fstride = (size_t)2 * nfn * nv;
#pragma omp parallel for schedule(static) reduction(max : lam)
    for (int64_t e = 0; e < c.ne; e++)
        for (int d = 0; d < dim; d++)
            lam = std::max(lam, face_vector(c, u, G, e, d, &c.facebuf[((size_t)e * dim + d) * fstride]));
#pragma omp parallel for schedule(static) reduction(max : lam)
    for (int64_t e = 0; e < c.ne; e++) {
        std::vector<double> el_u(nd * nv), el_d(nd * nv), el_g;
        for (int n = 0; n < nd; n++)
            for (int v = 0; v < nv; v++) el_u[n * nv + v] = u[idx(c, v, e, n)];
        if (c.p.parabolic) {
            el_g.resize((size_t)dim * nd * nv);
            for (int d = 0; d < dim; d++)
                for (int n = 0; n < nd; n++)
                    for (int v = 0; v < nv; v++)
                        el_g[((size_t)d * nd + n) * nv + v] = G[(size_t)d * c.size + idx(c, v, e, n)];
        }
        lam = std::max(lam, element_vector(c, el_u.data(), el_g.data(), c.alpha[e], el_d.data()));
        // dudt = 0 + element vector + face vectors (faces in -x,+x,-y,+y,-z,+z order).
        for (int n = 0; n < nd; n++)
            for (int v = 0; v < nv; v++) dudt[idx(c, v, e, n)] = 0.0 + el_d[n * nv + v];
        for (int d = 0; d < dim; d++) {
            // -d face: stored at (nbr_minus, d); this element is its "b" side.
            // A boundary -d face is evaluated here.
            int64_t em = c.nbr[e * 2 * dim + 2 * d];
            std::vector<double> bface;
            const double *mine;
            if (em < 0) {
                bface.resize((size_t)nfn * nv);
                lam = std::max(lam, bdr_face_vector(c, u, e, d, 0, (int)(-1 - em), bface.data()));
                mine = bface.data();
            } else {
                mine = &c.facebuf[((size_t)em * dim + d) * fstride] + (size_t)nfn * nv;
            }
            for (int t = 0; t < nfn; t++) {
                int n = face_node(c, d, 0, t);
                for (int v = 0; v < nv; v++) dudt[idx(c, v, e, n)] += mine[t * nv + v];
            }
            // +d face: stored at (e, d); this element is its "a" side.
            const double *mine2 = &c.facebuf[((size_t)e * dim + d) * fstride];
            for (int t = 0; t < nfn; t++) {
                int n = face_node(c, d, 1, t);
                for (int v = 0; v < nv; v++) dudt[idx(c, v, e, n)] += mine2[t * nv + v];
            }
        }
    }
    c.last_rhs_speed = lam;
    c.max_char_speed = std::max(c.max_char_speed, lam);
}

// ---------------------------------------------------------------------------
// Entropy filter, built from the intent of src/Filters/EntropyFilter.cpp
// (GetEntropyConstraints :81-158, FilterSolution :171-242, ComputeRoot
// :325-349): per-element bound = min of rho*log(p rho^-gamma) over the element
// and its face neighbours at the stage input; an element with min rho < 1e-8,
// min p < 1e-8 or min entropy < bound - 1e-4 has its modes of max degree j
// scaled by exp(-zeta j^2), zeta found by 20 bisection steps per violating
// node on [zeta, -ln 1e-10], visiting nodes in order.
// ---------------------------------------------------------------------------
static void filter_bounds(Ctx &c, const double *u)
{
    const int nv = c.nv, nd = c.ndof, dim = c.dim;
    std::vector<double> own(c.ne);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        double mn = std::numeric_limits<double>::infinity(), s[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = u[idx(c, v, e, n)];
            double rho = s[0], p = pressure(dim, c.p.gamma, s);
            mn = std::min(mn, entropy_fn(rho, p, c.p.gamma));
        }
        own[e] = mn;
    }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < c.ne; e++) {
        double mn = own[e];
        for (int f = 0; f < 2 * dim; f++)
            if (c.nbr[e * 2 * dim + f] >= 0) mn = std::min(mn, own[c.nbr[e * 2 * dim + f]]);
        c.emin[e] = mn;
    }
}

static void filter_apply(Ctx &c, double *x)
{
    const int nv = c.nv, nd = c.ndof, dim = c.dim, Np = c.Np;
    const double rho_min = 1e-8, p_min = 1e-8, ent_tol = 1e-4, epsilon = 1e-10;
    const int N_iter = 20;
    int64_t nf = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : nf)
    for (int64_t e = 0; e < c.ne; e++) {
        double s[5];
        double mr = std::numeric_limits<double>::infinity(), mp = mr, me = mr;
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = x[idx(c, v, e, n)];
            double rho = s[0], p = pressure(dim, c.p.gamma, s);
            me = std::min(me, entropy_fn(rho, p, c.p.gamma));
            mr = std::min(mr, rho);
            mp = std::min(mp, p);
        }
        const double bound = c.emin[e];
        if (!(mr < rho_min || mp < p_min || me < bound - ent_tol)) continue;
        nf++;
        std::vector<double> modes((size_t)nd * nv, 0.0), hs((size_t)Np * nv);
        for (int v = 0; v < nv; v++)
            for (int r = 0; r < nd; r++) {
                double acc = 0.0;
                for (int k = 0; k < nd; k++) acc += c.Vinv[r * nd + k] * x[idx(c, v, e, k)];
                modes[(size_t)r * nv + v] = acc;
            }
        auto violates = [&](const double *st) {
            double rho = st[0], p = pressure(dim, c.p.gamma, st);
            double en = entropy_fn(rho, p, c.p.gamma);
            return rho < rho_min || p < p_min || en < bound - ent_tol;
        };
        auto filter_modes = [&](double zeta, double *st) {  // FilterModes :160-169
            for (int v = 0; v < nv; v++) st[v] = hs[v];
            for (int j = 1; j < Np; j++) {
                double fac = std::exp(-zeta * std::pow(j, 2));
                for (int v = 0; v < nv; v++) st[v] += hs[(size_t)j * nv + v] * fac;
            }
        };
        double zeta = 0.0;
        for (int i = 0; i < nd; i++) {
            std::fill(hs.begin(), hs.end(), 0.0);  // ComputeHierarchStates :244-260
            for (int j = 0; j < Np; j++)
                for (int v = 0; v < nv; v++)
                    for (int l = 0; l < nd; l++)
                        if (c.max_order[l] == j) hs[(size_t)j * nv + v] += c.Vdm[i * nd + l] * modes[(size_t)l * nv + v];
            filter_modes(zeta, s);
            if (violates(s)) {  // ComputeRoot :325-349
                double z1 = zeta, z2 = -std::log(epsilon);
                for (int it = 0; it < N_iter; it++) {
                    double z3 = 0.5 * (z1 + z2);
                    filter_modes(z3, s);
                    if (violates(s)) z1 = z3;
                    else z2 = z3;
                }
                zeta = z2;
            }
        }
        std::vector<double> ffac(Np, 1.0);
        for (int d = 1; d < Np; d++) ffac[d] = std::exp(-zeta * std::pow(d, 2));
        for (int i = 0; i < nd; i++)
            for (int v = 0; v < nv; v++) {
                double tmp = 0.0;
                for (int j = 0; j < Np; j++)
                    for (int l = 0; l < nd; l++)
                        if (c.max_order[l] == j) tmp += ffac[j] * c.Vdm[i * nd + l] * modes[(size_t)l * nv + v];
                x[idx(c, v, e, i)] = tmp;
            }
    }
    c.filtered_elements += nf;
}

// ---------------------------------------------------------------------------
// Positivity-preserving limiter (params.filter & 2).  The reference's
// MinmodLimiter::LimitSolution limits nothing (src/Limiters/MinmodLimiter.cpp:
// 22-77) and no positivity limiter exists there; this restates the published
// one of Zhang & Shu (J. Comput. Phys. 229 (2010) 8918-8934): per element,
// with the LGL means u_bar and eps = min(1e-13, rho_bar, p(u_bar)),
//   (1) rho_i <- rho_bar + th1 (rho_i - rho_bar), th1 = (rho_bar - eps) /
//       (rho_bar - min rho_i), when min rho_i < eps;
//   (2) u_i <- u_bar + th2 (u_i - u_bar), th2 = min over nodes with
//       p(u_i) < eps of (p_bar - eps) / (p_bar - p(u_i)): p is concave in u,
//       so p(u_bar + th (u_i - u_bar)) >= (1 - th) p_bar + th p(u_i) = eps.
// Element means are unchanged, so the limiter conserves.
// ---------------------------------------------------------------------------
static void positivity_apply(Ctx &c, double *x)
{
    const int nv = c.nv, nd = c.ndof, dim = c.dim, Np = c.Np;
    int64_t nl = 0;
#pragma omp parallel for schedule(static) reduction(+ : nl)
    for (int64_t e = 0; e < c.ne; e++) {
        double m[5] = {0, 0, 0, 0, 0}, W = 0.0, rmin = std::numeric_limits<double>::infinity();
        for (int n = 0; n < nd; n++) {
            double wn = c.w[n % Np] * c.w[(n / Np) % Np];
            if (dim == 3) wn *= c.w[n / (Np * Np)];
            if (c.geo) wn *= c.gJ[(size_t)e * nd + n];  // general geometry: the J-weighted mean
            W += wn;
            for (int v = 0; v < nv; v++) m[v] += wn * x[idx(c, v, e, n)];
            rmin = std::min(rmin, x[idx(c, 0, e, n)]);
        }
        for (int v = 0; v < nv; v++) m[v] /= W;
        const double eps = std::min(1e-13, std::min(m[0], pressure(dim, c.p.gamma, m)));
        bool limited = false;
        if (rmin < eps) {
            const double th = (m[0] - eps) / (m[0] - rmin);
            for (int n = 0; n < nd; n++) x[idx(c, 0, e, n)] = m[0] + th * (x[idx(c, 0, e, n)] - m[0]);
            limited = true;
        }
        const double pbar = pressure(dim, c.p.gamma, m);
        double th2 = 1.0, s[5];
        for (int n = 0; n < nd; n++) {
            for (int v = 0; v < nv; v++) s[v] = x[idx(c, v, e, n)];
            const double p = pressure(dim, c.p.gamma, s);
            if (p < eps) th2 = std::min(th2, (pbar - eps) / (pbar - p));
        }
        if (th2 < 1.0) {
            for (int n = 0; n < nd; n++)
                for (int v = 0; v < nv; v++) x[idx(c, v, e, n)] = m[v] + th2 * (x[idx(c, v, e, n)] - m[v]);
            limited = true;
        }
        nl += limited;
    }
    c.limited_elements += nl;
}

// RK3SSPSolver::Step (Shu-Osher SSP-RK3), optionally filtering each stage.
static void rk3_step(Ctx &c, double dt, double *x)
{
    const int64_t n = c.size;
    double *k = c.k1.data(), *y = c.y1.data(), *z = c.z1.data();
    const bool ef = c.p.filter & 1, pl = c.p.filter & 2;
    if (ef) filter_bounds(c, x);
    rhs(c, x, k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) y[i] = x[i] + dt * k[i];
    if (ef) filter_apply(c, y);
    if (pl) positivity_apply(c, y);
    if (ef) filter_bounds(c, y);
    rhs(c, y, k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        z[i] = y[i] + dt * k[i];
        y[i] = 3. / 4 * x[i] + 1. / 4 * z[i];
    }
    if (ef) filter_apply(c, y);
    if (pl) positivity_apply(c, y);
    if (ef) filter_bounds(c, y);
    rhs(c, y, k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        z[i] = y[i] + dt * k[i];
        x[i] = 1. / 3 * x[i] + 2. / 3 * z[i];
    }
    if (ef) filter_apply(c, x);
    if (pl) positivity_apply(c, x);
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C interface (used only by tests/, smoke() and bench.py's CPU baseline)
// ---------------------------------------------------------------------------
using orc::Ctx;

extern "C" {

void *orc_create(const pdg_mesh *m, const pdg_params *p)
{
    if (!m || !p || (m->dim != 2 && m->dim != 3) || m->order < 1 || m->num_elements < 1) return nullptr;
    Ctx *c = new Ctx();
    c->p = *p;
    c->dim = m->dim;
    c->N = m->order;
    c->Np = m->order + 1;
    c->ndof = 1;
    for (int d = 0; d < c->dim; d++) c->ndof *= c->Np;
    c->nv = c->dim + 2;
    c->ne = m->num_elements;
    c->nnodes = c->ne * c->ndof;
    c->size = c->nnodes * c->nv;
    for (int d = 0; d < 3; d++) c->h[d] = d < c->dim ? m->h[d] : 1.0;
    c->nbr.assign(m->nbr, m->nbr + (size_t)c->ne * 2 * c->dim);
    for (int32_t nb : c->nbr)  // boundary faces: conditions 0..15
        if (nb >= c->ne || nb < -16) { delete c; return nullptr; }
    orc::gll(c->Np, c->x, c->w);
    orc::build_derivative_matrices(*c);
    if (c->dim == 2) {
        c->J = c->h[0] * c->h[1];
        c->adj[0] = c->h[1];
        c->adj[1] = c->h[0];
        c->area[0] = c->h[1];
        c->area[1] = c->h[0];
    } else {
        c->J = c->h[0] * (c->h[1] * c->h[2]);
        c->adj[0] = c->h[1] * c->h[2];
        c->adj[1] = c->h[0] * c->h[2];
        c->adj[2] = c->h[0] * c->h[1];
        c->area[0] = c->h[1] * c->h[2];
        c->area[1] = c->h[0] * c->h[2];
        c->area[2] = c->h[0] * c->h[1];
    }
    orc::build_subcell_normals(*c);
    orc::build_modal(*c);
    c->modalThreshold = 0.5 * std::pow(10.0, -1.8 * std::pow(c->N, 0.25));
    c->eta.assign(c->ne, 0.0);
    c->alpha.assign(c->ne, 0.0);
    if (c->p.parabolic) {
        c->grads.assign((size_t)c->dim * c->size, 0.0);
        c->went.assign(c->size, 0.0);
    }
    c->facebuf.assign((size_t)c->ne * c->dim * 2 * (c->ndof / c->Np) * c->nv, 0.0);
    c->emin.assign(c->ne, std::numeric_limits<double>::infinity());
    c->k1.assign(c->size, 0.0);
    c->y1.assign(c->size, 0.0);
    c->z1.assign(c->size, 0.0);
    c->max_char_speed = -1.0;
    c->last_rhs_speed = -1.0;
    c->filtered_elements = 0;
    c->limited_elements = 0;
    return c;
}

void orc_destroy(void *h) { delete (Ctx *)h; }

// General geometry (Euler): node coordinates x[k*nnodes + e*ndof + n] and
// face orientation codes (NULL: opposite faces, aligned axes), as
// pdg_set_geometry takes them.  J and the adjugate at every node from the
// LGL derivative of the coordinates (MFEM's element transformation at the
// integration points), the subcell metrics as ComputeSubcellMetrics forms
// them (DGSEMIntegrator.cpp:1199-1304).  Returns 0, or 1 on a bad input.
int orc_set_geometry(void *h, const double *x, const int32_t *face_orient)
{
    Ctx &c = *(Ctx *)h;
    const int dim = c.dim, Np = c.Np, N = c.N, nd = c.ndof, nf = 2 * dim, nfn = nd / Np;
    c.gJ.assign((size_t)c.ne * nd, 0.0);
    c.gadj.assign((size_t)c.ne * nd * 9, 0.0);
    for (int64_t e = 0; e < c.ne; e++)
        for (int n = 0; n < nd; n++) {
            const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            double A[3][3] = {};  // A[k][r] = dx_k / dxi_r
            for (int k = 0; k < dim; k++)
                for (int r = 0; r < dim; r++) {
                    double t = 0.0;
                    for (int l = 0; l < Np; l++) {
                        const int m = line_node(c, r, pos[0], pos[1], pos[2], l);
                        t += c.D[pos[r] * Np + l] * x[(size_t)k * c.nnodes + e * nd + m];
                    }
                    A[k][r] = t;
                }
            double adj[3][3] = {}, det;
            if (dim == 2) {
                adj[0][0] = A[1][1];
                adj[0][1] = -A[0][1];
                adj[1][0] = -A[1][0];
                adj[1][1] = A[0][0];
                det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
            } else {
                // cofactor transpose: adj[r][k] = (-1)^(r+k) minor(k, r)
                for (int r = 0; r < 3; r++)
                    for (int k = 0; k < 3; k++) {
                        const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, k1 = (k + 1) % 3, k2 = (k + 2) % 3;
                        adj[r][k] = A[k1][r1] * A[k2][r2] - A[k1][r2] * A[k2][r1];
                    }
                det = A[0][0] * adj[0][0] + A[0][1] * adj[1][0] + A[0][2] * adj[2][0];
            }
            if (!(det > 0.0)) return 1;
            c.gJ[(size_t)e * nd + n] = det;
            for (int r = 0; r < 3; r++)
                for (int k = 0; k < 3; k++) c.gadj[(((size_t)e * nd + n) * 3 + r) * 3 + k] = adj[r][k];
        }
    // subcell metrics: n_i = row(x_0) + sum_{l<i} w_l sum_m D(l, m) row(x_m)
    c.gsnor.assign((size_t)c.ne * dim * nfn * (Np + 1) * 3, 0.0);
    for (int64_t e = 0; e < c.ne; e++)
        for (int d = 0; d < dim; d++)
            for (int line = 0; line < nfn; line++) {
                int fi = 0, fj = 0, fk = 0;
                if (d == 0) { fj = line % Np; fk = line / Np; }
                else if (d == 1) { fi = line % Np; fk = line / Np; }
                else { fi = line % Np; fj = line / Np; }
                double *out = &c.gsnor[((((size_t)e * dim + d) * nfn + line) * (Np + 1)) * 3];
                const double *m0 = gadj_row(c, e, line_node(c, d, fi, fj, fk, 0), d);
                for (int i = 0; i < Np + 1; i++) {
                    double nor[3] = {0, 0, 0};
                    for (int k = 0; k < dim; k++) nor[k] = m0[k];
                    for (int l = 0; l < i; l++) {
                        double tmp[3] = {0, 0, 0};
                        for (int m = 0; m < Np; m++) {
                            const double *mr = gadj_row(c, e, line_node(c, d, fi, fj, fk, m), d);
                            for (int k = 0; k < dim; k++) {
                                double t = mr[k];
                                t *= c.D[l * Np + m];
                                tmp[k] += t;
                            }
                        }
                        for (int k = 0; k < dim; k++) {
                            tmp[k] *= c.w[l];
                            nor[k] += tmp[k];
                        }
                    }
                    for (int k = 0; k < dim; k++) out[(size_t)i * 3 + k] = nor[k];
                }
            }
    // faces: the neighbour's face and the node matching each face node
    c.gface.assign((size_t)c.ne * nf, 0);
    c.gnode.assign((size_t)c.ne * nf * nfn, 0);
    for (int64_t e = 0; e < c.ne; e++)
        for (int f = 0; f < nf; f++) {
            const int64_t nb = c.nbr[e * nf + f];
            if (nb < 0) continue;
            int f2 = f ^ 1, o = 0;
            if (face_orient) {
                f2 = face_orient[e * nf + f] & 7;
                o = face_orient[e * nf + f] >> 3;
            }
            if (f2 >= nf || c.nbr[nb * nf + f2] != e) return 1;
            c.gface[e * nf + f] = f2;
            for (int t = 0; t < nfn; t++) {
                int a = t % Np, b = dim == 3 ? t / Np : 0;
                if (o & 1) std::swap(a, b);
                if (o & 2) a = N - a;
                if (o & 4) b = N - b;
                c.gnode[((size_t)e * nf + f) * nfn + t] = face_node(c, f2 / 2, f2 % 2, a + Np * b);
            }
        }
    c.facebuf.assign((size_t)c.ne * nf * 2 * nfn * c.nv, 0.0);
    c.geo = true;
    return 0;
}

// Boundary condition `index`: its type and parameters as pdg_set_boundary
// takes them (types 1, 3: conserved state; 6: p; 7: rho, velocity; 8: cp,
// pt, Tt, theta, phi in degrees, stored as cp, pt, Tt, cos theta, sin theta;
// 9: primitive state rho, velocity, p; 10: wall velocity; 11: wall
// temperature and velocity, stored as velocity, 1/(R T)).
void orc_set_boundary(void *h, int index, int type, const double *state)
{
    Ctx &c = *(Ctx *)h;
    if (index < 0 || index >= 16) return;
    const int n = type == 6 ? 1 : type == 7 ? 1 + c.dim : type == 8 ? 5 : type == 10 ? c.dim : type == 11 ? 1 + c.dim : c.nv;
    c.bc[index][0] = type;
    for (int v = 0; v < 7; v++) c.bc[index][1 + v] = (state && v < n) ? state[v] : 0.0;
    if (type == 11 && state) {  // {T, V} -> V, 1/(R T)
        for (int q = 0; q < c.dim; q++) c.bc[index][1 + q] = state[1 + q];
        c.bc[index][1 + c.dim] = 1.0 / (c.p.R_gas * state[0]);
    }
    if (type == 8) {
        const double theta = c.bc[index][4];
        c.bc[index][4] = std::cos(theta * M_PI / 180.0);
        c.bc[index][5] = std::sin(theta * M_PI / 180.0);
    }
}

void orc_rhs(void *h, const double *u, double *dudt) { orc::rhs(*(Ctx *)h, u, dudt); }

void orc_rk3_step(void *h, double dt, double *u) { orc::rk3_step(*(Ctx *)h, dt, u); }

double orc_max_char_speed(void *h)
{
    Ctx *c = (Ctx *)h;
    return c->p.compat ? c->max_char_speed : c->last_rhs_speed;
}

void orc_get_blending(void *h, double *eta, double *alpha)
{
    Ctx *c = (Ctx *)h;
    if (eta) std::memcpy(eta, c->eta.data(), sizeof(double) * c->ne);
    if (alpha) std::memcpy(alpha, c->alpha.data(), sizeof(double) * c->ne);
}

void orc_get_gradients(void *h, double *g)
{
    Ctx *c = (Ctx *)h;
    if (c->p.parabolic) std::memcpy(g, c->grads.data(), sizeof(double) * c->grads.size());
}

int64_t orc_filtered_elements(void *h) { return ((Ctx *)h)->filtered_elements; }
int64_t orc_limited_elements(void *h) { return ((Ctx *)h)->limited_elements; }
void orc_positivity_apply(void *h, double *u) { orc::positivity_apply(*(Ctx *)h, u); }

void orc_filter_bounds(void *h, const double *u) { orc::filter_bounds(*(Ctx *)h, u); }
void orc_filter_apply(void *h, double *u) { orc::filter_apply(*(Ctx *)h, u); }

// Stage update of pdg_rk_stage: uout = a*un + b*(us + dt*L(us)).
void orc_rk_stage(void *h, int stage, double dt, const double *un, const double *us, double *uout)
{
    Ctx *c = (Ctx *)h;
    if (c->p.filter & 1) orc::filter_bounds(*c, us);
    orc::rhs(*c, us, c->k1.data());
    const double *k = c->k1.data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < c->size; i++) {
        double z = us[i] + dt * k[i];
        if (stage == 0) uout[i] = z;
        else if (stage == 1) uout[i] = 3. / 4 * un[i] + 1. / 4 * z;
        else uout[i] = 1. / 3 * un[i] + 2. / 3 * z;
    }
    if (c->p.filter & 1) orc::filter_apply(*c, uout);
    if (c->p.filter & 2) orc::positivity_apply(*c, uout);
}

void orc_gll(int Np, double *x, double *w)
{
    std::vector<double> xx, ww;
    orc::gll(Np, xx, ww);
    std::memcpy(x, xx.data(), sizeof(double) * Np);
    std::memcpy(w, ww.data(), sizeof(double) * Np);
}

void orc_derivative_matrices(int Np, double *D, double *Dhat, double *Dhat2)
{
    Ctx c;
    c.Np = Np;
    orc::gll(Np, c.x, c.w);
    orc::build_derivative_matrices(c);
    std::memcpy(D, c.D.data(), sizeof(double) * Np * Np);
    std::memcpy(Dhat, c.Dhat.data(), sizeof(double) * Np * Np);
    std::memcpy(Dhat2, c.Dhat2.data(), sizeof(double) * Np * Np);
}

double orc_logmean(double x, double y) { return orc::logmean(x, y); }

double orc_volume_flux(int dim, double gamma, const double *s1, const double *s2, const double *m1,
                       const double *m2, double *F)
{
    return orc::volume_flux(dim, gamma, s1, s2, m1, m2, F);
}

double orc_face_flux(int dim, double gamma, int compat, const double *s1, const double *s2,
                     const double *nor, double *F)
{
    return orc::face_flux(dim, gamma, compat, 1.0, s1, s2, nor, F);
}

void orc_viscous_flux(int dim, double gamma, double Pr, double mu, const double *state, const double *dq,
                      double *flux)
{
    orc::viscous_flux(dim, gamma, Pr, mu, state, dq, flux);
}

void orc_conserv2entropy(int dim, double gamma, const double *state, double *w)
{
    orc::conserv2entropy(dim, gamma, state, w);
}

void orc_entgrad2primgrad(int dim, double gamma, int compat, const double *state, double *g)
{
    orc::entgrad2primgrad(dim, gamma, compat, state, g);
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // extern "C"
