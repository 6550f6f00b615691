// physics.cuh — FP64 pointwise physics of the DGSEM right-hand side, device side.
//
// Each function restates one reference function (cited) for sm_100a, with the
// same quantities evaluated with fewer divisions: per-node reciprocals are
// computed once, and both log-means of a two-point flux share the reciprocal
// of the sum of their arguments.  All arithmetic is FP64 with CUDA's own
// division, sqrt and log; results differ from the reference's formulas by
// rounding only (the parity tests bound them at 1e-12 relative).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Pointwise functions compile for host and device, so that host-side checks
// can run them on the CPU.
#define PDG_FN __host__ __device__ __forceinline__

namespace pdg {

// Log-mean (y - x) / (ln y - ln x) of ComputeLogMean
// (src/BasicOperations/BasicOperations.cpp:6-12): with f = (y-x)/(y+x) and
// u = f^2 (equal to the reference's (xi-1)^2/(xi+1)^2, xi = y/x), the series
// branch u < 1e-4 is (x+y) 52.5 / (105 + u(35 + u(21 + 15u))), otherwise
// (y-x)/log(y/x).  Returns the mean and its reciprocal; `is` = 1/(x+y).
PDG_FN void logmean_inv(double x, double y, double s, double is, double &mean, double &inv)
{
    const double f = (y - x) * is;
    const double u = f * f;
    if (u < 1e-4) {
        const double P = 105.0 + u * (35.0 + u * (21.0 + 15.0 * u));
        mean = s * 52.5 / P;
        inv = P * is * (1.0 / 52.5);
    } else {
        const double L = log(y / x);
        mean = (y - x) / L;
        inv = L / (y - x);
    }
}
// Reciprocal of the log-mean only.
PDG_FN double logmean_recip(double x, double y, double is)
{
    const double f = (y - x) * is;
    const double u = f * f;
    if (u < 1e-4) return (105.0 + u * (35.0 + u * (21.0 + 15.0 * u))) * is * (1.0 / 52.5);
    return log(y / x) / (y - x);
}

// The means a two-point flux needs: rho_ln and 1/rho_ln, 1/beta_ln, 1/(beta_a
// + beta_b) and p_hat = (rho_a + rho_b) / (2 (beta_a + beta_b)), with the
// log-means of ComputeLogMean (BasicOperations.cpp:6-12).  One division
// gives both 1/(rho_a + rho_b) and 1/(beta_a + beta_b).  In the series branch
// (u < 1e-4) the mean 52.5 (x+y) / P(u), P = 105 + u(35 + u(21 + 15u)), is
// (x+y)/2 (1 + dlt)^-1 with dlt = P/105 - 1 < 3.4e-5, expanded to third order
// (the omitted dlt^4 is below 1.3e-18 relative), so that branch needs no
// further division; the log branch is as in logmean_inv.
PDG_FN void two_point_means(double ra, double rb, double ba, double bb, double &rho_ln, double &irho_ln,
                            double &ibeta_ln, double &isb, double &p_hat)
{
    const double s = ra + rb, B = ba + bb;
    const double r1 = 1.0 / (s * B);
    const double isr = B * r1;
    isb = s * r1;
    const double dr = rb - ra, db = bb - ba;
    const double fr = dr * isr, fb = db * isb;
    const double ur = fr * fr, ub = fb * fb;
    if (ur < 1e-4) {
        const double dlt = (ur * (35.0 + ur * (21.0 + 15.0 * ur))) * (1.0 / 105.0);
        rho_ln = (0.5 * s) * (1.0 - dlt * (1.0 - dlt * (1.0 - dlt)));
        irho_ln = (2.0 * isr) * (1.0 + dlt);
    } else {
        const double L = log(rb / ra);
        rho_ln = dr / L;
        irho_ln = L / dr;
    }
    if (ub < 1e-4) {
        const double dlt = (ub * (35.0 + ub * (21.0 + 15.0 * ub))) * (1.0 / 105.0);
        ibeta_ln = (2.0 * isb) * (1.0 + dlt);
    } else {
        ibeta_ln = log(bb / ba) / db;
    }
    p_hat = 0.5 * s * isb;
}

// Primitive quantities of one state, as the Chandrashekar flux derives them
// (ChandrashekarFlux.cpp:17-68): v = m / rho, p = (g-1)(E - rho |v|^2 / 2),
// beta = rho / (2p), plus 1/rho, 1/beta and the wave speed |v| + c.
template <int DIM> struct Prim {
    double rho, irho, v[DIM], p, beta, ib, lam;
};

template <int DIM> PDG_FN Prim<DIM> make_prim(const double *s, double gamma, double gm1)
{
    Prim<DIM> q;
    q.rho = s[0];
    q.irho = 1.0 / q.rho;
    double vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        q.v[d] = s[1 + d] * q.irho;
        vsq += q.v[d] * q.v[d];
    }
    q.p = gm1 * (s[DIM + 1] - 0.5 * q.rho * vsq);
    q.beta = 0.5 * q.rho / q.p;
    q.ib = 2.0 * q.p * q.irho;
    q.lam = sqrt(vsq) + sqrt(gamma * q.p * q.irho);
    return q;
}

// ChandrashekarFlux::ComputeVolumeFlux (ChandrashekarFlux.cpp:11-83) for a
// contravariant metric `metric` along axis DIR.
template <int DIM, int DIR>
PDG_FN void volume_flux(const Prim<DIM> &a, const Prim<DIM> &b, double metric, double gm1inv,
                                            double *F)
{
    double rho_ln, irho_ln, ibeta_ln, isb, p_hat;
    two_point_means(a.rho, b.rho, a.beta, b.beta, rho_ln, irho_ln, ibeta_ln, isb, p_hat);
    double vm[DIM];
    double h_hat = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    const double Vn = vm[DIR] * metric;
    const double fm = rho_ln * Vn;
    F[0] = fm;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = fm * vm[d] + (d == DIR ? p_hat * metric : 0.0);
    F[1 + DIM] = fm * h_hat;
}

// Same flux for a runtime direction d.
template <int DIM>
PDG_FN void volume_flux_rt(const Prim<DIM> &a, const Prim<DIM> &b, int dir, double metric,
                                               double gm1inv, double *F)
{
    double rho_ln, irho_ln, ibeta_ln, isb, p_hat;
    two_point_means(a.rho, b.rho, a.beta, b.beta, rho_ln, irho_ln, ibeta_ln, isb, p_hat);
    double vm[DIM];
    double h_hat = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    double vd = vm[0];
#pragma unroll
    for (int d = 1; d < DIM; d++) vd = dir == d ? vm[d] : vd;
    const double Vn = vd * metric;
    const double fm = rho_ln * Vn;
    F[0] = fm;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = fm * vm[d] + (d == dir ? p_hat * metric : 0.0);
    F[1 + DIM] = fm * h_hat;
}

// ChandrashekarFlux::ComputeFaceFlux (ChandrashekarFlux.cpp:85-161) for a
// normal of magnitude |nrm| along axis DIR (sign in nrm).  ma/mb are the
// momenta whose jump the Lax-Friedrichs term uses; compat keeps the 3D
// energy term as the reference writes it (`rho_mean * dw + w_mean`, :131).
template <int DIM, int DIR>
PDG_FN void face_flux(const Prim<DIM> &a, const Prim<DIM> &b, const double *ma, const double *mb,
                                          double nrm, double gm1inv, bool compat, double diss_scale, double *F)
{
    double rho_ln, irho_ln, ibeta_ln, isb, p_hat;
    two_point_means(a.rho, b.rho, a.beta, b.beta, rho_ln, irho_ln, ibeta_ln, isb, p_hat);
    const double rho_mean = 0.5 * (a.rho + b.rho), drho = b.rho - a.rho;
    double vm[DIM];
    double h_hat = 0.0, diss = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        const double dv = b.v[d] - a.v[d];
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
        if (DIM == 3 && d == 2 && compat)
            diss += 0.5 * drho * a.v[d] * b.v[d] + rho_mean * dv + vm[d];
        else
            diss += 0.5 * drho * a.v[d] * b.v[d] + rho_mean * dv * vm[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    diss += 0.5 * drho * gm1inv * ibeta_ln + 0.5 * rho_mean * gm1inv * (b.ib - a.ib);
    const double lam = 0.5 * fmax(a.lam, b.lam) * diss_scale * fabs(nrm);
    const double Vn = vm[DIR] * nrm;
    const double fm = rho_ln * Vn;
    F[0] = fm - lam * drho;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = fm * vm[d] + (d == DIR ? p_hat * nrm : 0.0) - lam * (mb[d] - ma[d]);
    F[1 + DIM] = fm * h_hat - lam * diss;
}

// volume_flux for a general contravariant metric vector n (the mean of the
// two nodes' metric rows on a curved element, ChandrashekarFlux.cpp:11-83):
// Vn = v_mean . n and the pressure term p_hat n.
template <int DIM>
PDG_FN void volume_flux_n(const Prim<DIM> &a, const Prim<DIM> &b, const double *n, double gm1inv, double *F)
{
    double rho_ln, irho_ln, ibeta_ln, isb, p_hat;
    two_point_means(a.rho, b.rho, a.beta, b.beta, rho_ln, irho_ln, ibeta_ln, isb, p_hat);
    double vm[DIM];
    double h_hat = 0.0, Vn = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
        Vn += vm[d] * n[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    const double fm = rho_ln * Vn;
    F[0] = fm;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = fm * vm[d] + p_hat * n[d];
    F[1 + DIM] = fm * h_hat;
}

// face_flux for a general normal vector n (ChandrashekarFlux.cpp:85-161): the
// Lax-Friedrichs term scales with |n|.
template <int DIM>
PDG_FN void face_flux_n(const Prim<DIM> &a, const Prim<DIM> &b, const double *ma, const double *mb,
                        const double *n, double gm1inv, bool compat, double diss_scale, double *F)
{
    double rho_ln, irho_ln, ibeta_ln, isb, p_hat;
    two_point_means(a.rho, b.rho, a.beta, b.beta, rho_ln, irho_ln, ibeta_ln, isb, p_hat);
    const double rho_mean = 0.5 * (a.rho + b.rho), drho = b.rho - a.rho;
    double vm[DIM];
    double h_hat = 0.0, diss = 0.0, Vn = 0.0, nn = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        const double dv = b.v[d] - a.v[d];
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
        if (DIM == 3 && d == 2 && compat)
            diss += 0.5 * drho * a.v[d] * b.v[d] + rho_mean * dv + vm[d];
        else
            diss += 0.5 * drho * a.v[d] * b.v[d] + rho_mean * dv * vm[d];
        Vn += vm[d] * n[d];
        nn += n[d] * n[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    diss += 0.5 * drho * gm1inv * ibeta_ln + 0.5 * rho_mean * gm1inv * (b.ib - a.ib);
    const double lam = 0.5 * fmax(a.lam, b.lam) * diss_scale * sqrt(nn);
    const double fm = rho_ln * Vn;
    F[0] = fm - lam * drho;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = fm * vm[d] + p_hat * n[d] - lam * (mb[d] - ma[d]);
    F[1 + DIM] = fm * h_hat - lam * diss;
}

// NavierStokesFlux::ComputeViscousFlux (src/Fluxes/NavierStokesFlux.cpp:12-90),
// constant mu, mu_bulk = 2/3, column `dir` only (flux along x_dir): momentum
// rows out[0..DIM-1] and the energy row out[DIM].  g(d, v) returns the
// primitive gradient of variable v along x_d.
template <int DIM, class Grad>
PDG_FN void viscous_col(const Prim<DIM> &q, const Grad &g, int dir, double gm1inv, double mu,
                                            double lambda_k, double *out)
{
    double div = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) div += g(d, 1 + d);
    const double mu_bulk = 2.0 / 3.0;
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < DIM; i++) {
        const double tau = (i == dir) ? mu * (2.0 * g(dir, 1 + i) - mu_bulk * div) : mu * (g(dir, 1 + i) + g(i, 1 + dir));
        out[i] = tau;
        e += q.v[i] * tau;
    }
    const double cv_dT = gm1inv * q.irho * (g(dir, DIM + 1) - q.p * q.irho * g(dir, 0));
    out[DIM] = e + lambda_k * cv_dT;
}

// Conserv2Entropy (BasicOperations.cpp:134-157): beta = rho / p,
// s = ln p - gamma ln rho.
template <int DIM>
PDG_FN void entropy_vars(const double *s, double gamma, double gm1, double gm1inv, double *w)
{
    const double rho = s[0], irho = 1.0 / rho;
    double vel[DIM], vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = s[1 + d] * irho;
        vv += vel[d] * vel[d];
    }
    const double v_sq = 0.5 * vv;
    const double p = gm1 * (s[DIM + 1] - rho * v_sq);
    const double beta = rho / p;
    const double sent = log(p) - gamma * log(rho);
    w[0] = (gamma - sent) * gm1inv - beta * v_sq;
#pragma unroll
    for (int d = 0; d < DIM; d++) w[1 + d] = beta * vel[d];
    w[DIM + 1] = -beta;
}

// EntropyGrad2PrimGrad (BasicOperations.cpp:179-223) for one direction: g
// holds the entropy-variable gradient on entry, the primitive gradient on
// exit.  compat keeps the reference's density term, which reads velocities
// where the formula means momenta (its row copy is divided in place, :190-191).
template <int DIM>
PDG_FN void entgrad_to_primgrad(const double *s, double gm1, double gm1inv, bool compat, double *g)
{
    const double rho = s[0], irho = 1.0 / rho;
    double vel[DIM], vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = s[1 + d] * irho;
        vv += vel[d] * vel[d];
    }
    const double v_sq = 0.5 * vv;
    const double p = gm1 * (s[DIM + 1] - rho * v_sq);
    const double KE = v_sq * rho;
    const double gl = g[DIM + 1];
    const double pr = p * irho;
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        g[1 + d] = pr * (g[1 + d] + vel[d] * gl);
        acc += (compat ? vel[d] : s[1 + d]) * g[1 + d];
    }
    g[0] = rho * g[0] - gl * (KE - p * gm1inv) + rho / p * acc;
    g[DIM + 1] = pr * (g[0] + p * gl);
}

// State quantities entgrad_to_primgrad and viscous_col derive from a node's
// conservative state, formed once per node when all directions need them.
template <int DIM> struct NodeState {
    double rho, irho, vel[DIM], v_sq, p, pr, rop, KE;
};
template <int DIM> PDG_FN NodeState<DIM> node_state(const double *s, double gm1)
{
    NodeState<DIM> q;
    q.rho = s[0];
    q.irho = 1.0 / q.rho;
    double vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        q.vel[d] = s[1 + d] * q.irho;
        vv += q.vel[d] * q.vel[d];
    }
    q.v_sq = 0.5 * vv;
    q.p = gm1 * (s[DIM + 1] - q.rho * q.v_sq);
    q.KE = q.v_sq * q.rho;
    q.pr = q.p * q.irho;
    q.rop = q.rho / q.p;
    return q;
}
// entgrad_to_primgrad with the node quantities formed beforehand (same
// arithmetic, so the same values).
template <int DIM>
PDG_FN void entgrad_to_primgrad_q(const NodeState<DIM> &q, const double *s, double gm1inv, bool compat, double *g)
{
    const double gl = g[DIM + 1];
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        g[1 + d] = q.pr * (g[1 + d] + q.vel[d] * gl);
        acc += (compat ? q.vel[d] : s[1 + d]) * g[1 + d];
    }
    g[0] = q.rho * g[0] - gl * (q.KE - q.p * gm1inv) + q.rop * acc;
    g[DIM + 1] = q.pr * (g[0] + q.p * gl);
}

}  // namespace pdg
