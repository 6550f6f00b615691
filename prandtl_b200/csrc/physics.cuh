// physics.cuh — FP64 pointwise physics of the DGSEM right-hand side, device side.
//
// Each function restates one reference function (cited) for sm_100a.  All
// arithmetic is FP64 with CUDA's own division, sqrt, log, pow and exp; the
// compiler may fuse multiply-adds (results then differ from the reference in
// the last bits only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pdg {

// ComputeLogMean, src/BasicOperations/BasicOperations.cpp:6-12 (eps = 1e-4).
__device__ __forceinline__ double logmean(double x, double y)
{
    const double xi = y / x;
    const double u = (xi * (xi - 2.0) + 1.0) / (xi * (xi + 2.0) + 1.0);
    if (u < 1e-4) return (x + y) * 52.5 / (105.0 + u * (35.0 + u * (21.0 + 15.0 * u)));
    return (y - x) / log(xi);
}

// Per-node primitive quantities used by the two-point fluxes.
template <int DIM> struct Prim {
    double rho, v[DIM], p, beta, vsq;
};

// Primitive state as the Chandrashekar flux computes it from a conservative
// state (ChandrashekarFlux.cpp:17-68): v = m / rho, p = (g-1)(E - rho |v|^2/2),
// beta = rho / (2 p).
template <int DIM> __device__ __forceinline__ Prim<DIM> make_prim(const double *s, double gm1)
{
    Prim<DIM> q;
    q.rho = s[0];
    double vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        q.v[d] = s[1 + d] / q.rho;
        vsq += q.v[d] * q.v[d];
    }
    q.vsq = vsq;
    q.p = gm1 * (s[DIM + 1] - 0.5 * q.rho * vsq);
    q.beta = 0.5 * q.rho / q.p;
    return q;
}

// Wave speed |v| + c of one state (ChandrashekarFlux.cpp:61-65).
template <int DIM> __device__ __forceinline__ double wave_speed(const Prim<DIM> &q, double gamma)
{
    return sqrt(q.vsq) + sqrt(gamma * q.p / q.rho);
}

// ChandrashekarFlux::ComputeVolumeFlux (ChandrashekarFlux.cpp:11-83) for an
// axis-aligned contravariant metric: the metric mean is `metric` along
// direction DIR and zero elsewhere.
template <int DIM>
__device__ __forceinline__ void volume_flux(const Prim<DIM> &a, const Prim<DIM> &b, int dir, double metric,
                                            double gm1inv, double *F)
{
    const double rho_ln = logmean(a.rho, b.rho);
    double vm[DIM];
    double h_hat = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
    }
    double vdir = vm[0];
#pragma unroll
    for (int d = 1; d < DIM; d++)
        if (dir == d) vdir = vm[d];
    const double Vn = vdir * metric;
    const double beta_ln = logmean(a.beta, b.beta);
    const double p_hat = 0.5 * (a.rho + b.rho) / (a.beta + b.beta);
    h_hat += 0.5 / beta_ln * gm1inv + p_hat / rho_ln;
    F[0] = rho_ln * Vn;
#pragma unroll
    for (int d = 0; d < DIM; d++) F[1 + d] = Vn * (rho_ln * vm[d]) + (d == dir ? p_hat * metric : 0.0);
    F[1 + DIM] = rho_ln * Vn * h_hat;
}

// ChandrashekarFlux::ComputeFaceFlux (ChandrashekarFlux.cpp:85-161) for a
// normal of magnitude |nrm| along axis DIR (sign included in nrm).  compat
// keeps the 3D energy term as the reference writes it (`rho_mean * dw +
// w_mean`, :131).  diss scales the Lax-Friedrichs term (1 = reference).
// s1/s2: conservative states; returns lambda_max.
template <int DIM>
__device__ __forceinline__ double face_flux(const double *s1, const double *s2, int dir, double nrm, double gamma,
                                            double gm1, double gm1inv, bool compat, double diss_scale, double *F)
{
    const double nor_mag = fabs(nrm);
    const double rho1 = s1[0], rho2 = s2[0];
    const double rho_mean = 0.5 * (rho1 + rho2);
    const double rho_ln = logmean(rho1, rho2);
    const double drho = rho2 - rho1;
    double v1[DIM], v2[DIM], vm[DIM];
    double Vsq1 = 0.0, Vsq2 = 0.0, h_hat = 0.0, diss = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        v1[d] = s1[1 + d] / rho1;
        v2[d] = s2[1 + d] / rho2;
        vm[d] = 0.5 * (v1[d] + v2[d]);
        const double dv = v2[d] - v1[d];
        Vsq1 += v1[d] * v1[d];
        Vsq2 += v2[d] * v2[d];
        h_hat += -0.25 * (v1[d] * v1[d] + v2[d] * v2[d]) + vm[d] * vm[d];
        if (DIM == 3 && d == 2 && compat)
            diss += 0.5 * drho * v1[d] * v2[d] + rho_mean * dv + vm[d];
        else
            diss += 0.5 * drho * v1[d] * v2[d] + rho_mean * dv * vm[d];
    }
    double vdir = vm[0];
#pragma unroll
    for (int d = 1; d < DIM; d++)
        if (dir == d) vdir = vm[d];
    const double Vn = vdir * nrm;
    const double p1 = gm1 * (s1[DIM + 1] - 0.5 * rho1 * Vsq1);
    const double p2 = gm1 * (s2[DIM + 1] - 0.5 * rho2 * Vsq2);
    const double lam1 = sqrt(Vsq1) + sqrt(gamma * p1 / rho1);
    const double lam2 = sqrt(Vsq2) + sqrt(gamma * p2 / rho2);
    const double lambda_max = fmax(lam1, lam2);
    const double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
    const double beta_ln = logmean(beta1, beta2);
    const double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
    h_hat += 0.5 / beta_ln * gm1inv + p_hat / rho_ln;
    diss += 0.5 * drho * gm1inv / beta_ln + 0.5 * rho_mean * gm1inv * (1.0 / beta2 - 1.0 / beta1);
    const double lam = 0.5 * lambda_max * diss_scale * nor_mag;
    F[0] = rho_ln * Vn - lam * (rho2 - rho1);
#pragma unroll
    for (int d = 0; d < DIM; d++)
        F[1 + d] = Vn * (rho_ln * vm[d]) + (d == dir ? p_hat * nrm : 0.0) - lam * (s2[1 + d] - s1[1 + d]);
    F[1 + DIM] = rho_ln * Vn * h_hat - lam * diss;
    return lambda_max;
}

// NavierStokesFlux::ComputeViscousFlux (src/Fluxes/NavierStokesFlux.cpp:12-90),
// constant mu, mu_bulk = 2/3.  dq[d][v]: primitive gradients along x_d.  Only
// the momentum and energy rows are returned: Fv[(v-1)][d] for v = 1..DIM+1.
template <int DIM>
__device__ __forceinline__ void viscous_flux(const double *s, const double (*dq)[DIM + 2], double gm1, double gm1inv,
                                             double mu, double lambda_k, double Fv[DIM + 1][DIM])
{
    const double rho = s[0];
    double vel[DIM], vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = s[1 + d] / rho;
        vsq += vel[d] * vel[d];
    }
    const double p = gm1 * (s[DIM + 1] - 0.5 * rho * vsq);
    double div = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) div += dq[d][1 + d];
    const double mu_bulk = 2.0 / 3.0;
#pragma unroll
    for (int j = 0; j < DIM; j++) {      // flux direction
        double e = 0.0;
#pragma unroll
        for (int i = 0; i < DIM; i++) {  // momentum component
            double tau = (i == j) ? mu * (2.0 * dq[j][1 + i] - mu_bulk * div) : mu * (dq[j][1 + i] + dq[i][1 + j]);
            Fv[i][j] = tau;
            e += vel[i] * tau;
        }
        const double cv_dT = gm1inv / rho * (dq[j][DIM + 1] - p / rho * dq[j][0]);
        Fv[DIM][j] = e + lambda_k * cv_dT;
    }
}

// Conserv2Entropy (BasicOperations.cpp:134-157): beta = rho / p.
template <int DIM>
__device__ __forceinline__ void entropy_vars(const double *s, double gamma, double gm1, double gm1inv, double *w)
{
    const double rho = s[0];
    double vel[DIM], vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = s[1 + d] / rho;
        vv += vel[d] * vel[d];
    }
    const double v_sq = 0.5 * vv;
    const double p = gm1 * (s[DIM + 1] - rho * v_sq);
    const double beta = rho / p;
    const double sent = log(p * pow(rho, -gamma));
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
__device__ __forceinline__ void entgrad_to_primgrad(const double *s, double gm1, double gm1inv, bool compat, double *g)
{
    const double rho = s[0];
    double vel[DIM], vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vel[d] = s[1 + d] / rho;
        vv += vel[d] * vel[d];
    }
    const double v_sq = 0.5 * vv;
    const double p = gm1 * (s[DIM + 1] - rho * v_sq);
    const double KE = v_sq * rho;
    const double gl = g[DIM + 1];
    const double pr = p / rho;
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        g[1 + d] = pr * (g[1 + d] + vel[d] * gl);
        acc += (compat ? vel[d] : s[1 + d]) * g[1 + d];
    }
    g[0] = rho * g[0] - gl * (KE - p * gm1inv) + rho / p * acc;
    g[DIM + 1] = pr * (g[0] + p * gl);
}

}  // namespace pdg
