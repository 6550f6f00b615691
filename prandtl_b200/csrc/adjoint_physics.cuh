// adjoint_physics.cuh — reverse-mode (vector-Jacobian) versions of the
// pointwise physics in physics.cuh, for the fixed (compat = 0) operator.
//
// Each *_vjp function takes the cotangent of a forward function's outputs and
// accumulates the cotangents of its inputs.  State cotangents are gathered in
// primitive form (PBar: rho, 1/rho, v, beta, p) and turned into conservative
// ones once per node by pbar_to_cons, following make_prim's own chain
// (v = m / rho, p = (g-1)(E - rho |v|^2 / 2), beta = rho / (2p)).
// The reference has no adjoint; the forward functions cite what they restate.
#pragma once

#include "physics.cuh"

namespace pdg {

template <int DIM> struct PBar {
    double rho, irho, v[DIM], beta, p;
};

template <int DIM> PDG_FN void pbar_zero(PBar<DIM> &b)
{
    b.rho = b.irho = b.beta = b.p = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) b.v[d] = 0.0;
}

// Log-mean L(x, y) and its partial derivatives, branch by branch as
// logmean_inv evaluates it (series for u = ((y-x)/(y+x))^2 < 1e-4).
PDG_FN void logmean_grad(double x, double y, double &L, double &dx, double &dy)
{
    const double s = x + y, is = 1.0 / s;
    const double f = (y - x) * is;
    const double u = f * f;
    if (u < 1e-4) {
        const double P = 105.0 + u * (35.0 + u * (21.0 + 15.0 * u));
        const double dP = 35.0 + u * (42.0 + 45.0 * u);
        L = s * 52.5 / P;
        const double dLdu = -L * dP / P;
        // f = (y - x)/s: df/dx = -2y/s^2, df/dy = 2x/s^2
        const double c = dLdu * 2.0 * f * is * is;
        dx = L * is - c * 2.0 * y;
        dy = L * is + c * 2.0 * x;
    } else {
        const double l = log(y / x);
        L = (y - x) / l;
        dx = (L / x - 1.0) / l;
        dy = (1.0 - L / y) / l;
    }
}

// Reverse of make_prim plus the state's direct momentum cotangent mbar
// (may be null): adds the conservative cotangent to sbar.
template <int DIM>
PDG_FN void pbar_to_cons(const double *s, const PBar<DIM> &b, const double *mbar, double gm1, double *sbar)
{
    const double rho = s[0], irho = 1.0 / rho;
    double v[DIM], vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        v[d] = s[1 + d] * irho;
        vsq += v[d] * v[d];
    }
    const double p = gm1 * (s[DIM + 1] - 0.5 * rho * vsq);
    const double beta = 0.5 * rho / p;
    double rb = b.rho, ib = b.irho, pb = b.p, vb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) vb[d] = b.v[d];
    // beta = rho / (2 p)
    rb += b.beta * (0.5 / p);
    pb -= b.beta * (beta / p);
    // p = (g-1)(E - rho vsq / 2)
    sbar[DIM + 1] += gm1 * pb;
    rb -= gm1 * 0.5 * vsq * pb;
#pragma unroll
    for (int d = 0; d < DIM; d++) vb[d] -= gm1 * rho * v[d] * pb;
    // v = m / rho (as m * (1/rho))
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        sbar[1 + d] += vb[d] * irho + (mbar ? mbar[d] : 0.0);
        ib += vb[d] * s[1 + d];
    }
    rb -= ib * irho * irho;
    sbar[0] += rb;
}

// Reverse of the shared part of the two-point fluxes: the log-means, p_hat,
// the mean velocities and h_hat.  In: cotangents of rho_ln, 1/rho_ln,
// 1/beta_ln, p_hat, vm[], h_hat.
template <int DIM>
PDG_FN void two_point_common_vjp(const Prim<DIM> &a, const Prim<DIM> &b, double rlnb, double irlnb, double iblnb,
                                 double phb, double *vmb, double hb, double gm1inv, PBar<DIM> &ab, PBar<DIM> &bb)
{
    const double sr = a.rho + b.rho, isb = 1.0 / (a.beta + b.beta);
    double rln, drx, dry, bln, dbx, dby;
    logmean_grad(a.rho, b.rho, rln, drx, dry);
    logmean_grad(a.beta, b.beta, bln, dbx, dby);
    const double irln = 1.0 / rln, ibln = 1.0 / bln;
    const double p_hat = 0.5 * sr * isb;
    // h_hat = sum(-(va^2 + vb^2)/4 + vm^2) + ibln gm1inv / 2 + p_hat irln
    iblnb += hb * 0.5 * gm1inv;
    phb += hb * irln;
    irlnb += hb * p_hat;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double vm = 0.5 * (a.v[d] + b.v[d]);
        ab.v[d] += hb * (-0.5 * a.v[d]);
        bb.v[d] += hb * (-0.5 * b.v[d]);
        const double t = vmb[d] + hb * 2.0 * vm;
        ab.v[d] += 0.5 * t;
        bb.v[d] += 0.5 * t;
    }
    // p_hat = sr / (2 (beta_a + beta_b))
    ab.rho += phb * 0.5 * isb;
    bb.rho += phb * 0.5 * isb;
    ab.beta -= phb * p_hat * isb;
    bb.beta -= phb * p_hat * isb;
    // rho_ln and its reciprocal
    const double rt = rlnb - irlnb * irln * irln;
    ab.rho += rt * drx;
    bb.rho += rt * dry;
    // 1 / beta_ln
    const double bt = -iblnb * ibln * ibln;
    ab.beta += bt * dbx;
    bb.beta += bt * dby;
}

// Reverse of volume_flux_rt (ChandrashekarFlux::ComputeVolumeFlux,
// ChandrashekarFlux.cpp:11-83) along a runtime direction.
template <int DIM>
PDG_FN void volume_flux_vjp(const Prim<DIM> &a, const Prim<DIM> &b, int dir, double metric, double gm1inv,
                            const double *Fb, PBar<DIM> &ab, PBar<DIM> &bb)
{
    const double sr = a.rho + b.rho, isr = 1.0 / sr;
    double rho_ln, irho_ln;
    logmean_inv(a.rho, b.rho, sr, isr, rho_ln, irho_ln);
    const double isb = 1.0 / (a.beta + b.beta);
    const double ibeta_ln = logmean_recip(a.beta, b.beta, isb);
    const double p_hat = 0.5 * sr * isb;
    double vm[DIM], h_hat = 0.0;
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
    double fmb = Fb[0] + Fb[DIM + 1] * h_hat, vmb[DIM], phb = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        fmb += Fb[1 + d] * vm[d];
        vmb[d] = Fb[1 + d] * fm;
        if (d == dir) phb += Fb[1 + d] * metric;
    }
    const double hb = Fb[DIM + 1] * fm;
    const double rlnb = fmb * Vn;
#pragma unroll
    for (int d = 0; d < DIM; d++)
        if (d == dir) vmb[d] += fmb * rho_ln * metric;
    two_point_common_vjp<DIM>(a, b, rlnb, 0.0, 0.0, phb, vmb, hb, gm1inv, ab, bb);
}

// Reverse of the wave speed |v| + sqrt(gamma p / rho), written as
// |v| + sqrt(gamma / (2 beta)) so that it holds for states whose pressure
// was not formed (the subcell line tasks keep rho, v and beta only).
template <int DIM> PDG_FN void wave_speed_vjp(const Prim<DIM> &q, double gamma, double lb, PBar<DIM> &qb)
{
    double vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) vsq += q.v[d] * q.v[d];
    const double vn = sqrt(vsq);
    if (vn > 0.0) {
#pragma unroll
        for (int d = 0; d < DIM; d++) qb.v[d] += lb * q.v[d] / vn;
    }
    const double c = sqrt(0.5 * gamma / q.beta);
    qb.beta -= lb * 0.5 * c / q.beta;
}

// Reverse of face_flux<DIM, D> (ChandrashekarFlux::ComputeFaceFlux,
// ChandrashekarFlux.cpp:85-161) in its fixed form: cotangents of the two
// states' primitives (ab, bb) and of the momenta the dissipation jump reads
// (mab, mbb, added).  D is a runtime direction here.
template <int DIM>
PDG_FN void face_flux_vjp(const Prim<DIM> &a, const Prim<DIM> &b, const double *ma, const double *mb, int D, double nrm,
                          double gamma, double gm1inv, double diss_scale, const double *Fb, PBar<DIM> &ab,
                          PBar<DIM> &bb, double *mab, double *mbb)
{
    const double sr = a.rho + b.rho, isr = 1.0 / sr;
    double rho_ln, irho_ln;
    logmean_inv(a.rho, b.rho, sr, isr, rho_ln, irho_ln);
    const double isb = 1.0 / (a.beta + b.beta);
    const double ibeta_ln = logmean_recip(a.beta, b.beta, isb);
    const double p_hat = 0.5 * sr * isb;
    const double rho_mean = 0.5 * sr, drho = b.rho - a.rho;
    double vm[DIM], dv[DIM], h_hat = 0.0, diss = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        vm[d] = 0.5 * (a.v[d] + b.v[d]);
        dv[d] = b.v[d] - a.v[d];
        h_hat += -0.25 * (a.v[d] * a.v[d] + b.v[d] * b.v[d]) + vm[d] * vm[d];
        diss += 0.5 * drho * a.v[d] * b.v[d] + rho_mean * dv[d] * vm[d];
    }
    h_hat += 0.5 * ibeta_ln * gm1inv + p_hat * irho_ln;
    diss += 0.5 * drho * gm1inv * ibeta_ln + 0.5 * rho_mean * gm1inv * (b.ib - a.ib);
    const bool a_max = a.lam >= b.lam;
    const double lfac = 0.5 * diss_scale * fabs(nrm);
    const double lam = (a_max ? a.lam : b.lam) * lfac;
    double vd = vm[0];
#pragma unroll
    for (int d = 1; d < DIM; d++) vd = D == d ? vm[d] : vd;
    const double Vn = vd * nrm;
    const double fm = rho_ln * Vn;
    // F0 = fm - lam drho; F_k = fm vm_k + [k = D] p_hat nrm - lam (mb_k - ma_k);
    // F_E = fm h_hat - lam diss
    double lamb = -Fb[0] * drho - Fb[DIM + 1] * diss;
    double drhob = -lam * Fb[0];
    const double dissb = -lam * Fb[DIM + 1];
    double fmb = Fb[0] + Fb[DIM + 1] * h_hat, vmb[DIM], phb = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        lamb -= Fb[1 + d] * (mb[d] - ma[d]);
        mbb[d] -= lam * Fb[1 + d];
        mab[d] += lam * Fb[1 + d];
        fmb += Fb[1 + d] * vm[d];
        vmb[d] = Fb[1 + d] * fm;
        if (d == D) phb += Fb[1 + d] * nrm;
    }
    const double hb = Fb[DIM + 1] * fm;
    const double rlnb = fmb * Vn;
#pragma unroll
    for (int d = 0; d < DIM; d++)
        if (d == D) vmb[d] += fmb * rho_ln * nrm;
    // dissipation energy term
    double rmb = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        drhob += dissb * 0.5 * a.v[d] * b.v[d];
        ab.v[d] += dissb * 0.5 * drho * b.v[d];
        bb.v[d] += dissb * 0.5 * drho * a.v[d];
        rmb += dissb * dv[d] * vm[d];
        const double dvb = dissb * rho_mean * vm[d];
        vmb[d] += dissb * rho_mean * dv[d];
        bb.v[d] += dvb;
        ab.v[d] -= dvb;
    }
    drhob += dissb * 0.5 * gm1inv * ibeta_ln;
    const double iblnb = dissb * 0.5 * drho * gm1inv;
    rmb += dissb * 0.5 * gm1inv * (b.ib - a.ib);
    const double ibb_b = dissb * 0.5 * rho_mean * gm1inv;
    // ib = 1 / beta
    bb.beta -= ibb_b / (b.beta * b.beta);
    ab.beta += ibb_b / (a.beta * a.beta);
    ab.rho += 0.5 * rmb - drhob;
    bb.rho += 0.5 * rmb + drhob;
    // lam = max(lam_a, lam_b) |nrm| diss_scale / 2
    if (a_max) wave_speed_vjp<DIM>(a, gamma, lamb * lfac, ab);
    else wave_speed_vjp<DIM>(b, gamma, lamb * lfac, bb);
    two_point_common_vjp<DIM>(a, b, rlnb, 0.0, iblnb, phb, vmb, hb, gm1inv, ab, bb);
}

// Reverse of entropy_vars (Conserv2Entropy, BasicOperations.cpp:134-157):
// adds the conservative cotangent for the entropy-variable cotangent wb.
template <int DIM>
PDG_FN void entropy_vars_vjp(const double *s, const double *wb, double gamma, double gm1, double gm1inv, double *sbar)
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
    double betab = -wb[DIM + 1] - wb[0] * v_sq;
    double vsqb = -wb[0] * beta;
    const double sentb = -wb[0] * gm1inv;
    double velb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        betab += wb[1 + d] * vel[d];
        velb[d] = wb[1 + d] * beta;
    }
    // s = ln p - gamma ln rho
    double pb = sentb / p;
    double rb = -gamma * sentb * irho;
    // beta = rho / p
    rb += betab / p;
    pb -= betab * beta / p;
    // p = (g-1)(E - rho v_sq)
    sbar[DIM + 1] += gm1 * pb;
    rb -= gm1 * v_sq * pb;
    vsqb -= gm1 * rho * pb;
    double ib = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        velb[d] += vsqb * vel[d];
        sbar[1 + d] += velb[d] * irho;
        ib += velb[d] * s[1 + d];
    }
    sbar[0] += rb - ib * irho * irho;
}

// Reverse of entgrad_to_primgrad in its fixed form (EntropyGrad2PrimGrad,
// BasicOperations.cpp:179-223, with momenta in the density term): g is the
// entropy-variable gradient the forward received, ob the cotangent of its
// output; writes gb (cotangent of g) and adds the state cotangent to sbar.
template <int DIM>
PDG_FN void entgrad_vjp(const double *s, const double *g, const double *ob, double gm1, double gm1inv, double *gb,
                        double *sbar)
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
    double o[DIM + 2], acc = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        o[1 + d] = pr * (g[1 + d] + vel[d] * gl);
        acc += s[1 + d] * o[1 + d];
    }
    o[0] = rho * g[0] - gl * (KE - p * gm1inv) + rho / p * acc;
    double prb = 0.0, pb = 0.0, rb = 0.0, KEb = 0.0, glb = 0.0, ib = 0.0;
    double o0b = ob[0], okb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) okb[d] = ob[1 + d];
    // oL = pr (o0 + p gl)
    const double oLb = ob[DIM + 1];
    prb += oLb * (o[0] + p * gl);
    o0b += oLb * pr;
    pb += oLb * pr * gl;
    glb += oLb * pr * p;
    // o0 = rho g0 - gl (KE - p gm1inv) + (rho / p) acc
    rb += o0b * g[0];
    gb[0] = o0b * rho;
    glb -= o0b * (KE - p * gm1inv);
    KEb -= o0b * gl;
    pb += o0b * gl * gm1inv;
    rb += o0b * acc / p;
    pb -= o0b * acc * rho / (p * p);
    const double accb = o0b * rho / p;
    double velb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        // acc = sum m_d o_d
        sbar[1 + d] += accb * o[1 + d];
        okb[d] += accb * s[1 + d];
        // o_d = pr (g_d + vel_d gl)
        prb += okb[d] * (g[1 + d] + vel[d] * gl);
        gb[1 + d] = okb[d] * pr;
        velb[d] = okb[d] * pr * gl;
        glb += okb[d] * pr * vel[d];
    }
    gb[DIM + 1] = glb;
    // KE = v_sq rho
    double vsqb = KEb * rho;
    rb += KEb * v_sq;
    // pr = p / rho (as p * irho)
    pb += prb * irho;
    ib += prb * p;
    // p = (g-1)(E - rho v_sq)
    sbar[DIM + 1] += gm1 * pb;
    rb -= gm1 * v_sq * pb;
    vsqb -= gm1 * rho * pb;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        velb[d] += vsqb * vel[d];
        sbar[1 + d] += velb[d] * irho;
        ib += velb[d] * s[1 + d];
    }
    sbar[0] += rb - ib * irho * irho;
}

// Reverse of viscous_col (NavierStokesFlux::ComputeViscousFlux,
// NavierStokesFlux.cpp:12-90) for column `dir`: cb = cotangent of the column
// (momentum rows, energy), adds to qb (v, p, 1/rho) and to gb[d][v], the
// cotangent of the primitive gradients.
template <int DIM>
PDG_FN void viscous_col_vjp(const Prim<DIM> &q, const double (*G)[DIM + 2], int dir, double gm1inv, double mu,
                            double lambda_k, const double *cb, PBar<DIM> &qb, double (*gb)[DIM + 2])
{
    double div = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) div += G[d][1 + d];
    const double eb = cb[DIM];
    double divb = 0.0;
#pragma unroll
    for (int i = 0; i < DIM; i++) {
        const double tau = (i == dir) ? mu * (2.0 * G[dir][1 + i] - (2.0 / 3.0) * div)
                                      : mu * (G[dir][1 + i] + G[i][1 + dir]);
        const double taub = cb[i] + eb * q.v[i];
        qb.v[i] += eb * tau;
        if (i == dir) {
            gb[dir][1 + i] += taub * mu * 2.0;
            divb -= taub * mu * (2.0 / 3.0);
        } else {
            gb[dir][1 + i] += taub * mu;
            gb[i][1 + dir] += taub * mu;
        }
    }
#pragma unroll
    for (int d = 0; d < DIM; d++) gb[d][1 + d] += divb;
    // cv_dT = gm1inv irho (g(dir, E) - p irho g(dir, rho))
    const double cvb = eb * lambda_k;
    const double gE = G[dir][DIM + 1], g0 = G[dir][0];
    gb[dir][DIM + 1] += cvb * gm1inv * q.irho;
    gb[dir][0] -= cvb * gm1inv * q.p * q.irho * q.irho;
    qb.irho += cvb * gm1inv * (gE - 2.0 * q.p * q.irho * g0);
    qb.p -= cvb * gm1inv * q.irho * q.irho * g0;
}

}  // namespace pdg
