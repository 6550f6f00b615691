// adjoint_kernels.cuh — vector-Jacobian product of the fixed (compat = 0)
// right-hand side: given a cotangent lam of dudt, ubar = (dL/du)^T lam.
//
// The kernels mirror the forward ones in reverse:
//   adj_rhs_kernel   flux-differencing volume terms, subcell FV blending and
//                    the blending coefficient (indicator) — stores ubar;
//   adj_lift_kernel  (Navier-Stokes) viscous volume divergence, face viscous
//                    columns, viscous fluxes, primitive-gradient conversion
//                    and the BR1 volume lifting — adds to ubar and leaves the
//                    cotangents of the face-normal entropy gradients in gcol;
//   adj_faces_kernel every direction's Riemann fluxes and (Navier-Stokes) the
//                    BR1 face jumps — stores both sides' cotangents per face
//                    node to a buffer;
//   adj_gather_kernel adds them to ubar, then (an RK stage's adjoint) the
//                    stage algebra.
// Order of a product: (NS: lift_face_kernel for the forward jumps,)
// adj_rhs_kernel, (NS: adj_lift_kernel,) adj_faces_kernel, adj_gather_kernel.
// The reference has no adjoint; each reversed step names the forward
// function it reverses.
#pragma once

#include "adjoint_physics.cuh"
#include "line_kernels.cuh"

namespace pdg {

// Launch shapes of the adjoint element kernels for 3D N = 3 (the adjoint
// benchmark's order): the lifting adjoint's 10 KB element slots pack an SM
// better in blocks of ADJ_LIFT_WPB warps, with the register budget that
// ADJ_LIFT_MIN_BLOCKS such blocks need.
#ifndef PDG_ADJ_LIFT_WPB
#define PDG_ADJ_LIFT_WPB 4
#endif
#ifndef PDG_ADJ_LIFT_MIN_BLOCKS
#define PDG_ADJ_LIFT_MIN_BLOCKS 1
#endif
#ifndef PDG_ADJ_RHS_MIN_BLOCKS
#define PDG_ADJ_RHS_MIN_BLOCKS 1
#endif
#ifndef PDG_ADJ_FACES_MIN_BLOCKS
#define PDG_ADJ_FACES_MIN_BLOCKS 2
#endif
template <int DIM, int N> struct AdjLiftLaunch {
    static constexpr bool tuned = DIM == 3 && N == 3;
    static constexpr int wpb = tuned ? PDG_ADJ_LIFT_WPB : 4;
    static constexpr int threads = 32 * wpb;
    static constexpr int min_blocks = tuned ? PDG_ADJ_LIFT_MIN_BLOCKS : 1;
};

template <int DIM, int N> struct AdjShape {
    using S = Shape<DIM, N>;
    // slot: primitives (rho, v, beta), cotangent lam, primitive cotangents,
    // two scratch fields (indicator input / modal buffers)
    static constexpr int EL = (3 * S::NV + 2) * S::NS_;
};

// Line index (within direction d) and position of node n = (i, j, k).
template <int DIM, int Np> __device__ __forceinline__ int line_of(int d, const int *idx)
{
    return d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                  : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
}

// Transposed 1D modal pass: dst[line, l] = sum_k Vinv(k, l) src[line, k].
template <int DIM, int N, int D>
__device__ __forceinline__ void modal_pass_t(const double *src, double *dst, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np;
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            double x[Np];
#pragma unroll
            for (int k = 0; k < Np; k++) x[k] = src[sp<DIM, Np>(line_node<DIM, Np, D>(line, k))];
#pragma unroll
            for (int l = 0; l < Np; l++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < Np; k++) s += Vinv[k * Np + l] * x[k];
                dst[sp<DIM, Np>(line_node<DIM, Np, D>(line, l))] = s;
            }
        }
    }
    __syncwarp();
}

// Reverse of the flux-differencing line tasks (ec_lines_rt) along d: pair
// (a, b) contributes scale (Dhat2(a,b) lam_a + Dhat2(b,a) lam_b) as the
// cotangent of its two-point flux.
template <int DIM, int N>
__device__ __forceinline__ void ec_lines_vjp(const KParams &P, int d, const double *pr, const double *lm, double *pb,
                                             const double *c, int gl, double scale)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    using PS = PSlot<DIM>;
    const double metric = C_ADJ(c)[d];
    const double *D2 = C_DHAT2(c);
#pragma unroll 1
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            Prim<DIM> q[Np];
            PBar<DIM> qb[Np];
#pragma unroll
            for (int l = 0; l < Np; l++) {
                q[l] = slot_prim<DIM>(pr, sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l)), ST);
                pbar_zero(qb[l]);
            }
#pragma unroll
            for (int a = 0; a < Np; a++)
#pragma unroll
                for (int b = a + 1; b < Np; b++) {
                    const int na = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, a));
                    const int nb = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, b));
                    const double cab = scale * D2[a * Np + b], cba = scale * D2[b * Np + a];
                    double Fb[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) Fb[v] = cab * lm[v * ST + na] + cba * lm[v * ST + nb];
                    volume_flux_vjp<DIM>(q[a], q[b], d, metric, P.gm1inv, Fb, qb[a], qb[b]);
                }
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l));
                pb[P_RHO * ST + n] += qb[l].rho;
#pragma unroll
                for (int k = 0; k < DIM; k++) pb[(P_V + k) * ST + n] += qb[l].v[k];
                pb[PS::BETA * ST + n] += qb[l].beta;
            }
        }
    }
    __syncwarp();
}

// Reverse of the subcell finite-volume line tasks (fv_lines) along D:
// interface flux F_{l+1/2} enters node l with -alpha fvs_l and node l+1 with
// +alpha fvs_{l+1}; its momenta are rho v of the slot primitives.
template <int DIM, int N, int D>
__device__ __forceinline__ void fv_lines_vjp(const KParams &P, const double *pr, const double *lm, double *pb,
                                             const double *c, int gl, double alpha)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    using PS = PSlot<DIM>;
    const double *sn = C_SNOR(c, D), *fvs = C_FVS(c);
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
#pragma unroll 1
            for (int l = 0; l < N; l++) {
                const int na = sp<DIM, Np>(line_node<DIM, Np, D>(line, l)), nb = sp<DIM, Np>(line_node<DIM, Np, D>(line, l + 1));
                Prim<DIM> qa = slot_prim<DIM>(pr, na, ST), qb = slot_prim<DIM>(pr, nb, ST);
                complete_prim<DIM>(qa, P.gamma);
                complete_prim<DIM>(qb, P.gamma);
                double ma[DIM], mb[DIM], mab[DIM], mbb[DIM];
#pragma unroll
                for (int k = 0; k < DIM; k++) {
                    ma[k] = qa.rho * qa.v[k];
                    mb[k] = qb.rho * qb.v[k];
                    mab[k] = mbb[k] = 0.0;
                }
                double Fb[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) Fb[v] = alpha * (fvs[l + 1] * lm[v * ST + nb] - fvs[l] * lm[v * ST + na]);
                PBar<DIM> ab, bb;
                pbar_zero(ab);
                pbar_zero(bb);
                face_flux_vjp<DIM>(qa, qb, ma, mb, D, sn[l + 1], P.gamma, P.gm1inv, P.diss_scale, Fb, ab, bb, mab, mbb);
#pragma unroll
                for (int k = 0; k < DIM; k++) {
                    ab.rho += mab[k] * qa.v[k];
                    ab.v[k] += mab[k] * qa.rho;
                    bb.rho += mbb[k] * qb.v[k];
                    bb.v[k] += mbb[k] * qb.rho;
                }
                pb[P_RHO * ST + na] += ab.rho;
                pb[P_RHO * ST + nb] += bb.rho;
#pragma unroll
                for (int k = 0; k < DIM; k++) {
                    pb[(P_V + k) * ST + na] += ab.v[k];
                    pb[(P_V + k) * ST + nb] += bb.v[k];
                }
                pb[PS::BETA * ST + na] += ab.beta;
                pb[PS::BETA * ST + nb] += bb.beta;
            }
        }
    }
    __syncwarp();
}

// This lane's share of lam . (d acc / d alpha) for the flux-differencing
// terms: sum over its lines' pairs of scale F (Dhat2(a,b) lam_a + Dhat2(b,a)
// lam_b), the forward volume sums contracted with lam without storing them.
template <int DIM, int N>
__device__ __forceinline__ double ec_lines_dot(const KParams &P, int d, const double *pr, const double *lm,
                                               const double *c, int gl, double scale)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    const double metric = C_ADJ(c)[d];
    const double *D2 = C_DHAT2(c);
    double dot = 0.0;
#pragma unroll 1
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            Prim<DIM> q[Np];
#pragma unroll
            for (int l = 0; l < Np; l++) q[l] = slot_prim<DIM>(pr, sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l)), ST);
#pragma unroll
            for (int a = 0; a < Np; a++)
#pragma unroll
                for (int b = a + 1; b < Np; b++) {
                    const int na = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, a));
                    const int nb = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, b));
                    double F[NV];
                    volume_flux_rt<DIM>(q[a], q[b], d, metric, P.gm1inv, F);
                    const double cab = scale * D2[a * Np + b], cba = scale * D2[b * Np + a];
#pragma unroll
                    for (int v = 0; v < NV; v++) dot += F[v] * (cab * lm[v * ST + na] + cba * lm[v * ST + nb]);
                }
        }
    }
    return dot;
}

// The same for the subcell FV terms along D (alpha = 1).
template <int DIM, int N, int D>
__device__ __forceinline__ double fv_lines_dot(const KParams &P, const double *pr, const double *lm, const double *c,
                                               int gl)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    const double *sn = C_SNOR(c, D), *fvs = C_FVS(c);
    double dot = 0.0;
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
#pragma unroll 1
            for (int l = 0; l < N; l++) {
                const int na = sp<DIM, Np>(line_node<DIM, Np, D>(line, l)), nb = sp<DIM, Np>(line_node<DIM, Np, D>(line, l + 1));
                Prim<DIM> qa = slot_prim<DIM>(pr, na, ST), qb = slot_prim<DIM>(pr, nb, ST);
                complete_prim<DIM>(qa, P.gamma);
                complete_prim<DIM>(qb, P.gamma);
                double ma[DIM], mb[DIM];
#pragma unroll
                for (int k = 0; k < DIM; k++) {
                    ma[k] = qa.rho * qa.v[k];
                    mb[k] = qb.rho * qb.v[k];
                }
                double F[NV];
                face_flux<DIM, D>(qa, qb, ma, mb, sn[l + 1], P.gm1inv, P.compat != 0, P.diss_scale, F);
#pragma unroll
                for (int v = 0; v < NV; v++) dot += F[v] * (fvs[l + 1] * lm[v * ST + nb] - fvs[l] * lm[v * ST + na]);
            }
        }
    }
    return dot;
}

// Reverse of the blending coefficient for one lane group (an element):
// etab is the cotangent of eta; adds the primitive cotangents of q = rho p to
// pb.  scr holds two modal buffers of the slot's scratch region.
template <int DIM, int N>
__device__ __forceinline__ void indicator_vjp(const double *pr, double *pb, double *scr, const double *c, int gl,
                                              double etab)
{
    using S = Shape<DIM, N>;
    using PS = PSlot<DIM>;
    constexpr int Np = S::Np, NDOF = S::NDOF, L = S::L, ST = S::NS_;
#pragma unroll
    for (int k = 0; k < S::NPL; k++) {
        const int n = gl + k * L;
        if (n < NDOF) {
            const int m = sp<DIM, Np>(n);
            const double rho = pr[P_RHO * ST + m], beta = pr[PS::BETA * ST + m];
            scr[m] = rho * (0.5 * rho / beta);
        }
    }
    __syncwarp();
    double *qa = scr, *qb = scr + ST;
    modal_pass<DIM, N, 0>(qa, qb, gl, C_VINV(c));
    modal_pass<DIM, N, 1>(qb, qa, gl, C_VINV(c));
    if (DIM == 3) modal_pass<DIM, N, (DIM == 3 ? 2 : 0)>(qa, qb, gl, C_VINV(c));
    double *mo = (DIM == 3) ? qb : qa, *other = (DIM == 3) ? qa : qb;
    double mm = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
    for (int k = 0; k < S::NPL; k++) {
        const int t = gl + k * L;
        if (t < NDOF) {
            const int i = t % Np, j = (t / Np) % Np, kk = DIM == 3 ? t / (Np * Np) : 0;
            int mx = i > j ? i : j;
            if (DIM == 3) mx = mx > kk ? mx : kk;
            const double v = mo[sp<DIM, Np>(t)] * mo[sp<DIM, Np>(t)];
            mm += v;
            if (mx <= N - 1) m1 += v;
            if (mx <= N - 2) m2 += v;
        }
    }
    mm = group_sum<L>(mm);
    m1 = group_sum<L>(m1);
    m2 = group_sum<L>(m2);
    // eta = max(1 - m1/mm, 1 - m2/m1)
    double mmb = 0.0, m1b = 0.0, m2b = 0.0;
    if (1.0 - m1 / mm >= 1.0 - m2 / m1) {
        mmb = etab * m1 / (mm * mm);
        m1b = -etab / mm;
    } else {
        m1b = etab * m2 / (m1 * m1);
        m2b = -etab / m1;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < S::NPL; k++) {
        const int t = gl + k * L;
        if (t < NDOF) {
            const int i = t % Np, j = (t / Np) % Np, kk = DIM == 3 ? t / (Np * Np) : 0;
            int mx = i > j ? i : j;
            if (DIM == 3) mx = mx > kk ? mx : kk;
            const double w = mmb + (mx <= N - 1 ? m1b : 0.0) + (mx <= N - 2 ? m2b : 0.0);
            mo[sp<DIM, Np>(t)] = 2.0 * mo[sp<DIM, Np>(t)] * w;
        }
    }
    __syncwarp();
    if (DIM == 3) {
        modal_pass_t<DIM, N, (DIM == 3 ? 2 : 0)>(mo, other, gl, C_VINV(c));
        modal_pass_t<DIM, N, 1>(other, mo, gl, C_VINV(c));
        modal_pass_t<DIM, N, 0>(mo, other, gl, C_VINV(c));
    } else {
        modal_pass_t<DIM, N, 1>(mo, other, gl, C_VINV(c));
        modal_pass_t<DIM, N, 0>(other, mo, gl, C_VINV(c));
    }
    const double *qbar = (DIM == 3) ? other : mo;
    // q = rho p with p = rho / (2 beta)
#pragma unroll
    for (int k = 0; k < S::NPL; k++) {
        const int n = gl + k * L;
        if (n < NDOF) {
            const int m = sp<DIM, Np>(n);
            const double rho = pr[P_RHO * ST + m], beta = pr[PS::BETA * ST + m];
            const double p = 0.5 * rho / beta, g = qbar[m];
            const double pbar = g * rho;
            pb[P_RHO * ST + m] += g * p + pbar * 0.5 / beta;
            pb[PS::BETA * ST + m] -= pbar * 0.5 * rho / (beta * beta);
        }
    }
    __syncwarp();
}

// Adjoint of the inviscid volume terms and the blending coefficient, the
// first kernel of a vector-Jacobian product: stores ubar = cotangent of u
// through those terms.
template <int DIM, int N>
__global__ void __launch_bounds__(128, (DIM == 3 && N == 3) ? PDG_ADJ_RHS_MIN_BLOCKS : 1) adj_rhs_kernel(const KParams P, const double *__restrict__ cot,
                                                      double *__restrict__ ubar)
{
    using S = Shape<DIM, N>;
    using PS = PSlot<DIM>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, L = S::L, EPW = S::EPW, ST = S::NS_;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / L, gl = lane % L;
    const int wpb = blockDim.x >> 5;
    // EPW * L = 32: every lane belongs to an element slot
    double *pr = smem + const_slots(Np) + (size_t)(warp * EPW + grp) * AdjShape<DIM, N>::EL;
    double *lm = pr + NV * ST, *pb = lm + NV * ST, *scr = pb + NV * ST;
    const int64_t nn = P.nnodes;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride) {
        const int64_t e0 = wt * EPW + grp;
        const bool valid = e0 < P.ne;
        const int64_t e = valid ? e0 : 0;
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                double s[NV];
#pragma unroll
                for (int v = 0; v < NV; v++)
                    s[v] = valid ? __ldg(P.u + v * nn + e * NDOF + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
                const Prim<DIM> q = make_prim<DIM>(s, P.gamma, P.gm1);
                const int m = sp<DIM, Np>(n);
                pr[P_RHO * ST + m] = q.rho;
#pragma unroll
                for (int d = 0; d < DIM; d++) pr[(P_V + d) * ST + m] = q.v[d];
                pr[PS::BETA * ST + m] = q.beta;
                scr[m] = q.rho * q.p;
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    lm[v * ST + m] = valid ? __ldg(cot + v * nn + e * NDOF + n) : 0.0;
                    pb[v * ST + m] = 0.0;
                }
            }
        }
        __syncwarp();
        double alpha = 0.0, dalpha = 0.0;
        if (P.blending) {
            const double eta = indicator_eta<DIM, N>(scr, gl, C_VINV(c));
            alpha = blending_alpha(eta, P);
            const double T = P.modal_threshold;
            const double a = 1.0 / (1.0 + exp(-9.21024 * (eta - T) / T));
            if (a >= P.alpha_min && a <= 1.0 - P.alpha_min && a < P.alpha_max) dalpha = a * (1.0 - a) * 9.21024 / T;
        }
        // blending coefficient: d(acc)/d(alpha) = invJ EC + FV; alpha <- eta <- rho p
        if (__any_sync(0xffffffffu, dalpha != 0.0)) {
            double abar = 0.0;
#pragma unroll 1
            for (int d = 0; d < DIM; d++) abar += ec_lines_dot<DIM, N>(P, d, pr, lm, c, gl, C_INVJ(c));
            abar += fv_lines_dot<DIM, N, 0>(P, pr, lm, c, gl);
            abar += fv_lines_dot<DIM, N, 1>(P, pr, lm, c, gl);
            if (DIM == 3) abar += fv_lines_dot<DIM, N, (DIM == 3 ? 2 : 0)>(P, pr, lm, c, gl);
            abar = group_sum<L>(abar);
            __syncwarp();
            indicator_vjp<DIM, N>(pr, pb, scr, c, gl, valid ? abar * dalpha : 0.0);
        }
        const double sc = -(1.0 - alpha) * C_INVJ(c);
#pragma unroll 1
        for (int d = 0; d < DIM; d++) ec_lines_vjp<DIM, N>(P, d, pr, lm, pb, c, gl, sc);
        if (P.blending && __any_sync(0xffffffffu, alpha > 0.0)) {
            fv_lines_vjp<DIM, N, 0>(P, pr, lm, pb, c, gl, alpha);
            fv_lines_vjp<DIM, N, 1>(P, pr, lm, pb, c, gl, alpha);
            if (DIM == 3) fv_lines_vjp<DIM, N, (DIM == 3 ? 2 : 0)>(P, pr, lm, pb, c, gl, alpha);
        }
        if (valid) {
#pragma unroll
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
                    const int m = sp<DIM, Np>(n);
                    double s[NV], sb[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        s[v] = __ldg(P.u + v * nn + e * NDOF + n);
                        sb[v] = 0.0;
                    }
                    PBar<DIM> b;
                    pbar_zero(b);
                    b.rho = pb[P_RHO * ST + m];
#pragma unroll
                    for (int d = 0; d < DIM; d++) b.v[d] = pb[(P_V + d) * ST + m];
                    b.beta = pb[PS::BETA * ST + m];
                    pbar_to_cons<DIM>(s, b, nullptr, P.gm1, sb);
#pragma unroll
                    for (int v = 0; v < NV; v++) ubar[v * nn + e * NDOF + n] = sb[v];
                }
            }
        }
        __syncwarp();
    }
}

// Adjoint of the viscous terms (lift_kernel in reverse): adds them to ubar.
// cot: cotangent of dudt; P.lbuf holds the forward BR1 face jumps
// (lift_face_kernel of u); gcol receives, at every face node, the cotangent
// of the face-normal entropy-variable gradient ([d][side][e][face node][v]).
template <int DIM, int N>
__global__ void __launch_bounds__(AdjLiftLaunch<DIM, N>::threads, AdjLiftLaunch<DIM, N>::min_blocks) adj_lift_kernel(const KParams P, const double *__restrict__ cot,
                                                       double *__restrict__ ubar, double *__restrict__ gcol)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, L = S::L, EPW = S::EPW, ST = S::NS_;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / L, gl = lane % L;
    const int wpb = blockDim.x >> 5;
    double *wv = smem + const_slots(Np) + (size_t)(warp * EPW + grp) * S::EL_LIFT;
    double *g = wv + NV * ST;
    const int64_t nn = P.nnodes;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    const double invJ = C_INVJ(c), fsc = C_FACE(c);
    const double *Dh = C_DHAT(c), *Dm = C_D(c);
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride) {
        const int64_t e0 = wt * EPW + grp;
        const bool valid = e0 < P.ne;
        const int64_t e = valid ? e0 : 0;
        // (i) entropy variables and their strong-form gradients
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                double s[NV], w[NV];
#pragma unroll
                for (int v = 0; v < NV; v++)
                    s[v] = valid ? __ldg(P.u + v * nn + e * NDOF + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
                entropy_vars<DIM>(s, P.gamma, P.gm1, P.gm1inv, w);
#pragma unroll
                for (int v = 0; v < NV; v++) wv[v * ST + sp<DIM, Np>(n)] = w[v];
            }
        }
        __syncwarp();
        grad_lines<DIM, N, 0>(wv, g, c, gl);
        grad_lines<DIM, N, 1>(wv, g, c, gl);
        if (DIM == 3) grad_lines<DIM, N, (DIM == 3 ? 2 : 0)>(wv, g, c, gl);
        __syncwarp();
        // (ii) the cotangent replaces the entropy variables in the slot
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
#pragma unroll
                for (int v = 0; v < NV; v++) wv[v * ST + sp<DIM, Np>(n)] = valid ? __ldg(cot + v * nn + e * NDOF + n) : 0.0;
            }
        }
        __syncwarp();
        // (iii) per node: viscous fluxes and gradient conversion in reverse
        int64_t enb[2 * DIM];
#pragma unroll
        for (int f = 0; f < 2 * DIM; f++) enb[f] = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + f) : 0;
        double sacc[S::NPL][NV];
#pragma unroll
        for (int k = 0; k < S::NPL; k++)
#pragma unroll
            for (int v = 0; v < NV; v++) sacc[k][v] = 0.0;
#pragma unroll 1
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n >= NDOF) break;
            const int m = sp<DIM, Np>(n);
            double s[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) s[v] = valid ? __ldg(P.u + v * nn + e * NDOF + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
            const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            // global operands of the node's face terms, loaded first: the
            // forward BR1 jumps and the neighbour's cotangent at each face
            double jf[DIM][NV], lo[DIM][DIM + 1];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const int pos = idx[d];
                const bool face = valid && (pos == 0 || pos == N);
                const int line = line_of<DIM, Np>(d, idx);
                const int64_t owner = pos == N ? e : enb[2 * d];
                const double *F = P.lbuf + ((d * P.ne + owner) * NFN + line) * NV;
#pragma unroll
                for (int v = 0; v < NV; v++) jf[d][v] = face ? __ldg(F + v) : 0.0;
                const int64_t other = enb[2 * d + (pos == N ? 1 : 0)];
                const int no = line_node_rt<DIM, Np>(d, line, pos == N ? 0 : N);
#pragma unroll
                for (int i = 0; i <= DIM; i++) lo[d][i] = face ? __ldg(cot + (int64_t)(1 + i) * nn + other * NDOF + no) : 0.0;
            }
            double gin[DIM][NV], dq[DIM][NV];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
#pragma unroll
                for (int v = 0; v < NV; v++) gin[d][v] = g[(d * NV + v) * ST + m];
                const int pos = idx[d];
                if (valid && (pos == 0 || pos == N)) {
#pragma unroll
                    for (int v = 0; v < NV; v++) gin[d][v] += jf[d][v];
                }
#pragma unroll
                for (int v = 0; v < NV; v++) dq[d][v] = gin[d][v];
                entgrad_to_primgrad<DIM>(s, P.gm1, P.gm1inv, false, dq[d]);
            }
            // cotangent of each viscous column: volume divergence (Dhat
            // transposed along the line through n) and the face terms
            double cb[DIM][DIM + 1];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                const int pos = idx[d];
                const double a = C_ADJ(c)[d] * invJ;
                const int line = line_of<DIM, Np>(d, idx);
#pragma unroll
                for (int i = 0; i <= DIM; i++) {
                    double acc = 0.0;
#pragma unroll
                    for (int p = 0; p < Np; p++)
                        acc += Dh[p * Np + pos] * wv[(1 + i) * ST + sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, p))];
                    cb[d][i] = a * acc;
                }
                if (valid && (pos == 0 || pos == N)) {
                    // the face column enters out_a with + fsc A / 2 and out_b with - fsc A / 2
                    const double h = 0.5 * fsc * C_AREA(c)[d];
#pragma unroll
                    for (int i = 0; i <= DIM; i++) {
                        const double le = wv[(1 + i) * ST + m];
                        cb[d][i] += pos == N ? h * (le - lo[d][i]) : h * (lo[d][i] - le);
                    }
                }
            }
            const Prim<DIM> q = make_prim<DIM>(s, P.gamma, P.gm1);
            PBar<DIM> qb;
            pbar_zero(qb);
            double dqb[DIM][NV];
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
                for (int v = 0; v < NV; v++) dqb[d][v] = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; d++) viscous_col_vjp<DIM>(q, dq, d, P.gm1inv, P.mu, P.lambda_k, cb[d], qb, dqb);
            double sk[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) sk[v] = 0.0;
            pbar_to_cons<DIM>(s, qb, nullptr, P.gm1, sk);
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double gb[NV];
                entgrad_vjp<DIM>(s, gin[d], dqb[d], P.gm1, P.gm1inv, gb, sk);
#pragma unroll
                for (int v = 0; v < NV; v++) g[(d * NV + v) * ST + m] = gb[v];
                const int pos = idx[d];
                if (valid && (pos == 0 || pos == N)) {
                    const int line = line_of<DIM, Np>(d, idx);
                    double *dst = gcol + (((int64_t)(d * 2 + (pos == N ? 1 : 0)) * P.ne + e) * NFN + line) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++) dst[v] = gb[v];
                }
            }
#pragma unroll
            for (int kk = 0; kk < S::NPL; kk++)
                if (kk == k)
#pragma unroll
                    for (int v = 0; v < NV; v++) sacc[kk][v] = sk[v];
        }
        __syncwarp();
        // (iv) volume lifting in reverse: wbar_l = sum_d adj_d / J sum_p D(p, l) gbar_d(p)
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    double acc = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        const int pos = idx[d];
                        const int line = line_of<DIM, Np>(d, idx);
                        double t = 0.0;
#pragma unroll
                        for (int p = 0; p < Np; p++)
                            t += Dm[p * Np + pos] * g[(d * NV + v) * ST + sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, p))];
                        acc += C_ADJ(c)[d] * invJ * t;
                    }
                    wv[v * ST + sp<DIM, Np>(n)] = acc;
                }
            }
        }
        __syncwarp();
        // (v) entropy variables in reverse, and the node's total
        if (valid) {
#pragma unroll
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
                    double s[NV], wb[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        s[v] = __ldg(P.u + v * nn + e * NDOF + n);
                        wb[v] = wv[v * ST + sp<DIM, Np>(n)];
                    }
                    entropy_vars_vjp<DIM>(s, wb, P.gamma, P.gm1, P.gm1inv, sacc[k]);
#pragma unroll
                    for (int v = 0; v < NV; v++) ubar[v * nn + e * NDOF + n] += sacc[k][v];
                }
            }
        }
        __syncwarp();
    }
}

// Adjoint of one face node's terms: element a's +D face node fn and its
// neighbour b's -D face node (face_node_terms in reverse), plus for
// Navier-Stokes the BR1 jump 0.5 fsc A (w_b - w_a) that lift_face_node adds to
// both sides' face gradients.  ga, gb: the cotangents of a's and b's states
// at the face node.
template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ void adj_face_node(const KParams &P, const double *c, const double *__restrict__ cot,
                                              const double *__restrict__ gcol, int64_t a, int64_t b, int fn,
                                              double *ga, double *gb)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t nn = P.nnodes;
    const int na = line_node<DIM, Np, D>(fn, N), nb = line_node<DIM, Np, D>(fn, 0);
    double sa[NV], sb[NV], la[NV], lb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        sa[v] = __ldg(P.u + v * nn + a * NDOF + na);
        sb[v] = __ldg(P.u + v * nn + b * NDOF + nb);
        la[v] = __ldg(cot + v * nn + a * NDOF + na);
        lb[v] = __ldg(cot + v * nn + b * NDOF + nb);
    }
    double hs[NV];
    if (NS) {  // loaded ahead of the flux arithmetic
        const double h = 0.5 * C_FACE(c) * C_AREA(c)[D];
#pragma unroll
        for (int v = 0; v < NV; v++)
            hs[v] = h * (__ldg(gcol + (((int64_t)(D * 2 + 1) * P.ne + a) * NFN + fn) * NV + v) +
                         __ldg(gcol + (((int64_t)(D * 2 + 0) * P.ne + b) * NFN + fn) * NV + v));
    }
    const Prim<DIM> qa = make_prim<DIM>(sa, P.gamma, P.gm1), qb = make_prim<DIM>(sb, P.gamma, P.gm1);
    const bool a_is_1 = a <= b;
    const double nrm = a_is_1 ? C_AREA(c)[D] : -C_AREA(c)[D];
    const double sc = C_FACE(c);
    // out_a += C, out_b -= C with C = sc (a_is_1 ? -F : F) (+ the viscous part)
    double Fb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) Fb[v] = (a_is_1 ? -sc : sc) * (la[v] - lb[v]);
    PBar<DIM> ab, bb;
    pbar_zero(ab);
    pbar_zero(bb);
    double mab[DIM], mbb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) mab[d] = mbb[d] = 0.0;
    if (a_is_1) face_flux_vjp<DIM>(qa, qb, sa + 1, sb + 1, D, nrm, P.gamma, P.gm1inv, P.diss_scale, Fb, ab, bb, mab, mbb);
    else face_flux_vjp<DIM>(qb, qa, sb + 1, sa + 1, D, nrm, P.gamma, P.gm1inv, P.diss_scale, Fb, bb, ab, mbb, mab);
#pragma unroll
    for (int v = 0; v < NV; v++) ga[v] = gb[v] = 0.0;
    pbar_to_cons<DIM>(sa, ab, mab, P.gm1, ga);
    pbar_to_cons<DIM>(sb, bb, mbb, P.gm1, gb);
    if (NS) {
        double wb[NV], wa[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
            wb[v] = hs[v];
            wa[v] = -hs[v];
        }
        entropy_vars_vjp<DIM>(sa, wa, P.gamma, P.gm1, P.gm1inv, ga);
        entropy_vars_vjp<DIM>(sb, wb, P.gamma, P.gm1, P.gm1inv, gb);
    }
}

// The adjoint face terms of every direction in one launch, each face node's
// two cotangents stored to gbuf[d][side][e][v][fn] (side 1: element a's +d
// face node, side 0: its +d neighbour's -d face node, under that
// neighbour's index); adj_rhs_kernel adds them to ubar.  Threads run
// direction-major inside chunks of 64 elements, as lift_face_kernel.
template <int DIM, int N, bool NS>
__global__ void __launch_bounds__(256, PDG_ADJ_FACES_MIN_BLOCKS) adj_faces_kernel(const KParams P, const double *__restrict__ cot,
                                                        double *__restrict__ gbuf, const double *__restrict__ gcol)
{
    using S = Shape<DIM, N>;
    constexpr int NV = S::NV, NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, S::Np);
    __syncthreads();
    constexpr int CH = 64, PER_CH = DIM * CH * NFN;
    const int64_t nch = (P.ne + CH - 1) / CH;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nch * PER_CH;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ch = t / PER_CH;
        const int r = (int)(t - ch * PER_CH);
        const int d = r / (CH * NFN);
        const int r2 = r - d * (CH * NFN);
        const int64_t a = ch * CH + r2 / NFN;
        const int fn = r2 % NFN;
        if (a >= P.ne) continue;
        const int64_t b = __ldg(P.nbr + a * 2 * DIM + 2 * d + 1);
        if (b < 0) continue;  // boundary face: adj_boundary_kernel
        double ga[NV], gb[NV];
        if (d == 0) adj_face_node<DIM, N, 0, NS>(P, c, cot, gcol, a, b, fn, ga, gb);
        else if (d == 1) adj_face_node<DIM, N, 1, NS>(P, c, cot, gcol, a, b, fn, ga, gb);
        else adj_face_node<DIM, N, (DIM == 3 ? 2 : 0), NS>(P, c, cot, gcol, a, b, fn, ga, gb);
        double *da = gbuf + (((int64_t)(d * 2 + 1) * P.ne + a) * NV) * NFN + fn;
        double *db = gbuf + (((int64_t)(d * 2 + 0) * P.ne + b) * NV) * NFN + fn;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            da[v * NFN] = ga[v];
            db[v * NFN] = gb[v];
        }
    }
}

// ubar += the face-term cotangents of gbuf at every face node (in the order
// x, y [, z] faces), one thread per node.  With P.stage >= 0 the RK stage's
// adjoint follows: for stage s of out = a_s un + b_s (us + dt L(us)) and the
// cotangent lam (cot) of out, with g = ubar = (dL/dus)^T lam,
//   stage 2: ubar = 2/3 (lam + dt g), bx = 1/3 lam;
//   stage 1: ubar = 1/4 (lam + dt g), bx += 3/4 lam;
//   stage 0 (us = un): bx += lam + dt g.
template <int DIM, int N>
__global__ void __launch_bounds__(256) adj_gather_kernel(const KParams P, const double *__restrict__ cot,
                                                         double *__restrict__ ubar)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t nn = P.nnodes;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / NDOF;
        const int n = (int)(t - e * NDOF);
        const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
        const double *src[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int pos = idx[d];
            src[d] = nullptr;
            if (pos == 0 || pos == N) {
                const int side = pos == N ? 1 : 0;
                if (__ldg(P.nbr + e * 2 * DIM + 2 * d + side) >= 0)  // boundary faces: adj_boundary_kernel
                    src[d] = P.gbuf + (((int64_t)(d * 2 + side) * P.ne + e) * NV) * NFN + line_of<DIM, Np>(d, idx);
            }
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const int64_t gi = v * nn + t;
            double x = ubar[gi];
#pragma unroll
            for (int d = 0; d < DIM; d++)
                if (src[d]) x += __ldg(src[d] + v * NFN);
            if (P.stage < 0) {
                ubar[gi] = x;
            } else {
                const double lam = __ldg(cot + gi);
                const double z = lam + P.dt * x;
                if (P.stage == 2) {
                    ubar[gi] = 2. / 3 * z;
                    P.bx[gi] = 1. / 3 * lam;
                } else if (P.stage == 1) {
                    ubar[gi] = 1. / 4 * z;
                    P.bx[gi] = P.bx[gi] + 3. / 4 * lam;
                } else {
                    P.bx[gi] = P.bx[gi] + z;
                }
            }
        }
    }
}

// Reverse of the slip wall's pressure flux F[1+D] = p* nrm (boundary_node_terms):
// p* of the interior density, normal velocity vn = sgn m_D / rho and pressure
// p = (g-1)(E - |m|^2 / (2 rho)); adds the conservative cotangent to g.
template <int DIM>
__device__ __forceinline__ void slip_wall_vjp(const KParams &P, const double *s, int D, double sgn, double psb,
                                              double *g)
{
    const double rho = s[0], irho = 1.0 / rho;
    double vsq = 0.0;
#pragma unroll
    for (int q = 0; q < DIM; q++) vsq += (s[1 + q] * irho) * (s[1 + q] * irho);
    const double gm1 = P.gm1, gamma = P.gamma;
    const double p = gm1 * (s[DIM + 1] - 0.5 * rho * vsq);
    const double vn = sgn * s[1 + D] * irho;
    const double an = sqrt(gamma * p * irho);
    double dp, dvn, drho;  // partial derivatives of p*
    if (vn > 0.0) {
        const double gp1 = 1.0 + gamma, A = 8.0 / gp1 * (gm1 / gp1 + 1.0);
        const double S = sqrt(vn * vn + A * p * irho);
        dp = 1.0 + 0.125 * gp1 * vn * A / S;
        dvn = 0.25 * gp1 * rho * (2.0 * vn + S + vn * vn / S);
        drho = 0.25 * gp1 * vn * (vn + S) - 0.125 * gp1 * vn * A * p * irho / S;
    } else {
        const double E = 2.0 * gamma / gm1;
        const double X0 = 1.0 + 0.5 * gm1 * vn / an;
        if (X0 > 0.0001) {
            const double XE1 = pow(X0, E - 1.0), pEX = p * E * XE1;
            dp = XE1 * X0 + pEX * (-0.25 * gm1 * vn / (an * p));
            dvn = pEX * 0.5 * gm1 / an;
            drho = pEX * 0.25 * gm1 * vn / (an * rho);
        } else {
            dp = pow(0.0001, E);
            dvn = drho = 0.0;
        }
    }
    // through p(rho, m, E) and vn(rho, m_D)
    g[0] += psb * (drho + dvn * (-vn * irho) + dp * 0.5 * gm1 * vsq);
#pragma unroll
    for (int q = 0; q < DIM; q++) g[1 + q] += psb * (dp * (-gm1 * s[1 + q] * irho) + (q == D ? dvn * sgn * irho : 0.0));
    g[DIM + 1] += psb * dp * gm1;
}

// Forward-mode number (value, derivative) for the Jacobian of the subsonic
// and Riemann-invariant outer states with respect to the interior state.
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double c, Dual a) { return {c * a.v, c * a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double c) { return {c * a.v, c * a.d}; }
__device__ __forceinline__ Dual operator+(double c, Dual a) { return {c + a.v, a.d}; }
__device__ __forceinline__ Dual operator-(double c, Dual a) { return {c - a.v, -a.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator/(Dual a, double c) { return {a.v / c, a.d / c}; }
__device__ __forceinline__ Dual dsqrt(Dual a)
{
    const double r = sqrt(a.v);
    return {r, r > 0.0 ? a.d * 0.5 / r : 0.0};
}
__device__ __forceinline__ Dual dpow(Dual a, double e)
{
    const double pv = pow(a.v, e);
    return {pv, a.d * e * pow(a.v, e - 1.0)};
}

// The fixed operator's outer states of conditions 6-9 (boundary_node_terms
// with compat = 0) in forward mode: type 6 subsonic outflow at a pressure, 7
// inflow from rho and V, 8 (2D) inflow from total pressure, temperature and
// direction, 9 Riemann invariants; prm as the boundary table stores it.
template <int DIM>
__device__ void outer_state_dual(const KParams &P, int type, const double *prm, int D, double sgn, const Dual *s1,
                                 Dual *s2)
{
    constexpr int NV = DIM + 2;
    const double gamma = P.gamma, gm1 = P.gm1, gm1inv = P.gm1inv;
    const Dual rho = s1[0];
    Dual V[DIM], vv = {0.0, 0.0}, msq = {0.0, 0.0};
    for (int q = 0; q < DIM; q++) {
        V[q] = s1[1 + q] / rho;
        vv = vv + V[q] * V[q];
        msq = msq + s1[1 + q] * s1[1 + q];
    }
    if (type == BC_SUBSONIC_OUTFLOW_P) {
        for (int v = 0; v < NV - 1; v++) s2[v] = s1[v];
        s2[NV - 1] = prm[0] * gm1inv + 0.5 * (rho * vv);
        return;
    }
    if (type == BC_SUBSONIC_INFLOW_RV) {
        const double r = prm[0];
        double uu = 0.0;
        s2[0] = {r, 0.0};
        for (int q = 0; q < DIM; q++) {
            s2[1 + q] = {r * prm[1 + q], 0.0};
            uu += prm[1 + q] * prm[1 + q];
        }
        s2[NV - 1] = s1[NV - 1] - 0.5 * (msq / rho) + Dual{0.5 * uu * r, 0.0};
        return;
    }
    const Dual p = gm1 * (s1[NV - 1] - 0.5 * (rho * vv));
    if (type == BC_SUBSONIC_INFLOW_PTTT) {
        const double cp = prm[0], p0 = prm[1], T0 = prm[2];
        Dual V_sq = (2.0 * cp * T0) * (1.0 - dpow(p / p0, gm1 / gamma));
        if (V_sq.v < 0.0) V_sq = {0.0, 0.0};
        const Dual r2 = (gamma * gm1inv) * p / ((cp * T0) - 0.5 * V_sq);
        const Dual sv = dsqrt(V_sq);
        s2[0] = r2;
        for (int q = 0; q < DIM; q++) s2[1 + q] = prm[3 + q] * (r2 * sv);
        s2[NV - 1] = gm1inv * p + 0.5 * (r2 * V_sq);
        return;
    }
    // BC_RIEMANN_INVARIANT
    const double rho_o = prm[0], p_o = prm[NV - 1];
    const Dual Vn_i = sgn * V[D];
    const double Vn_o = sgn * prm[1 + D];
    const double a_o = sqrt(gamma * p_o / rho_o);
    const Dual a_i = dsqrt(gamma * p / rho);
    const bool sup = fabs(Vn_o) >= a_o;
    const Dual R_minus = (sup && Vn_i.v >= 0.0) ? Vn_i - 2.0 * gm1inv * a_i : Dual{Vn_o - 2.0 * a_o * gm1inv, 0.0};
    const Dual R_plus = (sup && Vn_i.v < 0.0) ? Dual{Vn_o + 2.0 * a_o * gm1inv, 0.0} : Vn_i + 2.0 * gm1inv * a_i;
    const Dual Vn_b = 0.5 * (R_plus + R_minus), a_b = (0.25 * gm1) * (R_plus - R_minus);
    const Dual r2 = Vn_i.v < 0.0 ? rho_o * dpow((a_b * a_b) * (rho_o / (gamma * p_o)), gm1inv)
                                 : dpow((a_b * a_b) * rho / (gamma * p), gm1inv) * rho;
    Dual e2 = {0.0, 0.0};
    for (int q = 0; q < DIM; q++) {
        const double nq = q == D ? sgn : 0.0;
        s2[1 + q] = Vn_i.v >= 0.0 ? r2 * (V[q] + nq * (Vn_b - Vn_i)) : r2 * (prm[1 + q] + nq * (Vn_b - Dual{Vn_o, 0.0}));
        e2 = e2 + s2[1 + q] * s2[1 + q];
    }
    s2[0] = r2;
    s2[NV - 1] = 0.5 * (e2 / r2) + gm1inv * ((a_b * a_b) * r2 / gamma);
}

// Adjoint of the boundary faces (Euler, fixed operator): one thread per
// element walks its boundary faces, as boundary_kernel does forward, and
// adds (dC/du)^T cot at each boundary node, C = -F(s, s2(s)) / (w0 J):
// prescribed outer states are constants, outflow has s2 = s, symmetry
// s2 = s with the normal momentum reversed, the subsonic and Riemann-
// invariant states enter through their Jacobian (forward mode), and the slip
// wall's flux depends on s through p*.
template <int DIM, int N>
__global__ void __launch_bounds__(256) adj_boundary_kernel(const KParams P, const double *__restrict__ cot,
                                                           double *__restrict__ ubar, const double *__restrict__)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, Np);
    __syncthreads();
    const int64_t nn = P.nnodes;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < P.ne; a += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll 1
        for (int f = 0; f < 2 * DIM; f++) {
            const int32_t nb = __ldg(P.nbr + a * 2 * DIM + f);
            if (nb >= 0) continue;
            const int D = f >> 1, side = f & 1;
            const double sgn = side ? 1.0 : -1.0;
            const double *bc = P.bc + (-1 - nb) * BC_SLOT;
            const int type = (int)bc[0];
            const double nrm = sgn * C_AREA(c)[D];
#pragma unroll 1
            for (int fn = 0; fn < NFN; fn++) {
                const int n = line_node_rt<DIM, Np>(D, fn, side ? N : 0);
                double s1[NV], Fb[NV], g[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    s1[v] = __ldg(P.u + v * nn + a * NDOF + n);
                    Fb[v] = -C_FACE(c) * __ldg(cot + v * nn + a * NDOF + n);
                    g[v] = 0.0;
                }
                if (type == BC_SLIP_WALL || type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL) {
                    slip_wall_vjp<DIM>(P, s1, D, sgn, Fb[1 + D] * nrm, g);
                } else {
                    double s2[NV];
                    const bool given = type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE;
                    const bool sub = type >= BC_SUBSONIC_OUTFLOW_P && type <= BC_RIEMANN_INVARIANT;
                    // Jacobian of the outer state (columns by forward mode)
                    double Jm[NV][NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) s2[v] = given ? bc[1 + v] : s1[v];
                    if (type == BC_SYMMETRY) s2[1 + D] = -s1[1 + D];
                    if (sub) {
#pragma unroll 1
                        for (int j = 0; j < NV; j++) {
                            Dual x[NV], y[NV];
#pragma unroll
                            for (int v = 0; v < NV; v++) x[v] = {s1[v], v == j ? 1.0 : 0.0};
                            outer_state_dual<DIM>(P, type, bc + 1, D, sgn, x, y);
#pragma unroll
                            for (int i = 0; i < NV; i++) {
                                Jm[i][j] = y[i].d;
                                s2[i] = y[i].v;
                            }
                        }
                    }
                    const Prim<DIM> qa = make_prim<DIM>(s1, P.gamma, P.gm1), qb = make_prim<DIM>(s2, P.gamma, P.gm1);
                    PBar<DIM> ab, bb;
                    pbar_zero(ab);
                    pbar_zero(bb);
                    double mab[DIM], mbb[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; d++) mab[d] = mbb[d] = 0.0;
                    face_flux_vjp<DIM>(qa, qb, s1 + 1, s2 + 1, D, nrm, P.gamma, P.gm1inv, P.diss_scale, Fb, ab, bb, mab,
                                       mbb);
                    pbar_to_cons<DIM>(s1, ab, mab, P.gm1, g);
                    if (!given) {
                        double g2[NV];
#pragma unroll
                        for (int v = 0; v < NV; v++) g2[v] = 0.0;
                        pbar_to_cons<DIM>(s2, bb, mbb, P.gm1, g2);
                        if (type == BC_SYMMETRY) g2[1 + D] = -g2[1 + D];
                        if (sub) {
#pragma unroll
                            for (int j = 0; j < NV; j++) {
                                double a = 0.0;
#pragma unroll
                                for (int i = 0; i < NV; i++) a += g2[i] * Jm[i][j];
                                g[j] += a;
                            }
                        } else {
#pragma unroll
                            for (int v = 0; v < NV; v++) g[v] += g2[v];
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < NV; v++) ubar[v * nn + a * NDOF + n] += g[v];
            }
        }
    }
}

}  // namespace pdg
