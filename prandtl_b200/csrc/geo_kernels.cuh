// geo_kernels.cuh — the Euler and Navier-Stokes right-hand sides on meshes of
// general geometry (skewed, graded, curved or unstructured quadrilaterals and
// hexahedra): geo_rhs_kernel (Euler, or with NS the viscous terms as well)
// and geo_lift_kernel (BR1 gradients, Navier-Stokes).
//
// The reference evaluates every metric term from MFEM's element
// transformation at the integration points: the two-point volume fluxes use
// the mean of both nodes' contravariant metric rows (adj rows of the
// Jacobian, DGSEMIntegrator.cpp:252-266, ChandrashekarFlux.cpp:11-83), the
// volume term is divided by the node's own J (:427-431), the faces use the
// normal CalcOrtho gives out of the face's element 1 and each side's own
// J (:151-222), and the subcell finite-volume fluxes use the subcell normals
// n_i = adj(x_0) + sum_{l<i} w_l (D adj)_l along each line
// (ComputeSubcellMetrics, :1199-1304; ComputeFVFluxes, :972-1196) and
// divide by J w at the node.  Here the metric terms sit in HBM per node
// (P.geo: J and the adjugate rows), the face normals and the neighbour's
// matching node per element face node (P.fnor, P.fnode: conforming faces in
// any orientation), and the subcell normals are formed per line in the
// kernel from the metric rows, in the reference's order of operations.
//
// Work decomposition: as rhs_kernel — a lane group per element, line tasks
// per direction (each two-point flux evaluated once per line pair and added
// to both nodes), then each element evaluates its own face nodes with the
// element-1 rule (both elements of a face evaluate it from the same inputs
// in the same order and receive bit-identical fluxes) and stores the
// finished stage.  One launch per right-hand side or RK stage (Navier-Stokes:
// the lifting kernel first).
#pragma once

#include "line_kernels.cuh"

namespace pdg {

// Metric row r of node n of element e (dim components).
template <int DIM>
__device__ __forceinline__ void geo_row(const KParams &P, int64_t gnode, int r, double *m)
{
#pragma unroll
    for (int k = 0; k < DIM; k++) m[k] = __ldg(P.geo + (int64_t)(1 + r * DIM + k) * P.nnodes + gnode);
}
__device__ __forceinline__ double geo_J(const KParams &P, int64_t gnode) { return __ldg(P.geo + gnode); }
// Component c of metric row r of global node gnode.
template <int DIM>
__device__ __forceinline__ double geo_row1(const KParams &P, int64_t gnode, int r, int c)
{
    return __ldg(P.geo + (int64_t)(1 + r * DIM + c) * P.nnodes + gnode);
}

// Flux-differencing line tasks along direction d with per-node metrics: the
// pair (a < b) of a line takes the metric mean (m_a + m_b) / 2 of both nodes'
// row d, its flux contributes Dhat2(a,b) F to node a and Dhat2(b,a) F to
// node b, in ascending partner order.  The unscaled line sums are stored
// (d == 0) or added to acc.
template <int DIM, int N>
__device__ __forceinline__ void ec_lines_geo(const KParams &P, int d, const double *pr, double *acc,
                                             const double *c, int gl, int64_t e, bool valid)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, NDOF = S::NDOF;
    const double *D2 = C_DHAT2(c);
#pragma unroll 1
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            Prim<DIM> q[Np];
            double m[Np][DIM];
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = line_node_rt<DIM, Np>(d, line, l);
                q[l] = slot_prim<DIM>(pr, sp<DIM, Np>(n), S::NS_);
                if (valid) geo_row<DIM>(P, e * NDOF + n, d, m[l]);
                else
#pragma unroll
                    for (int k = 0; k < DIM; k++) m[l][k] = k == d ? 1.0 : 0.0;
            }
            double la[Np][NV];
#pragma unroll
            for (int l = 0; l < Np; l++)
#pragma unroll
                for (int v = 0; v < NV; v++) la[l][v] = 0.0;
#pragma unroll
            for (int a = 0; a < Np; a++)
#pragma unroll
                for (int b = a + 1; b < Np; b++) {
                    double mt[DIM], F[NV];
#pragma unroll
                    for (int k = 0; k < DIM; k++) mt[k] = (m[a][k] + m[b][k]) * 0.5;
                    volume_flux_n<DIM>(q[a], q[b], mt, P.gm1inv, F);
                    const double cab = D2[a * Np + b], cba = D2[b * Np + a];
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        la[a][v] += cab * F[v];
                        la[b][v] += cba * F[v];
                    }
                }
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l));
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    if (d == 0) acc[v * S::NS_ + n] = la[l][v];
                    else acc[v * S::NS_ + n] += la[l][v];
                }
            }
        }
    }
    __syncwarp();
}

// Subcell finite-volume line tasks along d: the interface normals of the
// line from its metric rows (n_0 = m_0, n_{i+1} = n_i + w_i sum_m D(i,m) m_m),
// the Chandrashekar face flux across each interior interface, and node l
// receiving alpha (f_{l-1/2} - f_{l+1/2}) / (J_l w_l).
template <int DIM, int N>
__device__ __forceinline__ void fv_lines_geo(const KParams &P, int d, const double *pr, double *acc,
                                             const double *c, int gl, int64_t e, bool valid, double alpha)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, NDOF = S::NDOF;
    const double *Dm = C_D(c), *w = C_W(c);
#pragma unroll 1
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            double m[Np][DIM], sc[Np];
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = line_node_rt<DIM, Np>(d, line, l);
                if (valid) {
                    geo_row<DIM>(P, e * NDOF + n, d, m[l]);
                    sc[l] = 1.0 / (geo_J(P, e * NDOF + n) * w[l]);
                } else {
#pragma unroll
                    for (int k = 0; k < DIM; k++) m[l][k] = k == d ? 1.0 : 0.0;
                    sc[l] = 1.0;
                }
            }
            double nor[DIM], prev[NV];
#pragma unroll
            for (int k = 0; k < DIM; k++) nor[k] = m[0][k];
#pragma unroll
            for (int v = 0; v < NV; v++) prev[v] = 0.0;
            Prim<DIM> qa = slot_prim<DIM>(pr, sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, 0)), S::NS_);
            complete_prim<DIM>(qa, P.gamma);
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l));
                double F[NV];
                Prim<DIM> qb;
                if (l < N) {
                    // interface l + 1/2: n_{l+1} = n_l + w_l (D m)_l
#pragma unroll
                    for (int k = 0; k < DIM; k++) {
                        double t = 0.0;
#pragma unroll
                        for (int j = 0; j < Np; j++) t += m[j][k] * Dm[l * Np + j];
                        nor[k] += t * w[l];
                    }
                    qb = slot_prim<DIM>(pr, sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l + 1)), S::NS_);
                    complete_prim<DIM>(qb, P.gamma);
                    double ma[DIM], mb[DIM];
#pragma unroll
                    for (int k = 0; k < DIM; k++) {
                        ma[k] = qa.rho * qa.v[k];
                        mb[k] = qb.rho * qb.v[k];
                    }
                    face_flux_n<DIM>(qa, qb, ma, mb, nor, P.gm1inv, P.compat != 0, P.diss_scale, F);
                } else {
#pragma unroll
                    for (int v = 0; v < NV; v++) F[v] = 0.0;
                }
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    acc[v * S::NS_ + n] += alpha * ((prev[v] - F[v]) * sc[l]);
                    prev[v] = F[v];
                }
                if (l < N) qa = qb;
            }
        }
    }
    __syncwarp();
}

// The normal and tangents of a boundary face (RotateState,
// src/BasicOperations/BasicOperations.cpp:238-258): the momentum of `s`
// expressed in the frame (n, t1[, t2]) of the unit normal n.
template <int DIM> __device__ __forceinline__ void rotate_momentum(double *s, const double *n)
{
    double t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
    if (DIM == 2) {
        t1[0] = -n[1];
        t1[1] = n[0];
    } else {
        const bool gen = fabs(n[0]) > 1e-10;
        const double q = gen ? n[1] / n[0] : 0.0;
        t1[0] = gen ? -q / sqrt(1.0 + q * q) : -1.0;
        t1[1] = gen ? 1.0 / sqrt(1.0 + q * q) : 0.0;
        t1[2] = 0.0;
        t2[0] = n[1] * t1[2] - n[2] * t1[1];
        t2[1] = n[2] * t1[0] - n[0] * t1[2];
        t2[2] = n[0] * t1[1] - n[1] * t1[0];
    }
    double ru = 0.0, rv = 0.0, rw = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        ru += s[1 + d] * n[d];
        rv += s[1 + d] * t1[d];
    }
    if (DIM == 3) {
#pragma unroll
        for (int d = 0; d < 3; d++) rw += s[1 + d] * t2[d];
        s[3] = rw;
    }
    s[1] = ru;
    s[2] = rv;
}

// Boundary face node with interior state s1 and outward normal nor (not
// normalised; |nor| is the face's area element): the normal flux F of
// condition b and the wave speed it reports (BdrFaceIntegrator::
// AssembleFaceVector and each condition's ComputeBdrFaceInviscidFlux /
// ComputeOuterInviscidState, src/Integrators/BoundaryConditions/).  Slip
// wall (and, without viscosity, both no-slip walls): the state rotated to the
// face frame, p* from the wall Riemann problem (SlipWallBdrFaceIntegrator.cpp:
// 15-58), flux p* nor in the momentum rows.  Other conditions: the outer
// state and the Chandrashekar face flux; the subsonic and Riemann-invariant
// conditions of the reference-value operator divide the interior momenta in
// place first, as the reference's Vector views do (ComputePressure,
// BasicOperations.cpp:31-37).
template <int DIM>
__device__ __noinline__ double geo_bdr_flux(const KParams &P, int b, const double *s_in, const double *nor, double *F,
                                            double *outer = nullptr)
{
    constexpr int NV = DIM + 2;
    const double *bc = P.bc + b * BC_SLOT;
    const int type = (int)bc[0];
    const double gamma = P.gamma, gm1 = P.gm1, gm1inv = P.gm1inv;
    const bool compat = P.compat != 0;
    double nn = 0.0, un[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) nn += nor[d] * nor[d];
    const double inv = 1.0 / sqrt(nn);
#pragma unroll
    for (int d = 0; d < DIM; d++) un[d] = nor[d] * inv;
    double s1[NV], s2[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) s1[v] = s2[v] = s_in[v];
    if (type == BC_SLIP_WALL || type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL) {
        rotate_momentum<DIM>(s2, un);
        const double rho = s2[0];
        double vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const double V = s2[1 + d] / rho;
            vv += V * V;
        }
        const double p = gm1 * (s2[NV - 1] - 0.5 * rho * vv);
        const double an = sqrt(gamma * p / rho);
        const double u = s2[1] / rho;
        const double gp1 = 1.0 + gamma, gp1inv = 1.0 / gp1;
        double ps;
        if (u > 0.0) ps = p + 0.25 * u * gp1 * rho * (u + sqrt(u * u + 8.0 * gp1inv / rho * p * (gm1 * gp1inv + 1.0)));
        else ps = p * pow(fmax(1.0 + 0.5 * gm1 * u / an, 0.0001), 2.0 * gamma * gm1inv);
        F[0] = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) F[1 + d] = ps * nor[d];
        F[NV - 1] = 0.0;
        return sqrt(vv) + an;
    }
    const double *prm = bc + 1;
    if (type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE) {
#pragma unroll
        for (int v = 0; v < NV; v++) s2[v] = prm[v];
    } else if (type == BC_SYMMETRY) {
        double mn = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) mn += s2[1 + d] * un[d];
#pragma unroll
        for (int d = 0; d < DIM; d++) s2[1 + d] += -2.0 * mn * un[d];
    } else if (type == BC_SUBSONIC_OUTFLOW_P || type == BC_SUBSONIC_INFLOW_PTTT) {
        const double rho = s_in[0], r1 = 1.0 / rho;
        double V[DIM], vv = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) V[d] = compat ? s_in[1 + d] * r1 : s_in[1 + d] / rho;
#pragma unroll
        for (int d = 0; d < DIM; d++) vv += V[d] * V[d];
        if (compat)
#pragma unroll
            for (int d = 0; d < DIM; d++) s1[1 + d] = V[d];
        if (type == BC_SUBSONIC_OUTFLOW_P) {
#pragma unroll
            for (int v = 0; v < NV; v++) s2[v] = s1[v];
            s2[NV - 1] = prm[0] * gm1inv + 0.5 * rho * vv;
        } else {
            const double cp = prm[0], p0 = prm[1], T0 = prm[2];
            const double p = gm1 * (s_in[NV - 1] - 0.5 * rho * vv);
            double V_sq = 2.0 * cp * T0 * (1.0 - pow(p / p0, gm1 / gamma));
            V_sq = fmax(0.0, V_sq);
            s2[0] = gamma * gm1inv * p / (cp * T0 - 0.5 * V_sq);
#pragma unroll
            for (int d = 0; d < DIM; d++) s2[1 + d] = s2[0] * sqrt(V_sq) * prm[3 + d];
            s2[NV - 1] = p * gm1inv + 0.5 * s2[0] * V_sq;
        }
    } else if (type == BC_SUBSONIC_INFLOW_RV) {
        const double r = prm[0];
        s2[0] = r;
        double dke = -s_in[1] * s_in[1], uu = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            s2[1 + d] = r * prm[1 + d];
            if (d > 0) dke -= s_in[1 + d] * s_in[1 + d];
            uu += prm[1 + d] * prm[1 + d];
        }
        dke *= 0.5 / s_in[0];
        dke += 0.5 * uu * r;
        s2[NV - 1] = s_in[NV - 1] + dke;
    } else if (type == BC_RIEMANN_INVARIANT) {
        const double ginv = 1.0 / gamma;
        const double rho = s_in[0], r1 = 1.0 / rho;
        const double rho_o = prm[0], p_o = prm[NV - 1];
        double V[DIM], Vn_i = 0.0, Vn_o = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) V[d] = compat ? s_in[1 + d] * r1 : s_in[1 + d] / rho;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            Vn_i += V[d] * un[d];
            Vn_o += prm[1 + d] * un[d];
        }
        double W[DIM], ww = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) W[d] = compat ? V[d] * r1 : V[d];
#pragma unroll
        for (int d = 0; d < DIM; d++) ww += W[d] * W[d];
        const double p_i = gm1 * (s_in[NV - 1] - 0.5 * rho * ww);
        if (compat)
#pragma unroll
            for (int d = 0; d < DIM; d++) V[d] = s1[1 + d] = W[d];
        const double a_o = sqrt(gamma * p_o / rho_o), a_i = sqrt(gamma * p_i / rho);
        const double R_minus = (fabs(Vn_o) >= a_o && Vn_i >= 0.0) ? Vn_i - 2.0 * a_i * gm1inv : Vn_o - 2.0 * a_o * gm1inv;
        const double R_plus = (fabs(Vn_o) >= a_o && Vn_i < 0.0) ? Vn_o + 2.0 * a_o * gm1inv : Vn_i + 2.0 * a_i * gm1inv;
        const double Vn_b = 0.5 * (R_plus + R_minus), a_b = 0.25 * gm1 * (R_plus - R_minus);
        const double dVn_i = Vn_b - Vn_i, dVn_o = Vn_b - Vn_o;
        s2[0] = (Vn_i < 0.0) ? pow(a_b * a_b * ginv * rho_o / p_o, gm1inv) * rho_o
                             : pow(a_b * a_b * ginv * rho / p_i, gm1inv) * rho;
        double e2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            s2[1 + d] = (Vn_i >= 0.0) ? s2[0] * (V[d] + dVn_i * un[d]) : s2[0] * (prm[1 + d] + dVn_o * un[d]);
            e2 = d == 0 ? s2[1] * s2[1] : e2 + s2[1 + d] * s2[1 + d];
        }
        const double p_b = a_b * a_b * s2[0] * ginv;
        e2 *= (0.5 / s2[0]);
        e2 += p_b * gm1inv;
        s2[NV - 1] = e2;
    }  // BC_SUPERSONIC_OUTFLOW: the interior state
    if (outer)
#pragma unroll
        for (int v = 0; v < NV; v++) outer[v] = s2[v];
    const Prim<DIM> qa = make_prim<DIM>(s1, gamma, gm1), qb = make_prim<DIM>(s2, gamma, gm1);
    double ma[DIM], mb[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        ma[d] = s1[1 + d];
        mb[d] = s2[1 + d];
    }
    face_flux_n<DIM>(qa, qb, ma, mb, nor, gm1inv, compat, P.diss_scale, F);
    return fmax(qa.lam, qb.lam);
}

// Element slot of geo_rhs_kernel: primitives and accumulator; Navier-Stokes
// adds the divergence of the contravariant viscous fluxes [row][node] (rows:
// momenta and energy).
template <int DIM, int N, bool NS> struct GeoShape {
    using S = Shape<DIM, N>;
    static constexpr int DV = S::EL_RHS_FB;  // offset of the viscous divergence
    static constexpr int EL = NS ? DV + (S::NV - 1) * S::NS_ : S::EL_RHS_FB;
};

// The viscous flux (NavierStokesFlux::ComputeViscousFlux, constant mu) of a
// state and its primitive gradients gr[k][v] (k: physical direction):
// fm[q][r], column q, rows r = momenta and energy.
template <int DIM>
__device__ __forceinline__ void viscous_flux_cols(const KParams &P, const double *s, const double (*gr)[DIM + 2],
                                                  double (*fm)[DIM + 1])
{
    Prim<DIM> q = make_prim<DIM>(s, P.gamma, P.gm1);
    auto G = [&](int d, int v) { return gr[d][v]; };
#pragma unroll
    for (int c = 0; c < DIM; c++) viscous_col<DIM>(q, G, c, P.gm1inv, P.mu, P.lambda_k, fm[c]);
}

// Divergence of the contravariant viscous fluxes geo_lift_kernel stored
// (MultABt(adj, flux) per node, DGSEMIntegrator.cpp:616-640, 764-786) along
// each direction's lines, dUv(l) = sum_m Dhat(l, m) F_d(m), accumulated over
// the directions into dv.
template <int DIM, int N>
__device__ __forceinline__ void viscous_volume_geo(const KParams &P, double *dv, const double *c, int gl, int64_t e,
                                                   bool valid)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NR = NV - 1, ST = S::NS_;
    const double *Dh = C_DHAT(c);
#pragma unroll 1
    for (int d = 0; d < DIM; d++) {
#pragma unroll 1
        for (int rr = 0; rr < S::LPL; rr++) {
            const int line = gl + rr * S::L;
            if (line < S::NFN) {
                double x[Np][NR];
#pragma unroll
                for (int l = 0; l < Np; l++)
#pragma unroll
                    for (int r = 0; r < NR; r++)
                        x[l][r] = valid ? __ldg(P.geo_fv + (int64_t)(d * NR + r) * P.nnodes + e * NDOF +
                                                line_node_rt<DIM, Np>(d, line, l))
                                        : 0.0;
#pragma unroll
                for (int l = 0; l < Np; l++) {
                    const int m = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l));
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        double t = d == 0 ? 0.0 : dv[r * ST + m];
#pragma unroll
                        for (int j = 0; j < Np; j++) t += x[j][r] * Dh[l * Np + j];
                        dv[r * ST + m] = t;
                    }
                }
            }
        }
        __syncwarp();
    }
}

// One warp tile of geo_rhs_kernel: EPW elements from e_base, one lane group
// each.  Volume terms into acc (flux differencing scaled by -(1 - alpha) / J
// per node, then the subcell FV terms), the stage combine, the face terms of
// every face node of the element (times the stage factor), the store.
template <int DIM, int N, bool NS>
__device__ __forceinline__ void geo_tile(const KParams &P, const double *c, double *pr, int64_t e_base, int grp, int gl,
                                         bool lane_used, unsigned int &flags, double &lam)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, L = S::L;
    constexpr int ST = S::NS_;
    double *acc = pr + S::NPRIM * ST, *scratch = acc;
    const int64_t e0 = e_base + grp;
    const bool valid = lane_used && e0 < range_end(P);
    const int64_t e = valid ? e0 : 0;
    const int64_t nn = P.nnodes;
    if (lane_used) {
        const double ls = stage_nodes<DIM, N>(P, e, valid, gl, pr, scratch, flags);
        if (valid) lam = fmax(lam, ls);
    }
    __syncwarp();
    double alpha = 0.0;
    if (P.blending) {
        const double eta = indicator_eta<DIM, N>(scratch, gl, C_VINV(c));
        alpha = blending_alpha(eta, P);
        if (valid && gl == 0) {
            P.eta_out[e] = eta;
            P.alpha_out[e] = alpha;
        }
    }
    if (lane_used) {
#pragma unroll 1
        for (int d = 0; d < DIM; d++) ec_lines_geo<DIM, N>(P, d, pr, acc, c, gl, e, valid);
    }
    double *dv = pr + GeoShape<DIM, N, NS>::DV;
    if (NS && lane_used) viscous_volume_geo<DIM, N>(P, dv, c, gl, e, valid);
    // (-(1 - alpha) dU [+ dUv]) / J at every node (DGSEMIntegrator.cpp:423-431, 840-860)
    if (lane_used) {
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                const double J = valid ? geo_J(P, e * NDOF + n) : 1.0;
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    double t = -acc[v * ST + sp<DIM, Np>(n)];
                    t *= (1.0 - alpha);
                    if (NS && v > 0) t = t + dv[(v - 1) * ST + sp<DIM, Np>(n)];
                    acc[v * ST + sp<DIM, Np>(n)] = t / J;
                }
            }
        }
    }
    __syncwarp();
    if (P.blending && __any_sync(0xffffffffu, alpha > 0.0)) {
        if (lane_used) {
#pragma unroll 1
            for (int d = 0; d < DIM; d++) fv_lines_geo<DIM, N>(P, d, pr, acc, c, gl, e, valid, alpha);
        }
    }
    const double coef = stage_coef(P);
    if (valid) {
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const int64_t gi = (int64_t)v * nn + e * NDOF + n;
                    acc[v * ST + sp<DIM, Np>(n)] = stage_combine(P, gi, acc[v * ST + sp<DIM, Np>(n)]);
                }
            }
        }
    }
    __syncwarp();
    // faces: direction by direction, so that no two lanes update one node at once
    const double iw0 = 1.0 / C_W(c)[0];
#pragma unroll 1
    for (int d = 0; d < DIM; d++) {
        if (valid) {
            for (int t = gl; t < 2 * NFN; t += L) {
                const int side = t >= NFN, fn = side ? t - NFN : t;
                const int f = 2 * d + side;
                const int n = line_node_rt<DIM, Np>(d, fn, side ? N : 0);
                const int64_t other = __ldg(P.nbr + e * 2 * DIM + f);
                const int64_t fi = (e * 2 * DIM + f) * NFN + fn;
                double nor[DIM], s[NV], F[NV];
#pragma unroll
                for (int k = 0; k < DIM; k++) nor[k] = __ldg(P.fnor + fi * DIM + k);
#pragma unroll
                for (int v = 0; v < NV; v++) s[v] = __ldg(P.u + (int64_t)v * nn + e * NDOF + n);
                const double J = geo_J(P, e * NDOF + n);
                double sgn, fnv[NV];  // fnv: the central viscous flux . n (Navier-Stokes)
#pragma unroll
                for (int v = 0; v < NV; v++) fnv[v] = 0.0;
                if (other >= 0) {
                    const int n2 = __ldg(P.fnode + fi);
                    double o[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) o[v] = __ldg(P.u + (int64_t)v * nn + other * NDOF + n2);
                    const bool is1 = e < other || (e == other && side == 1);
                    double s1[NV], s2[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        s1[v] = is1 ? s[v] : o[v];
                        s2[v] = is1 ? o[v] : s[v];
                    }
                    const Prim<DIM> qa = make_prim<DIM>(s1, P.gamma, P.gm1), qb = make_prim<DIM>(s2, P.gamma, P.gm1);
                    face_flux_n<DIM>(qa, qb, s1 + 1, s2 + 1, nor, P.gm1inv, P.compat != 0, P.diss_scale, F);
                    lam = fmax(lam, fmax(qa.lam, qb.lam));
                    sgn = is1 ? -1.0 : 1.0;
                    if (NS) {
                        // 0.5 (F_v(1) . n + F_v(2) . n) with element 1's normal
                        // (DGSEMIntegrator.cpp:435-549); both sides' F_v . n
                        // come from the lifting kernel
                        const int64_t pi = __ldg(P.fpart + fi);
#pragma unroll
                        for (int r = 0; r < NV - 1; r++) {
                            const double co = __ldg(P.geo_cf + fi * (NV - 1) + r);
                            const double cn = __ldg(P.geo_cf + pi * (NV - 1) + r);
                            fnv[1 + r] = 0.5 * (is1 ? co + cn : cn + co);
                        }
                    }
                } else {
                    lam = fmax(lam, geo_bdr_flux<DIM>(P, (int)(-1 - other), s, nor, F));
                    sgn = -1.0;
                    const double *bcv = P.bc + (-1 - other) * BC_SLOT;
                    const int bt = (int)bcv[0];
                    if (NS && (bt == BC_SUPERSONIC_OUTFLOW || bt == BC_NOSLIP_ADIABATIC || bt == BC_NOSLIP_ISOTHERMAL ||
                               bt == BC_SUBSONIC_INFLOW_PTTT)) {
                        // ComputeBdrFaceViscousFlux . n, formed by the lifting kernel: the
                        // interior state's own viscous flux (SupersonicOutflowBdrFaceIntegrator.cpp:15-20;
                        // the walls', whose adiabatic energy row is the wall velocity's work,
                        // NoSlipAdiabWallBdrFaceIntegrator.cpp:21-36), or the outer state's
                        // with the interior gradients (SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:88-92)
#pragma unroll
                        for (int r = 0; r < NV - 1; r++) fnv[1 + r] = __ldg(P.geo_cf + fi * (NV - 1) + r);
                        if (bt == BC_NOSLIP_ADIABATIC) {
                            double en = 0.0;
#pragma unroll
                            for (int q = 0; q < DIM; q++) en += bcv[1 + q] * fnv[1 + q];
                            fnv[NV - 1] = en + 0.0;
                        }
                    }
                }
                // AddMult_a_VWt(1 / (w0 J), shape, dU): dU = -+ (F - Fv.n) for element 1 / 2
                const double scale = NS ? 1.0 / (C_W(c)[0] * J) : iw0 / J;
                const int m = sp<DIM, Np>(n);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    double dU = sgn * F[v];
                    if (NS) dU = sgn < 0.0 ? dU + fnv[v] : dU - fnv[v];
                    acc[v * ST + m] += coef * (scale * dU);
                }
            }
        }
        __syncwarp();
    }
    if (valid) {
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
#pragma unroll
                for (int v = 0; v < NV; v++) P.out[(int64_t)v * nn + e * NDOF + n] = acc[v * ST + sp<DIM, Np>(n)];
            }
        }
    }
    __syncwarp();
}

// BR1 lifting on a general mesh (LiftingBR1.cpp:10-115 faces, :156-272
// elements; ComputeGlobalPrimitiveGradVector, DGSEMOperator.cpp:96-159): per
// node the entropy variables' derivatives along the reference directions,
// times the adjugate, times 1/J; every face node adds 0.5 (w2 - w1) n_k /
// (w0 J) with element 1's states and normal (a boundary face: the condition's
// outer state, supersonic inflow / outflow / specified state); then the
// primitive gradients per direction, stored to P.geo_grads [d][v][node].
// Slot: entropy variables [v][node], gradients [d][v][node].
template <int DIM, int N> struct GeoLiftShape {
    using S = Shape<DIM, N>;
    static constexpr int EL = (1 + DIM) * S::NV * S::NS_;
};

template <int DIM, int N>
__global__ void __launch_bounds__(128) geo_lift_kernel(const KParams P)
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
    double *W = smem + const_slots(Np) + (size_t)(warp * EPW + grp) * GeoLiftShape<DIM, N>::EL;
    double *Gs = W + NV * ST;
    const double *Dm = C_D(c);
    const int64_t nn = P.nnodes;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride) {
        const int64_t e0 = P.e_begin + wt * EPW + grp;
        const bool valid = e0 < range_end(P);
        const int64_t e = valid ? e0 : 0;
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                double sv[NV], w[NV];
#pragma unroll
                for (int v = 0; v < NV; v++)
                    sv[v] = valid ? __ldg(P.u + (int64_t)v * nn + e * NDOF + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
                entropy_vars<DIM>(sv, P.gamma, P.gm1, P.gm1inv, w);
#pragma unroll
                for (int v = 0; v < NV; v++) W[v * ST + sp<DIM, Np>(n)] = w[v];
            }
        }
        __syncwarp();
        // element part
#pragma unroll 1
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
                const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
                const int line[3] = {n / Np, DIM == 2 ? pos[0] : pos[0] + Np * pos[2], pos[0] + Np * pos[1]};
                double gr[NV][DIM];
#pragma unroll
                for (int r = 0; r < DIM; r++)
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        double acc = 0.0;
#pragma unroll
                        for (int l = 0; l < Np; l++)
                            acc += W[v * ST + sp<DIM, Np>(line_node_rt<DIM, Np>(r, line[r], l))] * Dm[pos[r] * Np + l];
                        gr[v][r] = acc;
                    }
                const int64_t g = e * NDOF + n;
                const double ij = 1.0 / (valid ? geo_J(P, g) : 1.0);
                double adj[DIM][DIM];
#pragma unroll
                for (int r = 0; r < DIM; r++)
#pragma unroll
                    for (int q = 0; q < DIM; q++) adj[r][q] = valid ? geo_row1<DIM>(P, g, r, q) : (r == q ? 1.0 : 0.0);
#pragma unroll
                for (int q = 0; q < DIM; q++)
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        double t = 0.0;
#pragma unroll
                        for (int r = 0; r < DIM; r++) t += gr[v][r] * adj[r][q];
                        Gs[(q * NV + v) * ST + sp<DIM, Np>(n)] = t * ij;
                    }
            }
        }
        __syncwarp();
        // faces, direction by direction (a node lies on one face per direction)
#pragma unroll 1
        for (int d = 0; d < DIM; d++) {
            if (valid) {
                for (int t = gl; t < 2 * NFN; t += L) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    const int f = 2 * d + side;
                    const int n = line_node_rt<DIM, Np>(d, fn, side ? N : 0);
                    const int m = sp<DIM, Np>(n);
                    const int64_t other = __ldg(P.nbr + e * 2 * DIM + f);
                    const int64_t fi = (e * 2 * DIM + f) * NFN + fn;
                    double nor[DIM], w1[NV], w2[NV], fl[NV];
#pragma unroll
                    for (int k = 0; k < DIM; k++) nor[k] = __ldg(P.fnor + fi * DIM + k);
                    if (other >= 0) {
                        const int n2 = __ldg(P.fnode + fi);
                        double o[NV], wo[NV];
#pragma unroll
                        for (int v = 0; v < NV; v++) o[v] = __ldg(P.u + (int64_t)v * nn + other * NDOF + n2);
                        entropy_vars<DIM>(o, P.gamma, P.gm1, P.gm1inv, wo);
                        const bool is1 = e < other || (e == other && side == 1);
#pragma unroll
                        for (int v = 0; v < NV; v++) {
                            w1[v] = is1 ? W[v * ST + m] : wo[v];
                            w2[v] = is1 ? wo[v] : W[v * ST + m];
                            fl[v] = 0.5 * (w2[v] - w1[v]);
                        }
                    } else {
                        // ComputeBdrFaceLiftingFlux (BdrFaceIntegrator.cpp:275-282): half the jump
                        // to the condition's outer state; the no-slip walls
                        // (NoSlipAdiabWallBdrFaceIntegrator.cpp:74-95, NoSlipIsothWallBdrFaceIntegrator.cpp:41-65):
                        // (w1_0, beta V_wall, -beta) - w1
                        const double *bc = P.bc + (-1 - other) * BC_SLOT;
                        const int type = (int)bc[0];
#pragma unroll
                        for (int v = 0; v < NV; v++) w1[v] = W[v * ST + m];
                        if (type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL) {
                            const double beta = type == BC_NOSLIP_ADIABATIC ? -w1[NV - 1] : bc[1 + DIM];
                            fl[0] = w1[0] - w1[0];
#pragma unroll
                            for (int q = 0; q < DIM; q++) fl[1 + q] = bc[1 + q] * beta - w1[1 + q];
                            fl[NV - 1] = -beta - w1[NV - 1];
                        } else {
                            double si[NV], so[NV];
#pragma unroll
                            for (int v = 0; v < NV; v++) si[v] = __ldg(P.u + (int64_t)v * nn + e * NDOF + n);
                            if (type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE) {
#pragma unroll
                                for (int v = 0; v < NV; v++) so[v] = bc[1 + v];
                            } else if (type == BC_SUPERSONIC_OUTFLOW) {
#pragma unroll
                                for (int v = 0; v < NV; v++) so[v] = si[v];
                            } else {
                                double Fd[NV];
                                geo_bdr_flux<DIM>(P, (int)(-1 - other), si, nor, Fd, so);
                            }
                            entropy_vars<DIM>(so, P.gamma, P.gm1, P.gm1inv, w2);
#pragma unroll
                            for (int v = 0; v < NV; v++) fl[v] = 0.5 * (w2[v] - w1[v]);
                        }
                    }
                    const double scale = 1.0 / (C_W(c)[0] * geo_J(P, e * NDOF + n));
#pragma unroll
                    for (int v = 0; v < NV; v++) {
#pragma unroll
                        for (int q = 0; q < DIM; q++) Gs[(q * NV + v) * ST + m] += scale * (fl[v] * nor[q]);
                    }
                }
            }
            __syncwarp();
        }
        // primitive gradients
        if (valid) {
#pragma unroll 1
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
                    double sv[NV];
#pragma unroll
                    for (int v = 0; v < NV; v++) sv[v] = __ldg(P.u + (int64_t)v * nn + e * NDOF + n);
                    const int64_t gn = e * NDOF + n;
                    double g[DIM][NV];
#pragma unroll
                    for (int q = 0; q < DIM; q++) {
#pragma unroll
                        for (int v = 0; v < NV; v++) g[q][v] = Gs[(q * NV + v) * ST + sp<DIM, Np>(n)];
                        entgrad_to_primgrad<DIM>(sv, P.gm1, P.gm1inv, false, g[q]);
                        if (P.geo_grads)
#pragma unroll
                            for (int v = 0; v < NV; v++) P.geo_grads[((int64_t)q * NV + v) * nn + gn] = g[q][v];
                    }
                    if (!P.geo_fv) continue;
                    // the viscous flux (NavierStokesFlux::ComputeViscousFlux), its
                    // contravariant rows MultABt(adj, flux) (DGSEMIntegrator.cpp:616-640,
                    // 764-786) and, at every face the node lies on, its product with
                    // the face normal (element 1's; a boundary face's outward one)
                    double fm[DIM][DIM + 1];
                    viscous_flux_cols<DIM>(P, sv, g, fm);
#pragma unroll
                    for (int a = 0; a < DIM; a++)
#pragma unroll
                        for (int r = 0; r < NV - 1; r++) {
                            double acc = 0.0;
#pragma unroll
                            for (int b = 0; b < DIM; b++) acc += geo_row1<DIM>(P, gn, a, b) * fm[b][r];
                            P.geo_fv[(int64_t)(a * (NV - 1) + r) * nn + gn] = acc;
                        }
                    const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
                    const int line[3] = {n / Np, DIM == 2 ? pos[0] : pos[0] + Np * pos[2], pos[0] + Np * pos[1]};
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        if (pos[d] != 0 && pos[d] != N) continue;
                        const int f = 2 * d + (pos[d] == N ? 1 : 0);
                        const int64_t fi = (e * 2 * DIM + f) * NFN + line[d];
                        double nor[DIM];
#pragma unroll
                        for (int k2 = 0; k2 < DIM; k2++) nor[k2] = __ldg(P.fnor + fi * DIM + k2);
                        const int64_t other = __ldg(P.nbr + e * 2 * DIM + f);
                        double fo[DIM][DIM + 1];
                        const double(*fx)[DIM + 1] = fm;
                        if (other < 0 && (int)P.bc[(-1 - other) * BC_SLOT] == BC_SUBSONIC_INFLOW_PTTT) {
                            // the outer state's viscous flux with the interior gradients
                            // (SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:88-92)
                            double so[NV], Fd[NV];
                            geo_bdr_flux<DIM>(P, (int)(-1 - other), sv, nor, Fd, so);
                            viscous_flux_cols<DIM>(P, so, g, fo);
                            fx = fo;
                        }
#pragma unroll
                        for (int r = 0; r < NV - 1; r++) {
                            double t = 0.0;
#pragma unroll
                            for (int q = 0; q < DIM; q++) t += fx[q][r] * nor[q];
                            P.geo_cf[fi * (NV - 1) + r] = t;
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
}

// Resident 4-warp blocks of the Navier-Stokes variant (its 7 KB element
// slots fit three per SM).
#ifndef PDG_GEONS_MIN_BLOCKS
#define PDG_GEONS_MIN_BLOCKS 3
#endif

// Resident 4-warp blocks the register budget must allow (3D N = 3).
#ifndef PDG_GEO3_MIN_BLOCKS
#define PDG_GEO3_MIN_BLOCKS 4
#endif
// (2D N = 4, the unstructured benchmark order: four blocks, 128 registers
// with 336 B of spills, measured 21 % faster than the two of 208 registers)
#ifndef PDG_GEO2_MIN_BLOCKS
#define PDG_GEO2_MIN_BLOCKS 4
#endif
template <int DIM, int N> struct GeoOccupancy {
    static constexpr int min_blocks = (DIM == 3 && N == 3) ? PDG_GEO3_MIN_BLOCKS : (DIM == 2 && N == 4) ? PDG_GEO2_MIN_BLOCKS : 1;
};

template <int DIM, int N, bool NS = false>
__global__ void __launch_bounds__(128, NS ? PDG_GEONS_MIN_BLOCKS : GeoOccupancy<DIM, N>::min_blocks)
    geo_rhs_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, L = S::L, EPW = S::EPW;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / L, gl = lane % L;
    const int wpb = blockDim.x >> 5;
    const bool lane_used = grp < EPW;
    double *pr = smem + const_slots(Np) + (size_t)(warp * EPW + (lane_used ? grp : 0)) * GeoShape<DIM, N, NS>::EL;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    unsigned int flags = 0;
    double lam = 0.0;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride)
        geo_tile<DIM, N, NS>(P, c, pr, P.e_begin + wt * EPW, grp, gl, lane_used, flags, lam);
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

}  // namespace pdg
