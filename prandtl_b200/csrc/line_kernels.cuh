// line_kernels.cuh — sm_100a FP64 kernels of the DGSEM right-hand side,
// organised by LGL lines.
//
// Work decomposition.  A group of L lanes (L = lines per direction rounded up
// to a power of two, at most 32) owns one element; a warp holds 32/L
// elements and synchronises only with __syncwarp.  Volume work is done by
// line tasks: for each direction the lane that owns a line loads its Np nodes
// and evaluates every two-point flux of that line (Np(Np-1)/2 independent
// evaluations, which the scheduler overlaps), sums the line's contributions
// in registers and adds them to a per-node accumulator in shared memory.
// Element faces are evaluated with the element-1 rule, either by separate
// face kernels (one thread per face node: the element on the -d side
// receives C and the one on the +d side -C) or, for the fixed operator,
// inside the volume kernel by each of the face's two elements from the same
// inputs in the same order; both sides therefore see bit-identical face
// fluxes.  Both receive the same BR1 lifting jump.  Boundary faces (a
// negative neighbour entry, Euler) take the boundary condition's flux.
//
// Kernels per right-hand side:
//   Euler, fixed:     rhs_kernel<false, faces>
//   NS, fixed:        lift_face_kernel -> lift_kernel (viscous volume term to vbuf) -> rhs_kernel<true, faces>
//   Euler, reference: rhs_kernel<false> -> face_kernel<x>, <y>[, <z>]
//   NS, reference:    lift_face_kernel -> rhs_kernel<true> -> lift_kernel -> face_kernel<x>, <y>[, <z>]
// lift_kernel turns the state into BR1 primitive gradients and from them the
// viscous terms the other kernels need (the volume divergence of the viscous
// flux at every node and its normal column at every face node), so neither
// the gradients nor the volume viscous fluxes travel through HBM.
//
// Reference mapping (paths relative to the reference tree):
//   indicator + blending   src/Indicators/PerssonPeraireIndicator.cpp:21-58,
//                          src/Operators/DGSEMOperator.cpp:60-80
//   subcell FV             src/Integrators/DGSEMIntegrator/DGSEMIntegrator.cpp:972-1196
//   flux differencing      DGSEMIntegrator.cpp:224-433 (Euler), 601-864 (NS)
//   faces                  DGSEMIntegrator.cpp:151-222 (Euler), 435-549 (NS)
//   BR1 lifting            src/Integrators/Lifting/LiftingBR1/LiftingBR1.cpp:10-272
//   primitive gradients    src/Operators/DGSEMOperator.cpp:82-159
//   RK stage               RK3SSPSolver::Step as called at src/Simulation/Simulation.cpp:1010
#pragma once

#include "physics.cuh"

namespace pdg {

constexpr unsigned int PDG_FLAG_NONFINITE_DEV = 1u;
constexpr unsigned int PDG_FLAG_NONPHYSICAL_DEV = 2u;

// Per-context constants (device memory, copied to shared memory per CTA).
struct DevConst {
    double D[36];       // D[i*Np+l] = l'_l(x_i)
    double Dhat[36];    // D + boundary corrections (viscous volume term)
    double Dhat2[36];   // 2D + boundary corrections (flux differencing)
    double Vinv1[36];   // 1D inverse Legendre Vandermonde (modal transform)
    double V1[36];      // 1D Legendre Vandermonde V1[i*Np + k] = L_k(x_i) (filter)
    double w[6];        // GLL weights on [0,1]
    double snor[3][7];  // subcell interface normals per direction
    double fv_scale[6]; // 1 / (J w_i)
    double J, invJ, face_scale;
    double adj[3], area[3];
};

// Kernel parameters shared by all kernels.
struct KParams {
    const double *u;      // stage input (us)
    const double *un;     // RK base state (stages 1, 2)
    double *out;          // dudt (plain) or next stage state
    double *lbuf;         // BR1 lifting jumps [d][e][face node][v]
    double *fcol;         // viscous flux normal columns at faces [d][side][e][face node][i]
    double *grads_out;    // optional: primitive gradients [d][v][node] (diagnostics)
    double *vbuf;         // NS with element-side faces: viscous volume term [v-1][node]
    const int32_t *nbr;   // [ne][2*dim]
    const DevConst *K;
    double *eta_out, *alpha_out;
    unsigned long long *lam_bits;  // running max wave speed (as ordered bits)
    unsigned int *err;
    double *ent_own;                    // filter: per-element entropy minimum at the stage input
    unsigned long long *filter_count;   // filter: elements filtered so far
    unsigned long long *limit_count;    // positivity limiter: elements limited so far
    int64_t ne, nnodes;
    int64_t nwt;          // number of warp tiles
    int stage;            // -1: plain RHS; 0, 1, 2: SSP-RK3 stage
    double dt;
    double gamma, gm1, gm1inv;
    double mu, lambda_k;  // NS: mu and mu*gamma/Pr
    double alpha_max, alpha_min, modal_threshold;
    double diss_scale;
    int blending, compat;
    int prefetch;         // L2-prefetch the next element's inputs
    const double *bc;     // boundary conditions, BC_SLOT doubles each (type, state)
    double *lbuf_lo;      // NS boundary faces: BR1 jumps of -d boundary faces [d][e][face node][v]
    int has_bdr;          // the neighbour table holds boundary faces (negative entries)
    // inviscid face flux of every interior face, evaluated once per face
    // node: [d][e][v][face node] for the face between e's +d face and its
    // +d neighbour, signed as element e receives it (see face_flux_oriented)
    double *fbuf;
    // adjoint: face-term cotangents [d][side][e][v][face node]
    // (adj_faces_kernel) and the RK base state's cotangent accumulator of an
    // adjoint stage
    const double *gbuf;
    double *bx;
    // elements [e_begin, e_end) that the face-node, lifting and volume
    // kernels process (e_end = 0: up to ne); nwt counts the range's tiles
    int64_t e_begin, e_end;
    // general geometry (geo_rhs_kernel): per node J and the adjugate rows,
    // geo[q * nnodes + node], q = 0: J, 1 + r * dim + k: adj(r, k); per
    // element face node the neighbour's matching node (local index) and the
    // face normal as the face's element 1 sees it, [e][face][face node](, k)
    const double *geo;
    const int32_t *fnode;
    const double *fnor;
    // general geometry, Navier-Stokes (written by geo_lift_kernel): the
    // primitive gradients [d][v][node] (when requested), the contravariant
    // viscous fluxes [d][row][node] and, per element face node, the viscous
    // flux dotted with the face normal [e][face][face node][row] (rows:
    // momenta and energy); fpart: the neighbour's slot of each face node in
    // that last array (-1 on boundary faces)
    double *geo_grads;
    double *geo_fv;
    double *geo_cf;
    const int32_t *fpart;
};

__device__ __forceinline__ int64_t range_end(const KParams &P) { return P.e_end ? P.e_end : P.ne; }

// Boundary conditions (src/Integrators/BoundaryConditions/): a neighbour
// entry -1 - b marks a boundary face with condition b of the table P.bc.
constexpr int BC_SLOT = 8;
constexpr int BC_SUPERSONIC_INFLOW = 1, BC_SUPERSONIC_OUTFLOW = 2, BC_SPECIFIED_STATE = 3, BC_SLIP_WALL = 4,
              BC_SYMMETRY = 5, BC_SUBSONIC_OUTFLOW_P = 6, BC_SUBSONIC_INFLOW_RV = 7, BC_SUBSONIC_INFLOW_PTTT = 8,
              BC_RIEMANN_INVARIANT = 9, BC_NOSLIP_ADIABATIC = 10, BC_NOSLIP_ISOTHERMAL = 11;

constexpr int pow2_at_least(int x) { return x <= 1 ? 1 : x <= 2 ? 2 : x <= 4 ? 4 : x <= 8 ? 8 : x <= 16 ? 16 : 32; }

template <int DIM, int N> struct Shape {
    static constexpr int Np = N + 1;
    static constexpr int NDOF = DIM == 2 ? Np * Np : Np * Np * Np;
    static constexpr int NV = DIM + 2;
    static constexpr int NFN = DIM == 2 ? Np : Np * Np;  // face nodes = lines per direction
    static constexpr int L = pow2_at_least(NFN);        // lanes per element
    static constexpr int EPW = 32 / L;                  // elements per warp
    static constexpr int NPL = (NDOF + L - 1) / L;      // nodes per lane
    static constexpr int LPL = (NFN + L - 1) / L;       // lines per lane per direction
    static constexpr int NPRIM = DIM + 2;               // rho, v[DIM], beta
    // per-variable stride in shared memory: swizzled (no padding) for 3D
    // Np = 4, one padding slot per x line otherwise
    static constexpr int NS_ = (DIM == 3 && Np == 4) ? NDOF : NDOF + NDOF / Np;
    // rhs element slot: primitives, accumulator (which also holds the modal
    // transform of the indicator before the first flux pass), and the compat
    // z-fill buffer
    static constexpr int ZFILL = NFN * N * NV;
    static constexpr int EL_RHS = NPRIM * NS_ + NV * NS_ + ZFILL;
    // the fixed operator's volume kernel reading the face buffer: no z-fill
    static constexpr int EL_RHS_FB = NPRIM * NS_ + NV * NS_;
    // adjoint lift slot: entropy variables, gradients along each direction
    static constexpr int EL_LIFT = NV * NS_ + DIM * NV * NS_;
    // forward lift slot: entropy variables (later the viscous RHS) and the
    // contravariant viscous fluxes (gradients are formed per node)
    static constexpr int EL_LIFTF = NV * NS_ + DIM * (NV - 1) * NS_;
};

// Shared-memory position of node n, chosen so that the lanes of a line task
// (one node of each line of a direction: a plane of the element) hit
// distinct banks.  3D Np = 4, n = i + 4j + 16k: row k, column
// 4((j + k) mod 4) + (i + k) mod 4 — a bijection on every x, y and z plane.
// Otherwise one padding slot per x line.
template <int DIM, int Np> __device__ __forceinline__ constexpr int sp(int n)
{
    if (DIM == 3 && Np == 4) {
        const int i = n & 3, j = (n >> 2) & 3, k = n >> 4;
        return (k << 4) + (((j + k) & 3) << 2) + ((i + k) & 3);
    }
    return n + n / Np;
}

// Prefetch a byte range into L2 (TMA bulk prefetch); the range is shrunk to
// whole 16-byte blocks inside it.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes)
{
    const uintptr_t a = (uintptr_t)p;
    const uintptr_t s = (a + 15) & ~(uintptr_t)15, e = (a + bytes) & ~(uintptr_t)15;
    if (e > s) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(s), "r"((unsigned)(e - s)) : "memory");
}

enum { P_RHO = 0, P_V = 1 };
template <int DIM> struct PSlot {
    static constexpr int BETA = P_V + DIM;
};

// Node index of position `pos` on line `line` of a runtime direction d.
template <int DIM, int Np> __device__ __forceinline__ int line_node_rt(int d, int line, int pos)
{
    if (DIM == 2) return d == 0 ? line * Np + pos : pos * Np + line;
    if (d == 0) return line * Np + pos;
    if (d == 1) return (line / Np) * Np * Np + pos * Np + (line % Np);
    return pos * Np * Np + line;
}

// Node index of position `pos` on line `line` of direction D (x fastest).
template <int DIM, int Np, int D> __device__ __forceinline__ int line_node(int line, int pos)
{
    if (DIM == 2) return D == 0 ? line * Np + pos : pos * Np + line;
    if (D == 0) return line * Np + pos;
    if (D == 1) return (line / Np) * Np * Np + pos * Np + (line % Np);
    return pos * Np * Np + line;
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *addr, double v)
{
    if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}
template <int G> __device__ __forceinline__ double group_sum(double x)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
template <int G> __device__ __forceinline__ double group_max(double x)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// ---- constants in shared memory ----
// Packed for the element's Np (each matrix Np x Np): D, Dhat, Dhat2, Vinv,
// w, subcell normals (Np + 1 per direction), 1/(J w), adj, area, J, 1/J,
// face scale.  The macros need a constant `Np` in scope.
__host__ __device__ constexpr int cs_snor(int Np) { return 4 * Np * Np + Np; }
__host__ __device__ constexpr int cs_fvs(int Np) { return cs_snor(Np) + 3 * (Np + 1); }
__host__ __device__ constexpr int cs_adj(int Np) { return cs_fvs(Np) + Np; }
__host__ __device__ constexpr int const_slots(int Np) { return (cs_adj(Np) + 9 + 1) & ~1; }
#define C_D(c) (c)
#define C_DHAT(c) ((c) + Np * Np)
#define C_DHAT2(c) ((c) + 2 * Np * Np)
#define C_VINV(c) ((c) + 3 * Np * Np)
#define C_W(c) ((c) + 4 * Np * Np)
#define C_SNOR(c, d) ((c) + cs_snor(Np) + (Np + 1) * (d))
#define C_FVS(c) ((c) + cs_fvs(Np))
#define C_ADJ(c) ((c) + cs_adj(Np))
#define C_AREA(c) ((c) + cs_adj(Np) + 3)
#define C_J(c) ((c)[cs_adj(Np) + 6])
#define C_INVJ(c) ((c)[cs_adj(Np) + 7])
#define C_FACE(c) ((c)[cs_adj(Np) + 8])
constexpr int CONST_SLOTS = 192;  // the largest packing (Np = 6) fits
static_assert(const_slots(6) <= CONST_SLOTS, "constant slots");

__device__ __forceinline__ void load_consts(const DevConst *K, double *c, int Np, int tid, int nth)
{
    const int n2 = Np * Np;
    for (int t = tid; t < n2; t += nth) {
        c[t] = K->D[t];
        c[n2 + t] = K->Dhat[t];
        c[2 * n2 + t] = K->Dhat2[t];
        c[3 * n2 + t] = K->Vinv1[t];
    }
    for (int t = tid; t < Np; t += nth) {
        c[4 * n2 + t] = K->w[t];
        c[cs_fvs(Np) + t] = K->fv_scale[t];
    }
    for (int t = tid; t < 3 * (Np + 1); t += nth) c[cs_snor(Np) + t] = K->snor[t / (Np + 1)][t % (Np + 1)];
    for (int t = tid; t < 3; t += nth) {
        c[cs_adj(Np) + t] = K->adj[t];
        c[cs_adj(Np) + 3 + t] = K->area[t];
    }
    if (tid == 0) {
        c[cs_adj(Np) + 6] = K->J;
        c[cs_adj(Np) + 7] = K->invJ;
        c[cs_adj(Np) + 8] = K->face_scale;
    }
}
__device__ __forceinline__ void load_consts(const DevConst *K, double *c, int Np)
{
    load_consts(K, c, Np, threadIdx.x, blockDim.x);
}

// Primitive quantities of a node from the shared slot (p and 1/rho are not
// kept: the two-point fluxes only need rho, v, beta, 1/beta and the speed).
template <int DIM> __device__ __forceinline__ Prim<DIM> slot_prim(const double *pr, int sn, int ST)
{
    using PS = PSlot<DIM>;
    Prim<DIM> q;
    q.rho = pr[P_RHO * ST + sn];
#pragma unroll
    for (int d = 0; d < DIM; d++) q.v[d] = pr[(P_V + d) * ST + sn];
    q.beta = pr[PS::BETA * ST + sn];
    q.ib = 0.0;
    q.lam = 0.0;
    q.p = 0.0;
    q.irho = 0.0;
    return q;
}
// Adds 1/beta and the wave speed |v| + sqrt(gamma p / rho) = |v| + sqrt(gamma / (2 beta)).
template <int DIM> __device__ __forceinline__ void complete_prim(Prim<DIM> &q, double gamma)
{
    double vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) vsq += q.v[d] * q.v[d];
    q.ib = 1.0 / q.beta;
    q.lam = sqrt(vsq) + sqrt(0.5 * gamma * q.ib);
}

__device__ __forceinline__ double blending_alpha(double eta, const KParams &P)
{
    const double T = P.modal_threshold;
    double a = 1.0 / (1.0 + exp(-9.21024 * (eta - T) / T));
    if (a < P.alpha_min) a = 0.0;
    else if (a > (1.0 - P.alpha_min)) a = 1.0;
    return fmin(a, P.alpha_max);
}

// One 1D pass of the modal transform: dst[line, k] = sum_l Vinv(k,l) src[line, l].
template <int DIM, int N, int D>
__device__ __forceinline__ void modal_pass(const double *src, double *dst, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np;
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            double x[Np];
#pragma unroll
            for (int l = 0; l < Np; l++) x[l] = src[sp<DIM, Np>(line_node<DIM, Np, D>(line, l))];
#pragma unroll
            for (int k = 0; k < Np; k++) {
                double s = 0.0;
#pragma unroll
                for (int l = 0; l < Np; l++) s += Vinv[k * Np + l] * x[l];
                dst[sp<DIM, Np>(line_node<DIM, Np, D>(line, k))] = s;
            }
        }
    }
    __syncwarp();
}

// Persson-Peraire indicator from q = rho p at the nodes (buf[0..NDOF)):
// modes = (V1^-1 x ... x V1^-1) q, eta = max(1 - |m1|^2/|m|^2,
// 1 - |m2|^2/|m1|^2), m1 without modes of 1D degree N, m2 without degree >= N-1.
template <int DIM, int N>
__device__ __forceinline__ double indicator_eta(double *buf, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF;
    double *a = buf, *b = buf + S::NS_;
    modal_pass<DIM, N, 0>(a, b, gl, Vinv);
    modal_pass<DIM, N, 1>(b, a, gl, Vinv);
    if (DIM == 3) modal_pass<DIM, N, (DIM == 3 ? 2 : 0)>(a, b, gl, Vinv);
    const double *m = (DIM == 3) ? b : a;
    double mm = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int t = gl + s * S::L;
        if (t < NDOF) {
            const int i = t % Np, j = (t / Np) % Np, k = DIM == 3 ? t / (Np * Np) : 0;
            int mx = i > j ? i : j;
            if (DIM == 3) mx = mx > k ? mx : k;
            const double v = m[sp<DIM, Np>(t)] * m[sp<DIM, Np>(t)];
            mm += v;
            if (mx <= N - 1) m1 += v;
            if (mx <= N - 2) m2 += v;
        }
    }
    mm = group_sum<S::L>(mm);
    m1 = group_sum<S::L>(m1);
    m2 = group_sum<S::L>(m2);
    const double eta = 1.0 - m1 / mm;
    return fmax(eta, 1.0 - m2 / m1);
}

// Loads the element's nodes, writes their primitives to the shared slot and
// rho*p to the scratch (indicator input).  Returns this lane's max speed.
template <int DIM, int N>
__device__ __forceinline__ double stage_nodes(const KParams &P, int64_t e, bool valid, int gl, double *pr,
                                              double *scratch, unsigned int &flags)
{
    using S = Shape<DIM, N>;
    using PS = PSlot<DIM>;
    constexpr int NDOF = S::NDOF, NV = S::NV;
    double lam = 0.0;
#pragma unroll
    for (int k = 0; k < S::NPL; k++) {
        const int n = gl + k * S::L;
        if (n < NDOF) {
            double s[NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                s[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + e * NDOF + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
            const Prim<DIM> q = make_prim<DIM>(s, P.gamma, P.gm1);
            constexpr int ST = S::NS_;
            const int m = sp<DIM, S::Np>(n);
            pr[P_RHO * ST + m] = q.rho;
#pragma unroll
            for (int d = 0; d < DIM; d++) pr[(P_V + d) * ST + m] = q.v[d];
            pr[PS::BETA * ST + m] = q.beta;
            scratch[m] = q.rho * q.p;
            lam = fmax(lam, q.lam);
            bool finite = true;
#pragma unroll
            for (int v = 0; v < NV; v++) finite = finite && isfinite(s[v]);
            if (!finite) flags |= PDG_FLAG_NONFINITE_DEV;
            else if (!(q.rho > 0.0) || !(q.p > 0.0)) flags |= PDG_FLAG_NONPHYSICAL_DEV;
        }
    }
    __syncwarp();
    return lam;
}

// Flux-differencing line tasks along direction d (a runtime value, so the
// two-point flux code exists once per kernel): every pair (a < b) of the line
// is evaluated once and contributes Dhat2(a,b) F to node a and Dhat2(b,a) F
// to node b; the line sums, scaled by `scale`, are stored (d == 0) or added
// to acc.  Node a receives its terms in ascending partner order, as the
// reference's row sum does.
// Compat NS 3D keeps the reference's z-direction fill (DGSEMIntegrator.cpp:
// 702): during the y pass (zsave) the flux of pair (j, N) of y line (i, m) is
// saved to zf[(i + Np m) * N + j]; during the z pass (zuse) node (i, j, k)
// takes Dhat2(k, m) * zf[(i + Np m) * N + j] (0 when j = N) for its partners
// m < k instead of the z flux.
template <int DIM, int N>
__device__ __forceinline__ void ec_lines_rt(const KParams &P, int d, const double *pr, double *acc, double *zf,
                                            const double *c, int gl, double scale, bool zsave, bool zuse)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV;
    const double metric = C_ADJ(c)[d];
    const double *D2 = C_DHAT2(c);
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            Prim<DIM> q[Np];
#pragma unroll
            for (int l = 0; l < Np; l++) q[l] = slot_prim<DIM>(pr, sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l)), S::NS_);
            double la[Np][NV];
#pragma unroll
            for (int l = 0; l < Np; l++)
#pragma unroll
                for (int v = 0; v < NV; v++) la[l][v] = 0.0;
#pragma unroll
            for (int a = 0; a < Np; a++)
#pragma unroll
                for (int b = a + 1; b < Np; b++) {
                    double F[NV];
                    volume_flux_rt<DIM>(q[a], q[b], d, metric, P.gm1inv, F);
                    const double cab = D2[a * Np + b], cba = D2[b * Np + a];
                    if (zsave && b == N) {
#pragma unroll
                        for (int v = 0; v < NV; v++) zf[(line * N + a) * NV + v] = F[v];
                    }
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        la[a][v] += cab * F[v];
                        if (!zuse) la[b][v] += cba * F[v];
                    }
                }
            if (zuse) {
                const int i = line % Np, j = line / Np;
                if (j < N) {
#pragma unroll
                    for (int k = 1; k < Np; k++)
#pragma unroll
                        for (int m = 0; m < k; m++) {
                            const double ckm = D2[k * Np + m];
                            const double *F = zf + ((i + Np * m) * N + j) * NV;
#pragma unroll
                            for (int v = 0; v < NV; v++) la[k][v] += ckm * F[v];
                        }
                }
            }
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = sp<DIM, Np>(line_node_rt<DIM, Np>(d, line, l));
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const double x = scale * la[l][v];
                    if (d == 0) acc[v * S::NS_ + n] = x;
                    else acc[v * S::NS_ + n] += x;
                }
            }
        }
    }
    __syncwarp();
}

// Subcell finite-volume line tasks along D (ComputeFVFluxes): node l of the
// line gets alpha (f_{l-1/2} - f_{l+1/2}) / (J w_l), interface fluxes being
// Chandrashekar face fluxes with the subcell normals.
template <int DIM, int N, int D>
__device__ __forceinline__ void fv_lines(const KParams &P, const double *pr, double *acc, const double *c, int gl,
                                         double alpha)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const double *sn = C_SNOR(c, D), *fvs = C_FVS(c);
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
            double prev[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) prev[v] = 0.0;
            Prim<DIM> qa = slot_prim<DIM>(pr, sp<DIM, Np>(line_node<DIM, Np, D>(line, 0)), S::NS_);
            complete_prim<DIM>(qa, P.gamma);
#pragma unroll
            for (int l = 0; l < Np; l++) {
                const int n = sp<DIM, Np>(line_node<DIM, Np, D>(line, l));
                double F[NV];
                Prim<DIM> qb;
                if (l < N) {
                    qb = slot_prim<DIM>(pr, sp<DIM, Np>(line_node<DIM, Np, D>(line, l + 1)), S::NS_);
                    complete_prim<DIM>(qb, P.gamma);
                    double ma[DIM], mb[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        ma[d] = qa.rho * qa.v[d];
                        mb[d] = qb.rho * qb.v[d];
                    }
                    face_flux<DIM, D>(qa, qb, ma, mb, sn[l + 1], P.gm1inv, P.compat != 0, P.diss_scale, F);
                } else {
#pragma unroll
                    for (int v = 0; v < NV; v++) F[v] = 0.0;
                }
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    acc[v * S::NS_ + n] += alpha * ((prev[v] - F[v]) * fvs[l]);
                    prev[v] = F[v];
                }
                if (l < N) qa = qb;
            }
        }
    }
    __syncwarp();
}

// Output of a volume kernel for node value gi with right-hand side x:
// plain RHS: x; SSP-RK3 stage: z = us + dt x and stage 0: z, 1: 3/4 un + 1/4 z,
// 2: 1/3 un + 2/3 z (RK3SSPSolver::Step).
__device__ __forceinline__ double stage_combine(const KParams &P, int64_t gi, double x)
{
    if (P.stage < 0) return x;
    const double z = __ldg(P.u + gi) + P.dt * x;
    if (P.stage == 0) return z;
    if (P.stage == 1) return 3. / 4 * __ldg(P.un + gi) + 1. / 4 * z;
    return 1. / 3 * __ldg(P.un + gi) + 2. / 3 * z;
}
// Factor with which a further right-hand-side term enters the output.
__device__ __forceinline__ double stage_coef(const KParams &P)
{
    if (P.stage < 0) return 1.0;
    if (P.stage == 0) return P.dt;
    if (P.stage == 1) return 1. / 4 * P.dt;
    return 2. / 3 * P.dt;
}

template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ double face_node_terms(const KParams &P, const double *c, int64_t a, int64_t b, int fn,
                                                  double coef, double *C);
template <int DIM, bool NS> struct FaceIn;
template <int DIM, int N, int D>
__device__ __noinline__ double boundary_node_terms(const KParams &P, const double *c, const double *s, int b,
                                                   double sgn, double coef, double *C);
template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ void load_face_in(const KParams &P, int64_t a, int64_t b, int fn, FaceIn<DIM, NS> &in);
template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ double face_terms_from(const KParams &P, const double *c, bool a_is_1,
                                                  const FaceIn<DIM, NS> &in, double coef, double *C);

// Face terms of direction D for one element e (its lane group): slot t <
// NFN is face node t of the -D face (element a = the -D neighbour), slot
// NFN + t face node t of the +D face (a = e).  Every slot of a lane is loaded
// before any is evaluated, so their load latencies overlap.  The inviscid
// flux comes first; NS then adds the central viscous flux, which for either
// orientation of the face is C_FACE coef (fa + fb)/2 |n_D| for element a and
// its negative for b (fixed operator only: the reference-value operator's
// face fluxes read velocities from the momentum slots).  BDR (a mesh with
// boundary faces): a slot whose neighbour entry is negative takes the
// boundary condition's inviscid flux (boundary_node_terms) and, NS, its
// viscous boundary flux, both for this element alone.
// FB: the inviscid fluxes come from P.fbuf (evaluated once per face by the
// face-flux kernel) instead of being evaluated here.
template <int DIM, int N, bool NS, int D, bool BDR, bool FB = false>
__device__ __forceinline__ void face_terms_dir(const KParams &P, const double *c, double *acc, int64_t e,
                                               const int32_t *enb, int gl, bool valid, double coef, double &lam)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, NFN = S::NFN, L = S::L, ST = S::NS_;
    constexpr int R = (2 * NFN + L - 1) / L;
    if (valid && FB) {
        double Fa[R][NV];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int t = gl + r * L;
            if (t < 2 * NFN) {
                const int side = t >= NFN, fn = side ? t - NFN : t;
                const int64_t a = side ? e : (int64_t)enb[2 * D];
                const double *src = P.fbuf + ((D * P.ne + a) * NV) * NFN + fn;
#pragma unroll
                for (int v = 0; v < NV; v++) Fa[r][v] = __ldg(src + v * NFN);
            }
        }
        const double sc = C_FACE(c) * coef;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int t = gl + r * L;
            if (t < 2 * NFN) {
                const int side = t >= NFN, fn = side ? t - NFN : t;
                const int n = sp<DIM, Np>(line_node<DIM, Np, D>(fn, side ? N : 0));
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const double C = sc * Fa[r][v];
                    if (side) acc[v * ST + n] += C;
                    else acc[v * ST + n] -= C;
                }
            }
        }
    }
    if (valid) {
        if (!FB) {
            FaceIn<DIM, false> in[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int t = gl + r * L;
                if (t < 2 * NFN) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    const int64_t other = enb[2 * D + side];
                    if (!BDR || other >= 0) {  // BDR: the mesh has boundary faces
                        load_face_in<DIM, N, D, false>(P, side ? e : other, side ? other : e, fn, in[r]);
                    } else {
                        // boundary face: this element's trace only
                        const int n = line_node<DIM, Np, D>(fn, side ? N : 0);
#pragma unroll
                        for (int v = 0; v < NV; v++) in[r].sa[v] = __ldg(P.u + v * P.nnodes + e * S::NDOF + n);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int t = gl + r * L;
                if (t < 2 * NFN) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    const int64_t other = enb[2 * D + side];
                    const int64_t a = side ? e : other, b = side ? other : e;
                    const int n = sp<DIM, Np>(line_node<DIM, Np, D>(fn, side ? N : 0));
                    double C[NV];
                    if (!BDR || other >= 0) {
                        face_terms_from<DIM, N, D, false>(P, c, a <= b, in[r], coef, C);
#pragma unroll
                        for (int v = 0; v < NV; v++) {
                            if (side) acc[v * ST + n] += C[v];
                            else acc[v * ST + n] -= C[v];
                        }
                    } else {
                        lam = fmax(lam, boundary_node_terms<DIM, N, D>(P, c, in[r].sa, (int)(-1 - other),
                                                                        side ? 1.0 : -1.0, coef, C));
#pragma unroll
                        for (int v = 0; v < NV; v++) acc[v * ST + n] += C[v];
                    }
                }
            }
        }
        if (NS) {
            const int64_t ne = P.ne;
            double fv[R][DIM + 1];
            bool bslot[R];  // boundary face: fv holds the element's whole viscous term
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int t = gl + r * L;
                bslot[r] = false;
                if (t < 2 * NFN) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    const int64_t other = enb[2 * D + side];
                    if (BDR && other < 0) {
                        // ComputeBdrFaceViscousFlux: the element's own column
                        // (outflow, no-slip wall) or nothing (prescribed
                        // states: the outer state with zero gradients)
                        bslot[r] = true;
                        const double *bc = P.bc + (-1 - other) * BC_SLOT;
                        const int type = (int)bc[0];
                        const double nrm = side ? C_AREA(c)[D] : -C_AREA(c)[D];
                        const double *fo = P.fcol + (((D * 2 + side) * ne + e) * NFN + fn) * (NV - 1);
                        const bool own = type == BC_SUPERSONIC_OUTFLOW || type == BC_NOSLIP_ADIABATIC ||
                                         type == BC_NOSLIP_ISOTHERMAL || type == BC_SUBSONIC_INFLOW_PTTT;
#pragma unroll
                        for (int i = 0; i <= DIM; i++) fv[r][i] = own ? __ldg(fo + i) * nrm : 0.0;
                        if (type == BC_NOSLIP_ADIABATIC) {  // energy row: the wall velocity's work, qn = 0
                            double en = 0.0;
#pragma unroll
                            for (int q = 0; q < DIM; q++) en += bc[1 + q] * fv[r][q];
                            fv[r][DIM] = en + 0.0;
                        }
                        continue;
                    }
                    const int64_t a = side ? e : other, b = side ? other : e;
                    const double *fa = P.fcol + (((D * 2 + 1) * ne + a) * NFN + fn) * (NV - 1);
                    const double *fb = P.fcol + (((D * 2 + 0) * ne + b) * NFN + fn) * (NV - 1);
#pragma unroll
                    for (int i = 0; i <= DIM; i++) fv[r][i] = __ldg(fa + i) + __ldg(fb + i);
                }
            }
            const double sc = (C_FACE(c) * coef) * (0.5 * C_AREA(c)[D]);
            const double sb = C_FACE(c) * coef;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int t = gl + r * L;
                if (t < 2 * NFN) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    const int n = sp<DIM, Np>(line_node<DIM, Np, D>(fn, side ? N : 0));
#pragma unroll
                    for (int i = 0; i <= DIM; i++) {
                        if (BDR && bslot[r]) {
                            acc[(1 + i) * ST + n] += sb * fv[r][i];
                            continue;
                        }
                        const double x = sc * fv[r][i];
                        if (side) acc[(1 + i) * ST + n] += x;
                        else acc[(1 + i) * ST + n] -= x;
                    }
                }
            }
        }
    }
    __syncwarp();
}

// One warp tile of the right-hand side element kernel: EPW elements from
// e_base, one lane group each.  Volume terms (flux differencing, subcell FV
// blending) into acc, then either the stage output is stored and the face
// terms are left to the face kernels (FACES = false), or (FACES = true) every
// element also adds the face terms of its own face nodes, evaluated with the
// same element-1 rule and in the same order (x faces, then y [, z]) as the
// face kernels use, and stores the finished stage.  With NS and FACES the
// lifting kernel has run first: its viscous volume term (P.vbuf) enters after
// the stage combine, where the other path's lifting kernel adds it, and the
// face terms include the central viscous flux of both sides' face columns.
// Each face is thus evaluated twice, once by each of its elements, on the
// same inputs in the same order, so both get the same value.
template <int DIM, int N, bool NS, bool FACES, bool PRELOAD = true, bool BDR = false, bool FB = false>
__device__ __forceinline__ void rhs_tile(const KParams &P, const double *c, double *pr, int64_t e_base, int grp,
                                         int gl, bool lane_used, unsigned int &flags, double &lam)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, L = S::L;
    constexpr int ST = S::NS_;
    double *acc = pr + S::NPRIM * ST, *scratch = acc, *zf = acc + NV * ST;
    const bool compat = P.compat != 0;
    const int64_t e0 = e_base + grp;
    const bool valid = lane_used && e0 < range_end(P);
    const int64_t e = valid ? e0 : 0;
    // the RK base state is first read by the final combine: bring the
    // element's block of each variable into L2 now
    if ((!FACES || NS) && valid && P.stage > 0 && gl < NV) prefetch_l2(P.un + (int64_t)gl * P.nnodes + e * NDOF, sizeof(double) * NDOF);
    if (FACES && NS && valid && gl >= NV && gl < 2 * NV - 1)
        prefetch_l2(P.vbuf + (int64_t)(gl - NV) * P.nnodes + e * NDOF, sizeof(double) * NDOF);
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
    const double sc = -(1.0 - alpha) * C_INVJ(c);
    if (lane_used) {
        // (the face-buffer variant's slot has no z-fill buffer; the host runs
        // it for the fixed operator only)
        const bool zfill = DIM == 3 && NS && compat && !FB;
#pragma unroll 1
        for (int d = 0; d < DIM; d++)
            ec_lines_rt<DIM, N>(P, d, pr, acc, zf, c, gl, sc, zfill && d == 1, zfill && d == 2);
    }
    if (P.blending && __any_sync(0xffffffffu, alpha > 0.0)) {
        if (lane_used) {
            fv_lines<DIM, N, 0>(P, pr, acc, c, gl, alpha);
            fv_lines<DIM, N, 1>(P, pr, acc, c, gl, alpha);
            if (DIM == 3) fv_lines<DIM, N, (DIM == 3 ? 2 : 0)>(P, pr, acc, c, gl, alpha);
        }
    }
    if (!FACES) {
        // store: out = a un + b (us + dt V); the viscous volume term and the
        // face terms are added afterwards by lift_kernel and face_kernel
        if (valid) {
#pragma unroll
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        const int64_t gi = (int64_t)v * P.nnodes + e * NDOF + n;
                        P.out[gi] = stage_combine(P, gi, acc[v * ST + sp<DIM, Np>(n)]);
                    }
                }
            }
        }
        __syncwarp();
        return;
    }
    // element-centric faces: combine first (plus the viscous volume term),
    // then add each direction's face terms in turn, then store
    const double coef = stage_coef(P);
    // the face neighbours, requested before the combine's loads
    int32_t enb[2 * DIM];
    if (PRELOAD) {
#pragma unroll
        for (int k = 0; k < 2 * DIM; k++) enb[k] = valid ? __ldg(P.nbr + e * 2 * DIM + k) : 0;
    }
    if (valid) {
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const int64_t gi = (int64_t)v * P.nnodes + e * NDOF + n;
                    double x = stage_combine(P, gi, acc[v * ST + sp<DIM, Np>(n)]);
                    if (NS && v > 0) x = x + coef * __ldg(P.vbuf + gi - P.nnodes);
                    acc[v * ST + sp<DIM, Np>(n)] = x;
                }
            }
        }
    }
    __syncwarp();
    if (PRELOAD) {
        face_terms_dir<DIM, N, NS, 0, BDR, FB>(P, c, acc, e, enb, gl, valid, coef, lam);
        face_terms_dir<DIM, N, NS, 1, BDR, FB>(P, c, acc, e, enb, gl, valid, coef, lam);
        if (DIM == 3) face_terms_dir<DIM, N, NS, (DIM == 3 ? 2 : 0), BDR, FB>(P, c, acc, e, enb, gl, valid, coef, lam);
    } else {
        // one face node at a time (Euler): the batched sweep's register
        // variants are tuned for this form
#pragma unroll 1
        for (int d = 0; d < DIM; d++) {
            if (valid) {
                for (int t = gl; t < 2 * NFN; t += L) {
                    const int side = t >= NFN, fn = side ? t - NFN : t;
                    // side 1: this element's +d face (it is element a); side
                    // 0: its -d face, whose element a is the -d neighbour
                    const int64_t other = __ldg(P.nbr + e * 2 * DIM + 2 * d + side);
                    const int64_t a = side ? e : other, b = side ? other : e;
                    double C[NV];
                    if (d == 0) face_node_terms<DIM, N, 0, false>(P, c, a, b, fn, coef, C);
                    else if (d == 1) face_node_terms<DIM, N, 1, false>(P, c, a, b, fn, coef, C);
                    else face_node_terms<DIM, N, (DIM == 3 ? 2 : 0), false>(P, c, a, b, fn, coef, C);
                    const int n = sp<DIM, Np>(line_node_rt<DIM, Np>(d, fn, side ? N : 0));
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        if (side) acc[v * ST + n] += C[v];
                        else acc[v * ST + n] -= C[v];
                    }
                }
            }
            __syncwarp();
        }
    }
    if (valid) {
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
            if (n < NDOF) {
#pragma unroll
                for (int v = 0; v < NV; v++) P.out[(int64_t)v * P.nnodes + e * NDOF + n] = acc[v * ST + sp<DIM, Np>(n)];
            }
        }
    }
    __syncwarp();
}

// Right-hand side element kernel (Euler or Navier-Stokes volume terms,
// optional SSP-RK3 stage).
// Resident blocks the register budget must allow: 4 for 3D N = 3 (whose
// swizzled slots let four 4-warp blocks share an SM), 1 otherwise.
#ifndef PDG_RHS3_MIN_BLOCKS
#define PDG_RHS3_MIN_BLOCKS 4
#endif
#ifndef PDG_LIFT3_MIN_BLOCKS
#define PDG_LIFT3_MIN_BLOCKS 4
#endif
template <int DIM, int N> struct RhsOccupancy {
    static constexpr int min_blocks = (DIM == 3 && N == 3) ? PDG_RHS3_MIN_BLOCKS : 1;
};
template <int DIM, int N> struct LiftOccupancy {
    static constexpr int min_blocks = (DIM == 3 && N == 3) ? PDG_LIFT3_MIN_BLOCKS : 1;
};

// BDR: a variant for meshes with boundary faces (Euler), whose boundary
// branch would otherwise cost registers in every face loop.  FB: the
// inviscid face fluxes come from P.fbuf (periodic meshes, FACES only).
template <int DIM, int N, bool NS, bool FACES = false, bool BDR = false, bool FB = false>
__global__ void __launch_bounds__(128, RhsOccupancy<DIM, N>::min_blocks) rhs_kernel(const KParams P)
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
    constexpr int EL = FB ? S::EL_RHS_FB : S::EL_RHS;
    double *pr = smem + const_slots(Np) + (size_t)(warp * EPW + (lane_used ? grp : 0)) * EL;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    unsigned int flags = 0;
    double lam = 0.0;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride)
        rhs_tile<DIM, N, NS, FACES, true, BDR, FB>(P, c, pr, P.e_begin + wt * EPW, grp, gl, lane_used, flags, lam);
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

// Primitive quantities of a state whose momentum slots hold velocities (the
// reference's NS face states after ComputeViscousFlux divided them in place):
// velocities v' = v / rho, pressure from E with v', and the derived terms.
template <int DIM>
__device__ __forceinline__ Prim<DIM> velocity_slot_prim(const Prim<DIM> &q, double E, double gamma, double gm1,
                                                        double *mom)
{
    Prim<DIM> r;
    r.rho = q.rho;
    r.irho = q.irho;
    double vsq = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        mom[d] = q.v[d];
        r.v[d] = q.v[d] * q.irho;
        vsq += r.v[d] * r.v[d];
    }
    r.p = gm1 * (E - 0.5 * r.rho * vsq);
    r.beta = 0.5 * r.rho / r.p;
    r.ib = 2.0 * r.p * r.irho;
    r.lam = sqrt(vsq) + sqrt(gamma * r.p * r.irho);
    return r;
}

// One face node: the face between element a's +D face and its neighbour b's
// -D face, evaluated once with the element-1 rule (element 1 = the
// lower-numbered element, normal out of it).  Element a's contribution is
// C = scale * (-/+ F* [+/- Fv.n]); b's is -C.  Both are added (times the
// stage factor) to the output, which the volume kernel has already written.
// NS adds the central (BR1) viscous flux from the normal columns lift_kernel
// wrote, and in compat mode evaluates the inviscid flux with velocities in
// the momentum slots, as the reference does (its ComputeViscousFlux divides
// the face states' momenta in place before ComputeFaceFlux reads them,
// BasicOperations.cpp:33-34, DGSEMIntegrator.cpp:467-481).
// Inputs of one face node: both traces and (NS) both normal viscous columns.
template <int DIM, bool NS> struct FaceIn {
    double sa[DIM + 2], sb[DIM + 2];
    double fa[NS ? DIM + 1 : 1], fb[NS ? DIM + 1 : 1];
};

template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ void load_face_in(const KParams &P, int64_t a, int64_t b, int fn, FaceIn<DIM, NS> &in)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t nn = P.nnodes;
    const int na = line_node<DIM, Np, D>(fn, N), nb = line_node<DIM, Np, D>(fn, 0);
#pragma unroll
    for (int v = 0; v < NV; v++) {
        in.sa[v] = __ldg(P.u + v * nn + a * NDOF + na);
        in.sb[v] = __ldg(P.u + v * nn + b * NDOF + nb);
    }
    if (NS) {
#pragma unroll
        for (int i = 0; i <= DIM; i++) {
            in.fa[i] = __ldg(P.fcol + (((D * 2 + 1) * P.ne + a) * NFN + fn) * (NV - 1) + i);
            in.fb[i] = __ldg(P.fcol + (((D * 2 + 0) * P.ne + b) * NFN + fn) * (NV - 1) + i);
        }
    }
}

// Inviscid flux of one face node between element a's +D trace sa and its
// +D neighbour b's -D trace sb, signed as element a receives it: Fa = -F for
// a = element 1 (the lower index, normal out of it), +F otherwise, F being
// the Chandrashekar + LLF flux with the element-1 normal.  NSC: the
// reference-value Navier-Stokes face states, whose momentum slots hold
// velocities (returns their wave speed; 0 otherwise).
template <int DIM, int N, int D, bool NSC>
__device__ __forceinline__ double face_flux_oriented(const KParams &P, const double *c, bool a_is_1, const double *sa,
                                                     const double *sb, double *Fa)
{
    constexpr int NV = DIM + 2, Np = N + 1;  // Np: constant layout
    Prim<DIM> qa = make_prim<DIM>(sa, P.gamma, P.gm1), qb = make_prim<DIM>(sb, P.gamma, P.gm1);
    double ma[DIM], mb[DIM];
    double lam = 0.0;
    const bool compat = P.compat != 0;
    if (NSC && compat) {
        qa = velocity_slot_prim<DIM>(qa, sa[DIM + 1], P.gamma, P.gm1, ma);
        qb = velocity_slot_prim<DIM>(qb, sb[DIM + 1], P.gamma, P.gm1, mb);
        lam = fmax(qa.lam, qb.lam);
    } else {
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            ma[d] = sa[1 + d];
            mb[d] = sb[1 + d];
        }
    }
    const double nrm = a_is_1 ? C_AREA(c)[D] : -C_AREA(c)[D];
    double F[NV];
    if (a_is_1) face_flux<DIM, D>(qa, qb, ma, mb, nrm, P.gm1inv, compat, P.diss_scale, F);
    else face_flux<DIM, D>(qb, qa, mb, ma, nrm, P.gm1inv, compat, P.diss_scale, F);
#pragma unroll
    for (int v = 0; v < NV; v++) Fa[v] = a_is_1 ? -F[v] : F[v];
    return lam;
}

// Element a's face terms C (element b receives -C) from the signed inviscid
// flux Fa and, NS, both sides' normal viscous columns: C = C_FACE coef
// (Fa +/- (fa + fb)/2 n).
template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ void face_terms_signed(const double *c, bool a_is_1, const double *Fa, const double *fa,
                                                  const double *fb, double coef, double *C)
{
    constexpr int Np = N + 1;  // Np: constant layout
    const double nrm = a_is_1 ? C_AREA(c)[D] : -C_AREA(c)[D];
    const double sc = C_FACE(c) * coef;
    C[0] = sc * Fa[0];
#pragma unroll
    for (int i = 0; i <= DIM; i++) {
        double du = Fa[1 + i];
        if (NS) {
            const double fvn = ((fa[i] + fb[i]) * 0.5) * nrm;
            du = a_is_1 ? du + fvn : du - fvn;
        }
        C[1 + i] = sc * du;
    }
}

template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ double face_terms_from(const KParams &P, const double *c, bool a_is_1,
                                                  const FaceIn<DIM, NS> &in, double coef, double *C)
{
    constexpr int NV = DIM + 2;
    double Fa[NV];
    const double lam = face_flux_oriented<DIM, N, D, NS>(P, c, a_is_1, in.sa, in.sb, Fa);
    face_terms_signed<DIM, N, D, NS>(c, a_is_1, Fa, in.fa, in.fb, coef, C);
    return lam;
}

// Outer states of the subsonic conditions and the Riemann-invariant
// condition; s1 enters as the interior state and leaves as the face flux
// will see it (momenta divided in place for the reference-value operator).
// prm: 6 p; 7 rho, velocity; 8 (2D) cp, pt, Tt, cos theta, sin theta;
// 9 primitive outer state rho, velocity, p.  The normal is sgn e_D.
//   6  SubsonicOutflowPBdrFaceIntegrator.cpp:17-31: interior state with
//      E = p / (g-1) + rho |v|^2 / 2
//   7  SubsonicInflowRVBdrFaceIntegrator.cpp:20-50: (rho, rho V) with the
//      interior's E less its kinetic energy plus the outer one
//   8  SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:52-80: |V|^2 = 2 cp Tt
//      (1 - (p/pt)^((g-1)/g)) along the flow angle, rho from p and
//      cp Tt - |V|^2/2
//   9  RiemannInvariantBdrFaceIntegrator.cpp:43-112: boundary normal speed
//      and sound speed from the outgoing and incoming invariants
template <int DIM, int D>
__device__ __noinline__ void subsonic_outer_state(const KParams &P, int type, const double *prm, double sgn,
                                                  double *s1, double *s2)
{
    constexpr int NV = DIM + 2;
    const bool compat = P.compat != 0;
    const double gm1 = P.gm1, gm1inv = P.gm1inv, gamma = P.gamma;
    const double rho = s1[0], r1 = 1.0 / rho;
    double V[DIM], vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) V[d] = compat ? s1[1 + d] * r1 : s1[1 + d] / rho;
    if (type == BC_SUBSONIC_INFLOW_RV) {
        const double r = prm[0];
        s2[0] = r;
        double dke = -s1[1] * s1[1], uu = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            s2[1 + d] = r * prm[1 + d];
            if (d > 0) dke -= s1[1 + d] * s1[1 + d];
            uu += prm[1 + d] * prm[1 + d];
        }
        dke *= 0.5 / rho;
        dke += 0.5 * uu * r;
        s2[NV - 1] = s1[NV - 1] + dke;
        return;
    }
    if (type == BC_RIEMANN_INVARIANT) {
        const double ginv = 1.0 / gamma;
        const double rho_o = prm[0], p_o = prm[NV - 1];
        const double Vn_i = sgn * V[D], Vn_o = sgn * prm[1 + D];
        // ComputePressure(state1): once more through the view for compat
        double W[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            W[d] = compat ? V[d] * r1 : V[d];
            vv += W[d] * W[d];
        }
        const double p_i = gm1 * (s1[NV - 1] - 0.5 * rho * vv);
        if (compat) {
#pragma unroll
            for (int d = 0; d < DIM; d++) V[d] = s1[1 + d] = W[d];
        }
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
            const double nd = d == D ? sgn : 0.0;
            s2[1 + d] = (Vn_i >= 0.0) ? s2[0] * (V[d] + dVn_i * nd) : s2[0] * (prm[1 + d] + dVn_o * nd);
            e2 = d == 0 ? s2[1] * s2[1] : e2 + s2[1 + d] * s2[1 + d];
        }
        const double p_b = a_b * a_b * s2[0] * ginv;
        e2 *= (0.5 / s2[0]);
        e2 += p_b * gm1inv;
        s2[NV - 1] = e2;
        return;
    }
#pragma unroll
    for (int d = 0; d < DIM; d++) vv += V[d] * V[d];
    if (compat) {
#pragma unroll
        for (int d = 0; d < DIM; d++) s1[1 + d] = V[d];
    }
    if (type == BC_SUBSONIC_OUTFLOW_P) {
#pragma unroll
        for (int v = 0; v < NV; v++) s2[v] = s1[v];
        s2[NV - 1] = prm[0] * gm1inv + 0.5 * rho * vv;
        return;
    }
    // BC_SUBSONIC_INFLOW_PTTT
    const double cp = prm[0], p0 = prm[1], T0 = prm[2];
    const double p = gm1 * (s1[NV - 1] - 0.5 * rho * vv);
    double V_sq = 2.0 * cp * T0 * (1.0 - pow(p / p0, gm1 / gamma));
    V_sq = fmax(0.0, V_sq);
    s2[0] = gamma * gm1inv * p / (cp * T0 - 0.5 * V_sq);
#pragma unroll
    for (int d = 0; d < DIM; d++) s2[1 + d] = s2[0] * sqrt(V_sq) * prm[3 + d];
    s2[NV - 1] = p * gm1inv + 0.5 * s2[0] * V_sq;
}

// Boundary face node of an element with interior trace s on its +D (sgn = 1)
// or -D (sgn = -1) face, boundary condition b (BdrFaceIntegrator::
// AssembleFaceVector, src/Integrators/BoundaryConditions/BdrFaceIntegrator.cpp:
// 64-130): the outer state of the condition and the face flux with the
// outward normal sgn |n_D| e_D, or the slip wall's pressure flux; the element
// receives C = -F / (w0 J) times the stage factor.  Returns the wave speed the
// condition reports.  Outer states: supersonic inflow and specified state the
// prescribed state (SupersonicInflowBdrFaceIntegrator.cpp:22-35,
// SpecifiedStateBdrFaceIntegrator.cpp:21-35), supersonic outflow the interior
// state (SupersonicOutflowBdrFaceIntegrator.cpp:10-13), symmetry the interior
// state with its normal momentum reversed (SymmetryBdrFaceIntegrator.cpp:
// 12-37).  Slip wall (SlipWallBdrFaceIntegrator.cpp:15-58): with the normal
// velocity vn and pressure p of the interior state rotated to the face frame,
// p* = p + (g+1)/4 rho vn (vn + sqrt(vn^2 + 8 p / ((g+1) rho) ((g-1)/(g+1) +
// 1))) for vn > 0, else p max(1 + (g-1)/2 vn/c, 1e-4)^(2g/(g-1)), and the
// flux is p* n in the momentum rows only.  The rotation to the face frame
// lists the normal component first and the others in ascending order, so
// |v|^2 is summed in that order.
// Not inlined: a rare path that would otherwise raise the register demand
// of every face loop.
template <int DIM, int N, int D>
__device__ __noinline__ double boundary_node_terms(const KParams &P, const double *c, const double *s, int b,
                                                   double sgn, double coef, double *C)
{
    constexpr int NV = DIM + 2, Np = N + 1;  // Np: constant layout
    const double *bc = P.bc + b * BC_SLOT;
    const int type = (int)bc[0];
    const double nrm = sgn * C_AREA(c)[D];
    double F[NV];
    double lam;
    if (type == BC_SLIP_WALL || type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL) {  // no-slip walls derive from the slip wall
        const double rho = s[0];
        double vsq = 0.0;
        {
            const double vD = s[1 + D] / rho;
            vsq += vD * vD;
#pragma unroll
            for (int q = 0; q < DIM; q++)
                if (q != D) {
                    const double vq = s[1 + q] / rho;
                    vsq += vq * vq;
                }
        }
        const double p = P.gm1 * (s[DIM + 1] - 0.5 * rho * vsq);
        const double vn = (sgn * s[1 + D]) / rho;
        const double an = sqrt(P.gamma * p / rho);
        const double gp1 = 1.0 + P.gamma, gp1inv = 1.0 / gp1;
        double ps;
        if (vn > 0.0) {
            ps = p + 0.25 * vn * gp1 * rho * (vn + sqrt(vn * vn + 8.0 * gp1inv / rho * p * (P.gm1 * gp1inv + 1.0)));
        } else {
            ps = p * pow(fmax(1.0 + 0.5 * P.gm1 * vn / an, 0.0001), 2.0 * P.gamma * P.gm1inv);
        }
#pragma unroll
        for (int v = 0; v < NV; v++) F[v] = 0.0;
        F[1 + D] = ps * nrm;
        lam = sqrt(vsq) + an;
    } else {
        // s1: the interior state as the face flux sees it.  The reference's
        // subsonic conditions divide its momenta in place through Vector
        // views (ComputePressure, BasicOperations.cpp:31-37, and their own
        // velocity views); the reference-value operator keeps that.
        double s1[NV], s2[NV];
        const bool given = type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            s1[v] = s[v];
            s2[v] = given ? bc[1 + v] : s[v];
        }
        if (type == BC_SYMMETRY) s2[1 + D] = -s[1 + D];
        if (type >= BC_SUBSONIC_OUTFLOW_P && type <= BC_RIEMANN_INVARIANT)
            subsonic_outer_state<DIM, D>(P, type, bc + 1, sgn, s1, s2);
        const Prim<DIM> qa = make_prim<DIM>(s1, P.gamma, P.gm1), qb = make_prim<DIM>(s2, P.gamma, P.gm1);
        double ma[DIM], mb[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            ma[d] = s1[1 + d];
            mb[d] = s2[1 + d];
        }
        face_flux<DIM, D>(qa, qb, ma, mb, nrm, P.gm1inv, P.compat != 0, P.diss_scale, F);
        lam = fmax(qa.lam, qb.lam);
    }
    const double sc = C_FACE(c) * coef;
#pragma unroll
    for (int v = 0; v < NV; v++) C[v] = sc * (-F[v]);
    return lam;
}

template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ double face_node_terms(const KParams &P, const double *c, int64_t a, int64_t b, int fn,
                                                  double coef, double *C)
{
    FaceIn<DIM, NS> in;
    load_face_in<DIM, N, D, NS>(P, a, b, fn, in);
    return face_terms_from<DIM, N, D, NS>(P, c, a <= b, in, coef, C);
}

template <int DIM, int N, int D, bool NS>
__device__ __forceinline__ double face_node(const KParams &P, const double *c, int64_t a, int64_t b, int fn,
                                            double coef)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const int64_t nn = P.nnodes;
    const int na = line_node<DIM, Np, D>(fn, N), nb = line_node<DIM, Np, D>(fn, 0);
    // the output values are loaded before the flux arithmetic, so that their
    // latency overlaps it
    double oa[NV], ob[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        oa[v] = P.out[v * nn + a * NDOF + na];
        ob[v] = P.out[v * nn + b * NDOF + nb];
    }
    double C[NV];
    const double lam = face_node_terms<DIM, N, D, NS>(P, c, a, b, fn, coef, C);
#pragma unroll
    for (int v = 0; v < NV; v++) {
        P.out[v * nn + a * NDOF + na] = oa[v] + C[v];
        P.out[v * nn + b * NDOF + nb] = ob[v] - C[v];
    }
    return lam;
}


// Boundary face node fn of element a's +D (side 1) or -D (side 0) face:
// read-modify-write of a's output node.  NS adds the viscous boundary flux
// from a's own face column (outflow, no-slip walls; none for prescribed
// states), as the element-side path does.
template <int DIM, int N, int D, bool NS = false>
__device__ __forceinline__ double boundary_node(const KParams &P, const double *c, int64_t a, int fn, int side, int b,
                                                double coef)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const int64_t nn = P.nnodes;
    const int n = line_node<DIM, Np, D>(fn, side ? N : 0);
    double s[NV], o[NV], C[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        s[v] = __ldg(P.u + v * nn + a * NDOF + n);
        o[v] = P.out[v * nn + a * NDOF + n];
    }
    const double lam = boundary_node_terms<DIM, N, D>(P, c, s, b, side ? 1.0 : -1.0, coef, C);
#pragma unroll
    for (int v = 0; v < NV; v++) o[v] = o[v] + C[v];
    if (NS) {
        const double *bc = P.bc + b * BC_SLOT;
        const int type = (int)bc[0];
        if (type == BC_SUPERSONIC_OUTFLOW || type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL ||
            type == BC_SUBSONIC_INFLOW_PTTT) {
            const double nrm = side ? C_AREA(c)[D] : -C_AREA(c)[D];
            const double *fo = P.fcol + (((D * 2 + side) * P.ne + a) * S::NFN + fn) * (NV - 1);
            double fv[DIM + 1];
#pragma unroll
            for (int i = 0; i <= DIM; i++) fv[i] = __ldg(fo + i) * nrm;
            if (type == BC_NOSLIP_ADIABATIC) {
                double en = 0.0;
#pragma unroll
                for (int q = 0; q < DIM; q++) en += bc[1 + q] * fv[q];
                fv[DIM] = en + 0.0;
            }
            const double sb = C_FACE(c) * coef;
#pragma unroll
            for (int i = 0; i <= DIM; i++) o[1 + i] += sb * fv[i];
        }
    }
#pragma unroll
    for (int v = 0; v < NV; v++) P.out[v * nn + a * NDOF + n] = o[v];
    return lam;
}

// Face kernel of direction D: one thread per (element, face node).  Within one
// direction every output entry belongs to exactly one face, so the
// read-modify-write updates need no atomics.  Boundary faces are left to
// boundary_kernel.
template <int DIM, int N, int D, bool NS>
__global__ void __launch_bounds__(256, 3) face_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, S::Np);
    __syncthreads();
    const double coef = stage_coef(P);
    double lam = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < P.ne * NFN;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = t / NFN;
        const int fn = (int)(t - a * NFN);
        const int64_t b = __ldg(P.nbr + a * 2 * DIM + 2 * D + 1);
        if (b >= 0) lam = fmax(lam, face_node<DIM, N, D, NS>(P, c, a, b, fn, coef));  // else: boundary_kernel
    }
    lam = group_max<32>(lam);
    if ((threadIdx.x & 31) == 0) atomic_max_pos(P.lam_bits, lam);
}

// Boundary faces for the separate-face path (Euler): one thread per element
// walks its boundary faces one after another, so an edge or corner node on
// two boundary faces is updated by one thread; threads of interior elements
// return at once.  Launched after the face kernels, so its
// read-modify-writes do not overlap theirs.
template <int DIM, int N, bool NS = false>
__global__ void __launch_bounds__(256) boundary_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, S::Np);
    __syncthreads();
    const double coef = stage_coef(P);
    double lam = 0.0;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < P.ne; a += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll 1
        for (int f = 0; f < 2 * DIM; f++) {
            const int32_t nb = __ldg(P.nbr + a * 2 * DIM + f);
            if (nb >= 0) continue;
            const int d = f >> 1, side = f & 1;
#pragma unroll 1
            for (int fn = 0; fn < NFN; fn++) {
                if (d == 0) lam = fmax(lam, boundary_node<DIM, N, 0, NS>(P, c, a, fn, side, -1 - nb, coef));
                else if (d == 1) lam = fmax(lam, boundary_node<DIM, N, 1, NS>(P, c, a, fn, side, -1 - nb, coef));
                else lam = fmax(lam, boundary_node<DIM, N, (DIM == 3 ? 2 : 0), NS>(P, c, a, fn, side, -1 - nb, coef));
            }
        }
    }
    lam = group_max<32>(lam);
    if ((threadIdx.x & 31) == 0) atomic_max_pos(P.lam_bits, lam);
}

// Face-node kernel modes: the BR1 jump (lift_face_node) and/or the signed
// inviscid face flux to P.fbuf (the fixed operator's element-side faces then
// read it instead of evaluating each face from both sides).
constexpr int FACE_JUMP = 1, FACE_FLUX = 2;

// BR1 lifting face node: 0.5 (w2 - w1) n1_D / (w0 J), the same value for both
// sides (LiftingBR1.cpp:10-115).  Written to P.lbuf for the -D-side element a.
// MODE & FACE_FLUX: also the inviscid flux of the face node, signed for a
// (face_flux_oriented), to P.fbuf[D][a][v][fn].
template <int DIM, int N, int D, int MODE = FACE_JUMP>
__device__ __forceinline__ void lift_face_node(const KParams &P, const double *c, int64_t a, int fn)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t nn = P.nnodes;
    const int64_t b = __ldg(P.nbr + a * 2 * DIM + 2 * D + 1);
    const int na = line_node<DIM, Np, D>(fn, N), nb = line_node<DIM, Np, D>(fn, 0);
    double sa[NV], sb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        sa[v] = __ldg(P.u + v * nn + a * NDOF + na);
        sb[v] = __ldg(P.u + v * nn + b * NDOF + nb);
    }
    const bool a_is_1 = a <= b;
    if (MODE & FACE_JUMP) {
        double wa[NV], wb[NV];
        entropy_vars<DIM>(sa, P.gamma, P.gm1, P.gm1inv, wa);
        entropy_vars<DIM>(sb, P.gamma, P.gm1, P.gm1inv, wb);
        const double nrm = a_is_1 ? C_AREA(c)[D] : -C_AREA(c)[D];
        const double sc = C_FACE(c);
        double *dst = P.lbuf + ((D * P.ne + a) * NFN + fn) * NV;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const double w1 = a_is_1 ? wa[v] : wb[v], w2 = a_is_1 ? wb[v] : wa[v];
            dst[v] = sc * ((0.5 * (w2 - w1)) * nrm);
        }
    }
    if (MODE & FACE_FLUX) {
        double Fa[NV];
        face_flux_oriented<DIM, N, D, false>(P, c, a_is_1, sa, sb, Fa);
        double *dst = P.fbuf + ((D * P.ne + a) * NV) * NFN + fn;
#pragma unroll
        for (int v = 0; v < NV; v++) dst[v * NFN] = Fa[v];
    }
}

// BR1 jump of a boundary face node (LiftingBR1::AssembleLiftingBdrFaceVector,
// LiftingBR1.cpp:311-345, with ComputeBdrFaceLiftingFlux): the element is
// element 1 and the normal points out of it; 0.5 (w(s2) - w1) for the
// prescribed states and the outer states of the subsonic conditions and the
// Riemann invariants (BdrFaceIntegrator.cpp:275-282), 0 for the outflow,
// (w1_0, beta V, -beta) - w1 for the no-slip wall
// (NoSlipAdiabWallBdrFaceIntegrator.cpp:74-95); the reference-value operator
// keeps the reference's in-place division (below).
template <int DIM, int N, int D>
__device__ __noinline__ void lift_boundary_node(const KParams &P, const double *c, int64_t a, int fn, int side, int b,
                                                double *dst)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const int64_t nn = P.nnodes;
    const int n = line_node<DIM, Np, D>(fn, side ? N : 0);
    double s[NV], w1[NV], f[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) s[v] = __ldg(P.u + v * nn + a * NDOF + n);
    entropy_vars<DIM>(s, P.gamma, P.gm1, P.gm1inv, w1);
    const double *bc = P.bc + b * BC_SLOT;
    const int type = (int)bc[0];
    if (type == BC_NOSLIP_ADIABATIC || type == BC_NOSLIP_ISOTHERMAL) {
        // the isothermal wall (NoSlipIsothWallBdrFaceIntegrator.cpp:41-65)
        // takes 1/(R T_wall), stored after the wall velocity, for beta
        const double beta = type == BC_NOSLIP_ADIABATIC ? -w1[NV - 1] : bc[1 + DIM];
        f[0] = w1[0] - w1[0];
#pragma unroll
        for (int q = 0; q < DIM; q++) f[1 + q] = bc[1 + q] * beta - w1[1 + q];
        f[NV - 1] = -beta - w1[NV - 1];
    } else if (P.compat) {
        // the reference reaches the outer state through Entropy2Conserv(w1)
        // (BasicOperations.cpp:106-124), whose velocity view divides w1's
        // momentum entries by beta in place before they are subtracted
        const double beta = -w1[NV - 1], ib = 1.0 / beta;
        double vv = 0.0;
#pragma unroll
        for (int q = 0; q < DIM; q++) {
            w1[1 + q] *= ib;
            vv += w1[1 + q] * w1[1 + q];
        }
        double s2[NV], w2[NV];
        if (type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE) {
#pragma unroll
            for (int v = 0; v < NV; v++) s2[v] = bc[1 + v];
        } else {
            const double sent = P.gamma - (w1[0] + 0.5 * beta * vv) * P.gm1;
            s2[0] = pow(exp(-sent) / beta, P.gm1inv);
#pragma unroll
            for (int q = 0; q < DIM; q++) s2[1 + q] = s2[0] * w1[1 + q];
            s2[NV - 1] = s2[0] * (1.0 / beta * P.gm1inv + 0.5 * vv);
            if (type == BC_SUBSONIC_OUTFLOW_P || type == BC_SUBSONIC_INFLOW_RV || type == BC_SUBSONIC_INFLOW_PTTT) {
                // ComputeOuterInviscidState of that state (BdrFaceIntegrator.cpp:278)
                double so[NV];
                subsonic_outer_state<DIM, D>(P, type, bc + 1, side ? 1.0 : -1.0, s2, so);
#pragma unroll
                for (int v = 0; v < NV; v++) s2[v] = so[v];
            }
        }
        entropy_vars<DIM>(s2, P.gamma, P.gm1, P.gm1inv, w2);
#pragma unroll
        for (int v = 0; v < NV; v++) f[v] = (w2[v] - w1[v]) * 0.5;
    } else if (type == BC_SUPERSONIC_INFLOW || type == BC_SPECIFIED_STATE) {
        double w2[NV];
        entropy_vars<DIM>(bc + 1, P.gamma, P.gm1, P.gm1inv, w2);
#pragma unroll
        for (int v = 0; v < NV; v++) f[v] = (w2[v] - w1[v]) * 0.5;
    } else if (type == BC_SUBSONIC_OUTFLOW_P || type == BC_SUBSONIC_INFLOW_RV || type == BC_RIEMANN_INVARIANT ||
               type == BC_SUBSONIC_INFLOW_PTTT) {
        // the outer state of the inviscid flux (BdrFaceIntegrator.cpp:275-282)
        double so[NV], w2[NV];
        subsonic_outer_state<DIM, D>(P, type, bc + 1, side ? 1.0 : -1.0, s, so);
        entropy_vars<DIM>(so, P.gamma, P.gm1, P.gm1inv, w2);
#pragma unroll
        for (int v = 0; v < NV; v++) f[v] = (w2[v] - w1[v]) * 0.5;
    } else {
#pragma unroll
        for (int v = 0; v < NV; v++) f[v] = 0.0;
    }
    const double nrm = side ? C_AREA(c)[D] : -C_AREA(c)[D];
#pragma unroll
    for (int v = 0; v < NV; v++) dst[v] = C_FACE(c) * (f[v] * nrm);
}

// BDR: the mesh has boundary faces (Navier-Stokes): a face towards the
// boundary takes its jump from lift_boundary_node, the -D boundary faces into
// P.lbuf_lo.  MODE: FACE_JUMP (the jumps), FACE_FLUX (the inviscid face
// fluxes, periodic meshes) or both.
#ifndef PDG_FACE_NODE_MIN_BLOCKS
#define PDG_FACE_NODE_MIN_BLOCKS 1
#endif
template <int DIM, int N, bool BDR = false, int MODE = FACE_JUMP>
__global__ void __launch_bounds__(256, (MODE & FACE_FLUX) ? PDG_FACE_NODE_MIN_BLOCKS : 1) lift_face_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, S::Np);
    __syncthreads();
    // chunks of CH elements, direction-major inside a chunk: a warp works on
    // one direction of consecutive elements, and a chunk's traces are still
    // in L2 for its later directions (direction-major order over the whole
    // mesh read the state from DRAM about twice per launch)
    constexpr int CH = 64, PER_CH = DIM * CH * NFN;
    const int64_t e_end = range_end(P);
    const int64_t nch = (e_end - P.e_begin + CH - 1) / CH;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nch * PER_CH;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ch = t / PER_CH;
        const int r = (int)(t - ch * PER_CH);
        const int d = r / (CH * NFN);
        const int r2 = r - d * (CH * NFN);
        const int64_t a = P.e_begin + ch * CH + r2 / NFN;
        const int fn = r2 % NFN;
        if (a >= e_end) continue;
        if (BDR) {
            const int32_t bp = __ldg(P.nbr + a * 2 * DIM + 2 * d + 1), bm = __ldg(P.nbr + a * 2 * DIM + 2 * d);
            double *dp = P.lbuf + ((d * P.ne + a) * NFN + fn) * (DIM + 2);
            double *dm = P.lbuf_lo + ((d * P.ne + a) * NFN + fn) * (DIM + 2);
            if (bp < 0) {
                if (d == 0) lift_boundary_node<DIM, N, 0>(P, c, a, fn, 1, -1 - bp, dp);
                else if (d == 1) lift_boundary_node<DIM, N, 1>(P, c, a, fn, 1, -1 - bp, dp);
                else lift_boundary_node<DIM, N, (DIM == 3 ? 2 : 0)>(P, c, a, fn, 1, -1 - bp, dp);
            }
            if (bm < 0) {
                if (d == 0) lift_boundary_node<DIM, N, 0>(P, c, a, fn, 0, -1 - bm, dm);
                else if (d == 1) lift_boundary_node<DIM, N, 1>(P, c, a, fn, 0, -1 - bm, dm);
                else lift_boundary_node<DIM, N, (DIM == 3 ? 2 : 0)>(P, c, a, fn, 0, -1 - bm, dm);
            }
            if (bp < 0) continue;
        }
        if (d == 0) lift_face_node<DIM, N, 0, MODE>(P, c, a, fn);
        else if (d == 1) lift_face_node<DIM, N, 1, MODE>(P, c, a, fn);
        else lift_face_node<DIM, N, (DIM == 3 ? 2 : 0), MODE>(P, c, a, fn);
    }
}

// Strong-form entropy-variable gradient along D by line tasks:
// g_D[v][n] = (sum_l D(pos,l) w_l) adj_D / J.
template <int DIM, int N, int D>
__device__ __forceinline__ void grad_lines(const double *wv, double *g, const double *c, int gl)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    const double *Dm = C_D(c);
    const double sc = C_ADJ(c)[D], invJ = C_INVJ(c);
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
#pragma unroll
            for (int v = 0; v < NV; v++) {
                double x[Np];
#pragma unroll
                for (int l = 0; l < Np; l++) x[l] = wv[v * ST + sp<DIM, Np>(line_node<DIM, Np, D>(line, l))];
#pragma unroll
                for (int p = 0; p < Np; p++) {
                    double a = 0.0;
#pragma unroll
                    for (int l = 0; l < Np; l++) a += Dm[p * Np + l] * x[l];
                    g[(D * NV + v) * ST + sp<DIM, Np>(line_node<DIM, Np, D>(line, p))] = (a * sc) * invJ;
                }
            }
        }
    }
}

// Viscous volume divergence along D by line tasks: node p of the line gets
// (1/J) sum_l Dhat(p, l) Fv_D[l] (momentum and energy rows), Fv_D being the
// contravariant fluxes stored in the gradient slots (slot D*(NV-1)+i).
template <int DIM, int N, int D, bool FIRST>
__device__ __forceinline__ void divergence_lines(const double *fvs, double *dv, const double *c, int gl)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NV = S::NV, ST = S::NS_;
    const double *Dh = C_DHAT(c);
    const double invJ = C_INVJ(c);
#pragma unroll
    for (int r = 0; r < S::LPL; r++) {
        const int line = gl + r * S::L;
        if (line < S::NFN) {
#pragma unroll
            for (int i = 0; i < NV - 1; i++) {
                double x[Np];
#pragma unroll
                for (int l = 0; l < Np; l++) x[l] = fvs[(D * (NV - 1) + i) * ST + sp<DIM, Np>(line_node<DIM, Np, D>(line, l))];
#pragma unroll
                for (int p = 0; p < Np; p++) {
                    double a = 0.0;
#pragma unroll
                    for (int l = 0; l < Np; l++) a += Dh[p * Np + l] * x[l];
                    const int m = i * ST + sp<DIM, Np>(line_node<DIM, Np, D>(line, p));
                    if (FIRST) dv[m] = invJ * a;
                    else dv[m] += invJ * a;
                }
            }
        }
    }
    __syncwarp();
}

// BR1 lifting element kernel: entropy variables, strong-form gradients, face
// jumps from lbuf, conversion to primitive gradients, then the viscous fluxes:
// contravariant volume fluxes at every node (with the state of the element's
// last node in compat mode, as the reference's member id1 gives,
// DGSEMIntegrator.cpp:620, :770), their divergence (the viscous volume term:
// added to the output the volume kernel wrote, times the stage factor, or
// stored to P.vbuf when the volume kernel with element-side faces runs after
// this one) and the normal column at every face node (with the node's own
// state, DGSEMIntegrator.cpp:467-477, written to P.fcol).
// Viscous column of the total-pressure inflow's outer state with the
// interior's primitive gradients dq[d * NV + v]
// (SubsonicInflowPtTtAngBdrFaceIntegrator.cpp:88-92), stored in place of the
// element's own column at that boundary face node.
template <int DIM, int D>
__device__ __noinline__ void outer_viscous_col(const KParams &P, const double *s, int b, double sgn,
                                               const double *dq, double *col)
{
    constexpr int NV = DIM + 2;
    double s1[NV], so[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) s1[v] = s[v];
    subsonic_outer_state<DIM, D>(P, BC_SUBSONIC_INFLOW_PTTT, P.bc + b * BC_SLOT + 1, sgn, s1, so);
    const NodeState<DIM> ns = node_state<DIM>(so, P.gm1);
    Prim<DIM> q;
    q.rho = ns.rho;
    q.irho = ns.irho;
#pragma unroll
    for (int d = 0; d < DIM; d++) q.v[d] = ns.vel[d];
    q.p = ns.p;
    q.beta = q.ib = q.lam = 0.0;
    auto G = [&](int d, int v) { return dq[d * NV + v]; };
    viscous_col<DIM>(q, G, D, P.gm1inv, P.mu, P.lambda_k, col);
}

// BDR: jumps of -d boundary faces come from P.lbuf_lo (Navier-Stokes meshes
// with boundary faces).  PTTT (2D, a mesh with a total-pressure inflow): the
// face columns of those boundary faces come from outer_viscous_col; a
// separate instantiation, since the out-of-line call gives the kernel a stack
// frame that slowed the other boundary meshes by ~8 %.
template <int DIM, int N, bool BDR = false, bool PTTT = false>
__global__ void __launch_bounds__(128, LiftOccupancy<DIM, N>::min_blocks) lift_kernel(const KParams P)
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
    const bool lane_used = grp < EPW;
    double *wv = smem + const_slots(Np) + (size_t)(warp * EPW + (lane_used ? grp : 0)) * S::EL_LIFTF;
    double *g = wv + NV * ST;
    const int64_t nn = P.nnodes;
    const bool compat = P.compat != 0;
    const int64_t wstride = (int64_t)gridDim.x * wpb;
    unsigned int flags = 0;
    const int64_t e_end = range_end(P);
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += wstride) {
        const int64_t e0 = P.e_begin + wt * EPW + grp;
        const bool valid = lane_used && e0 < e_end;
        const int64_t e = valid ? e0 : 0;
        {
            const int64_t en = P.e_begin + (wt + wstride) * EPW + grp;
            if (P.prefetch && lane_used && en < e_end && gl < NV) prefetch_l2(P.u + (int64_t)gl * nn + en * NDOF, sizeof(double) * NDOF);
        }
        if (lane_used) {
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
        }
        __syncwarp();
        if (lane_used) {
            // state of the element's last node (compat volume viscous flux)
            double sl[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) sl[v] = valid ? __ldg(P.u + v * nn + e * NDOF + NDOF - 1) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
            const Prim<DIM> ql = make_prim<DIM>(sl, P.gamma, P.gm1);
            // the -d neighbours (owners of the -d faces' jumps)
            int64_t enb[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) enb[d] = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + 2 * d) : 0;
            // the next node's state is loaded one node ahead
            double snext[NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                snext[v] = (valid && gl < NDOF) ? __ldg(P.u + v * nn + e * NDOF + gl) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
#pragma unroll 1
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n >= NDOF) break;
                const int m = sp<DIM, Np>(n);
                double s[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) s[v] = snext[v];
                const int nn2 = n + L;
#pragma unroll
                for (int v = 0; v < NV; v++)
                    if (valid && k + 1 < S::NPL && nn2 < NDOF) snext[v] = __ldg(P.u + v * nn + e * NDOF + nn2);
                const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
                double dq[DIM][NV];
                const double *Dm = C_D(c);
                const NodeState<DIM> ns = node_state<DIM>(s, P.gm1);
                // BR1 face jumps of the node's faces, loaded before the
                // gradient arithmetic so that their latency overlaps it
                double jf[DIM][NV];
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    const int pos = idx[d];
                    const bool face = valid && (pos == 0 || pos == N);
                    const int line = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                            : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
                    const int64_t owner = pos == N ? e : enb[d];
                    const double *F = (BDR && owner < 0) ? P.lbuf_lo + ((d * P.ne + e) * NFN + line) * NV
                                                         : P.lbuf + ((d * P.ne + owner) * NFN + line) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++) jf[d][v] = face ? __ldg(F + v) : 0.0;
                }
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    // strong-form gradient along d at this node:
                    // (sum_l D(pos, l) w_l) adj_d / J along the node's d line
                    const int pos = idx[d];
                    const int gline = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                             : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        double a = 0.0;
#pragma unroll
                        for (int l = 0; l < Np; l++)
                            a += Dm[pos * Np + l] * wv[v * ST + sp<DIM, Np>(line_node_rt<DIM, Np>(d, gline, l))];
                        dq[d][v] = (a * C_ADJ(c)[d]) * C_INVJ(c);
                    }
                    if (valid && (pos == 0 || pos == N)) {
#pragma unroll
                        for (int v = 0; v < NV; v++) dq[d][v] += jf[d][v];
                    }
                    entgrad_to_primgrad_q<DIM>(ns, s, P.gm1inv, compat, dq[d]);
                    if (valid) {
#pragma unroll
                        for (int v = 0; v < NV; v++) {
                            if (!isfinite(dq[d][v])) flags |= PDG_FLAG_NONFINITE_DEV;
                            if (P.grads_out) P.grads_out[(int64_t)d * NV * nn + v * nn + e * NDOF + n] = dq[d][v];
                        }
                    }
                }
                auto GQ = [&](int d, int v) { return dq[d][v]; };
                // the viscous flux reads v, p and 1/rho only
                Prim<DIM> qn;
                qn.rho = ns.rho;
                qn.irho = ns.irho;
#pragma unroll
                for (int d = 0; d < DIM; d++) qn.v[d] = ns.vel[d];
                qn.p = ns.p;
                qn.beta = qn.ib = qn.lam = 0.0;
                const Prim<DIM> &qv = compat ? ql : qn;
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    double col[DIM + 1];
                    viscous_col<DIM>(qv, GQ, d, P.gm1inv, P.mu, P.lambda_k, col);
                    const double a = C_ADJ(c)[d];
                    // contravariant flux into the (now consumed) gradient slots of node n
#pragma unroll
                    for (int i = 0; i <= DIM; i++) g[(d * (NV - 1) + i) * ST + m] = a * col[i];
                    const int pos = idx[d];
                    if (valid && (pos == 0 || pos == N)) {
                        if (compat) viscous_col<DIM>(qn, GQ, d, P.gm1inv, P.mu, P.lambda_k, col);
                        if constexpr (BDR && PTTT && DIM == 2) {
                            const int64_t nbf = pos == N ? (int64_t)__ldg(P.nbr + e * 2 * DIM + 2 * d + 1) : enb[d];
                            if (nbf < 0 && (int)P.bc[(-1 - nbf) * BC_SLOT] == BC_SUBSONIC_INFLOW_PTTT) {
                                // a copy, so that dq itself stays in registers
                                double dqc[DIM * NV];
#pragma unroll
                                for (int q = 0; q < DIM; q++)
#pragma unroll
                                    for (int v = 0; v < NV; v++) dqc[q * NV + v] = dq[q][v];
                                const double sgn = pos == N ? 1.0 : -1.0;
                                if (d == 0) outer_viscous_col<DIM, 0>(P, s, (int)(-1 - nbf), sgn, dqc, col);
                                else outer_viscous_col<DIM, (DIM > 1 ? 1 : 0)>(P, s, (int)(-1 - nbf), sgn, dqc, col);
                            }
                        }
                        const int line = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                                : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
                        const int side = pos == N ? 1 : 0;
                        double *dst = P.fcol + (((d * 2 + side) * P.ne + e) * NFN + line) * (NV - 1);
#pragma unroll
                        for (int i = 0; i <= DIM; i++) dst[i] = col[i];
                    }
                }
            }
        }
        __syncwarp();
        // the output values the divergence is added to, loaded before the
        // divergence line tasks (none when it goes to vbuf)
        const bool add_out = valid && P.out && !P.vbuf;
        double oprev[S::NPL][NV - 1];
#pragma unroll
        for (int k = 0; k < S::NPL; k++) {
            const int n = gl + k * L;
#pragma unroll
            for (int i = 0; i < NV - 1; i++)
                oprev[k][i] = (add_out && n < NDOF) ? P.out[(int64_t)(1 + i) * nn + e * NDOF + n] : 0.0;
        }
        if (lane_used) {
            divergence_lines<DIM, N, 0, true>(g, wv, c, gl);
            divergence_lines<DIM, N, 1, false>(g, wv, c, gl);
            if (DIM == 3) divergence_lines<DIM, N, (DIM == 3 ? 2 : 0), false>(g, wv, c, gl);
        } else {
            __syncwarp();
            __syncwarp();
            if (DIM == 3) __syncwarp();
        }
        if (valid && P.vbuf) {
            // element-side faces: the right-hand side kernel adds it
#pragma unroll
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
#pragma unroll
                    for (int i = 0; i < NV - 1; i++) P.vbuf[(int64_t)i * nn + e * NDOF + n] = wv[i * ST + sp<DIM, Np>(n)];
                }
            }
        } else if (add_out) {
            const double coef = stage_coef(P);
#pragma unroll
            for (int k = 0; k < S::NPL; k++) {
                const int n = gl + k * L;
                if (n < NDOF) {
#pragma unroll
                    for (int i = 0; i < NV - 1; i++)
                        P.out[(int64_t)(1 + i) * nn + e * NDOF + n] = oprev[k][i] + coef * wv[i * ST + sp<DIM, Np>(n)];
                }
            }
        }
        __syncwarp();
    }
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

}  // namespace pdg
