// dgsem_kernels.cuh — sm_100a FP64 kernels of the DGSEM right-hand side.
//
// Work decomposition: one group of G lanes (G = 16 or 32, a half or a full
// warp) owns one element at a time; groups never synchronise beyond their
// warp (__syncwarp), so a CTA is just a bag of independent warps and the
// grid is persistent over "warp tiles" of 32/G consecutive elements.  The
// element's conservative state and per-node primitives are staged in shared
// memory with coalesced loads (consecutive lanes read consecutive nodes of
// one variable; consecutive elements are contiguous in the byNODES layout).
// Each lane accumulates the right-hand side of the nodes it owns (n = lane,
// lane + G, ...) in registers; fluxes shared by several nodes (two-point
// volume pairs, subcell interfaces, element faces) are computed once per
// element into a shared buffer and then gathered by the owners.  Directions
// are template parameters so line and pair index arithmetic folds at compile
// time.
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
    double w[6];        // GLL weights on [0,1]
    double snor[3][7];  // subcell interface normals per direction
    double fv_scale[6]; // 1 / (J w_i)
    double J, invJ, face_scale;
    double adj[3], area[3];
};

// Kernel parameters shared by all element kernels.
struct KParams {
    const double *u;      // stage input (us)
    const double *un;     // RK base state (stages 1, 2)
    double *out;          // dudt (plain) or next stage state
    const double *grads;  // NS: primitive gradients [d][v][node]
    double *grads_out;    // NS lifting output
    double *fbuf;         // NS face contributions [d][e][face node][v] of the element on the -d side
    const int32_t *nbr;   // [ne][2*dim]
    const DevConst *K;
    double *eta_out, *alpha_out;
    unsigned long long *lam_bits;  // running max wave speed (as ordered bits)
    unsigned int *err;
    int64_t ne, nnodes;
    int64_t nwt;          // number of warp tiles
    int stage;            // -1: plain RHS; 0, 1, 2: SSP-RK3 stage
    double dt;
    double gamma, gm1, gm1inv;
    double mu, lambda_k;  // NS: mu and mu*gamma/Pr
    double alpha_max, alpha_min, modal_threshold;
    double diss_scale;
    int blending, compat;
};

template <int DIM, int N> struct Shape {
    static constexpr int Np = N + 1;
    static constexpr int NDOF = DIM == 2 ? Np * Np : Np * Np * Np;
    static constexpr int NV = DIM + 2;
    static constexpr int NFN = DIM == 2 ? Np : Np * Np;     // face nodes = lines per direction
    static constexpr int NPAIR = Np * (Np - 1) / 2;
    static constexpr int G = (DIM == 2 && NDOF <= 16) ? 16 : 32;
    static constexpr int EPW = 32 / G;                      // elements per warp
    static constexpr int NPL = (NDOF + G - 1) / G;          // owned nodes per lane
    static constexpr int NPRIM = DIM + 6;                   // rho, 1/rho, v[DIM], p, beta, 1/beta, speed
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int BUF_PAIR = NFN * NPAIR * NV;
    static constexpr int BUF_FACE = 2 * DIM * NFN * NV;
    static constexpr int BUF_FV = NFN * N * NV;
    static constexpr int BUF_MODAL = 2 * NDOF;
    static constexpr int BUF = cmax(cmax(BUF_PAIR, BUF_FACE), cmax(BUF_FV, BUF_MODAL));
    static constexpr int BUF_NS = cmax(BUF, DIM * (NV - 1) * NDOF);  // + contravariant viscous fluxes
    static constexpr int EL_EULER = NV * NDOF + NPRIM * NDOF + BUF;
    static constexpr int EL_NS = NV * NDOF + NPRIM * NDOF + BUF_NS;
    static constexpr int EL_LIFT = NV * NDOF + NV * NDOF + DIM * NV * NDOF + BUF_FACE;
};

// primitive slots in shared memory (each NDOF long)
enum { P_RHO = 0, P_IRHO = 1, P_V = 2 };
template <int DIM> struct PSlot {
    static constexpr int P = P_V + DIM, BETA = P_V + DIM + 1, IB = P_V + DIM + 2, LAM = P_V + DIM + 3;
};

// Node index of position `pos` on line `line` of direction D (x fastest).
template <int DIM, int Np, int D> __device__ __forceinline__ int line_node(int line, int pos)
{
    if (DIM == 2) return D == 0 ? line * Np + pos : pos * Np + line;
    if (D == 0) return line * Np + pos;
    if (D == 1) return (line / Np) * Np * Np + pos * Np + (line % Np);
    return pos * Np * Np + line;
}
// Position and line of node n along direction D.
template <int DIM, int Np, int D> __device__ __forceinline__ void node_pos(int n, int &pos, int &line)
{
    const int i = n % Np, j = (n / Np) % Np, k = n / (Np * Np);
    if (D == 0) { pos = i; line = DIM == 2 ? j : j + Np * k; }
    else if (D == 1) { pos = j; line = DIM == 2 ? i : i + Np * k; }
    else { pos = k; line = i + Np * j; }
}
template <int Np> __device__ __forceinline__ int pair_index(int a, int b)
{
    return a * Np - a * (a + 1) / 2 + (b - a - 1);
}
template <int Np> __device__ __forceinline__ void pair_decode(int p, int &a, int &b)
{
    int aa = 0, rem = p;
#pragma unroll
    for (int q = 0; q < Np - 1; q++)
        if (rem >= Np - 1 - aa) { rem -= Np - 1 - aa; aa++; }
    a = aa;
    b = aa + 1 + rem;
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
#define C_D(c) (c)
#define C_DHAT(c) ((c) + 36)
#define C_DHAT2(c) ((c) + 72)
#define C_VINV(c) ((c) + 108)
#define C_W(c) ((c) + 144)
#define C_SNOR(c, d) ((c) + 150 + 7 * (d))
#define C_FVS(c) ((c) + 171)
#define C_ADJ(c) ((c) + 177)
#define C_AREA(c) ((c) + 180)
#define C_J(c) ((c)[183])
#define C_INVJ(c) ((c)[184])
#define C_FACE(c) ((c)[185])
constexpr int CONST_SLOTS = 192;

__device__ __forceinline__ void load_consts(const DevConst *K, double *c, int Np)
{
    for (int t = threadIdx.x; t < Np * Np; t += blockDim.x) {
        c[t] = K->D[t];
        c[36 + t] = K->Dhat[t];
        c[72 + t] = K->Dhat2[t];
        c[108 + t] = K->Vinv1[t];
    }
    for (int t = threadIdx.x; t < Np; t += blockDim.x) {
        c[144 + t] = K->w[t];
        c[171 + t] = K->fv_scale[t];
    }
    for (int t = threadIdx.x; t < 3 * 7; t += blockDim.x) c[150 + t] = (&K->snor[0][0])[t];
    if (threadIdx.x < 3) {
        c[177 + threadIdx.x] = K->adj[threadIdx.x];
        c[180 + threadIdx.x] = K->area[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        c[183] = K->J;
        c[184] = K->invJ;
        c[185] = K->face_scale;
    }
}

template <int DIM> __device__ __forceinline__ Prim<DIM> load_prim(const double *pr, int n, int NDOF)
{
    using PS = PSlot<DIM>;
    Prim<DIM> q;
    q.rho = pr[P_RHO * NDOF + n];
    q.irho = pr[P_IRHO * NDOF + n];
#pragma unroll
    for (int d = 0; d < DIM; d++) q.v[d] = pr[(P_V + d) * NDOF + n];
    q.p = pr[PS::P * NDOF + n];
    q.beta = pr[PS::BETA * NDOF + n];
    q.ib = pr[PS::IB * NDOF + n];
    q.lam = pr[PS::LAM * NDOF + n];
    return q;
}

// Persson-Peraire indicator of one element from q = rho * p at its nodes
// (in buf[0..NDOF)): modes = (V1^-1 x ... x V1^-1) q by sum factorisation, then
// eta = max(1 - |m1|^2/|m|^2, 1 - |m2|^2/|m1|^2) where m1 drops modes with a
// 1D degree of N and m2 those with a 1D degree >= N - 1.
template <int DIM, int N, int G, int D>
__device__ __forceinline__ void modal_pass(const double *src, double *dst, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF;
    for (int t = gl; t < NDOF; t += G) {
        int pos, line;
        node_pos<DIM, Np, D>(t, pos, line);
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < Np; l++) s += Vinv[pos * Np + l] * src[line_node<DIM, Np, D>(line, l)];
        dst[t] = s;
    }
    __syncwarp();
}
template <int DIM, int N, int G>
__device__ __forceinline__ double indicator_eta(double *buf, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF;
    double *a = buf, *b = buf + NDOF;
    modal_pass<DIM, N, G, 0>(a, b, gl, Vinv);
    modal_pass<DIM, N, G, 1>(b, a, gl, Vinv);
    if (DIM == 3) modal_pass<DIM, N, G, (DIM == 3 ? 2 : 0)>(a, b, gl, Vinv);
    const double *m = (DIM == 3) ? b : a;
    double mm = 0.0, m1 = 0.0, m2 = 0.0;
    for (int t = gl; t < NDOF; t += G) {
        const int i = t % Np, j = (t / Np) % Np, k = DIM == 3 ? t / (Np * Np) : 0;
        int mx = i > j ? i : j;
        if (DIM == 3) mx = mx > k ? mx : k;
        const double v = m[t] * m[t];
        mm += v;
        if (mx <= N - 1) m1 += v;
        if (mx <= N - 2) m2 += v;
    }
    mm = group_sum<G>(mm);
    m1 = group_sum<G>(m1);
    m2 = group_sum<G>(m2);
    const double eta = 1.0 - m1 / mm;
    return fmax(eta, 1.0 - m2 / m1);
}

__device__ __forceinline__ double blending_alpha(double eta, const KParams &P)
{
    const double T = P.modal_threshold;
    double a = 1.0 / (1.0 + exp(-9.21024 * (eta - T) / T));
    if (a < P.alpha_min) a = 0.0;
    else if (a > (1.0 - P.alpha_min)) a = 1.0;
    return fmin(a, P.alpha_max);
}

// Stages the element (or a uniform dummy state for the idle tail) and its
// node primitives in shared memory; returns this lane's max wave speed.
template <int DIM, int N, int G>
__device__ __forceinline__ double stage_element(const KParams &P, int64_t e, bool valid, int gl, double *us,
                                                double *pr, unsigned int &flags)
{
    using S = Shape<DIM, N>;
    using PS = PSlot<DIM>;
    constexpr int NDOF = S::NDOF, NV = S::NV;
    const double *src = P.u + e * NDOF;
    for (int t = gl; t < NV * NDOF; t += G) {
        const int v = t / NDOF, n = t - v * NDOF;
        double x;
        if (valid) x = __ldg(src + (int64_t)v * P.nnodes + n);
        else x = (v == 0) ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0);
        us[t] = x;
    }
    __syncwarp();
    double lam = 0.0;
    for (int n = gl; n < NDOF; n += G) {
        double s[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) s[v] = us[v * NDOF + n];
        const Prim<DIM> q = make_prim<DIM>(s, P.gamma, P.gm1);
        pr[P_RHO * NDOF + n] = q.rho;
        pr[P_IRHO * NDOF + n] = q.irho;
#pragma unroll
        for (int d = 0; d < DIM; d++) pr[(P_V + d) * NDOF + n] = q.v[d];
        pr[PS::P * NDOF + n] = q.p;
        pr[PS::BETA * NDOF + n] = q.beta;
        pr[PS::IB * NDOF + n] = q.ib;
        pr[PS::LAM * NDOF + n] = q.lam;
        lam = fmax(lam, q.lam);
        bool finite = true;
#pragma unroll
        for (int v = 0; v < NV; v++) finite = finite && isfinite(s[v]);
        if (!finite) flags |= PDG_FLAG_NONFINITE_DEV;
        else if (!(q.rho > 0.0) || !(q.p > 0.0)) flags |= PDG_FLAG_NONPHYSICAL_DEV;
    }
    __syncwarp();
    return lam;
}

// Flux differencing along direction D: every unordered node pair of every
// line once into buf, then each owner adds sum_m Dhat2(pos, m) F(pos, m).
// Q2FILL (compat NS 3D, y direction) also adds the z-direction terms the
// reference fills from the last y flux (DGSEMIntegrator.cpp:702): for node
// (i, j, k) and every m < k, Dhat2(k, m) F_y((i,j,m), (i,N,m)) (zero when
// j = N).  SKIPLOW (same path, z direction) then omits the m < k terms.
template <int DIM, int N, int G, int D, bool Q2FILL, bool SKIPLOW>
__device__ __forceinline__ void flux_differencing(const KParams &P, const double *pr, double *buf, const double *c,
                                                  int gl, double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NPAIR = S::NPAIR, NFN = S::NFN;
    constexpr int TOTAL = NFN * NPAIR, ROUNDS = (TOTAL + G - 1) / G;
    const double metric = C_ADJ(c)[D];
#pragma unroll
    for (int r = 0; r < ROUNDS; r++) {
        const int t = gl + r * G;
        if (TOTAL % G == 0 || t < TOTAL) {
            const int line = t / NPAIR, p = t - line * NPAIR;
            int a, b;
            pair_decode<Np>(p, a, b);
            const Prim<DIM> qa = load_prim<DIM>(pr, line_node<DIM, Np, D>(line, a), NDOF);
            const Prim<DIM> qb = load_prim<DIM>(pr, line_node<DIM, Np, D>(line, b), NDOF);
            double F[NV];
            volume_flux<DIM, D>(qa, qb, metric, P.gm1inv, F);
#pragma unroll
            for (int v = 0; v < NV; v++) buf[t * NV + v] = F[v];
        }
    }
    __syncwarp();
    const double *D2 = C_DHAT2(c);
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        int pos, line;
        node_pos<DIM, Np, D>(n, pos, line);
#pragma unroll
        for (int m = 0; m < Np; m++) {
            if (m == pos || (SKIPLOW && m < pos)) continue;
            const int pidx = m > pos ? pair_index<Np>(pos, m) : pair_index<Np>(m, pos);
            const double cf = D2[pos * Np + m];
            const double *F = buf + (line * NPAIR + pidx) * NV;
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] += cf * F[v];
        }
        if (DIM == 3 && Q2FILL) {
            const int i = n % Np, j = (n / Np) % Np, k = n / (Np * Np);
            if (j < N) {
#pragma unroll
                for (int m = 0; m < Np - 1; m++) {
                    if (m >= k) break;
                    const double cf = D2[k * Np + m];
                    const double *F = buf + ((i + Np * m) * NPAIR + pair_index<Np>(j, N)) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++) acc[s][v] += cf * F[v];
                }
            }
        }
    }
    __syncwarp();
}

// Subcell finite-volume update of ComputeFVFluxes along direction D: adds
// (f_{pos-1/2} - f_{pos+1/2}) / (J w_pos) to fv for the owned nodes.
template <int DIM, int N, int G, int D>
__device__ __forceinline__ void subcell_fv(const KParams &P, const double *us, const double *pr, double *buf,
                                           const double *c, int gl, double (&fv)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const double *sn = C_SNOR(c, D);
    for (int t = gl; t < NFN * N; t += G) {
        const int line = t / N, iface = t - line * N + 1;  // between nodes iface-1 and iface
        const int n1 = line_node<DIM, Np, D>(line, iface - 1), n2 = line_node<DIM, Np, D>(line, iface);
        const Prim<DIM> q1 = load_prim<DIM>(pr, n1, NDOF), q2 = load_prim<DIM>(pr, n2, NDOF);
        double m1[DIM], m2[DIM], F[NV];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            m1[d] = us[(1 + d) * NDOF + n1];
            m2[d] = us[(1 + d) * NDOF + n2];
        }
        face_flux<DIM, D>(q1, q2, m1, m2, sn[iface], P.gm1inv, P.compat != 0, P.diss_scale, F);
#pragma unroll
        for (int v = 0; v < NV; v++) buf[t * NV + v] = F[v];
    }
    __syncwarp();
    const double *fvs = C_FVS(c);
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        int pos, line;
        node_pos<DIM, Np, D>(n, pos, line);
#pragma unroll
        for (int v = 0; v < NV; v++) {
            double du = pos > 0 ? buf[(line * N + pos - 1) * NV + v] : 0.0;
            if (pos < N) du -= buf[(line * N + pos) * NV + v];
            fv[s][v] += du * fvs[pos];
        }
    }
    __syncwarp();
}

// Face orientation: face on side `side` (0: -d, 1: +d) of element e with
// neighbour nb.  Element 1 is the lower-numbered element; its outward normal
// is +d when it sits on the -d side of the face.
struct FaceOrient {
    bool own_is_1;
    double nrm;  // signed normal of element 1 along d, magnitude = face area
};
__device__ __forceinline__ FaceOrient face_orient(int64_t e, int64_t nb, int side, double area)
{
    const int64_t a = side ? e : nb, b = side ? nb : e;  // a: element on the -d side
    FaceOrient o;
    o.own_is_1 = side ? (e <= nb) : (nb > e);
    o.nrm = (a <= b) ? area : -area;
    return o;
}

// Gathers face contributions (buf[((2d+side)*NFN + line)*NV + v]) into owners.
template <int DIM, int N, int G>
__device__ __forceinline__ void gather_faces(const double *buf, int gl, double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int pos = idx[d];
            if (pos == 0 || pos == N) {
                const int line = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                        : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
                const double *F = buf + ((2 * d + (pos == N ? 1 : 0)) * NFN + line) * NV;
#pragma unroll
                for (int v = 0; v < NV; v++) acc[s][v] += F[v];
            }
        }
    }
}

// Stores the owned nodes' right-hand side, optionally as an SSP-RK3 stage:
// z = us + dt L; stage 0: z, 1: 3/4 un + 1/4 z, 2: 1/3 un + 2/3 z.
template <int DIM, int N, int G>
__device__ __forceinline__ void store_owned(const KParams &P, int64_t e, int gl, const double *us,
                                            const double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int NDOF = S::NDOF, NV = S::NV;
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const int64_t gi = (int64_t)v * P.nnodes + e * NDOF + n;
            double r = acc[s][v];
            if (P.stage >= 0) {
                const double z = us[v * NDOF + n] + P.dt * r;
                if (P.stage == 0) r = z;
                else if (P.stage == 1) r = 3. / 4 * __ldg(P.un + gi) + 1. / 4 * z;
                else r = 1. / 3 * __ldg(P.un + gi) + 2. / 3 * z;
            }
            P.out[gi] = r;
        }
    }
}

// Element faces of direction D, recomputed from this side with the element-1
// rule so both sides of a face evaluate the same flux.  NS adds the central
// (BR1) viscous flux; in compat mode the inviscid flux there sees velocities
// in the momentum slots, as in the reference (its ComputeViscousFlux divides
// the face states' momenta in place before ComputeFaceFlux reads them,
// BasicOperations.cpp:33-34, DGSEMIntegrator.cpp:467-481).
template <int DIM, int N, int G, int D, bool NS>
__device__ __forceinline__ double element_faces(const KParams &P, int64_t e, bool valid, int gl, const double *us,
                                                const double *pr, double *buf, const double *c)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t size = (int64_t)NV * P.nnodes;
    const bool compat = P.compat != 0;
    double lam = 0.0;
    for (int t = gl; t < 2 * NFN; t += G) {
        const int side = t / NFN, fn = t - side * NFN;
        const int nown = line_node<DIM, Np, D>(fn, side ? N : 0);
        const int nnb = line_node<DIM, Np, D>(fn, side ? 0 : N);
        const int64_t nb = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + 2 * D + side) : e;
        double sn[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
            sn[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + nb * NDOF + nnb) : us[v * NDOF + nown];
        const FaceOrient o = face_orient(e, nb, side, C_AREA(c)[D]);
        Prim<DIM> qo = load_prim<DIM>(pr, nown, NDOF);
        Prim<DIM> qn = make_prim<DIM>(sn, P.gamma, P.gm1);
        double mo[DIM], mn[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            mo[d] = us[(1 + d) * NDOF + nown];
            mn[d] = sn[1 + d];
        }
        double fo[DIM + 1], fnb[DIM + 1];
        if (NS) {
            const double *go = P.grads + e * NDOF + nown;
            const double *gn = P.grads + nb * NDOF + nnb;
            const int64_t nn = P.nnodes;
            auto GO = [&](int d, int v) { return __ldg(go + d * size + v * nn); };
            auto GN = [&](int d, int v) { return valid ? __ldg(gn + d * size + v * nn) : 0.0; };
            viscous_col<DIM>(qo, GO, D, P.gm1inv, P.mu, P.lambda_k, fo);
            viscous_col<DIM>(qn, GN, D, P.gm1inv, P.mu, P.lambda_k, fnb);
            if (!valid)
#pragma unroll
                for (int i = 0; i <= DIM; i++) fnb[i] = fo[i];
            if (compat) {
                double so[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) so[v] = us[v * NDOF + nown];
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    so[1 + d] = so[1 + d] / so[0];
                    sn[1 + d] = sn[1 + d] / sn[0];
                    mo[d] = so[1 + d];
                    mn[d] = sn[1 + d];
                }
                qo = make_prim<DIM>(so, P.gamma, P.gm1);
                qn = make_prim<DIM>(sn, P.gamma, P.gm1);
                lam = fmax(lam, fmax(qo.lam, qn.lam));
            }
        }
        double F[NV];
        if (o.own_is_1) face_flux<DIM, D>(qo, qn, mo, mn, o.nrm, P.gm1inv, compat, P.diss_scale, F);
        else face_flux<DIM, D>(qn, qo, mn, mo, o.nrm, P.gm1inv, compat, P.diss_scale, F);
        const double sc = C_FACE(c);
        double *dst = buf + ((2 * D + side) * NFN + fn) * NV;
        dst[0] = sc * (o.own_is_1 ? -F[0] : F[0]);
#pragma unroll
        for (int i = 0; i <= DIM; i++) {
            double du = o.own_is_1 ? -F[1 + i] : F[1 + i];
            if (NS) {
                const double fvn = ((fo[i] + fnb[i]) * 0.5) * o.nrm;
                du = o.own_is_1 ? du + fvn : du - fvn;
            }
            dst[1 + i] = sc * du;
        }
    }
    return lam;
}

// Blending coefficient of the staged element (writes eta/alpha outputs).
template <int DIM, int N, int G>
__device__ __forceinline__ double element_alpha(const KParams &P, int64_t e, bool valid, int gl, const double *pr,
                                                double *buf, const double *c)
{
    using S = Shape<DIM, N>;
    using PS = PSlot<DIM>;
    constexpr int NDOF = S::NDOF;
    if (!P.blending) return 0.0;
    for (int n = gl; n < NDOF; n += G) buf[n] = pr[P_RHO * NDOF + n] * pr[PS::P * NDOF + n];
    __syncwarp();
    const double eta = indicator_eta<DIM, N, G>(buf, gl, C_VINV(c));
    const double alpha = blending_alpha(eta, P);
    if (valid && gl == 0) {
        P.eta_out[e] = eta;
        P.alpha_out[e] = alpha;
    }
    __syncwarp();
    return alpha;
}

// Adds alpha * subcell-FV update to acc when any element of the warp blends.
template <int DIM, int N, int G>
__device__ __forceinline__ void blend_fv(const KParams &P, double alpha, const double *us, const double *pr,
                                        double *buf, const double *c, int gl,
                                        double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int NPL = S::NPL, NV = S::NV;
    if (!(P.blending && __any_sync(0xffffffffu, alpha > 0.0))) return;
    double fv[NPL][NV];
#pragma unroll
    for (int s = 0; s < NPL; s++)
#pragma unroll
        for (int v = 0; v < NV; v++) fv[s][v] = 0.0;
    subcell_fv<DIM, N, G, 0>(P, us, pr, buf, c, gl, fv);
    subcell_fv<DIM, N, G, 1>(P, us, pr, buf, c, gl, fv);
    if (DIM == 3) subcell_fv<DIM, N, G, (DIM == 3 ? 2 : 0)>(P, us, pr, buf, c, gl, fv);
#pragma unroll
    for (int s = 0; s < NPL; s++)
#pragma unroll
        for (int v = 0; v < NV; v++) acc[s][v] = alpha * fv[s][v] + acc[s][v];
}

template <int DIM, int N, int G, bool NS>
__device__ __forceinline__ double all_faces(const KParams &P, int64_t e, bool valid, int gl, const double *us,
                                            const double *pr, double *buf, const double *c)
{
    double lam = element_faces<DIM, N, G, 0, NS>(P, e, valid, gl, us, pr, buf, c);
    lam = fmax(lam, element_faces<DIM, N, G, 1, NS>(P, e, valid, gl, us, pr, buf, c));
    if (DIM == 3) lam = fmax(lam, element_faces<DIM, N, G, (DIM == 3 ? 2 : 0), NS>(P, e, valid, gl, us, pr, buf, c));
    __syncwarp();
    return lam;
}

// Occupancy target: 4 CTAs of 4 warps per SM (128 registers per thread) for
// elements of up to 64 nodes; larger elements keep more registers per thread.
#define PDG_MIN_BLOCKS ((Shape<DIM, N>::NDOF > 64) ? 2 : 4)

// Euler right-hand side (plain or fused into an SSP-RK3 stage).
template <int DIM, int N>
__global__ void __launch_bounds__(128, PDG_MIN_BLOCKS) euler_rhs_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NDOF = S::NDOF, NV = S::NV, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, S::Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int wpb = blockDim.x >> 5;
    double *us = smem + CONST_SLOTS + (size_t)(warp * EPW + grp) * S::EL_EULER;
    double *pr = us + NV * NDOF, *buf = pr + S::NPRIM * NDOF;
    unsigned int flags = 0;
    double lam = 0.0;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += (int64_t)gridDim.x * wpb) {
        const int64_t e0 = wt * EPW + grp;
        const bool valid = e0 < P.ne;
        const int64_t e = valid ? e0 : 0;
        const double ls = stage_element<DIM, N, G>(P, e, valid, gl, us, pr, flags);
        if (valid) lam = fmax(lam, ls);
        const double alpha = element_alpha<DIM, N, G>(P, e, valid, gl, pr, buf, c);
        double acc[NPL][NV];
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = 0.0;
        flux_differencing<DIM, N, G, 0, false, false>(P, pr, buf, c, gl, acc);
        flux_differencing<DIM, N, G, 1, false, false>(P, pr, buf, c, gl, acc);
        if (DIM == 3) flux_differencing<DIM, N, G, (DIM == 3 ? 2 : 0), false, false>(P, pr, buf, c, gl, acc);
        const double invJ = C_INVJ(c), oma = 1.0 - alpha;
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = (-acc[s][v] * oma) * invJ;
        blend_fv<DIM, N, G>(P, alpha, us, pr, buf, c, gl, acc);
        const double lf = all_faces<DIM, N, G, false>(P, e, valid, gl, us, pr, buf, c);
        if (valid) lam = fmax(lam, lf);
        gather_faces<DIM, N, G>(buf, gl, acc);
        if (valid) store_owned<DIM, N, G>(P, e, gl, us, acc);
        __syncwarp();
    }
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

// BR1 lifting faces of direction D: 0.5 (w2 - w1) n1_d / (w0 J) on both sides.
template <int DIM, int N, int G, int D>
__device__ __forceinline__ void lift_faces(const KParams &P, int64_t e, bool valid, int gl, const double *us,
                                           const double *wv, double *fb, const double *c)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    for (int t = gl; t < 2 * NFN; t += G) {
        const int side = t / NFN, fn = t - side * NFN;
        const int nown = line_node<DIM, Np, D>(fn, side ? N : 0);
        const int nnb = line_node<DIM, Np, D>(fn, side ? 0 : N);
        const int64_t nb = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + 2 * D + side) : e;
        double sn[NV], wn[NV];
#pragma unroll
        for (int v = 0; v < NV; v++)
            sn[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + nb * NDOF + nnb) : us[v * NDOF + nown];
        entropy_vars<DIM>(sn, P.gamma, P.gm1, P.gm1inv, wn);
        const FaceOrient o = face_orient(e, nb, side, C_AREA(c)[D]);
        const double sc = C_FACE(c);
        double *dst = fb + ((2 * D + side) * NFN + fn) * NV;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const double wo = wv[v * NDOF + nown];
            const double w1 = o.own_is_1 ? wo : wn[v], w2 = o.own_is_1 ? wn[v] : wo;
            dst[v] = sc * ((0.5 * (w2 - w1)) * o.nrm);
        }
    }
}

// Strong-form gradient along D: (sum_l D(pos,l) w_l) adj_D / J.
template <int DIM, int N, int G, int D>
__device__ __forceinline__ void lift_volume(int gl, const double *wv, double *gacc, const double *c)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const double *Dm = C_D(c);
    const double sc = C_ADJ(c)[D], invJ = C_INVJ(c);
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        int pos, line;
        node_pos<DIM, Np, D>(n, pos, line);
#pragma unroll
        for (int v = 0; v < NV; v++) {
            double a = 0.0;
#pragma unroll
            for (int l = 0; l < Np; l++) a += Dm[pos * Np + l] * wv[v * NDOF + line_node<DIM, Np, D>(line, l)];
            gacc[(D * NV + v) * NDOF + n] = (a * sc) * invJ;
        }
    }
}

// BR1 lifting: entropy variables, strong-form gradient, 1/2-jump face lifting,
// conversion to primitive gradients (written to P.grads_out).
template <int DIM, int N>
__global__ void __launch_bounds__(128, PDG_MIN_BLOCKS) lift_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int wpb = blockDim.x >> 5;
    double *us = smem + CONST_SLOTS + (size_t)(warp * EPW + grp) * S::EL_LIFT;
    double *wv = us + NV * NDOF, *gacc = wv + NV * NDOF, *fb = gacc + DIM * NV * NDOF;
    const int64_t size = (int64_t)NV * P.nnodes;
    unsigned int flags = 0;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += (int64_t)gridDim.x * wpb) {
        const int64_t e0 = wt * EPW + grp;
        const bool valid = e0 < P.ne;
        const int64_t e = valid ? e0 : 0;
        const double *src = P.u + e * NDOF;
        for (int t = gl; t < NV * NDOF; t += G) {
            const int v = t / NDOF, n = t - v * NDOF;
            us[t] = valid ? __ldg(src + (int64_t)v * P.nnodes + n) : (v == 0 ? 1.0 : (v == NV - 1 ? P.gm1inv : 0.0));
        }
        __syncwarp();
        for (int n = gl; n < NDOF; n += G) {
            double s[NV], w[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) s[v] = us[v * NDOF + n];
            entropy_vars<DIM>(s, P.gamma, P.gm1, P.gm1inv, w);
#pragma unroll
            for (int v = 0; v < NV; v++) wv[v * NDOF + n] = w[v];
        }
        __syncwarp();
        lift_volume<DIM, N, G, 0>(gl, wv, gacc, c);
        lift_volume<DIM, N, G, 1>(gl, wv, gacc, c);
        if (DIM == 3) lift_volume<DIM, N, G, (DIM == 3 ? 2 : 0)>(gl, wv, gacc, c);
        lift_faces<DIM, N, G, 0>(P, e, valid, gl, us, wv, fb, c);
        lift_faces<DIM, N, G, 1>(P, e, valid, gl, us, wv, fb, c);
        if (DIM == 3) lift_faces<DIM, N, G, (DIM == 3 ? 2 : 0)>(P, e, valid, gl, us, wv, fb, c);
        __syncwarp();
#pragma unroll
        for (int s = 0; s < NPL; s++) {
            const int n = gl + s * G;
            if (n >= NDOF) break;
            double st[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) st[v] = us[v * NDOF + n];
            const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double g[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) g[v] = gacc[(d * NV + v) * NDOF + n];
                const int pos = idx[d];
                if (pos == 0 || pos == N) {
                    const int line = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                            : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
                    const double *F = fb + ((2 * d + (pos == N ? 1 : 0)) * NFN + line) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++) g[v] += F[v];
                }
                entgrad_to_primgrad<DIM>(st, P.gm1, P.gm1inv, P.compat != 0, g);
                if (valid) {
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        if (!isfinite(g[v])) flags |= PDG_FLAG_NONFINITE_DEV;
                        P.grads_out[d * size + (int64_t)v * P.nnodes + e * NDOF + n] = g[v];
                    }
                }
            }
        }
        __syncwarp();
    }
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

// One Navier-Stokes face node: the face between element a's +D face and its
// neighbour b's -D face, evaluated once with the element-1 rule (element 1 =
// the lower-numbered element, normal out of it).  Writes a's contribution
// C = scale * (-/+ F* +/- Fv.n) (b's contribution is -C) to P.fbuf.
template <int DIM, int N, int D>
__device__ __forceinline__ double ns_face_node(const KParams &P, const double *c, int64_t a, int fn)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    const int64_t size = (int64_t)NV * P.nnodes, nn = P.nnodes;
    const int64_t b = __ldg(P.nbr + a * 2 * DIM + 2 * D + 1);
    const int na = line_node<DIM, Np, D>(fn, N), nb = line_node<DIM, Np, D>(fn, 0);
    double sa[NV], sb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        sa[v] = __ldg(P.u + v * nn + a * NDOF + na);
        sb[v] = __ldg(P.u + v * nn + b * NDOF + nb);
    }
    const double *ga = P.grads + a * NDOF + na, *gb = P.grads + b * NDOF + nb;
    auto GA = [&](int d, int v) { return __ldg(ga + d * size + v * nn); };
    auto GB = [&](int d, int v) { return __ldg(gb + d * size + v * nn); };
    Prim<DIM> qa = make_prim<DIM>(sa, P.gamma, P.gm1), qb = make_prim<DIM>(sb, P.gamma, P.gm1);
    double fa[DIM + 1], fb[DIM + 1];
    viscous_col<DIM>(qa, GA, D, P.gm1inv, P.mu, P.lambda_k, fa);
    viscous_col<DIM>(qb, GB, D, P.gm1inv, P.mu, P.lambda_k, fb);
    double ma[DIM], mb[DIM];
    double lam = 0.0;
    if (P.compat) {
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
    const bool a_is_1 = a <= b;
    const double nrm = a_is_1 ? C_AREA(c)[D] : -C_AREA(c)[D];
    double F[NV];
    if (a_is_1) face_flux<DIM, D>(qa, qb, ma, mb, nrm, P.gm1inv, P.compat != 0, P.diss_scale, F);
    else face_flux<DIM, D>(qb, qa, mb, ma, nrm, P.gm1inv, P.compat != 0, P.diss_scale, F);
    const double sc = C_FACE(c);
    double *dst = P.fbuf + ((D * P.ne + a) * NFN + fn) * NV;
    dst[0] = sc * (a_is_1 ? -F[0] : F[0]);
#pragma unroll
    for (int i = 0; i <= DIM; i++) {
        const double fvn = ((fa[i] + fb[i]) * 0.5) * nrm;
        dst[1 + i] = sc * (a_is_1 ? -F[1 + i] + fvn : F[1 + i] - fvn);
    }
    return lam;
}

// Face kernel: one thread per (direction, element, face node), direction
// slowest so a warp's threads share one direction.
template <int DIM, int N>
__global__ void __launch_bounds__(256) ns_face_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NFN = S::NFN;
    __shared__ double c[CONST_SLOTS];
    load_consts(P.K, c, S::Np);
    __syncthreads();
    const int64_t per_dir = P.ne * NFN;
    double lam = 0.0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < DIM * per_dir;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int d = (int)(t / per_dir);
        const int64_t r = t - d * per_dir;
        const int64_t a = r / NFN;
        const int fn = (int)(r - a * NFN);
        if (d == 0) lam = fmax(lam, ns_face_node<DIM, N, 0>(P, c, a, fn));
        else if (d == 1) lam = fmax(lam, ns_face_node<DIM, N, 1>(P, c, a, fn));
        else lam = fmax(lam, ns_face_node<DIM, N, (DIM == 3 ? 2 : 0)>(P, c, a, fn));
    }
    lam = group_max<32>(lam);
    if ((threadIdx.x & 31) == 0) atomic_max_pos(P.lam_bits, lam);
}

// Adds the precomputed face contributions to the owned nodes: +C from the
// element's +d faces (it is their "a" side), -C from its -d faces.
template <int DIM, int N, int G>
__device__ __forceinline__ void gather_face_buffer(const KParams &P, int64_t e, bool valid, int gl,
                                                   double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
    if (!valid) return;
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        const int idx[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const int pos = idx[d];
            if (pos == 0 || pos == N) {
                const int line = d == 0 ? (DIM == 2 ? idx[1] : idx[1] + Np * idx[2])
                                        : (d == 1 ? (DIM == 2 ? idx[0] : idx[0] + Np * idx[2]) : idx[0] + Np * idx[1]);
                const int64_t owner = pos == N ? e : (int64_t)__ldg(P.nbr + e * 2 * DIM + 2 * d);
                const double *F = P.fbuf + ((d * P.ne + owner) * NFN + line) * NV;
                if (pos == N) {
#pragma unroll
                    for (int v = 0; v < NV; v++) acc[s][v] += __ldg(F + v);
                } else {
#pragma unroll
                    for (int v = 0; v < NV; v++) acc[s][v] -= __ldg(F + v);
                }
            }
        }
    }
}

// dv[s][i] += sum_l Dhat(pos, l) fvc[D][i][line node l] for the owned nodes.
template <int DIM, int N, int G, int D>
__device__ __forceinline__ void viscous_divergence_dir(int gl, const double *fvc, const double *c,
                                                       double (&dv)[Shape<DIM, N>::NPL][DIM + 1])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    const double *Dh = C_DHAT(c);
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        int pos, line;
        node_pos<DIM, Np, D>(n, pos, line);
#pragma unroll
        for (int l = 0; l < Np; l++) {
            const double cf = Dh[pos * Np + l];
            const int nl = line_node<DIM, Np, D>(line, l);
#pragma unroll
            for (int i = 0; i < NV - 1; i++) dv[s][i] += cf * fvc[(D * (NV - 1) + i) * NDOF + nl];
        }
    }
}

// Navier-Stokes right-hand side (plain or fused into an SSP-RK3 stage).
template <int DIM, int N>
__global__ void __launch_bounds__(128, PDG_MIN_BLOCKS) ns_rhs_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NDOF = S::NDOF, NV = S::NV, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts(P.K, c, S::Np);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int wpb = blockDim.x >> 5;
    double *us = smem + CONST_SLOTS + (size_t)(warp * EPW + grp) * S::EL_NS;
    double *pr = us + NV * NDOF, *buf = pr + S::NPRIM * NDOF;
    const int64_t size = (int64_t)NV * P.nnodes;
    const bool compat = P.compat != 0;
    unsigned int flags = 0;
    double lam = 0.0;
    for (int64_t wt = (int64_t)blockIdx.x * wpb + warp; wt < P.nwt; wt += (int64_t)gridDim.x * wpb) {
        const int64_t e0 = wt * EPW + grp;
        const bool valid = e0 < P.ne;
        const int64_t e = valid ? e0 : 0;
        const double ls = stage_element<DIM, N, G>(P, e, valid, gl, us, pr, flags);
        if (valid) lam = fmax(lam, ls);
        const double alpha = element_alpha<DIM, N, G>(P, e, valid, gl, pr, buf, c);
        // Contravariant viscous fluxes at the nodes into buf[d][i][n].  The
        // reference evaluates them with the state of its member id1, the
        // element's last node (DGSEMIntegrator.cpp:620, :770); compat keeps it.
        const double *gsrc = P.grads + e * NDOF;
        for (int n = gl; n < NDOF; n += G) {
            const Prim<DIM> q = load_prim<DIM>(pr, compat ? NDOF - 1 : n, NDOF);
            auto GG = [&](int d, int v) { return valid ? __ldg(gsrc + d * size + (int64_t)v * P.nnodes + n) : 0.0; };
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double col[DIM + 1];
                viscous_col<DIM>(q, GG, d, P.gm1inv, P.mu, P.lambda_k, col);
#pragma unroll
                for (int i = 0; i <= DIM; i++) buf[(d * (NV - 1) + i) * NDOF + n] = C_ADJ(c)[d] * col[i];
            }
        }
        __syncwarp();
        double dv[NPL][NV - 1];
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int i = 0; i < NV - 1; i++) dv[s][i] = 0.0;
        viscous_divergence_dir<DIM, N, G, 0>(gl, buf, c, dv);
        viscous_divergence_dir<DIM, N, G, 1>(gl, buf, c, dv);
        if (DIM == 3) viscous_divergence_dir<DIM, N, G, (DIM == 3 ? 2 : 0)>(gl, buf, c, dv);
        __syncwarp();
        double acc[NPL][NV];
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = 0.0;
        flux_differencing<DIM, N, G, 0, false, false>(P, pr, buf, c, gl, acc);
        if (DIM == 3 && compat) {
            flux_differencing<DIM, N, G, 1, (DIM == 3), false>(P, pr, buf, c, gl, acc);
            flux_differencing<DIM, N, G, (DIM == 3 ? 2 : 0), false, (DIM == 3)>(P, pr, buf, c, gl, acc);
        } else {
            flux_differencing<DIM, N, G, 1, false, false>(P, pr, buf, c, gl, acc);
            if (DIM == 3) flux_differencing<DIM, N, G, (DIM == 3 ? 2 : 0), false, false>(P, pr, buf, c, gl, acc);
        }
        const double invJ = C_INVJ(c), oma = 1.0 - alpha;
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) {
                double t = -acc[s][v] * oma;
                if (v > 0) t = t + dv[s][v - 1];
                acc[s][v] = t * invJ;
            }
        blend_fv<DIM, N, G>(P, alpha, us, pr, buf, c, gl, acc);
        gather_face_buffer<DIM, N, G>(P, e, valid, gl, acc);
        if (valid) store_owned<DIM, N, G>(P, e, gl, us, acc);
        __syncwarp();
    }
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

}  // namespace pdg
