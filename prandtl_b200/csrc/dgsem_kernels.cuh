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
// element into a shared buffer and then gathered by the owners.
//
// Reference mapping (all paths relative to the reference tree):
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
    static constexpr int NPRIM = DIM + 3;                   // rho, v[DIM], p, beta
    static constexpr int BUF_PAIR = NFN * NPAIR * NV;
    static constexpr int BUF_FACE = 2 * DIM * NFN * NV;
    static constexpr int BUF_FV = NFN * N * NV;
    static constexpr int BUF_MODAL = 2 * NDOF;
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int BUF = cmax(cmax(BUF_PAIR, BUF_FACE), cmax(BUF_FV, BUF_MODAL));
    // per-element shared doubles: state, primitives, flux buffer
    static constexpr int EL_EULER = NV * NDOF + NPRIM * NDOF + BUF;
    // NS adds the contravariant viscous fluxes [DIM][NV-1][NDOF]
    static constexpr int EL_NS = EL_EULER + DIM * (NV - 1) * NDOF;
    // lifting: state, entropy variables, gradient accumulators, face buffer
    static constexpr int EL_LIFT = NV * NDOF + NV * NDOF + DIM * NV * NDOF + BUF_FACE;
    static constexpr int CONST_D = 4 * 36 + 6 + 21 + 6;     // D, Dhat, Dhat2, Vinv1, w, snor, fv_scale
};

// Node index of position `pos` on line `line` of direction d (x fastest).
template <int DIM, int Np> __device__ __forceinline__ int line_node(int d, int line, int pos)
{
    if (DIM == 2) return d == 0 ? line * Np + pos : pos * Np + line;
    if (d == 0) return line * Np + pos;
    if (d == 1) return (line / Np) * Np * Np + pos * Np + (line % Np);
    return pos * Np * Np + line;
}
// Position and line of node n along direction d.
template <int DIM, int Np> __device__ __forceinline__ void node_pos(int n, int d, int &pos, int &line)
{
    const int i = n % Np, j = (n / Np) % Np, k = n / (Np * Np);
    if (d == 0) { pos = i; line = DIM == 2 ? j : j + Np * k; }
    else if (d == 1) { pos = j; line = DIM == 2 ? i : i + Np * k; }
    else { pos = k; line = i + Np * j; }
}
// Index of the unordered pair (a, b), a < b, among Np*(Np-1)/2 pairs.
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

// Order-preserving map of a non-negative double to uint64 for atomicMax.
__device__ __forceinline__ void atomic_max_pos(unsigned long long *addr, double v)
{
    if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// Sum over the G lanes of one group (G divides 32; xor offsets stay inside).
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

// Copies the constants a kernel needs into shared memory.
template <int DIM, int N> __device__ __forceinline__ void load_consts(const DevConst *K, double *c)
{
    constexpr int Np = N + 1;
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

// Persson-Peraire indicator of one element from q = rho * p at its nodes:
// modes = (V1^-1 x ... x V1^-1) q by sum factorisation, then
// eta = max(1 - |m1|^2/|m|^2, 1 - |m2|^2/|m1|^2) where m1 drops modes with a
// 1D degree of N and m2 those with a 1D degree >= N - 1.
template <int DIM, int N, int G>
__device__ __forceinline__ double indicator_eta(double *buf, int gl, const double *Vinv)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF;
    double *a = buf, *b = buf + NDOF;
    // contract the 1D index of each direction in turn: a -> b -> a (-> b)
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double *src = (d % 2 == 0) ? a : b;
        double *dst = (d % 2 == 0) ? b : a;
        for (int t = gl; t < NDOF; t += G) {
            int pos, line;
            node_pos<DIM, Np>(t, d, pos, line);
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < Np; l++) s += Vinv[pos * Np + l] * src[line_node<DIM, Np>(d, line, l)];
            dst[t] = s;
        }
        __syncwarp();
    }
    const double *m = (DIM % 2 == 0) ? a : b;
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
    double eta = 1.0 - m1 / mm;
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

// Fills an element slot of shared memory with its state (or a harmless
// uniform state for the idle tail) and computes the node primitives.
// Returns this lane's max wave speed.
template <int DIM, int N, int G>
__device__ __forceinline__ double stage_element(const KParams &P, int64_t e, bool valid, int gl, double *us,
                                                double *pr, unsigned int &flags)
{
    using S = Shape<DIM, N>;
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
        Prim<DIM> q = make_prim<DIM>(s, P.gm1);
        pr[n] = q.rho;
#pragma unroll
        for (int d = 0; d < DIM; d++) pr[(1 + d) * NDOF + n] = q.v[d];
        pr[(DIM + 1) * NDOF + n] = q.p;
        pr[(DIM + 2) * NDOF + n] = q.beta;
        lam = fmax(lam, wave_speed<DIM>(q, P.gamma));
        bool finite = true;
#pragma unroll
        for (int v = 0; v < NV; v++) finite = finite && isfinite(s[v]);
        if (!finite) flags |= PDG_FLAG_NONFINITE_DEV;
        else if (!(q.rho > 0.0) || !(q.p > 0.0)) flags |= PDG_FLAG_NONPHYSICAL_DEV;
    }
    __syncwarp();
    return lam;
}

template <int DIM> __device__ __forceinline__ Prim<DIM> load_prim(const double *pr, int n, int NDOF)
{
    Prim<DIM> q;
    q.rho = pr[n];
#pragma unroll
    for (int d = 0; d < DIM; d++) q.v[d] = pr[(1 + d) * NDOF + n];
    q.p = pr[(DIM + 1) * NDOF + n];
    q.beta = pr[(DIM + 2) * NDOF + n];
    q.vsq = 0.0;
    return q;
}

// Flux differencing along direction d: computes every unordered node pair of
// every line once into buf, then each owner adds sum_m Dhat2(pos, m) F(pos, m).
// With q2 set (compat NS 3D, y direction), it also adds the z-direction terms
// the reference fills from the last y flux (DGSEMIntegrator.cpp:702): for
// node (i, j, k) and every m < k, Dhat2(k, m) * F_y((i,j,m), (i,N,m)) (zero
// when j = N).  With skip_lower set (same path, z direction) the m < k terms
// are omitted because they were added that way.
template <int DIM, int N, int G>
__device__ __forceinline__ void flux_differencing(const KParams &P, int d, const double *pr, double *buf,
                                                  const double *c, int gl, double (&acc)[Shape<DIM, N>::NPL][DIM + 2],
                                                  bool q2_fill, bool skip_lower)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NPAIR = S::NPAIR, NFN = S::NFN;
    const double metric = C_ADJ(c)[d];
    for (int t = gl; t < NFN * NPAIR; t += G) {
        const int line = t / NPAIR, p = t - line * NPAIR;
        int a, b;
        pair_decode<Np>(p, a, b);
        const Prim<DIM> qa = load_prim<DIM>(pr, line_node<DIM, Np>(d, line, a), NDOF);
        const Prim<DIM> qb = load_prim<DIM>(pr, line_node<DIM, Np>(d, line, b), NDOF);
        double F[NV];
        volume_flux<DIM>(qa, qb, d, metric, P.gm1inv, F);
#pragma unroll
        for (int v = 0; v < NV; v++) buf[t * NV + v] = F[v];
    }
    __syncwarp();
    const double *D2 = C_DHAT2(c);
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
        int pos, line;
        node_pos<DIM, Np>(n, d, pos, line);
#pragma unroll
        for (int m = 0; m < Np; m++) {
            if (m == pos || (skip_lower && m < pos)) continue;
            const int pidx = m > pos ? pair_index<Np>(pos, m) : pair_index<Np>(m, pos);
            const double cf = D2[pos * Np + m];
            const double *F = buf + (line * NPAIR + pidx) * NV;
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] += cf * F[v];
        }
        if (DIM == 3 && q2_fill) {
            // node (i, j, k): y line index is i + Np*k, position j
            const int i = n % Np, j = (n / Np) % Np, k = n / (Np * Np);
            if (j < N) {
#pragma unroll
                for (int m = 0; m < Np; m++) {
                    if (m >= k) break;
                    const int lz = i + Np * m;  // y line through (i, *, m)
                    const double cf = D2[k * Np + m];
                    const double *F = buf + (lz * NPAIR + pair_index<Np>(j, N)) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++) acc[s][v] += cf * F[v];
                }
            }
        }
    }
    __syncwarp();
}

// Subcell finite-volume update of ComputeFVFluxes: adds
// sum_d (f_{pos-1/2} - f_{pos+1/2}) / (J w_pos) to fv for the owned nodes.
template <int DIM, int N, int G>
__device__ __forceinline__ void subcell_fv(const KParams &P, const double *us, double *buf, const double *c, int gl,
                                           double (&fv)[Shape<DIM, N>::NPL][DIM + 2], double &lam)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
#pragma unroll 1
    for (int d = 0; d < DIM; d++) {
        const double *sn = C_SNOR(c, d);
        for (int t = gl; t < NFN * N; t += G) {
            const int line = t / N, iface = t - line * N + 1;  // interface between iface-1 and iface
            const int n1 = line_node<DIM, Np>(d, line, iface - 1), n2 = line_node<DIM, Np>(d, line, iface);
            double s1[NV], s2[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                s1[v] = us[v * NDOF + n1];
                s2[v] = us[v * NDOF + n2];
            }
            lam = fmax(lam, face_flux<DIM>(s1, s2, d, sn[iface], P.gamma, P.gm1, P.gm1inv, P.compat != 0,
                                           P.diss_scale, F));
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
            node_pos<DIM, Np>(n, d, pos, line);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                double du = pos > 0 ? buf[(line * N + pos - 1) * NV + v] : 0.0;
                if (pos < N) du -= buf[(line * N + pos) * NV + v];
                fv[s][v] += du * fvs[pos];
            }
        }
        __syncwarp();
    }
}

// Gathers face contributions (buf[(f*NFN + fn)*NV + v]) into the owners.
template <int DIM, int N, int G>
__device__ __forceinline__ void gather_faces(const double *buf, int gl, double (&acc)[Shape<DIM, N>::NPL][DIM + 2])
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN;
#pragma unroll
    for (int s = 0; s < S::NPL; s++) {
        const int n = gl + s * G;
        if (n >= NDOF) break;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            int pos, line;
            node_pos<DIM, Np>(n, d, pos, line);
            if (pos == 0 || pos == N) {
                const int f = 2 * d + (pos == N ? 1 : 0);
                const double *F = buf + (f * NFN + line) * NV;
#pragma unroll
                for (int v = 0; v < NV; v++) acc[s][v] += F[v];
            }
        }
    }
}

// Face orientation: the face on side `side` (0: -d, 1: +d) of element e with
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

// Stores the finished right-hand side of the owned nodes, optionally as an
// SSP-RK3 stage: z = us + dt L; stage 0: z, 1: 3/4 un + 1/4 z, 2: 1/3 un + 2/3 z.
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

}  // namespace pdg

namespace pdg {

// One column (flux direction `dir`) of the viscous flux: momentum rows and the
// energy row of NavierStokesFlux::ComputeViscousFlux (NavierStokesFlux.cpp:12-90).
// g[d*gsd + v*gsv] is the primitive gradient of variable v along x_d.
template <int DIM>
__device__ __forceinline__ void viscous_flux_col(const double *s, const double *g, int64_t gsd, int64_t gsv, int dir,
                                                 double gm1, double gm1inv, double mu, double lambda_k, double *out)
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
    for (int d = 0; d < DIM; d++) div += __ldg(g + d * gsd + (1 + d) * gsv);
    const double *gd = g + dir * gsd;
    const double mu_bulk = 2.0 / 3.0;
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < DIM; i++) {
        double tau;
        if (i == dir) tau = mu * (2.0 * __ldg(gd + (1 + i) * gsv) - mu_bulk * div);
        else tau = mu * (__ldg(gd + (1 + i) * gsv) + __ldg(g + i * gsd + (1 + dir) * gsv));
        out[i] = tau;
        e += vel[i] * tau;
    }
    const double cv_dT = gm1inv / rho * (__ldg(gd + (DIM + 1) * gsv) - p / rho * __ldg(gd));
    out[DIM] = e + lambda_k * cv_dT;
}

// Euler right-hand side (plain or fused into an SSP-RK3 stage).
template <int DIM, int N>
__global__ void __launch_bounds__(128) euler_rhs_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts<DIM, N>(P.K, c);
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
        double alpha = 0.0;
        if (P.blending) {
            for (int n = gl; n < NDOF; n += G) buf[n] = pr[n] * pr[(DIM + 1) * NDOF + n];
            __syncwarp();
            const double eta = indicator_eta<DIM, N, G>(buf, gl, C_VINV(c));
            alpha = blending_alpha(eta, P);
            if (valid && gl == 0) {
                P.eta_out[e] = eta;
                P.alpha_out[e] = alpha;
            }
            __syncwarp();
        }
        double acc[NPL][NV];
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = 0.0;
#pragma unroll 1
        for (int d = 0; d < DIM; d++) flux_differencing<DIM, N, G>(P, d, pr, buf, c, gl, acc, false, false);
        const double invJ = C_INVJ(c), oma = 1.0 - alpha;
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = (-acc[s][v] * oma) * invJ;
        if (P.blending && __any_sync(0xffffffffu, alpha > 0.0)) {
            double fv[NPL][NV];
#pragma unroll
            for (int s = 0; s < NPL; s++)
#pragma unroll
                for (int v = 0; v < NV; v++) fv[s][v] = 0.0;
            double lfv = 0.0;
            subcell_fv<DIM, N, G>(P, us, buf, c, gl, fv, lfv);
#pragma unroll
            for (int s = 0; s < NPL; s++)
#pragma unroll
                for (int v = 0; v < NV; v++) acc[s][v] = alpha * fv[s][v] + acc[s][v];
        }
        // element faces, recomputed from this side with the element-1 rule
        for (int t = gl; t < 2 * DIM * NFN; t += G) {
            const int f = t / NFN, fn = t - f * NFN, d = f >> 1, side = f & 1;
            const int nown = line_node<DIM, Np>(d, fn, side ? N : 0);
            const int nnb = line_node<DIM, Np>(d, fn, side ? 0 : N);
            const int64_t nb = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + f) : e;
            double so[NV], sn[NV], s1[NV], s2[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                so[v] = us[v * NDOF + nown];
                sn[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + nb * NDOF + nnb) : so[v];
            }
            const FaceOrient o = face_orient(e, nb, side, C_AREA(c)[d]);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                s1[v] = o.own_is_1 ? so[v] : sn[v];
                s2[v] = o.own_is_1 ? sn[v] : so[v];
            }
            const double lf = face_flux<DIM>(s1, s2, d, o.nrm, P.gamma, P.gm1, P.gm1inv, P.compat != 0, P.diss_scale, F);
            if (valid) lam = fmax(lam, lf);
            const double sc = C_FACE(c);
#pragma unroll
            for (int v = 0; v < NV; v++) buf[t * NV + v] = sc * (o.own_is_1 ? -F[v] : F[v]);
        }
        __syncwarp();
        gather_faces<DIM, N, G>(buf, gl, acc);
        if (valid) store_owned<DIM, N, G>(P, e, gl, us, acc);
        __syncwarp();
    }
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

// BR1 lifting: entropy variables, strong-form gradient, 1/2-jump face
// lifting, conversion to primitive gradients (written to P.grads_out).
template <int DIM, int N>
__global__ void __launch_bounds__(128) lift_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts<DIM, N>(P.K, c);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int wpb = blockDim.x >> 5;
    double *us = smem + CONST_SLOTS + (size_t)(warp * EPW + grp) * S::EL_LIFT;
    double *wv = us + NV * NDOF, *gacc = wv + NV * NDOF, *fb = gacc + DIM * NV * NDOF;
    const int64_t size = (int64_t)NV * P.nnodes;
    const double *D = C_D(c);
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
        // element part: (sum_l D(pos,l) w_l) * adj_d * (1/J)
#pragma unroll
        for (int s = 0; s < NPL; s++) {
            const int n = gl + s * G;
            if (n >= NDOF) break;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                int pos, line;
                node_pos<DIM, Np>(n, d, pos, line);
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    double a = 0.0;
#pragma unroll
                    for (int l = 0; l < Np; l++) a += D[pos * Np + l] * wv[v * NDOF + line_node<DIM, Np>(d, line, l)];
                    gacc[(d * NV + v) * NDOF + n] = (a * C_ADJ(c)[d]) * C_INVJ(c);
                }
            }
        }
        // faces: 0.5 (w2 - w1) n1_d / (w0 J), the same value on both sides
        for (int t = gl; t < 2 * DIM * NFN; t += G) {
            const int f = t / NFN, fn = t - f * NFN, d = f >> 1, side = f & 1;
            const int nown = line_node<DIM, Np>(d, fn, side ? N : 0);
            const int nnb = line_node<DIM, Np>(d, fn, side ? 0 : N);
            const int64_t nb = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + f) : e;
            double sn[NV], wn[NV];
#pragma unroll
            for (int v = 0; v < NV; v++)
                sn[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + nb * NDOF + nnb) : us[v * NDOF + nown];
            entropy_vars<DIM>(sn, P.gamma, P.gm1, P.gm1inv, wn);
            const FaceOrient o = face_orient(e, nb, side, C_AREA(c)[d]);
            const double sc = C_FACE(c);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const double wo = wv[v * NDOF + nown];
                const double w1 = o.own_is_1 ? wo : wn[v], w2 = o.own_is_1 ? wn[v] : wo;
                fb[t * NV + v] = sc * ((0.5 * (w2 - w1)) * o.nrm);
            }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < NPL; s++) {
            const int n = gl + s * G;
            if (n >= NDOF) break;
            double st[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) st[v] = us[v * NDOF + n];
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                int pos, line;
                node_pos<DIM, Np>(n, d, pos, line);
                double g[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) g[v] = gacc[(d * NV + v) * NDOF + n];
                if (pos == 0 || pos == N) {
                    const int f = 2 * d + (pos == N ? 1 : 0);
#pragma unroll
                    for (int v = 0; v < NV; v++) g[v] += fb[(f * NFN + line) * NV + v];
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

// Navier-Stokes right-hand side (plain or fused into an SSP-RK3 stage).
template <int DIM, int N>
__global__ void __launch_bounds__(128) ns_rhs_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV, NFN = S::NFN, G = S::G, EPW = S::EPW, NPL = S::NPL;
    extern __shared__ double smem[];
    double *c = smem;
    load_consts<DIM, N>(P.K, c);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const int wpb = blockDim.x >> 5;
    double *us = smem + CONST_SLOTS + (size_t)(warp * EPW + grp) * S::EL_NS;
    double *pr = us + NV * NDOF, *buf = pr + S::NPRIM * NDOF, *fvc = buf + S::BUF;
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
        double alpha = 0.0;
        if (P.blending) {
            for (int n = gl; n < NDOF; n += G) buf[n] = pr[n] * pr[(DIM + 1) * NDOF + n];
            __syncwarp();
            const double eta = indicator_eta<DIM, N, G>(buf, gl, C_VINV(c));
            alpha = blending_alpha(eta, P);
            if (valid && gl == 0) {
                P.eta_out[e] = eta;
                P.alpha_out[e] = alpha;
            }
            __syncwarp();
        }
        // contravariant viscous fluxes at the nodes; the reference evaluates
        // them with the state of its member id1, the element's last node
        // (DGSEMIntegrator.cpp:620, :770) — compat keeps that.
        const double *gsrc = P.grads + e * NDOF;
        for (int n = gl; n < NDOF; n += G) {
            const int sn = compat ? NDOF - 1 : n;
            double st[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) st[v] = us[v * NDOF + sn];
            double dq[DIM][NV];
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
                for (int v = 0; v < NV; v++) dq[d][v] = valid ? __ldg(gsrc + d * size + (int64_t)v * P.nnodes + n) : 0.0;
            double Fv[DIM + 1][DIM];
            viscous_flux<DIM>(st, dq, P.gm1, P.gm1inv, P.mu, P.lambda_k, Fv);
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
                for (int i = 0; i <= DIM; i++) fvc[(d * (NV - 1) + i) * NDOF + n] = C_ADJ(c)[d] * Fv[i][d];
        }
        __syncwarp();
        double dv[NPL][NV - 1];
        const double *Dh = C_DHAT(c);
#pragma unroll
        for (int s = 0; s < NPL; s++) {
#pragma unroll
            for (int i = 0; i < NV - 1; i++) dv[s][i] = 0.0;
            const int n = gl + s * G;
            if (n >= NDOF) continue;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                int pos, line;
                node_pos<DIM, Np>(n, d, pos, line);
#pragma unroll
                for (int l = 0; l < Np; l++) {
                    const double cf = Dh[pos * Np + l];
                    const int nl = line_node<DIM, Np>(d, line, l);
#pragma unroll
                    for (int i = 0; i < NV - 1; i++) dv[s][i] += cf * fvc[(d * (NV - 1) + i) * NDOF + nl];
                }
            }
        }
        double acc[NPL][NV];
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) acc[s][v] = 0.0;
        const bool q2 = DIM == 3 && compat;
#pragma unroll 1
        for (int d = 0; d < DIM; d++)
            flux_differencing<DIM, N, G>(P, d, pr, buf, c, gl, acc, q2 && d == 1, q2 && d == 2);
        const double invJ = C_INVJ(c), oma = 1.0 - alpha;
#pragma unroll
        for (int s = 0; s < NPL; s++)
#pragma unroll
            for (int v = 0; v < NV; v++) {
                double t = -acc[s][v] * oma;
                if (v > 0) t = t + dv[s][v - 1];
                acc[s][v] = t * invJ;
            }
        if (P.blending && __any_sync(0xffffffffu, alpha > 0.0)) {
            double fv[NPL][NV];
#pragma unroll
            for (int s = 0; s < NPL; s++)
#pragma unroll
                for (int v = 0; v < NV; v++) fv[s][v] = 0.0;
            double lfv = 0.0;
            subcell_fv<DIM, N, G>(P, us, buf, c, gl, fv, lfv);
#pragma unroll
            for (int s = 0; s < NPL; s++)
#pragma unroll
                for (int v = 0; v < NV; v++) acc[s][v] = alpha * fv[s][v] + acc[s][v];
        }
        // faces: Chandrashekar flux + central (BR1) viscous flux
        for (int t = gl; t < 2 * DIM * NFN; t += G) {
            const int f = t / NFN, fn = t - f * NFN, d = f >> 1, side = f & 1;
            const int nown = line_node<DIM, Np>(d, fn, side ? N : 0);
            const int nnb = line_node<DIM, Np>(d, fn, side ? 0 : N);
            const int64_t nb = valid ? (int64_t)__ldg(P.nbr + e * 2 * DIM + f) : e;
            double so[NV], sn[NV], s1[NV], s2[NV], F[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                so[v] = us[v * NDOF + nown];
                sn[v] = valid ? __ldg(P.u + (int64_t)v * P.nnodes + nb * NDOF + nnb) : so[v];
            }
            const FaceOrient o = face_orient(e, nb, side, C_AREA(c)[d]);
            double fo[DIM + 1], fnb[DIM + 1];
            viscous_flux_col<DIM>(so, P.grads + e * NDOF + nown, size, P.nnodes, d, P.gm1, P.gm1inv, P.mu,
                                  P.lambda_k, fo);
            if (valid)
                viscous_flux_col<DIM>(sn, P.grads + nb * NDOF + nnb, size, P.nnodes, d, P.gm1, P.gm1inv, P.mu,
                                      P.lambda_k, fnb);
            else
#pragma unroll
                for (int i = 0; i <= DIM; i++) fnb[i] = fo[i];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                s1[v] = o.own_is_1 ? so[v] : sn[v];
                s2[v] = o.own_is_1 ? sn[v] : so[v];
            }
            if (compat) {
                // ComputeViscousFlux divides the momenta of the reference's
                // face states in place before ComputeFaceFlux reads them
                // (BasicOperations.cpp:33-34, DGSEMIntegrator.cpp:467-481).
#pragma unroll
                for (int dd = 0; dd < DIM; dd++) {
                    s1[1 + dd] = s1[1 + dd] / s1[0];
                    s2[1 + dd] = s2[1 + dd] / s2[0];
                }
            }
            const double lf = face_flux<DIM>(s1, s2, d, o.nrm, P.gamma, P.gm1, P.gm1inv, compat, P.diss_scale, F);
            if (valid) lam = fmax(lam, lf);
            const double sc = C_FACE(c);
            buf[t * NV] = sc * (o.own_is_1 ? -F[0] : F[0]);
#pragma unroll
            for (int i = 0; i <= DIM; i++) {
                const double avg = (fo[i] + fnb[i]) * 0.5;
                const double fvn = avg * o.nrm;
                const double du = o.own_is_1 ? (-F[1 + i] + fvn) : (F[1 + i] - fvn);
                buf[t * NV + 1 + i] = sc * du;
            }
        }
        __syncwarp();
        gather_faces<DIM, N, G>(buf, gl, acc);
        if (valid) store_owned<DIM, N, G>(P, e, gl, us, acc);
        __syncwarp();
    }
    lam = group_max<32>(lam);
    if (lane == 0) atomic_max_pos(P.lam_bits, lam);
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(P.err, flags);
}

}  // namespace pdg
