// filter_kernels.cuh — entropy/positivity filter applied after an RK stage.
//
// Restates the intent of Prandtl's EntropyFilter (src/Filters/EntropyFilter.cpp:
// GetEntropyConstraints :81-158, FilterModes :160-169, FilterSolution :171-242,
// ComputeHierarchStates :244-260, ComputeRoot :325-349), which the reference
// declares but never constructs: the element bound is the minimum of the
// specific-entropy function rho log(p rho^-gamma) over the element and its
// face neighbours at the stage input; an element whose new state has
// min rho < 1e-8, min p < 1e-8 or min entropy < bound - 1e-4 has its modes of
// maximum 1D degree j scaled by exp(-zeta j^2), with zeta grown node by node
// (in node order) by 20 bisection steps on [zeta, -ln 1e-10] wherever the
// filtered node state still violates a constraint.
#pragma once

#include "line_kernels.cuh"

namespace pdg {

constexpr double FILTER_RHO_MIN = 1e-8, FILTER_P_MIN = 1e-8, FILTER_ENT_TOL = 1e-4, FILTER_EPS = 1e-10;
constexpr int FILTER_ITERS = 20;

// Pressure and entropy function as the filter evaluates them
// (EntropyFilter.cpp:95-110): velocities by division, +inf entropy for a
// non-positive density or pressure so that such nodes never lower a bound.
template <int DIM> __device__ __forceinline__ double filter_pressure(const double *s, double gm1)
{
    double vv = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const double v = s[1 + d] / s[0];
        vv += v * v;
    }
    return gm1 * (s[DIM + 1] - 0.5 * s[0] * vv);
}
__device__ __forceinline__ double filter_entropy(double rho, double p, double gamma)
{
    return (rho > 0.0 && p > 0.0) ? rho * log(p * pow(rho, -gamma)) : __longlong_as_double(0x7ff0000000000000LL);
}

template <int DIM, int N> struct FilterShape {
    using S = Shape<DIM, N>;
    // per-warp slot: state [NV][NDOF], ping-pong buffer [NV][NDOF],
    // hierarchical states [NDOF][Np][NV]
    static constexpr int EL = 2 * S::NV * S::NDOF + S::NDOF * S::Np * S::NV;
};

// Per-element minimum of the entropy function at the stage input (one warp
// per element) — the element's own part of the filter bound.
template <int DIM, int N>
__global__ void __launch_bounds__(256) filter_bounds_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int NDOF = S::NDOF, NV = S::NV;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t e = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < P.ne; e += warps) {
        double mn = __longlong_as_double(0x7ff0000000000000LL);
        for (int n = lane; n < NDOF; n += 32) {
            double s[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) s[v] = __ldg(P.u + (int64_t)v * P.nnodes + e * NDOF + n);
            mn = fmin(mn, filter_entropy(s[0], filter_pressure<DIM>(s, P.gm1), P.gamma));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        if (lane == 0) P.ent_own[e] = mn;
    }
}

// Filtered state of one node: hs[0] + sum_j hs[j] exp(-zeta j^2).
template <int DIM, int N>
__device__ __forceinline__ void filter_node_state(const double *hs, double zeta, double *st)
{
    constexpr int Np = N + 1, NV = DIM + 2;
#pragma unroll
    for (int v = 0; v < NV; v++) st[v] = hs[v];
#pragma unroll
    for (int j = 1; j < Np; j++) {
        const double fac = exp(-zeta * (double)(j * j));
#pragma unroll
        for (int v = 0; v < NV; v++) st[v] += hs[j * NV + v] * fac;
    }
}

template <int DIM>
__device__ __forceinline__ bool filter_violates(const double *st, double bound, double gamma, double gm1)
{
    const double rho = st[0], p = filter_pressure<DIM>(st, gm1);
    const double en = filter_entropy(rho, p, gamma);
    return rho < FILTER_RHO_MIN || p < FILTER_P_MIN || en < bound - FILTER_ENT_TOL;
}

// One warp per element over the stage output P.out (in place).
template <int DIM, int N>
__global__ void __launch_bounds__(128) filter_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    using F = FilterShape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *V1 = smem;                      // 1D Legendre Vandermonde V1[i*Np + k] = L_k(x_i)
    double *Vi = smem + 36;                 // its inverse, Vi[k*Np + i]
    for (int t = threadIdx.x; t < 36; t += blockDim.x) {
        V1[t] = P.K->V1[t];
        Vi[t] = P.K->Vinv1[t];
    }
    __syncthreads();
    double *xs = smem + CONST_SLOTS + (size_t)warp * F::EL;  // [NV][NDOF]
    double *tb = xs + NV * NDOF;                              // [NV][NDOF]
    double *hs = tb + NV * NDOF;                              // [NDOF][Np][NV]
    const int64_t nn = P.nnodes;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    for (int64_t e = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; e < P.ne; e += warps) {
        double mr = inf, mp = inf, me = inf;
        for (int n = lane; n < NDOF; n += 32) {
            double s[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                s[v] = P.out[v * nn + e * NDOF + n];
                xs[v * NDOF + n] = s[v];
            }
            const double p = filter_pressure<DIM>(s, P.gm1);
            me = fmin(me, filter_entropy(s[0], p, P.gamma));
            mr = fmin(mr, s[0]);
            mp = fmin(mp, p);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mr = fmin(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            mp = fmin(mp, __shfl_xor_sync(0xffffffffu, mp, o));
            me = fmin(me, __shfl_xor_sync(0xffffffffu, me, o));
        }
        double bound = P.ent_own[e];
#pragma unroll
        for (int f = 0; f < 2 * DIM; f++) {
            const int32_t nb = P.nbr[e * 2 * DIM + f];
            if (nb >= 0) bound = fmin(bound, P.ent_own[nb]);  // boundary faces have no neighbour
        }
        // NaN-safe: the element is filtered only when a constraint is met as false
        if (!(mr < FILTER_RHO_MIN || mp < FILTER_P_MIN || me < bound - FILTER_ENT_TOL)) {
            __syncwarp();
            continue;
        }
        if (lane == 0) atomicAdd(P.filter_count, 1ull);
        __syncwarp();
        // modes m = (Vi x Vi [x Vi]) x per variable, one 1D pass per direction
        double *src = xs, *dst = tb;
#pragma unroll 1
        for (int d = 0; d < DIM; d++) {
            const int stride = d == 0 ? 1 : (d == 1 ? Np : Np * Np);
            for (int t = lane; t < NV * NDOF; t += 32) {
                const int v = t / NDOF, n = t - v * NDOF;
                const int k = (n / stride) % Np, base = n - k * stride;
                double acc = 0.0;
#pragma unroll
                for (int l = 0; l < Np; l++) acc += Vi[k * Np + l] * src[v * NDOF + base + l * stride];
                dst[v * NDOF + n] = acc;
            }
            __syncwarp();
            double *tmp = src;
            src = dst;
            dst = tmp;
        }
        const double *m = src;
        // hierarchical states of every node: hs[n][j] = sum over modes t of
        // maximum degree j of V(n, t) m(t)
        for (int n = lane; n < NDOF; n += 32) {
            const int ni = n % Np, nj = (n / Np) % Np, nk = DIM == 3 ? n / (Np * Np) : 0;
            double *h = hs + n * Np * NV;
            for (int t = 0; t < Np * NV; t++) h[t] = 0.0;
            for (int t = 0; t < NDOF; t++) {
                const int ti = t % Np, tj = (t / Np) % Np, tk = DIM == 3 ? t / (Np * Np) : 0;
                int j = ti > tj ? ti : tj;
                double w = V1[ni * Np + ti] * V1[nj * Np + tj];
                if (DIM == 3) {
                    j = j > tk ? j : tk;
                    w *= V1[nk * Np + tk];
                }
#pragma unroll
                for (int v = 0; v < NV; v++) h[j * NV + v] += w * m[v * NDOF + t];
            }
        }
        __syncwarp();
        // zeta grows node by node in node order; the first node (at or after
        // `start`) that violates at the current zeta is bisected by every
        // lane alike, so zeta stays warp-uniform
        double zeta = 0.0;
        int start = 0;
        for (int guard = 0; guard <= NDOF; guard++) {
            int first = NDOF;
            for (int n = lane; n < NDOF; n += 32) {
                if (n < start || first < NDOF) continue;
                double st[NV];
                filter_node_state<DIM, N>(hs + n * Np * NV, zeta, st);
                if (filter_violates<DIM>(st, bound, P.gamma, P.gm1)) first = n;
            }
            first = __reduce_min_sync(0xffffffffu, first);
            if (first >= NDOF) break;
            double z1 = zeta, z2 = -log(FILTER_EPS);
            for (int it = 0; it < FILTER_ITERS; it++) {
                const double z3 = 0.5 * (z1 + z2);
                double st[NV];
                filter_node_state<DIM, N>(hs + first * Np * NV, z3, st);
                if (filter_violates<DIM>(st, bound, P.gamma, P.gm1)) z1 = z3;
                else z2 = z3;
            }
            zeta = z2;
            start = first + 1;
        }
        for (int n = lane; n < NDOF; n += 32) {
            double st[NV];
            filter_node_state<DIM, N>(hs + n * Np * NV, zeta, st);
#pragma unroll
            for (int v = 0; v < NV; v++) P.out[v * nn + e * NDOF + n] = st[v];
        }
        __syncwarp();
    }
}

}  // namespace pdg

namespace pdg {

// ---------------------------------------------------------------------------
// Positivity-preserving limiter after an RK stage (params.filter & 2).  The
// reference's MinmodLimiter::LimitSolution limits nothing
// (src/Limiters/MinmodLimiter.cpp:22-77) and it has no positivity limiter;
// this is the published limiter of Zhang & Shu (J. Comput. Phys. 229 (2010)
// 8918-8934).  Per element, with the LGL means u_bar and
// eps = min(1e-13, rho_bar, p(u_bar)):
//   (1) rho_i <- rho_bar + th1 (rho_i - rho_bar), th1 = (rho_bar - eps) /
//       (rho_bar - min rho_i), when min rho_i < eps;
//   (2) u_i <- u_bar + th2 (u_i - u_bar), th2 = min over nodes with
//       p(u_i) < eps of (p_bar - eps) / (p_bar - p(u_i)), which the concavity
//       of p in u makes a lower bound of p along the contraction (the exact
//       root of p = eps is ill-conditioned where step (1) left a node almost
//       empty, and its rounding can leave p below zero).
// The means are unchanged, so the limiter conserves; nodes of an element it
// leaves alone keep their bits.
// ---------------------------------------------------------------------------
constexpr double POSITIVITY_EPS = 1e-13;

// One warp per element over the stage output P.out (in place); counts the
// elements it changes in P.limit_count.
template <int DIM, int N>
__global__ void __launch_bounds__(256) positivity_kernel(const KParams P)
{
    using S = Shape<DIM, N>;
    constexpr int Np = S::Np, NDOF = S::NDOF, NV = S::NV;
    __shared__ double w[8];
    if (threadIdx.x < Np) w[threadIdx.x] = P.K->w[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t nn = P.nnodes;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    unsigned long long limited = 0;
    for (int64_t e = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < P.ne; e += warps) {
        double *x = P.out + e * NDOF;
        double m[NV], W = 0.0, rmin = inf;
#pragma unroll
        for (int v = 0; v < NV; v++) m[v] = 0.0;
        for (int n = lane; n < NDOF; n += 32) {
            double wn = w[n % Np] * w[(n / Np) % Np];
            if (DIM == 3) wn *= w[n / (Np * Np)];
            if (P.geo) wn *= __ldg(P.geo + e * NDOF + n);  // general geometry: the J-weighted mean
            W += wn;
#pragma unroll
            for (int v = 0; v < NV; v++) m[v] += wn * x[v * nn + n];
            rmin = fmin(rmin, x[n]);
        }
        W = group_sum<32>(W);
#pragma unroll
        for (int v = 0; v < NV; v++) m[v] = group_sum<32>(m[v]) / W;
        rmin = group_max<32>(-rmin) * -1.0;
        const double pbar = filter_pressure<DIM>(m, P.gm1);
        const double eps = fmin(POSITIVITY_EPS, fmin(m[0], pbar));
        bool lim = false;
        if (rmin < eps) {
            const double th = (m[0] - eps) / (m[0] - rmin);
            for (int n = lane; n < NDOF; n += 32) x[n] = m[0] + th * (x[n] - m[0]);
            lim = true;
        }
        double th2 = 1.0;
        for (int n = lane; n < NDOF; n += 32) {
            double s[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) s[v] = x[v * nn + n];
            const double p = filter_pressure<DIM>(s, P.gm1);
            if (p < eps) th2 = fmin(th2, (pbar - eps) / (pbar - p));
        }
        th2 = -group_max<32>(-th2);
        if (th2 < 1.0) {
            for (int n = lane; n < NDOF; n += 32)
#pragma unroll
                for (int v = 0; v < NV; v++) x[v * nn + n] = m[v] + th2 * (x[v * nn + n] - m[v]);
            lim = true;
        }
        if (lane == 0 && lim) limited++;
        __syncwarp();
    }
    if (lane == 0 && limited) atomicAdd(P.limit_count, limited);
}

}  // namespace pdg
