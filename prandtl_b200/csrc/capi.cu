// capi.cu — host side of the C ABI declared in include/prandtl_b200.h.
//
// A pdg_ctx plays the role of the reference's DGSEMOperator + DGSEMIntegrator
// + PerssonPeraireIndicator objects (src/Operators/DGSEMOperator.cpp:5-50,
// src/Integrators/DGSEMIntegrator/DGSEMIntegrator.cpp:8-149): it owns the
// LGL operators, the subcell metrics, the modal transform, the neighbour
// table and all scratch (blending coefficients, gradient fields, RK stage
// buffers, the running wave-speed maximum and the error word) in device
// memory.  Every call is asynchronous on the caller's stream unless stated.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/prandtl_b200.h"
#include "line_kernels.cuh"
#include "host_common.h"
#include "kernel_table.h"

using namespace pdg;

struct pdg_ctx {
    pdg_params p;
    int dim, N, Np, ndof, nv;
    int64_t ne, nnodes, size;
    double h[3];
    double hmin;
    double modal_threshold;
    DevConst hK;
    // device memory
    DevConst *K = nullptr;
    int32_t *nbr = nullptr;
    double *eta = nullptr, *alpha = nullptr;
    double *lbuf = nullptr;                         // BR1 lifting jumps [d][e][fn][v]
    double *fcol = nullptr;                         // viscous normal columns at faces
    double *vbuf = nullptr;                         // viscous volume term [v-1][node] (element-side faces)
    double *fbuf = nullptr;                         // inviscid face fluxes [d][e][v][fn] (element-side faces)
    // boundary conditions: host table, its device copy, which entries the
    // mesh uses and which pdg_set_boundary has set
    double bc_host[PDG_MAX_BOUNDARIES * BC_SLOT] = {};
    double *bc = nullptr;
    unsigned int bc_used = 0, bc_set = 0;
    double *lbuf_lo = nullptr;  // NS boundary faces: BR1 jumps of -d boundary faces
    double *stage_a = nullptr, *stage_b = nullptr;  // RK stage buffers
    double *io_a = nullptr, *io_b = nullptr;        // host-path staging
    unsigned long long *lam_bits = nullptr;
    unsigned int *err = nullptr;
    double *ent_own = nullptr;                // filter: per-element entropy minimum at the stage input
    unsigned long long *filter_count = nullptr;
    unsigned long long *limit_count = nullptr;  // positivity limiter applications
    double *gcol = nullptr;   // adjoint: cotangents of the face-normal entropy gradients
    double *gbuf = nullptr;   // adjoint: face-term cotangents of both sides of every face node
    // pdg_rk3_steps: one step captured in a CUDA graph for a (state, dt) pair
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double *graph_u = nullptr;
    double graph_dt = 0.0;
    int64_t graph_launches = 0;
    bool adj_ready = false;
    // launch configuration per kernel kind
    KernelInfo kinfo[KIND_COUNT];
    int wpb[KIND_COUNT];
    int grid[KIND_COUNT];
    size_t smem[KIND_COUNT];
    int64_t launches = 0;
    int prefetch = 1;  // PDG_PREFETCH=0 in the environment turns the L2 prefetch off
    // fixed operator: face terms inside the volume kernel, each face evaluated
    // by both of its elements (PDG_ELEMENT_FACES=0: separate face kernels)
    bool element_faces = true;
    // periodic fixed operator: every face's inviscid flux evaluated once into
    // fbuf by the face-node kernel, read by both elements' volume kernels
    // (PDG_FACE_BUFFER=0: each element evaluates its faces itself)
    bool face_buffer = true;
    bool profile = false;
    struct TimedLaunch { int kind; cudaEvent_t a, b; };
    std::vector<TimedLaunch> timed;
    std::vector<cudaEvent_t> event_pool;
    cudaStream_t last_stream = 0;
    // pdg_rk3_step_host's pipeline: element chunks, the chunks holding each
    // chunk's face neighbours, copy and compute streams and their events
    struct HostPipe {
        bool ready = false, usable = false;
        std::vector<int64_t> bounds;          // chunk k = elements [bounds[k], bounds[k + 1])
        std::vector<std::vector<int>> near;   // chunks holding chunk k's elements and their face neighbours
        cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
        std::vector<cudaEvent_t> ev_in, ev_done;
        cudaEvent_t ev_start = nullptr;
    } pipe;
    int device = 0;
    std::string last_error;
    std::vector<int32_t> nbr_host;  // the neighbour table as given (the host step's pipeline reads it)
    // general geometry (pdg_set_geometry): per node J and adjugate rows, per
    // element face node the neighbour's matching node and element 1's normal
    bool geo = false;
    double *geo_d = nullptr;
    int32_t *fnode_d = nullptr;
    double *fnor_d = nullptr;
    double *geo_grads = nullptr;  // (unused: the primitive gradients go only to pdg_gradients' buffer)
    double *geo_fv = nullptr;     // Navier-Stokes: contravariant viscous fluxes [d][row][node]
    double *geo_cf = nullptr;     // Navier-Stokes: viscous flux . face normal [e][face][face node][row]
    int32_t *fpart_d = nullptr;   // the neighbour's face-node slot of every face node (-1: boundary)
};

namespace {

int fail(pdg_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->last_error = buf;
    }
    return code;
}

int cuda_fail(pdg_ctx *c, cudaError_t e, const char *what)
{
    return fail(c, PDG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                                                                             \
    do {                                                                                                           \
        cudaError_t _e = (call);                                                                                   \
        if (_e != cudaSuccess) return cuda_fail(c, _e, what);                                                      \
    } while (0)

// ---- one-dimensional operators (same mathematics as the reference's
// DGSEMIntegrator constructor, DGSEMIntegrator.cpp:41-82) ----

void legendre(int n, long double x, long double &P, long double &dP)
{
    long double p0 = 1.0L, p1 = x;
    if (n == 0) { P = 1.0L; dP = 0.0L; return; }
    for (int k = 1; k < n; k++) {
        long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
        p0 = p1;
        p1 = p2;
    }
    P = p1;
    dP = (std::fabs(x) == 1.0L) ? 0.0L : n * (x * p1 - p0) / (x * x - 1.0L);
}

// Gauss-Lobatto nodes/weights on [0,1]: interior nodes are the roots of P_N'
// (Newton's method in long double from Chebyshev-Lobatto guesses), weights
// 1/(N(N+1) P_N^2); mirrored so x[N-i] = 1 - x[i].
void gauss_lobatto(int Np, double *x, double *w)
{
    const int N = Np - 1;
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i <= N / 2; i++) {
        long double t = -1.0L;
        if (i > 0) {
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
        x[i] = (double)(0.5L * (1.0L + t));
        w[i] = (double)(1.0L / (N * (N + 1) * P * P));
        x[N - i] = 1.0 - x[i];
        w[N - i] = w[i];
    }
    if (N % 2 == 0) x[N / 2] = 0.5;
}

}  // namespace

namespace pdg_host {

void fill_constants(int dim, int N, const double *h, DevConst &K, double &modal_threshold)
{
    std::memset(&K, 0, sizeof(K));
    const int Np = N + 1;
    double x[6], w[6];
    gauss_lobatto(Np, x, w);
    // barycentric weights and the differentiation matrix D_il = l_l'(x_i)
    double wb[6];
    for (int i = 0; i < Np; i++) wb[i] = 1.0;
    for (int i = 1; i < Np; i++)
        for (int j = 0; j < i; j++) {
            wb[j] *= (x[j] - x[i]);
            wb[i] *= (x[i] - x[j]);
        }
    for (int i = 0; i < Np; i++) wb[i] = 1.0 / wb[i];
    double D[36] = {0};
    for (int l = 0; l < Np; l++)
        for (int i = 0; i < Np; i++)
            if (l != i) {
                D[i * Np + l] = wb[l] / wb[i] / (x[i] - x[l]);
                D[i * Np + i] -= D[i * Np + l];
            }
    for (int t = 0; t < Np * Np; t++) {
        K.D[t] = D[t];
        K.Dhat[t] = D[t];
        K.Dhat2[t] = D[t] * 2.0;
    }
    K.Dhat[0] += 1.0 / w[0];
    K.Dhat[Np * Np - 1] -= 1.0 / w[Np - 1];
    K.Dhat2[0] += 1.0 / w[0];
    K.Dhat2[Np * Np - 1] -= 1.0 / w[Np - 1];
    for (int i = 0; i < Np; i++) K.w[i] = w[i];
    // affine element: J = prod h, adj = diag(J / h_d), face area = J / h_d
    if (dim == 2) {
        K.J = h[0] * h[1];
        K.adj[0] = h[1];
        K.adj[1] = h[0];
    } else {
        K.J = h[0] * (h[1] * h[2]);
        K.adj[0] = h[1] * h[2];
        K.adj[1] = h[0] * h[2];
        K.adj[2] = h[0] * h[1];
    }
    for (int d = 0; d < dim; d++) K.area[d] = K.adj[d];
    K.invJ = 1.0 / K.J;
    K.face_scale = 1.0 / (w[0] * K.J);
    for (int i = 0; i < Np; i++) K.fv_scale[i] = 1.0 / (K.J * w[i]);
    // subcell interface normals (ComputeSubcellMetrics, DGSEMIntegrator.cpp:
    // 1199-1304): adj_d + sum_{l<i} w_l sum_m D(l,m) adj_d on an affine element
    for (int d = 0; d < dim; d++)
        for (int i = 0; i <= Np; i++) {
            double nor = K.adj[d];
            for (int l = 0; l < i; l++) {
                double tmp = 0.0;
                for (int m = 0; m < Np; m++) tmp += K.adj[d] * D[l * Np + m];
                nor += tmp * w[l];
            }
            K.snor[d][i] = nor;
        }
    // 1D Legendre Vandermonde on the nodes and its inverse; the tensor-product
    // modal transform of ModalBasis (ModalBasis.cpp:110-150) factors into it.
    double V[36], I[36] = {0};
    for (int i = 0; i < Np; i++) {
        double z = 2.0 * x[i] - 1.0, L[6];
        L[0] = 1.0;
        if (Np > 1) L[1] = z;
        for (int n = 1; n + 1 < Np; n++) L[n + 1] = ((2 * n + 1) * z * L[n] - n * L[n - 1]) / (n + 1);
        for (int k = 0; k < Np; k++) V[i * Np + k] = L[k];
    }
    for (int t = 0; t < Np * Np; t++) K.V1[t] = V[t];
    for (int i = 0; i < Np; i++) I[i * Np + i] = 1.0;
    for (int col = 0; col < Np; col++) {  // Gauss-Jordan with partial pivoting
        int piv = col;
        for (int r = col + 1; r < Np; r++)
            if (std::fabs(V[r * Np + col]) > std::fabs(V[piv * Np + col])) piv = r;
        for (int k = 0; k < Np; k++) {
            std::swap(V[piv * Np + k], V[col * Np + k]);
            std::swap(I[piv * Np + k], I[col * Np + k]);
        }
        const double inv = 1.0 / V[col * Np + col];
        for (int k = 0; k < Np; k++) {
            V[col * Np + k] *= inv;
            I[col * Np + k] *= inv;
        }
        for (int r = 0; r < Np; r++)
            if (r != col) {
                const double f = V[r * Np + col];
                for (int k = 0; k < Np; k++) {
                    V[r * Np + k] -= f * V[col * Np + k];
                    I[r * Np + k] -= f * I[col * Np + k];
                }
            }
    }
    for (int t = 0; t < Np * Np; t++) K.Vinv1[t] = I[t];  // Vinv1[k*Np + i]: mode k from node i
    modal_threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)N, 0.25));
}

int kernel_config(int dim, int N, int kind, int64_t ne, int device, LaunchCfg *cfg, const char **why)
{
    KernelInfo &ki = cfg->ki;
    const bool ok = dim == 2 ? kernel_info_2d(N, kind, &ki) : kernel_info_3d(N, kind, &ki);
    if (!ok) { *why = "no kernel for this dimension and order"; return PDG_ERR_UNSUPPORTED; }
    int max_smem = 0, sms = 0;
    if (cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        *why = "device attribute query failed";
        return PDG_ERR_CUDA;
    }
    const int Np = N + 1, nfn = dim == 2 ? Np : Np * Np;
    if (ki.el_doubles == 0) {  // thread-per-face-node kernel
        const int64_t threads = (kind == KIND_FILTER_BOUNDS || kind == KIND_POSITIVITY) ? 32 * ne
                                : (kind == KIND_BOUNDARY || kind == KIND_ADJ_BOUNDARY || kind == KIND_BOUNDARY_NS) ? ne
                                : kind == KIND_ADJ_GATHER ? ne * nfn * (N + 1)  // thread per node
                                : ((kind == KIND_LIFT_FACE || kind == KIND_LIFT_FACE_BDR || kind == KIND_LIFT_FACE_FLUX ||
                                    kind == KIND_FACE_FLUX || kind == KIND_ADJ_FACE_E0 || kind == KIND_ADJ_FACE_NS0)
                                       ? (int64_t)dim : 1) * ne * nfn;
        // 256-thread blocks; 128 when that gives fewer than four blocks per
        // SM, so that a small mesh still spreads evenly over the SMs
        cfg->wpb = threads < 4LL * 256 * sms ? 4 : 8;
        const int bs = 32 * cfg->wpb;
        int blocks_per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, ki.fn, bs, 0) != cudaSuccess) {
            *why = "occupancy query failed";
            return PDG_ERR_CUDA;
        }
        cfg->grid = (int)std::max<int64_t>(1, std::min<int64_t>((threads + bs - 1) / bs, (int64_t)sms * std::max(1, blocks_per_sm)));
        cfg->smem = 0;
        return PDG_OK;
    }
    const size_t per_warp = (size_t)ki.epw * ki.el_doubles * sizeof(double);
    const size_t base = (size_t)(kind == KIND_FILTER ? CONST_SLOTS : const_slots(Np)) * sizeof(double);
    int wpb = std::max(1, std::min(4, ki.wpb));
    while (wpb > 1 && base + wpb * per_warp > (size_t)max_smem) wpb--;
    if (base + wpb * per_warp > (size_t)max_smem) { *why = "element does not fit in shared memory"; return PDG_ERR_UNSUPPORTED; }
    const size_t smem = base + wpb * per_warp;
    if (cudaFuncSetAttribute(ki.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        *why = "shared-memory attribute failed";
        return PDG_ERR_CUDA;
    }
    int blocks_per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, ki.fn, 32 * wpb, smem) != cudaSuccess) {
        *why = "occupancy query failed";
        return PDG_ERR_CUDA;
    }
    if (blocks_per_sm < 1) { *why = "kernel cannot be resident"; return PDG_ERR_UNSUPPORTED; }
    const int64_t nwt = (ne + ki.epw - 1) / ki.epw;
    const int64_t need = (nwt + wpb - 1) / wpb;
    cfg->wpb = wpb;
    cfg->grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms * blocks_per_sm));
    cfg->smem = smem;
    return PDG_OK;
}

bool kind_used(int kind, int dim, bool parabolic, int filter)
{
    if (kind == KIND_FILTER_BOUNDS || kind == KIND_FILTER) return filter & 1;
    if (kind == KIND_POSITIVITY) return (filter & 2) != 0;
    if (kind == KIND_GEO || kind == KIND_GEO_LIFT || kind == KIND_GEO_NS) return false;  // configured by pdg_set_geometry
    if ((kind >= KIND_ADJ_RHS && kind <= KIND_ADJ_FACE_NS2) || kind == KIND_ADJ_BOUNDARY)
        return false;  // configured by the first pdg_rhs_vjp
    const bool ns_kind = kind == KIND_NS || kind == KIND_NS_FACES || kind == KIND_LIFT || kind == KIND_LIFT_FACE ||
                         (kind >= KIND_FACE_NS0 && kind <= KIND_FACE_NS2) || kind == KIND_LIFT_FACE_BDR ||
                         kind == KIND_NS_FACES_FB || kind == KIND_LIFT_FACE_FLUX ||
                         kind == KIND_LIFT_BDR || kind == KIND_NS_FACES_BDR || kind == KIND_BOUNDARY_NS ||
                         kind == KIND_LIFT_BDR_PTTT;
    if (ns_kind != parabolic) return false;
    if (kind == KIND_LIFT_BDR_PTTT && dim != 2) return false;
    if ((kind == KIND_FACE_E2 || kind == KIND_FACE_NS2) && dim < 3) return false;
    return true;
}

int launch_kernel(const LaunchCfg &cfg, KParams P, int64_t ne, cudaStream_t s)
{
    P.nwt = (ne + cfg.ki.epw - 1) / cfg.ki.epw;
    void *args[] = {&P};
    return cudaLaunchKernel(cfg.ki.fn, dim3(cfg.grid), dim3(32 * cfg.wpb), args, cfg.smem, s) == cudaSuccess
               ? PDG_OK
               : PDG_ERR_CUDA;
}

}  // namespace pdg_host

namespace {
using namespace pdg_host;

void build_constants(pdg_ctx *c)
{
    fill_constants(c->dim, c->N, c->h, c->hK, c->modal_threshold);
}

int configure_launch(pdg_ctx *c, int kind)
{
    LaunchCfg cfg;
    const char *why = "";
    const int r = kernel_config(c->dim, c->N, kind, c->ne, c->device, &cfg, &why);
    if (r) return fail(c, r, "%s (dim=%d order=%d kernel %d)", why, c->dim, c->N, kind);
    c->kinfo[kind] = cfg.ki;
    c->wpb[kind] = cfg.wpb;
    c->grid[kind] = cfg.grid;
    c->smem[kind] = cfg.smem;
    return PDG_OK;
}

KParams base_params(pdg_ctx *c)
{
    KParams P;
    std::memset(&P, 0, sizeof(P));
    P.nbr = c->nbr;
    P.lbuf = c->lbuf;
    P.fcol = c->fcol;
    P.K = c->K;
    P.eta_out = c->eta;
    P.alpha_out = c->alpha;
    P.lam_bits = c->lam_bits;
    P.err = c->err;
    P.ent_own = c->ent_own;
    P.filter_count = c->filter_count;
    P.limit_count = c->limit_count;
    P.ne = c->ne;
    P.nnodes = c->nnodes;
    P.stage = -1;
    P.gamma = c->p.gamma;
    P.gm1 = c->p.gamma - 1.0;
    P.gm1inv = 1.0 / P.gm1;
    P.mu = c->p.mu;
    P.lambda_k = c->p.mu * c->p.gamma * (1.0 / c->p.Pr);
    P.alpha_max = c->p.alpha_max;
    P.alpha_min = c->p.alpha_min;
    P.modal_threshold = c->modal_threshold;
    P.diss_scale = c->p.face_dissipation;
    P.blending = c->p.blending;
    P.compat = c->p.compat;
    P.prefetch = c->prefetch;
    P.bc = c->bc;
    P.has_bdr = c->bc_used != 0;
    P.lbuf_lo = c->lbuf_lo;
    P.fbuf = c->fbuf;
    P.geo = c->geo_d;
    P.fnode = c->fnode_d;
    P.fnor = c->fnor_d;
    P.geo_grads = c->geo_grads;
    P.geo_fv = c->geo_fv;
    P.geo_cf = c->geo_cf;
    P.fpart = c->fpart_d;
    return P;
}

cudaEvent_t pooled_event(pdg_ctx *c)
{
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

int launch(pdg_ctx *c, int kind, KParams P, cudaStream_t s)
{
    const KernelInfo &ki = c->kinfo[kind];
    if (!ki.fn || ki.epw < 1) return fail(c, PDG_ERR_UNSUPPORTED, "kernel %d is not configured", kind);
    const int64_t range = (P.e_end ? P.e_end : c->ne) - P.e_begin;  // element range (whole mesh by default)
    P.nwt = (range + ki.epw - 1) / ki.epw;
    void *args[] = {&P};
    cudaEvent_t ea = nullptr, eb = nullptr;
    if (c->profile) {
        ea = pooled_event(c);
        eb = pooled_event(c);
        if (!ea || !eb) return fail(c, PDG_ERR_CUDA, "event creation failed");
        CK(cudaEventRecord(ea, s), "event record");
    }
    CK(cudaLaunchKernel(ki.fn, dim3(c->grid[kind]), dim3(32 * c->wpb[kind]), args, c->smem[kind], s), "kernel launch");
    if (c->profile) {
        CK(cudaEventRecord(eb, s), "event record");
        c->timed.push_back({kind, ea, eb});
    }
    c->launches++;
    return PDG_OK;
}

// Launch of a kernel whose arguments follow the KParams (adjoint kernels).
int launch_with(pdg_ctx *c, int kind, KParams P, void *a1, void *a2, void *a3, cudaStream_t s)
{
    const KernelInfo &ki = c->kinfo[kind];
    if (!ki.fn || ki.epw < 1) return fail(c, PDG_ERR_UNSUPPORTED, "kernel %d is not configured", kind);
    P.nwt = (c->ne + ki.epw - 1) / ki.epw;
    void *args[] = {&P, a1, a2, a3};
    cudaEvent_t ea = nullptr, eb = nullptr;
    if (c->profile) {
        ea = pooled_event(c);
        eb = pooled_event(c);
        if (!ea || !eb) return fail(c, PDG_ERR_CUDA, "event creation failed");
        CK(cudaEventRecord(ea, s), "event record");
    }
    CK(cudaLaunchKernel(ki.fn, dim3(c->grid[kind]), dim3(32 * c->wpb[kind]), args, c->smem[kind], s), "kernel launch");
    if (c->profile) {
        CK(cudaEventRecord(eb, s), "event record");
        c->timed.push_back({kind, ea, eb});
    }
    c->launches++;
    return PDG_OK;
}

// BR1 lifting of state u: face jumps, then gradients (to grads_out when it
// is not null) and, with P.out set, the viscous volume term added to the
// output and the face columns of the viscous flux.
// The lifting kernel of a Navier-Stokes mesh with boundary faces: the
// total-pressure inflow has its own instantiation.
int lift_bdr_kind(const pdg_ctx *c)
{
    for (int b = 0; b < PDG_MAX_BOUNDARIES; b++)
        if ((c->bc_used >> b & 1u) && (int)c->bc_host[b * BC_SLOT] == PDG_BC_SUBSONIC_INFLOW_PTTT)
            return KIND_LIFT_BDR_PTTT;
    return KIND_LIFT_BDR;
}

int lift(pdg_ctx *c, KParams P, const double *u, double *grads_out, cudaStream_t s)
{
    P.u = u;
    P.grads_out = grads_out;
    if (c->bc_used && (c->bc_used & ~c->bc_set))
        return fail(c, PDG_ERR_ARG, "a boundary condition the mesh uses is not set (pdg_set_boundary)");
    int r = launch(c, c->bc_used ? KIND_LIFT_FACE_BDR : KIND_LIFT_FACE, P, s);
    if (r) return r;
    return launch(c, c->bc_used ? lift_bdr_kind(c) : KIND_LIFT, P, s);
}

// RHS (stage < 0) or fused SSP-RK3 stage of the operator on device buffers.
// Fixed operator: (NS: BR1 face jumps, then the lifting kernel, which stores
// the viscous volume term to vbuf and the face columns to fcol) one volume
// kernel that also evaluates every face from both sides and writes the
// finished output.  Reference-value operator (or PDG_ELEMENT_FACES=0): the
// volume kernel writes the output, the lifting kernel (NS) and the face
// kernels of each direction add their terms.
int evaluate(pdg_ctx *c, int stage, double dt, const double *un, const double *us, double *out, cudaStream_t s)
{
    if (c->bc_used & ~c->bc_set) {
        for (int b = 0; b < PDG_MAX_BOUNDARIES; b++)
            if ((c->bc_used & ~c->bc_set) >> b & 1u)
                return fail(c, PDG_ERR_ARG, "boundary condition %d is used by the mesh but not set (pdg_set_boundary)", b);
    }
    if (!c->p.compat) CK(cudaMemsetAsync(c->lam_bits, 0, sizeof(unsigned long long), s), "reset wave speed");
    KParams P = base_params(c);
    P.u = us;
    P.un = un;
    P.out = out;
    P.stage = stage;
    P.dt = dt;
    c->last_stream = s;
    int r;
    if (c->geo) {
        // general geometry: one kernel (Navier-Stokes: the lifting kernel
        // first), with the filter's bounds before and the filter and the
        // positivity limiter after it, as on box meshes
        if (c->p.parabolic)
            for (int b = 0; b < PDG_MAX_BOUNDARIES; b++) {
                const int t = (int)c->bc_host[b * BC_SLOT];
                // as on box meshes: the reference has no viscous flux for the slip wall and the symmetry plane
                if ((c->bc_used >> b & 1u) && (t == PDG_BC_SLIP_WALL || t == PDG_BC_SYMMETRY))
                    return fail(c, PDG_ERR_UNSUPPORTED,
                                "boundary condition %d: type %d has no viscous boundary flux here", b, t);
            }
        if ((c->p.filter & 1) && stage >= 0 && (r = launch(c, KIND_FILTER_BOUNDS, P, s))) return r;
        if (!c->p.parabolic) {
            if ((r = launch(c, KIND_GEO, P, s))) return r;
        } else {
            if ((r = launch(c, KIND_GEO_LIFT, P, s))) return r;
            if ((r = launch(c, KIND_GEO_NS, P, s))) return r;
        }
        if ((c->p.filter & 1) && stage >= 0 && (r = launch(c, KIND_FILTER, P, s))) return r;
        if ((c->p.filter & 2) && stage >= 0 && (r = launch(c, KIND_POSITIVITY, P, s))) return r;
        return PDG_OK;
    }
    const bool element_faces = c->element_faces && !c->p.compat;
    if (c->p.parabolic) {
        if ((c->p.filter & 1) && stage >= 0 && (r = launch(c, KIND_FILTER_BOUNDS, P, s))) return r;
        if (c->bc_used) {
            // Navier-Stokes boundary faces: the conditions with a viscous boundary flux
            // slip wall and symmetry have no viscous flux in the reference
            // (BdrFaceIntegrator.cpp:260-273 raise mfem_error); the
            // reference-value Riemann invariants' lifting (a normal left from
            // another face) is not built
            for (int b = 0; b < PDG_MAX_BOUNDARIES; b++) {
                const int t = (int)c->bc_host[b * BC_SLOT];
                const bool ok = t == PDG_BC_SUPERSONIC_INFLOW || t == PDG_BC_SUPERSONIC_OUTFLOW ||
                                t == PDG_BC_SPECIFIED_STATE || t == PDG_BC_NOSLIP_ADIABATIC ||
                                t == PDG_BC_NOSLIP_ISOTHERMAL || t == PDG_BC_SUBSONIC_OUTFLOW_P ||
                                t == PDG_BC_SUBSONIC_INFLOW_RV || t == PDG_BC_SUBSONIC_INFLOW_PTTT ||
                                (t == PDG_BC_RIEMANN_INVARIANT && !c->p.compat);
                if ((c->bc_used >> b & 1u) && !ok)
                    return fail(c, PDG_ERR_UNSUPPORTED,
                                "boundary condition %d: type %d has no viscous boundary flux here", b, t);
            }
            if ((r = launch(c, KIND_LIFT_FACE_BDR, P, s))) return r;
            if (element_faces) {
                P.vbuf = c->vbuf;
                if ((r = launch(c, lift_bdr_kind(c), P, s))) return r;
                if ((r = launch(c, KIND_NS_FACES_BDR, P, s))) return r;
            } else {  // separate face passes, then the boundary faces
                if ((r = launch(c, KIND_NS, P, s))) return r;
                if ((r = launch(c, lift_bdr_kind(c), P, s))) return r;
                for (int d = 0; d < c->dim; d++)
                    if ((r = launch(c, KIND_FACE_NS0 + d, P, s))) return r;
                if ((r = launch(c, KIND_BOUNDARY_NS, P, s))) return r;
            }
        } else if (element_faces) {
            const bool fb = c->fbuf != nullptr;
            if ((r = launch(c, fb ? KIND_LIFT_FACE_FLUX : KIND_LIFT_FACE, P, s))) return r;
            P.vbuf = c->vbuf;
            if ((r = launch(c, KIND_LIFT, P, s))) return r;
            if ((r = launch(c, fb ? KIND_NS_FACES_FB : KIND_NS_FACES, P, s))) return r;
        } else {
            if ((r = launch(c, KIND_LIFT_FACE, P, s))) return r;
            if ((r = launch(c, KIND_NS, P, s))) return r;
            if ((r = launch(c, KIND_LIFT, P, s))) return r;
            for (int d = 0; d < c->dim; d++)
                if ((r = launch(c, KIND_FACE_NS0 + d, P, s))) return r;
        }
    } else {
        if ((c->p.filter & 1) && stage >= 0 && (r = launch(c, KIND_FILTER_BOUNDS, P, s))) return r;
        if (element_faces && c->fbuf) {
            if ((r = launch(c, KIND_FACE_FLUX, P, s))) return r;
            if ((r = launch(c, KIND_EULER_FACES_FB, P, s))) return r;
        } else if (element_faces) {
            if ((r = launch(c, c->bc_used ? KIND_EULER_FACES_BDR : KIND_EULER_FACES, P, s))) return r;
        } else {
            if ((r = launch(c, KIND_EULER, P, s))) return r;
            for (int d = 0; d < c->dim; d++)
                if ((r = launch(c, KIND_FACE_E0 + d, P, s))) return r;
            if (c->bc_used && (r = launch(c, KIND_BOUNDARY, P, s))) return r;
        }
    }
    // entropy filter of the stage output (EntropyFilter::FilterSolution), then
    // the positivity limiter
    if ((c->p.filter & 1) && stage >= 0 && (r = launch(c, KIND_FILTER, P, s))) return r;
    if ((c->p.filter & 2) && stage >= 0 && (r = launch(c, KIND_POSITIVITY, P, s))) return r;
    return PDG_OK;
}

}  // namespace

extern "C" {

void pdg_default_params(pdg_params *p)
{
    if (!p) return;
    p->parabolic = 0;
    p->blending = 1;
    p->compat = 1;
    p->filter = 0;
    p->gamma = 1.4;
    p->Pr = 0.72;
    p->mu = 0.0;
    p->R_gas = 287.0;
    p->alpha_max = 0.5;
    p->alpha_min = 0.001;
    p->face_dissipation = 1.0;
}

int pdg_create(const pdg_mesh *mesh, const pdg_params *params, pdg_ctx **out)
{
    if (!out) return PDG_ERR_ARG;
    *out = nullptr;
    if (!mesh || !params || !mesh->nbr) return PDG_ERR_ARG;
    if ((mesh->dim != 2 && mesh->dim != 3) || mesh->order < 1 || mesh->order > 5 || mesh->num_elements < 1)
        return PDG_ERR_ARG;
    if (!(params->gamma > 1.0) || (params->parabolic && !(params->Pr > 0.0))) return PDG_ERR_ARG;
    if (params->filter < 0 || params->filter > 3) return PDG_ERR_ARG;
    pdg_ctx *c = new pdg_ctx();
    c->p = *params;
    c->dim = mesh->dim;
    c->N = mesh->order;
    c->Np = c->N + 1;
    c->ndof = c->dim == 2 ? c->Np * c->Np : c->Np * c->Np * c->Np;
    c->nv = c->dim + 2;
    c->ne = mesh->num_elements;
    c->nnodes = c->ne * c->ndof;
    c->size = c->nnodes * c->nv;
    c->hmin = 1e300;
    for (int d = 0; d < 3; d++) {
        c->h[d] = d < c->dim ? mesh->h[d] : 1.0;
        if (d < c->dim) {
            if (!(c->h[d] > 0.0)) { delete c; return PDG_ERR_ARG; }
            c->hmin = std::min(c->hmin, c->h[d]);
        }
    }
    for (int64_t i = 0; i < c->ne * 2 * c->dim; i++) {
        const int32_t nb = mesh->nbr[i];
        if (nb >= c->ne || nb < -PDG_MAX_BOUNDARIES) { delete c; return PDG_ERR_ARG; }
        if (nb < 0) c->bc_used |= 1u << (-1 - nb);
    }
    c->nbr_host.assign(mesh->nbr, mesh->nbr + c->ne * 2 * c->dim);
    auto cleanup = [&](int code) {
        pdg_destroy(c);
        return code;
    };
    if (cudaGetDevice(&c->device) != cudaSuccess) return cleanup(PDG_ERR_CUDA);
    if (const char *pf = std::getenv("PDG_PREFETCH")) c->prefetch = std::atoi(pf) != 0;
    if (const char *ef = std::getenv("PDG_ELEMENT_FACES")) c->element_faces = std::atoi(ef) != 0;
    if (const char *fb = std::getenv("PDG_FACE_BUFFER")) c->face_buffer = std::atoi(fb) != 0;
    build_constants(c);
    const size_t fbytes = sizeof(double) * (size_t)c->size;
    if (cudaMalloc(&c->K, sizeof(DevConst)) != cudaSuccess || cudaMalloc(&c->nbr, sizeof(int32_t) * c->ne * 2 * c->dim) ||
        cudaMalloc(&c->eta, sizeof(double) * c->ne) || cudaMalloc(&c->alpha, sizeof(double) * c->ne) ||
        cudaMalloc(&c->lam_bits, sizeof(unsigned long long)) || cudaMalloc(&c->err, sizeof(unsigned int)) ||
        cudaMalloc(&c->stage_a, fbytes) || cudaMalloc(&c->stage_b, fbytes) ||
        cudaMalloc(&c->bc, sizeof(double) * PDG_MAX_BOUNDARIES * BC_SLOT))
        return cleanup(PDG_ERR_NOMEM);
    if (cudaMemset(c->bc, 0, sizeof(double) * PDG_MAX_BOUNDARIES * BC_SLOT) != cudaSuccess) return cleanup(PDG_ERR_CUDA);
    if (c->p.filter & 1) {
        if (cudaMalloc(&c->ent_own, sizeof(double) * c->ne) != cudaSuccess ||
            cudaMalloc(&c->filter_count, sizeof(unsigned long long)) != cudaSuccess ||
            cudaMemset(c->filter_count, 0, sizeof(unsigned long long)) != cudaSuccess)
            return cleanup(PDG_ERR_NOMEM);
    }
    if (c->p.filter & 2) {
        if (cudaMalloc(&c->limit_count, sizeof(unsigned long long)) != cudaSuccess ||
            cudaMemset(c->limit_count, 0, sizeof(unsigned long long)) != cudaSuccess)
            return cleanup(PDG_ERR_NOMEM);
    }
    if (c->element_faces && c->face_buffer && !c->p.compat && !c->bc_used) {
        const size_t nfn = c->dim == 2 ? c->Np : c->Np * c->Np;
        if (cudaMalloc(&c->fbuf, sizeof(double) * c->dim * c->ne * nfn * c->nv) != cudaSuccess)
            return cleanup(PDG_ERR_NOMEM);
    }
    if (c->p.parabolic) {
        const size_t nfn = c->dim == 2 ? c->Np : c->Np * c->Np;
        if (cudaMalloc(&c->lbuf, sizeof(double) * c->dim * c->ne * nfn * c->nv) != cudaSuccess ||
            cudaMalloc(&c->fcol, sizeof(double) * 2 * c->dim * c->ne * nfn * (c->nv - 1)) != cudaSuccess ||
            cudaMalloc(&c->vbuf, sizeof(double) * (c->nv - 1) * c->nnodes) != cudaSuccess ||
            (c->bc_used && cudaMalloc(&c->lbuf_lo, sizeof(double) * c->dim * c->ne * nfn * c->nv) != cudaSuccess))
            return cleanup(PDG_ERR_NOMEM);
    }
    if (cudaMemcpy(c->K, &c->hK, sizeof(DevConst), cudaMemcpyHostToDevice) ||
        cudaMemcpy(c->nbr, mesh->nbr, sizeof(int32_t) * c->ne * 2 * c->dim, cudaMemcpyHostToDevice) ||
        cudaMemset(c->eta, 0, sizeof(double) * c->ne) || cudaMemset(c->alpha, 0, sizeof(double) * c->ne) ||
        cudaMemset(c->lam_bits, 0, sizeof(unsigned long long)) || cudaMemset(c->err, 0, sizeof(unsigned int)))
        return cleanup(PDG_ERR_CUDA);
    for (int kind = 0; kind < KIND_COUNT; kind++) {
        if (!kind_used(kind, c->dim, c->p.parabolic != 0, c->p.filter)) continue;
        int r = configure_launch(c, kind);
        if (r) return cleanup(r);
    }
    *out = c;
    return PDG_OK;
}

int pdg_set_boundary(pdg_ctx *c, int index, int type, const double *state)
{
    if (!c) return PDG_ERR_ARG;
    if (index < 0 || index >= PDG_MAX_BOUNDARIES)
        return fail(c, PDG_ERR_ARG, "pdg_set_boundary: index %d outside [0, %d)", index, PDG_MAX_BOUNDARIES);
    if (type < PDG_BC_SUPERSONIC_INFLOW || type > PDG_BC_NOSLIP_ISOTHERMAL)
        return fail(c, PDG_ERR_ARG, "pdg_set_boundary: unknown boundary type %d", type);
    if (type == PDG_BC_SUBSONIC_INFLOW_PTTT && c->dim != 2)
        return fail(c, PDG_ERR_UNSUPPORTED, "pdg_set_boundary: the total-pressure inflow is 2D only");
    double slot[BC_SLOT] = {(double)type};
    const int n = type == PDG_BC_SUBSONIC_OUTFLOW_P ? 1
                  : type == PDG_BC_SUBSONIC_INFLOW_RV ? 1 + c->dim
                  : type == PDG_BC_NOSLIP_ADIABATIC ? c->dim
                  : type == PDG_BC_NOSLIP_ISOTHERMAL ? 1 + c->dim
                  : type == PDG_BC_SUBSONIC_INFLOW_PTTT ? 5
                  : (type == PDG_BC_SUPERSONIC_INFLOW || type == PDG_BC_SPECIFIED_STATE || type == PDG_BC_RIEMANN_INVARIANT)
                      ? c->nv : 0;
    if (n > 0) {
        if (!state) return fail(c, PDG_ERR_ARG, "pdg_set_boundary: type %d needs its data", type);
        bool ok = true;
        for (int v = 0; v < n; v++) ok = ok && std::isfinite(state[v]);
        if (type == PDG_BC_SUPERSONIC_INFLOW || type == PDG_BC_SPECIFIED_STATE) {
            double msq = 0.0;
            for (int d = 0; d < c->dim; d++) msq += state[1 + d] * state[1 + d];
            const double p = (c->p.gamma - 1.0) * (state[c->dim + 1] - 0.5 * msq / state[0]);
            ok = ok && state[0] > 0.0 && p > 0.0;
        } else if (type == PDG_BC_RIEMANN_INVARIANT) {
            ok = ok && state[0] > 0.0 && state[c->nv - 1] > 0.0;
        } else if (type == PDG_BC_SUBSONIC_INFLOW_PTTT) {
            ok = ok && state[0] > 0.0 && state[1] > 0.0 && state[2] > 0.0;
        } else if (type == PDG_BC_NOSLIP_ADIABATIC) {
            // any wall velocity
        } else if (type == PDG_BC_NOSLIP_ISOTHERMAL) {
            ok = ok && state[0] > 0.0 && c->p.R_gas > 0.0;
        } else {
            ok = ok && state[0] > 0.0;
        }
        if (!ok) return fail(c, PDG_ERR_ARG, "pdg_set_boundary: the data of condition %d is not physical", index);
        for (int v = 0; v < n; v++) slot[1 + v] = state[v];
        if (type == PDG_BC_NOSLIP_ISOTHERMAL) {  // {T, V} -> V, 1/(R T) (the integrator's constructor)
            for (int q = 0; q < c->dim; q++) slot[1 + q] = state[1 + q];
            slot[1 + c->dim] = 1.0 / (c->p.R_gas * state[0]);
        }
        if (type == PDG_BC_SUBSONIC_INFLOW_PTTT) {  // flow angle -> direction (the integrator's constructor)
            const double theta = state[3];
            slot[4] = std::cos(theta * M_PI / 180.0);
            slot[5] = std::sin(theta * M_PI / 180.0);
        }
    }
    std::memcpy(c->bc_host + index * BC_SLOT, slot, sizeof(slot));
    CK(cudaMemcpy(c->bc + index * BC_SLOT, slot, sizeof(slot), cudaMemcpyHostToDevice), "boundary table upload");
    c->bc_set |= 1u << index;
    return PDG_OK;
}

}  // extern "C"

namespace {

// Node index of position `pos` along direction d on line `line` (x fastest).
inline int host_line_node(int dim, int Np, int d, int line, int pos)
{
    if (dim == 2) return d == 0 ? line * Np + pos : pos * Np + line;
    if (d == 0) return line * Np + pos;
    if (d == 1) return (line / Np) * Np * Np + pos * Np + (line % Np);
    return pos * Np * Np + line;
}

// Smallest singular value of a dim x dim matrix A (row-major): the square
// root of the smallest eigenvalue of A^T A, in closed form (2D) or by the
// trigonometric solution of the symmetric 3 x 3 eigenproblem (Smith, 1961).
double min_singular_value(int dim, const double *A)
{
    double B[9] = {};
    for (int i = 0; i < dim; i++)
        for (int j = 0; j < dim; j++)
            for (int k = 0; k < dim; k++) B[i * 3 + j] += A[k * dim + i] * A[k * dim + j];
    if (dim == 2) {
        const double a = B[0], b = B[1], cc = B[4];
        const double m = 0.5 * (a + cc), r = std::sqrt(0.25 * (a - cc) * (a - cc) + b * b);
        return std::sqrt(std::max(m - r, 0.0));
    }
    const double p1 = B[1] * B[1] + B[2] * B[2] + B[5] * B[5];
    if (p1 == 0.0) return std::sqrt(std::max(0.0, std::min(B[0], std::min(B[4], B[8]))));
    const double q = (B[0] + B[4] + B[8]) / 3.0;
    const double p2 = (B[0] - q) * (B[0] - q) + (B[4] - q) * (B[4] - q) + (B[8] - q) * (B[8] - q) + 2.0 * p1;
    const double p = std::sqrt(p2 / 6.0);
    double C[9];
    for (int i = 0; i < 9; i++) C[i] = (B[i] - ((i % 4) == 0 ? q : 0.0)) / p;
    const double det = C[0] * (C[4] * C[8] - C[5] * C[7]) - C[1] * (C[3] * C[8] - C[5] * C[6]) +
                       C[2] * (C[3] * C[7] - C[4] * C[6]);
    const double r = std::max(-1.0, std::min(1.0, 0.5 * det));
    const double phi = std::acos(r) / 3.0;
    const double lmin = q + 2.0 * p * std::cos(phi + 2.0 * 3.14159265358979323846 / 3.0);
    return std::sqrt(std::max(lmin, 0.0));
}

}  // namespace

extern "C" {

int pdg_set_geometry(pdg_ctx *c, const double *x, const int32_t *face_orient)
{
    if (!c) return PDG_ERR_ARG;
    if (!x) return fail(c, PDG_ERR_ARG, "pdg_set_geometry: null coordinates");
    if (c->geo) return fail(c, PDG_ERR_ARG, "pdg_set_geometry: the geometry is already set");
    if (c->launches > 0 || c->graph_exec)
        return fail(c, PDG_ERR_ARG, "pdg_set_geometry: must precede the first evaluation");
    if (c->p.parabolic && c->p.compat)
        return fail(c, PDG_ERR_UNSUPPORTED, "pdg_set_geometry: Navier-Stokes on general geometry takes compat = 0");
    const int dim = c->dim, Np = c->Np, N = c->N, nd = c->ndof, nf = 2 * dim;
    const int nfn = dim == 2 ? Np : Np * Np;
    const int64_t ne = c->ne, nn = c->nnodes;
    const int nq = 1 + dim * dim;
    const double *D = c->hK.D;  // D[i * Np + l] = l'_l(x_i)
    std::vector<double> geo((size_t)nq * nn);
    // Jacobian dx_k / dxi_r at every node from the node coordinates (the
    // derivative of the element's degree-N interpolant of its geometry, what
    // MFEM's element transformation evaluates at the LGL points), its
    // adjugate (MFEM's AdjugateJacobian) and determinant (Weight)
    for (int64_t e = 0; e < ne; e++)
        for (int n = 0; n < nd; n++) {
            const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            double Jm[9] = {};
            for (int k = 0; k < dim; k++)
                for (int r = 0; r < dim; r++) {
                    const int line = r == 0 ? n / Np : r == 1 ? (dim == 2 ? pos[0] : pos[0] + Np * pos[2]) : pos[0] + Np * pos[1];
                    double t = 0.0;
                    for (int l = 0; l < Np; l++)
                        t += D[pos[r] * Np + l] * x[(int64_t)k * nn + e * nd + host_line_node(dim, Np, r, line, l)];
                    Jm[k * 3 + r] = t;
                }
            auto J_ = [&](int i, int j) { return Jm[i * 3 + j]; };
            double adj[9] = {}, det;
            if (dim == 2) {
                adj[0] = J_(1, 1);
                adj[1] = -J_(0, 1);
                adj[3] = -J_(1, 0);
                adj[4] = J_(0, 0);
                det = J_(0, 0) * J_(1, 1) - J_(0, 1) * J_(1, 0);
            } else {
                // row r of the adjugate: the cross product of Jacobian columns r+1 and r+2
                for (int r = 0; r < 3; r++) {
                    const int a = (r + 1) % 3, b = (r + 2) % 3;
                    adj[r * 3 + 0] = J_(1, a) * J_(2, b) - J_(2, a) * J_(1, b);
                    adj[r * 3 + 1] = J_(2, a) * J_(0, b) - J_(0, a) * J_(2, b);
                    adj[r * 3 + 2] = J_(0, a) * J_(1, b) - J_(1, a) * J_(0, b);
                }
                det = J_(0, 0) * (J_(1, 1) * J_(2, 2) - J_(1, 2) * J_(2, 1)) -
                      J_(0, 1) * (J_(1, 0) * J_(2, 2) - J_(1, 2) * J_(2, 0)) +
                      J_(0, 2) * (J_(1, 0) * J_(2, 1) - J_(1, 1) * J_(2, 0));
            }
            if (!(det > 0.0))
                return fail(c, PDG_ERR_ARG, "pdg_set_geometry: element %lld node %d has Jacobian %g (not positive)",
                            (long long)e, n, det);
            const int64_t g = e * nd + n;
            geo[g] = det;
            for (int r = 0; r < dim; r++)
                for (int k = 0; k < dim; k++) geo[(size_t)(1 + r * dim + k) * nn + g] = adj[r * 3 + k];
        }
    auto row = [&](int64_t e, int n, int r, int k) { return geo[(size_t)(1 + r * dim + k) * nn + e * nd + n]; };
    // faces: the neighbour's matching node and the normal out of the face's
    // element 1 (the lower-numbered element; its +d or -d adjugate row)
    std::vector<int32_t> fnode((size_t)ne * nf * nfn, 0);
    std::vector<int32_t> fpart((size_t)ne * nf * nfn, -1);
    if ((int64_t)ne * nf * nfn >= (int64_t)INT32_MAX)
        return fail(c, PDG_ERR_ARG, "pdg_set_geometry: too many face nodes for the face tables");
    std::vector<double> fnor((size_t)ne * nf * nfn * dim, 0.0);
    for (int64_t e = 0; e < ne; e++)
        for (int f = 0; f < nf; f++) {
            const int d = f / 2, side = f % 2;
            const int64_t nb = c->nbr_host[e * nf + f];
            int f2 = f ^ 1, o = 0;
            if (nb >= 0 && face_orient) {
                const int32_t code = face_orient[e * nf + f];
                f2 = code & 7;
                o = code >> 3;
                if (f2 >= nf || o > 7 || (dim == 2 && (o & 5)))
                    return fail(c, PDG_ERR_ARG, "pdg_set_geometry: element %lld face %d: bad orientation code %d",
                                (long long)e, f, code);
            }
            if (nb >= 0 && c->nbr_host[nb * nf + f2] != e)
                return fail(c, PDG_ERR_ARG, "pdg_set_geometry: element %lld face %d: the neighbour's face %d does not point back",
                            (long long)e, f, f2);
            for (int t = 0; t < nfn; t++) {
                const int n = host_line_node(dim, Np, d, t, side ? N : 0);
                const size_t fi = ((size_t)e * nf + f) * nfn + t;
                double own[3];
                for (int k = 0; k < dim; k++) own[k] = (side ? 1.0 : -1.0) * row(e, n, d, k);
                if (nb < 0) {
                    for (int k = 0; k < dim; k++) fnor[fi * dim + k] = own[k];
                    continue;
                }
                int a = t % Np, b = dim == 3 ? t / Np : 0;
                if (o & 1) std::swap(a, b);
                if (o & 2) a = N - a;
                if (o & 4) b = N - b;
                const int t2 = a + Np * b, d2 = f2 / 2, side2 = f2 % 2;
                const int n2 = host_line_node(dim, Np, d2, t2, side2 ? N : 0);
                fnode[fi] = n2;
                fpart[fi] = (int32_t)(((int64_t)nb * nf + f2) * nfn + t2);
                // matching nodes sit at the same point, up to one periodic
                // shift per face
                {
                    const int nlast = host_line_node(dim, Np, d, nfn - 1, side ? N : 0);
                    const int nfirst = host_line_node(dim, Np, d, 0, side ? N : 0);
                    double ext = 0.0, dev = 0.0;
                    for (int k = 0; k < dim; k++) {
                        const double *xk = x + (int64_t)k * nn;
                        const double shift0 = xk[e * nd + nfirst] - xk[nb * nd + fnode[((size_t)e * nf + f) * nfn]];
                        const double dk = (xk[e * nd + n] - xk[nb * nd + n2]) - shift0;
                        const double ek = xk[e * nd + nlast] - xk[e * nd + nfirst];
                        dev += dk * dk;
                        ext += ek * ek;
                    }
                    if (!(dev <= 1e-18 * ext))
                        return fail(c, PDG_ERR_ARG,
                                    "pdg_set_geometry: element %lld face %d node %d does not meet the neighbour's "
                                    "matching node (a non-conforming face or a wrong orientation code)",
                                    (long long)e, f, t);
                }
                double other[3], sq = 0.0, dsq = 0.0;
                for (int k = 0; k < dim; k++) {
                    other[k] = (side2 ? 1.0 : -1.0) * row(nb, n2, d2, k);
                    sq += own[k] * own[k];
                    dsq += (own[k] + other[k]) * (own[k] + other[k]);
                }
                if (!(dsq <= 1e-12 * sq))
                    return fail(c, PDG_ERR_ARG,
                                "pdg_set_geometry: element %lld face %d node %d: the neighbour's normal does not match "
                                "(a non-conforming face or a wrong orientation code)",
                                (long long)e, f, t);
                const bool is1 = e < nb || (e == nb && side == 1);
                // element 1's outward normal: this element's, or the neighbour's
                for (int k = 0; k < dim; k++) fnor[fi * dim + k] = is1 ? own[k] : other[k];
            }
        }
    // CFL length: the smallest singular value of the Jacobian at an element
    // centre (MFEM's GetElementSize(e, 1), as Simulation.cpp:896-906 uses)
    std::vector<double> xg(Np), wg(Np), Lc(Np), dLc(Np);
    gauss_lobatto(Np, xg.data(), wg.data());
    for (int j = 0; j < Np; j++) {
        double v = 1.0, dv = 0.0;
        for (int m = 0; m < Np; m++) {
            if (m == j) continue;
            double prod = 1.0 / (xg[j] - xg[m]);
            for (int q = 0; q < Np; q++)
                if (q != j && q != m) prod *= (0.5 - xg[q]) / (xg[j] - xg[q]);
            dv += prod;
            v *= (0.5 - xg[m]) / (xg[j] - xg[m]);
        }
        Lc[j] = v;
        dLc[j] = dv;
    }
    double hmin = 1e300;
    for (int64_t e = 0; e < ne; e++) {
        double Jc[9] = {};
        for (int n = 0; n < nd; n++) {
            const int pos[3] = {n % Np, (n / Np) % Np, n / (Np * Np)};
            for (int r = 0; r < dim; r++) {
                double wgt = 1.0;
                for (int q = 0; q < dim; q++) wgt *= q == r ? dLc[pos[q]] : Lc[pos[q]];
                for (int k = 0; k < dim; k++) Jc[k * dim + r] += wgt * x[(int64_t)k * nn + e * nd + n];
            }
        }
        hmin = std::min(hmin, min_singular_value(dim, Jc));
    }
    if (cudaMalloc(&c->geo_d, sizeof(double) * geo.size()) != cudaSuccess ||
        cudaMalloc(&c->fnode_d, sizeof(int32_t) * fnode.size()) != cudaSuccess ||
        cudaMalloc(&c->fnor_d, sizeof(double) * fnor.size()) != cudaSuccess)
        return fail(c, PDG_ERR_NOMEM, "pdg_set_geometry: allocation failed");
    CK(cudaMemcpy(c->geo_d, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice), "geometry upload");
    CK(cudaMemcpy(c->fnode_d, fnode.data(), sizeof(int32_t) * fnode.size(), cudaMemcpyHostToDevice), "geometry upload");
    CK(cudaMemcpy(c->fnor_d, fnor.data(), sizeof(double) * fnor.size(), cudaMemcpyHostToDevice), "geometry upload");
    int r = configure_launch(c, c->p.parabolic ? KIND_GEO_NS : KIND_GEO);
    if (r) return r;
    if (c->p.parabolic) {
        if ((r = configure_launch(c, KIND_GEO_LIFT))) return r;
        if (cudaMalloc(&c->geo_fv, sizeof(double) * dim * (c->nv - 1) * nn) != cudaSuccess ||
            cudaMalloc(&c->geo_cf, sizeof(double) * fpart.size() * (c->nv - 1)) != cudaSuccess ||
            cudaMalloc(&c->fpart_d, sizeof(int32_t) * fpart.size()) != cudaSuccess)
            return fail(c, PDG_ERR_NOMEM, "pdg_set_geometry: allocation failed");
        CK(cudaMemcpy(c->fpart_d, fpart.data(), sizeof(int32_t) * fpart.size(), cudaMemcpyHostToDevice),
           "geometry upload");
    }
    cudaFree(c->fbuf);  // the box path's face buffer is not used
    c->fbuf = nullptr;
    c->hmin = hmin;
    c->geo = true;
    return PDG_OK;
}

int pdg_destroy(pdg_ctx *c)
{
    if (!c) return PDG_OK;
    cudaFree(c->K);
    cudaFree(c->nbr);
    cudaFree(c->eta);
    cudaFree(c->alpha);
    cudaFree(c->lbuf);
    cudaFree(c->fcol);
    cudaFree(c->vbuf);
    cudaFree(c->fbuf);
    cudaFree(c->bc);
    cudaFree(c->lbuf_lo);
    cudaFree(c->stage_a);
    cudaFree(c->stage_b);
    cudaFree(c->io_a);
    cudaFree(c->io_b);
    cudaFree(c->lam_bits);
    cudaFree(c->err);
    cudaFree(c->ent_own);
    cudaFree(c->gcol);
    cudaFree(c->gbuf);
    cudaFree(c->geo_d);
    cudaFree(c->fnode_d);
    cudaFree(c->fnor_d);
    cudaFree(c->geo_grads);
    cudaFree(c->geo_fv);
    cudaFree(c->geo_cf);
    cudaFree(c->fpart_d);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->cap) cudaStreamDestroy(c->cap);
    cudaFree(c->filter_count);
    cudaFree(c->limit_count);
    for (auto &t : c->timed) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    for (auto e : c->pipe.ev_in) cudaEventDestroy(e);
    for (auto e : c->pipe.ev_done) cudaEventDestroy(e);
    if (c->pipe.ev_start) cudaEventDestroy(c->pipe.ev_start);
    if (c->pipe.in) cudaStreamDestroy(c->pipe.in);
    if (c->pipe.comp) cudaStreamDestroy(c->pipe.comp);
    if (c->pipe.out) cudaStreamDestroy(c->pipe.out);
    delete c;
    return PDG_OK;
}

int64_t pdg_size(const pdg_ctx *c) { return c ? c->size : -1; }

int pdg_rhs(pdg_ctx *c, const double *u, double *dudt, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!u || !dudt || u == dudt) return fail(c, PDG_ERR_ARG, "pdg_rhs: null or aliased buffers");
    return evaluate(c, -1, 0.0, nullptr, u, dudt, (cudaStream_t)stream);
}

int pdg_rhs_host(pdg_ctx *c, const double *u_host, double *dudt_host)
{
    if (!c) return PDG_ERR_ARG;
    if (!u_host || !dudt_host) return fail(c, PDG_ERR_ARG, "pdg_rhs_host: null buffer");
    const size_t bytes = sizeof(double) * (size_t)c->size;
    if (!c->io_a) {
        if (cudaMalloc(&c->io_a, bytes) != cudaSuccess || cudaMalloc(&c->io_b, bytes) != cudaSuccess)
            return fail(c, PDG_ERR_NOMEM, "pdg_rhs_host: staging allocation failed");
    }
    cudaStream_t s = 0;
    CK(cudaMemcpyAsync(c->io_a, u_host, bytes, cudaMemcpyHostToDevice, s), "copy in");
    int r = evaluate(c, -1, 0.0, nullptr, c->io_a, c->io_b, s);
    if (r) return r;
    CK(cudaMemcpyAsync(dudt_host, c->io_b, bytes, cudaMemcpyDeviceToHost, s), "copy out");
    CK(cudaStreamSynchronize(s), "synchronize");
    return PDG_OK;
}

int pdg_rk_stage(pdg_ctx *c, int stage, double dt, const double *un, const double *us, double *uout, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (stage < 0 || stage > 2) return fail(c, PDG_ERR_ARG, "pdg_rk_stage: stage must be 0, 1 or 2");
    if (!us || !uout || uout == us) return fail(c, PDG_ERR_ARG, "pdg_rk_stage: null or aliased buffers");
    if (stage > 0 && !un) return fail(c, PDG_ERR_ARG, "pdg_rk_stage: stage %d needs un", stage);
    return evaluate(c, stage, dt, stage > 0 ? un : us, us, uout, (cudaStream_t)stream);
}

int pdg_rk3_step(pdg_ctx *c, double dt, double *u, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!u) return fail(c, PDG_ERR_ARG, "pdg_rk3_step: null state");
    cudaStream_t s = (cudaStream_t)stream;
    int r = evaluate(c, 0, dt, u, u, c->stage_a, s);
    if (!r) r = evaluate(c, 1, dt, u, c->stage_a, c->stage_b, s);
    // stage 2 reads un and writes the same entry from the same thread, so the
    // result can overwrite u in place
    if (!r) r = evaluate(c, 2, dt, u, c->stage_b, u, s);
    return r;
}

int pdg_rk3_steps(pdg_ctx *c, double dt, double *u, int nsteps, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!u || nsteps < 0) return fail(c, PDG_ERR_ARG, "pdg_rk3_steps: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (!c->graph_exec || c->graph_u != u || c->graph_dt != dt) {
        if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
        if (c->graph) cudaGraphDestroy(c->graph);
        c->graph_exec = nullptr;
        c->graph = nullptr;
        if (!c->cap && cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking) != cudaSuccess)
            return fail(c, PDG_ERR_CUDA, "pdg_rk3_steps: stream creation failed");
        const bool prof = c->profile;
        c->profile = false;  // no timing events inside the graph
        const int64_t l0 = c->launches;
        CK(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        int r = evaluate(c, 0, dt, u, u, c->stage_a, c->cap);
        if (!r) r = evaluate(c, 1, dt, u, c->stage_a, c->stage_b, c->cap);
        if (!r) r = evaluate(c, 2, dt, u, c->stage_b, u, c->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->cap, &g);
        c->profile = prof;
        c->graph_launches = c->launches - l0;
        c->launches = l0;
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "end capture");
        c->graph = g;
        CK(cudaGraphInstantiate(&c->graph_exec, c->graph, 0), "graph instantiate");
        c->graph_u = u;
        c->graph_dt = dt;
    }
    c->last_stream = s;
    for (int i = 0; i < nsteps; i++) {
        CK(cudaGraphLaunch(c->graph_exec, s), "graph launch");
        c->launches += c->graph_launches;
    }
    return PDG_OK;
}

}  // extern "C"

namespace {

// pdg_rk3_step_host's pipeline (the fixed operator with the face buffer, no
// filter, at least PIPE_CHUNKS x PIPE_MIN_CHUNK elements): the state crosses
// PCIe in chunks of consecutive elements on a copy stream.  At four
// milestones of the copy, stage 0's kernels are launched over the runs of
// consecutive chunks whose reads have landed (a face-node kernel reads its
// chunk and the chunks of the face neighbours, a lifting kernel the
// face-node results of its neighbours' chunks, a volume kernel the lifting
// results of its neighbours' chunks; on a periodic mesh the last chunks to
// land hold up their neighbours, so only part of stage 0 overlaps the copy);
// stage 1 runs whole; stage 2 runs its face-node and lifting kernels whole
// and its volume kernel in four runs, each copied back on a second copy
// stream while the next is computed.  Per element the arithmetic is that of
// the unchunked step, so the result is the same to the bit.
constexpr int PIPE_CHUNKS = 32, PIPE_MILESTONES = 4;
constexpr int64_t PIPE_MIN_CHUNK = 128;

int pipe_setup(pdg_ctx *c)
{
    auto &q = c->pipe;
    if (q.ready) return PDG_OK;
    q.ready = true;
    q.usable = c->fbuf && !c->geo && !c->p.filter && c->ne >= PIPE_CHUNKS * PIPE_MIN_CHUNK;
    if (const char *hp = std::getenv("PDG_HOST_PIPELINE")) q.usable = q.usable && std::atoi(hp) != 0;
    if (!q.usable) return PDG_OK;
    const int C = PIPE_CHUNKS, nf = 2 * c->dim;
    q.bounds.resize(C + 1);
    for (int k = 0; k <= C; k++) q.bounds[k] = c->ne * k / C;
    auto chunk_of = [&](int64_t e) {
        return (int)(std::upper_bound(q.bounds.begin(), q.bounds.end(), e) - q.bounds.begin()) - 1;
    };
    q.near.assign(C, {});
    for (int k = 0; k < C; k++) {
        std::vector<char> hit(C, 0);
        hit[k] = 1;
        for (int64_t e = q.bounds[k]; e < q.bounds[k + 1]; e++)
            for (int f = 0; f < nf; f++) {
                const int32_t nb = c->nbr_host[e * nf + f];
                if (nb >= 0) hit[chunk_of(nb)] = 1;
            }
        for (int j = 0; j < C; j++)
            if (hit[j]) q.near[k].push_back(j);
    }
    q.ev_in.assign(PIPE_MILESTONES, nullptr);
    q.ev_done.assign(PIPE_MILESTONES, nullptr);
    bool ok = cudaStreamCreateWithFlags(&q.in, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&q.comp, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&q.out, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&q.ev_start, cudaEventDisableTiming) == cudaSuccess;
    for (int m = 0; m < PIPE_MILESTONES && ok; m++)
        ok = cudaEventCreateWithFlags(&q.ev_in[m], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&q.ev_done[m], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) return fail(c, PDG_ERR_CUDA, "pdg_rk3_step_host: stream or event creation failed");
    return PDG_OK;
}

// Copies chunks [k0, k1) of every variable between the device state and the
// host state (same byNODES offsets).
int pipe_copy(pdg_ctx *c, int k0, int k1, double *dst, const double *src, cudaMemcpyKind kind, cudaStream_t s)
{
    const auto &q = c->pipe;
    const int64_t first = q.bounds[k0] * c->ndof, count = (q.bounds[k1] - q.bounds[k0]) * c->ndof;
    for (int v = 0; v < c->nv; v++)
        CK(cudaMemcpyAsync(dst + v * c->nnodes + first, src + v * c->nnodes + first, sizeof(double) * count, kind, s),
           "chunk copy");
    return PDG_OK;
}

int step_host_pipelined(pdg_ctx *c, double dt, double *u_host)
{
    auto &q = c->pipe;
    const int C = PIPE_CHUNKS, M = PIPE_MILESTONES, per = C / M;
    const bool ns = c->p.parabolic != 0;
    const int kinds[3] = {ns ? KIND_LIFT_FACE_FLUX : KIND_FACE_FLUX, KIND_LIFT, ns ? KIND_NS_FACES_FB : KIND_EULER_FACES_FB};
    int r;
    // after the caller's earlier work on the legacy default stream
    CK(cudaEventRecord(q.ev_start, 0), "event record");
    CK(cudaStreamWaitEvent(q.in, q.ev_start, 0), "stream wait");
    CK(cudaStreamWaitEvent(q.comp, q.ev_start, 0), "stream wait");
    for (int m = 0; m < M; m++) {
        if ((r = pipe_copy(c, m * per, (m + 1) * per, c->io_a, u_host, cudaMemcpyHostToDevice, q.in))) return r;
        CK(cudaEventRecord(q.ev_in[m], q.in), "event record");
    }
    // readiness of stage 0's kernels: the last chunk (copy order) each reads
    std::vector<int> t[3];
    for (auto &v : t) v.assign(C, 0);
    for (int k = 0; k < C; k++) t[0][k] = *std::max_element(q.near[k].begin(), q.near[k].end());
    for (int k = 0; k < C; k++)
        for (int j : q.near[k]) t[1][k] = std::max(t[1][k], t[0][j]);
    for (int k = 0; k < C; k++)
        for (int j : q.near[k]) t[2][k] = std::max(t[2][k], ns ? std::max(t[0][j], t[1][j]) : t[0][j]);
    CK(cudaMemsetAsync(c->lam_bits, 0, sizeof(unsigned long long), q.comp), "reset wave speed");
    KParams P = base_params(c);
    P.u = c->io_a;
    P.un = c->io_a;
    P.out = c->stage_a;
    P.stage = 0;
    P.dt = dt;
    P.vbuf = c->vbuf;
    std::vector<char> done[3];
    for (auto &v : done) v.assign(C, 0);
    for (int m = 0; m < M; m++) {
        CK(cudaStreamWaitEvent(q.comp, q.ev_in[m], 0), "stream wait");
        const int landed = (m + 1) * per - 1;
        for (int type = 0; type < 3; type++) {
            if (type == 1 && !ns) continue;
            // runs of consecutive ready chunks, one launch each
            for (int k = 0; k < C;) {
                if (done[type][k] || t[type][k] > landed) { k++; continue; }
                int k1 = k;
                while (k1 < C && !done[type][k1] && t[type][k1] <= landed) done[type][k1++] = 1;
                P.e_begin = q.bounds[k];
                P.e_end = q.bounds[k1];
                if ((r = launch(c, kinds[type], P, q.comp))) return r;
                k = k1;
            }
        }
    }
    // stage 1 on the whole mesh
    if ((r = evaluate(c, 1, dt, c->io_a, c->stage_a, c->stage_b, q.comp))) return r;
    // stage 2: face nodes and lifting on the whole mesh, the volume kernel in
    // M runs, each run's result back to the host behind it
    CK(cudaMemsetAsync(c->lam_bits, 0, sizeof(unsigned long long), q.comp), "reset wave speed");
    P = base_params(c);
    P.u = c->stage_b;
    P.un = c->io_a;
    P.out = c->io_a;  // stage 2 reads un and writes the same entries from the same thread
    P.stage = 2;
    P.dt = dt;
    P.vbuf = c->vbuf;
    if ((r = launch(c, kinds[0], P, q.comp))) return r;
    if (ns && (r = launch(c, KIND_LIFT, P, q.comp))) return r;
    for (int m = 0; m < M; m++) {
        P.e_begin = q.bounds[m * per];
        P.e_end = q.bounds[(m + 1) * per];
        if ((r = launch(c, kinds[2], P, q.comp))) return r;
        CK(cudaEventRecord(q.ev_done[m], q.comp), "event record");
        CK(cudaStreamWaitEvent(q.out, q.ev_done[m], 0), "stream wait");
        if ((r = pipe_copy(c, m * per, (m + 1) * per, u_host, c->io_a, cudaMemcpyDeviceToHost, q.out))) return r;
    }
    c->last_stream = q.comp;
    CK(cudaStreamSynchronize(q.out), "synchronize");
    CK(cudaStreamSynchronize(q.comp), "synchronize");
    return PDG_OK;
}

}  // namespace

extern "C" {

int pdg_rk3_step_host(pdg_ctx *c, double dt, double *u_host)
{
    if (!c) return PDG_ERR_ARG;
    if (!u_host) return fail(c, PDG_ERR_ARG, "pdg_rk3_step_host: null state");
    const size_t bytes = sizeof(double) * (size_t)c->size;
    if (!c->io_a) {
        if (cudaMalloc(&c->io_a, bytes) != cudaSuccess || cudaMalloc(&c->io_b, bytes) != cudaSuccess)
            return fail(c, PDG_ERR_NOMEM, "pdg_rk3_step_host: staging allocation failed");
    }
    int r = pipe_setup(c);
    if (r) return r;
    if (c->pipe.usable && !c->profile) return step_host_pipelined(c, dt, u_host);
    cudaStream_t s = 0;
    CK(cudaMemcpyAsync(c->io_a, u_host, bytes, cudaMemcpyHostToDevice, s), "copy in");
    r = pdg_rk3_step(c, dt, c->io_a, s);
    if (r) return r;
    CK(cudaMemcpyAsync(u_host, c->io_a, bytes, cudaMemcpyDeviceToHost, s), "copy out");
    CK(cudaStreamSynchronize(s), "synchronize");
    return PDG_OK;
}

int pdg_rk_stage_part(pdg_ctx *c, int part, int stage, double dt, const double *un, const double *us, double *uout,
                      int64_t e_begin, int64_t e_end, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!c->fbuf || c->geo || c->p.filter)
        return fail(c, PDG_ERR_UNSUPPORTED, "pdg_rk_stage_part: needs the fixed operator on a periodic box mesh, no filter");
    if (part < PDG_PART_START || part > PDG_PART_VOLUME) return fail(c, PDG_ERR_ARG, "pdg_rk_stage_part: bad part");
    if (stage < -1 || stage > 2) return fail(c, PDG_ERR_ARG, "pdg_rk_stage_part: stage must be -1, 0, 1 or 2");
    if (e_begin < 0 || e_end > c->ne || e_begin > e_end) return fail(c, PDG_ERR_ARG, "pdg_rk_stage_part: bad range");
    cudaStream_t s = (cudaStream_t)stream;
    c->last_stream = s;
    if (part == PDG_PART_START) {
        CK(cudaMemsetAsync(c->lam_bits, 0, sizeof(unsigned long long), s), "reset wave speed");
        return PDG_OK;
    }
    if (!us || (part == PDG_PART_VOLUME && (!uout || uout == us || (stage > 0 && !un))))
        return fail(c, PDG_ERR_ARG, "pdg_rk_stage_part: null or aliased buffers");
    if (e_begin == e_end) return PDG_OK;
    const bool ns = c->p.parabolic != 0;
    if (part == PDG_PART_LIFT && !ns) return PDG_OK;  // Euler has no lifting kernel
    KParams P = base_params(c);
    P.u = us;
    P.un = stage > 0 ? un : us;
    P.out = uout;
    P.stage = stage;
    P.dt = dt;
    P.vbuf = c->vbuf;
    P.e_begin = e_begin;
    P.e_end = e_end;
    const int kind = part == PDG_PART_FACES ? (ns ? KIND_LIFT_FACE_FLUX : KIND_FACE_FLUX)
                     : part == PDG_PART_LIFT ? KIND_LIFT
                                             : (ns ? KIND_NS_FACES_FB : KIND_EULER_FACES_FB);
    return launch(c, kind, P, s);
}

int pdg_face_columns(pdg_ctx *c, double **cols, int64_t *count)
{
    if (!c || !cols || !count) return PDG_ERR_ARG;
    if (!c->p.parabolic) return fail(c, PDG_ERR_ARG, "pdg_face_columns: operator is not parabolic");
    const int64_t nfn = c->dim == 2 ? c->Np : c->Np * c->Np;
    *cols = c->fcol;
    *count = 2 * c->dim * c->ne * nfn * (c->nv - 1);
    return PDG_OK;
}

int pdg_profile_enable(pdg_ctx *c, int on)
{
    if (!c) return PDG_ERR_ARG;
    c->profile = on != 0;
    return PDG_OK;
}

int pdg_profile_read(pdg_ctx *c, int kind, double *total_ms, int64_t *launches)
{
    if (!c || !total_ms || !launches) return PDG_ERR_ARG;
    double ms = 0.0;
    int64_t n = 0;
    std::vector<pdg_ctx::TimedLaunch> keep;
    for (auto &t : c->timed) {
        if (t.kind != kind) { keep.push_back(t); continue; }
        CK(cudaEventSynchronize(t.b), "event synchronize");
        float dt = 0.0f;
        CK(cudaEventElapsedTime(&dt, t.a, t.b), "event elapsed");
        ms += dt;
        n++;
        c->event_pool.push_back(t.a);
        c->event_pool.push_back(t.b);
    }
    c->timed.swap(keep);
    *total_ms = ms;
    *launches = n;
    return PDG_OK;
}

int pdg_max_char_speed(pdg_ctx *c, double *out)
{
    if (!c || !out) return PDG_ERR_ARG;
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, c->lam_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->last_stream), "read wave speed");
    CK(cudaStreamSynchronize(c->last_stream), "synchronize");
    double v;
    std::memcpy(&v, &bits, sizeof(v));
    *out = bits ? v : -1.0;
    return PDG_OK;
}

int pdg_cfl_dt(pdg_ctx *c, double cfl, double *dt_out)
{
    if (!c || !dt_out) return PDG_ERR_ARG;
    double lam;
    int r = pdg_max_char_speed(c, &lam);
    if (r) return r;
    if (!(lam > 0.0)) return fail(c, PDG_ERR_ARG, "pdg_cfl_dt: no wave speed yet (evaluate a RHS first)");
    *dt_out = cfl * c->hmin / (lam * std::pow((double)(c->N + 1), 2));
    return PDG_OK;
}

int pdg_get_blending(pdg_ctx *c, double *eta_host, double *alpha_host)
{
    if (!c) return PDG_ERR_ARG;
    CK(cudaStreamSynchronize(c->last_stream), "synchronize");
    if (eta_host) CK(cudaMemcpy(eta_host, c->eta, sizeof(double) * c->ne, cudaMemcpyDeviceToHost), "copy eta");
    if (alpha_host) CK(cudaMemcpy(alpha_host, c->alpha, sizeof(double) * c->ne, cudaMemcpyDeviceToHost), "copy alpha");
    return PDG_OK;
}

int pdg_gradients(pdg_ctx *c, const double *u, double *grads, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!c->p.parabolic) return fail(c, PDG_ERR_ARG, "pdg_gradients: operator is not parabolic");
    if (!u || !grads) return fail(c, PDG_ERR_ARG, "pdg_gradients: null buffer");
    c->last_stream = (cudaStream_t)stream;
    KParams P = base_params(c);
    P.out = nullptr;
    if (c->geo) {  // general geometry: the lifting kernel writes the caller's buffer
        P.u = u;
        P.geo_grads = grads;
        return launch(c, KIND_GEO_LIFT, P, (cudaStream_t)stream);
    }
    return lift(c, P, u, grads, (cudaStream_t)stream);
}

int pdg_check(pdg_ctx *c, uint32_t *flags)
{
    if (!c || !flags) return PDG_ERR_ARG;
    unsigned int f = 0;
    CK(cudaStreamSynchronize(c->last_stream), "synchronize");
    CK(cudaMemcpy(&f, c->err, sizeof(f), cudaMemcpyDeviceToHost), "read error word");
    CK(cudaMemset(c->err, 0, sizeof(unsigned int)), "clear error word");
    *flags = f;
    if (f & PDG_FLAG_NONFINITE) return fail(c, PDG_ERR_NONFINITE, "non-finite value in a state");
    if (f & PDG_FLAG_NONPHYSICAL) return fail(c, PDG_ERR_NONPHYSICAL, "non-positive density or pressure");
    return PDG_OK;
}

const char *pdg_last_error(const pdg_ctx *c) { return c ? c->last_error.c_str() : "null context"; }

int64_t pdg_launch_count(const pdg_ctx *c) { return c ? c->launches : -1; }

}  // extern "C"

namespace {

// Configures the adjoint kernels and their scratch on the first use.
int vjp_setup(pdg_ctx *c)
{
    if (c->adj_ready) return PDG_OK;
    int r;
    const int kinds[] = {KIND_ADJ_RHS, KIND_ADJ_LIFT, KIND_ADJ_FACE_E0, KIND_ADJ_FACE_NS0, KIND_ADJ_GATHER};
    for (int kind : kinds) {
        const bool ns_kind = kind == KIND_ADJ_LIFT || kind == KIND_ADJ_FACE_NS0;
        if ((ns_kind && !c->p.parabolic) || (kind == KIND_ADJ_FACE_E0 && c->p.parabolic)) continue;
        if ((r = configure_launch(c, kind))) return r;
    }
    if (!c->p.parabolic && (r = configure_launch(c, KIND_ADJ_BOUNDARY))) return r;
    const size_t nfn = c->dim == 2 ? c->Np : c->Np * c->Np;
    if (c->p.parabolic && cudaMalloc(&c->gcol, sizeof(double) * 2 * c->dim * c->ne * nfn * c->nv) != cudaSuccess)
        return fail(c, PDG_ERR_NOMEM, "pdg_rhs_vjp: scratch allocation failed");
    if (cudaMalloc(&c->gbuf, sizeof(double) * 2 * c->dim * c->ne * nfn * c->nv) != cudaSuccess)
        return fail(c, PDG_ERR_NOMEM, "pdg_rhs_vjp: scratch allocation failed");
    c->adj_ready = true;
    return PDG_OK;
}

// (NS: the forward BR1 jumps,) the volume terms to ubar, (NS: the viscous
// terms added,) every face's adjoint terms to gbuf, then their sum into ubar
// with, for stage >= 0, the RK stage's adjoint (adj_gather_kernel).  Boundary
// faces (Euler, stage < 0 only) are added to ubar last.
int vjp(pdg_ctx *c, int stage, double dt, const double *u, const double *cot, double *ubar, double *bx,
        cudaStream_t s)
{
    int r;
    if ((r = vjp_setup(c))) return r;
    KParams P = base_params(c);
    P.u = u;
    P.gbuf = c->gbuf;
    P.stage = stage;
    P.dt = dt;
    P.bx = bx;
    c->last_stream = s;
    void *a_cot = (void *)&cot, *a_bar = (void *)&ubar, *a_g = (void *)&c->gcol, *a_gb = (void *)&c->gbuf;
    if (c->p.parabolic && (r = launch(c, KIND_LIFT_FACE, P, s))) return r;
    if ((r = launch_with(c, KIND_ADJ_RHS, P, a_cot, a_bar, nullptr, s))) return r;
    if (c->p.parabolic && (r = launch_with(c, KIND_ADJ_LIFT, P, a_cot, a_bar, a_g, s))) return r;
    if ((r = launch_with(c, c->p.parabolic ? KIND_ADJ_FACE_NS0 : KIND_ADJ_FACE_E0, P, a_cot, a_gb, a_g, s))) return r;
    if ((r = launch_with(c, KIND_ADJ_GATHER, P, a_cot, a_bar, nullptr, s))) return r;
    if (!c->p.parabolic && c->bc_used && (r = launch_with(c, KIND_ADJ_BOUNDARY, P, a_cot, a_bar, a_g, s))) return r;
    return PDG_OK;
}

int vjp_check(pdg_ctx *c, const char *what)
{
    if (c->geo) return fail(c, PDG_ERR_UNSUPPORTED, "%s: the adjoint takes box meshes only", what);
    if (c->p.compat) return fail(c, PDG_ERR_UNSUPPORTED, "%s: the adjoint is of the fixed operator (compat = 0)", what);
    if (c->p.parabolic && c->bc_used)
        return fail(c, PDG_ERR_UNSUPPORTED, "%s: Navier-Stokes boundary faces are not differentiated", what);
    if (c->bc_used & ~c->bc_set) return fail(c, PDG_ERR_ARG, "%s: a boundary condition is not set", what);
    return PDG_OK;
}

}  // namespace

extern "C" {

int pdg_rhs_vjp(pdg_ctx *c, const double *u, const double *cot, double *ubar, void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (!u || !cot || !ubar || ubar == u || ubar == cot) return fail(c, PDG_ERR_ARG, "pdg_rhs_vjp: null or aliased buffers");
    int r;
    if ((r = vjp_check(c, "pdg_rhs_vjp"))) return r;
    return vjp(c, -1, 0.0, u, cot, ubar, nullptr, (cudaStream_t)stream);
}

int pdg_rk_stage_vjp(pdg_ctx *c, int stage, double dt, const double *us, const double *lam, double *out, double *bx,
                     void *stream)
{
    if (!c) return PDG_ERR_ARG;
    if (stage < 0 || stage > 2) return fail(c, PDG_ERR_ARG, "pdg_rk_stage_vjp: stage must be 0, 1 or 2");
    if (!us || !lam || !out || !bx || out == us || out == lam || out == bx || bx == us || bx == lam)
        return fail(c, PDG_ERR_ARG, "pdg_rk_stage_vjp: null or aliased buffers");
    int r;
    if ((r = vjp_check(c, "pdg_rk_stage_vjp"))) return r;
    if (c->bc_used)  // their adjoint is added after the volume kernel's store
        return fail(c, PDG_ERR_UNSUPPORTED, "pdg_rk_stage_vjp: boundary faces (use pdg_rhs_vjp)");
    return vjp(c, stage, dt, us, lam, out, bx, (cudaStream_t)stream);
}

int pdg_limiter_count(pdg_ctx *c, int64_t *limited)
{
    if (!c || !limited) return PDG_ERR_ARG;
    if (!(c->p.filter & 2)) {
        *limited = 0;
        return PDG_OK;
    }
    unsigned long long n = 0;
    CK(cudaStreamSynchronize(c->last_stream), "synchronize");
    CK(cudaMemcpy(&n, c->limit_count, sizeof(n), cudaMemcpyDeviceToHost), "read limiter count");
    *limited = (int64_t)n;
    return PDG_OK;
}

int pdg_filter_count(pdg_ctx *c, int64_t *filtered)
{
    if (!c || !filtered) return PDG_ERR_ARG;
    if (!(c->p.filter & 1)) {
        *filtered = 0;
        return PDG_OK;
    }
    unsigned long long n = 0;
    CK(cudaStreamSynchronize(c->last_stream), "synchronize");
    CK(cudaMemcpy(&n, c->filter_count, sizeof(n), cudaMemcpyDeviceToHost), "read filter count");
    *filtered = (int64_t)n;
    return PDG_OK;
}

}  // extern "C"
