// noalloc.cu — the allocation-free right-hand side, pdg_rhs_noalloc.
//
// Some callers cannot allocate device memory at the moment they need the
// right-hand side: code that runs where another allocator owns the whole
// device (a solver framework that pre-reserves HBM and hands out slices), or
// a host integrator that must not grow its footprint mid-run.  For them this
// file keeps every piece of device state the operator needs — constants,
// neighbour table, blending outputs, wave-speed and error words and the
// Navier-Stokes lifting scratch — in one file-scope device array of fixed
// size.  The caller passes the state and the output; nothing is allocated.
//
// The array lives in the module, so every GPU that loads this library holds
// PDG_NOALLOC_SCRATCH_DOUBLES doubles (24 MiB) of it until the process exits.
// All calls on one device share it: calls that overlap on the GPU (two
// streams, or two host threads) race on its contents.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/prandtl_b200.h"
#include "host_common.h"
#include "kernel_table.h"

using namespace pdg;
using namespace pdg_host;

namespace {

// Host code sees this name as a stand-in symbol; its device address comes
// from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) double noalloc_scratch[PDG_NOALLOC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex setup_mutex;
double *scratch_ptr[MAX_DEVICES] = {};

// Device address of the scratch array on `device` (the current device),
// looked up on the first call for that device.
int scratch_on(int device, double **out)
{
    if (device < 0 || device >= MAX_DEVICES) return PDG_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (!scratch_ptr[device]) {
        double *p = nullptr;
        if (cudaGetSymbolAddress((void **)&p, noalloc_scratch) != cudaSuccess || !p) return PDG_ERR_CUDA;
        scratch_ptr[device] = p;
    }
    *out = scratch_ptr[device];
    return PDG_OK;
}

// Region sizes are rounded up to 32 doubles so every region starts on a
// 256-byte boundary.
constexpr int64_t round32(int64_t n) { return (n + 31) & ~int64_t(31); }

}  // namespace

extern "C" int pdg_rhs_noalloc(const pdg_mesh *mesh, const pdg_params *params, const double *u, double *dudt,
                               void *stream)
{
    if (!mesh || !params || !mesh->nbr || !u || !dudt || u == dudt) return PDG_ERR_ARG;
    const int dim = mesh->dim, N = mesh->order;
    if ((dim != 2 && dim != 3) || N < 1 || N > 5 || mesh->num_elements < 1) return PDG_ERR_ARG;
    if (!(params->gamma > 1.0) || (params->parabolic && !(params->Pr > 0.0))) return PDG_ERR_ARG;
    double h[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < dim; d++) {
        if (!(mesh->h[d] > 0.0)) return PDG_ERR_ARG;
        h[d] = mesh->h[d];
    }
    const int64_t ne = mesh->num_elements;
    for (int64_t i = 0; i < ne * 2 * dim; i++)
        if (mesh->nbr[i] < 0 || mesh->nbr[i] >= ne) return PDG_ERR_ARG;
    const bool ns = params->parabolic != 0;
    const int Np = N + 1, nv = dim + 2;
    const int64_t ndof = dim == 2 ? Np * Np : Np * Np * Np, nfn = dim == 2 ? Np : Np * Np;

    // scratch layout (doubles): constants | wave speed + error word |
    // neighbour table | eta | alpha | [lifting jumps | viscous face columns]
    const int64_t o_words = round32((int64_t)((sizeof(DevConst) + 7) / 8));
    const int64_t o_nbr = o_words + 32;
    const int64_t o_eta = o_nbr + round32((ne * 2 * dim + 1) / 2);
    const int64_t o_alpha = o_eta + round32(ne);
    const int64_t o_lbuf = o_alpha + round32(ne);
    const int64_t o_fcol = o_lbuf + (ns ? round32(dim * ne * nfn * nv) : 0);
    const int64_t total = o_fcol + (ns ? round32(2 * dim * ne * nfn * (nv - 1)) : 0);
    if (total > PDG_NOALLOC_SCRATCH_DOUBLES) return PDG_ERR_CAPACITY;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return PDG_ERR_CUDA;
    double *base = nullptr;
    int r = scratch_on(device, &base);
    if (r) return r;

    DevConst K;
    double modal_threshold = 0.0;
    fill_constants(dim, N, h, K, modal_threshold);
    cudaStream_t s = (cudaStream_t)stream;
    // the wave-speed maximum and the error word must start at zero; every
    // other region is written in full before it is read
    if (cudaMemcpyAsync(base, &K, sizeof(DevConst), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemsetAsync(base + o_words, 0, 2 * sizeof(double), s) != cudaSuccess ||
        cudaMemcpyAsync(base + o_nbr, mesh->nbr, sizeof(int32_t) * ne * 2 * dim, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
        return PDG_ERR_CUDA;

    KParams P;
    std::memset(&P, 0, sizeof(P));
    P.u = u;
    P.out = dudt;
    P.K = (const DevConst *)base;
    P.lam_bits = (unsigned long long *)(base + o_words);
    P.err = (unsigned int *)(base + o_words + 1);
    P.nbr = (const int32_t *)(base + o_nbr);
    P.eta_out = base + o_eta;
    P.alpha_out = base + o_alpha;
    P.lbuf = ns ? base + o_lbuf : nullptr;
    P.fcol = ns ? base + o_fcol : nullptr;
    P.ne = ne;
    P.nnodes = ne * ndof;
    P.stage = -1;
    P.gamma = params->gamma;
    P.gm1 = params->gamma - 1.0;
    P.gm1inv = 1.0 / P.gm1;
    P.mu = params->mu;
    P.lambda_k = params->mu * params->gamma * (1.0 / (ns ? params->Pr : 1.0));
    P.alpha_max = params->alpha_max;
    P.alpha_min = params->alpha_min;
    P.modal_threshold = modal_threshold;
    P.diss_scale = params->face_dissipation;
    P.blending = params->blending;
    P.compat = params->compat;
    P.prefetch = 1;

    // same kernel sequence as pdg_rhs
    const int seq_ns[] = {KIND_LIFT_FACE, KIND_NS, KIND_LIFT, KIND_FACE_NS0, KIND_FACE_NS0 + 1, KIND_FACE_NS0 + 2};
    const int seq_eu[] = {KIND_EULER, KIND_FACE_E0, KIND_FACE_E0 + 1, KIND_FACE_E0 + 2};
    const int *seq = ns ? seq_ns : seq_eu;
    const int count = (ns ? 3 : 1) + dim;
    for (int i = 0; i < count; i++) {
        LaunchCfg cfg;
        const char *why = "";
        if ((r = kernel_config(dim, N, seq[i], ne, device, &cfg, &why))) return r;
        if ((r = launch_kernel(cfg, P, ne, s))) return r;
    }
    return PDG_OK;
}
