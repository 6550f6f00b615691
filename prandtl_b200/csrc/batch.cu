// batch.cu — many independent periodic 2D Euler cases of uneven size and
// order in one persistent launch per SSP-RK3 stage.
//
// The reference runs one case per process (Simulation::Run, src/Simulation/
// Simulation.cpp:800-1020); a parameter sweep there is a loop of runs.  Here
// the cases' states are concatenated (each in its own byNODES block), every
// case keeps its own mesh constants, neighbour table, time step and running
// wave-speed maximum, and one kernel launch walks a tile list covering all
// cases: a warp takes tiles (case, EPW elements of it) from a global counter,
// computes the volume terms, the subcell blending and — element-centrically —
// the face terms of its own face nodes, and stores the finished stage.  One
// step is three such launches, captured once in a CUDA graph.  The warps per
// block, the tiles taken per counter fetch and the tile order are chosen by
// pdg_batch_tune, which times each candidate on the caller's state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prandtl_b200.h"
#include "host_common.h"
#include "line_kernels.cuh"

namespace pdg {

// Highest order the batched kernel is compiled for (its register budget is
// that of its largest instantiation).
#ifndef PDG_BATCH_MAX_N
#define PDG_BATCH_MAX_N 5
#endif

template <int N> constexpr int batch_slot_n() { return N <= PDG_BATCH_MAX_N ? Shape<2, N>::EPW * Shape<2, N>::EL_RHS : 0; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }
// per-warp shared memory: the case's constants and the largest tile slot
constexpr int BATCH_SLOT = cmax(cmax(cmax(batch_slot_n<1>(), batch_slot_n<2>()), cmax(batch_slot_n<3>(), batch_slot_n<4>())),
                                batch_slot_n<5>());
constexpr int BATCH_WARP_DOUBLES = CONST_SLOTS + BATCH_SLOT;

struct BatchArgs {
    const KParams *__restrict__ params;  // per case, for this launch
    const int2 *tiles;      // (case, first element)
    const int *order;       // polynomial order per case
    unsigned int *counter;  // next tile; zero at launch
    unsigned int *err;
    int ntiles, chunk;
};

template <int N>
__device__ __forceinline__ void batch_tile(const KParams &P, const double *c, double *slot, int64_t e_base, int lane,
                                           unsigned int &flags, double &lam)
{
    using S = Shape<2, N>;
    const int grp = lane / S::L, gl = lane % S::L;
    const bool lane_used = grp < S::EPW;
    double *pr = slot + (lane_used ? grp : 0) * S::EL_RHS;
    rhs_tile<2, N, false, true, false>(P, c, pr, e_base, grp, gl, lane_used, flags, lam);
}

// MINB = minimum resident blocks per SM the compiler must allow (register
// budget): MINB = 1 with 256 threads gives up to 255 registers, MINB = 3 with
// 128 threads 170, MINB = 4 with 128 threads 128.  The autotuner chooses.
template <int MINB>
__global__ void __launch_bounds__(MINB == 1 ? 256 : 128, MINB) batch_stage_kernel(const BatchArgs A)
{
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *c = smem + (size_t)warp * BATCH_WARP_DOUBLES;
    double *slot = c + CONST_SLOTS;
    int cur = -1;
    unsigned int flags = 0;
    for (;;) {
        unsigned int t0 = 0;
        if (lane == 0) t0 = atomicAdd(A.counter, (unsigned int)A.chunk);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        if (t0 >= (unsigned int)A.ntiles) break;
        const unsigned int t1 = min(t0 + (unsigned int)A.chunk, (unsigned int)A.ntiles);
        for (unsigned int t = t0; t < t1; t++) {
            const int2 tile = A.tiles[t];
            const KParams &P = A.params[tile.x];
            const int N = A.order[tile.x];
            if (tile.x != cur) {
                __syncwarp();
                load_consts(P.K, c, N + 1, lane, 32);
                __syncwarp();
                cur = tile.x;
            }
            double lam = 0.0;
            switch (N) {
            case 1: batch_tile<1>(P, c, slot, tile.y, lane, flags, lam); break;
#if PDG_BATCH_MAX_N >= 2
            case 2: batch_tile<2>(P, c, slot, tile.y, lane, flags, lam); break;
#endif
#if PDG_BATCH_MAX_N >= 3
            case 3: batch_tile<3>(P, c, slot, tile.y, lane, flags, lam); break;
#endif
#if PDG_BATCH_MAX_N >= 4
            case 4: batch_tile<4>(P, c, slot, tile.y, lane, flags, lam); break;
#endif
#if PDG_BATCH_MAX_N >= 5
            case 5: batch_tile<5>(P, c, slot, tile.y, lane, flags, lam); break;
#endif
            default: break;
            }
            lam = group_max<32>(lam);
            if (lane == 0) atomic_max_pos(P.lam_bits, lam);
        }
    }
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(A.err, flags);
}

struct BatchVariant {
    const void *fn;
    int max_wpb;
};
static const BatchVariant BATCH_VARIANTS[] = {{(const void *)&batch_stage_kernel<1>, 8},
                                              {(const void *)&batch_stage_kernel<3>, 4},
                                              {(const void *)&batch_stage_kernel<4>, 4}};
constexpr int BATCH_NVARIANTS = 3;

}  // namespace pdg

using namespace pdg;
using namespace pdg_host;

struct pdg_batch {
    pdg_params p;
    int ncases = 0, device = 0, sms = 0;
    std::vector<int> order;
    std::vector<int64_t> ne, off, eoff;  // per case: elements, state offset, element offset
    std::vector<double> hmin, dt, modal_threshold;
    int64_t total = 0, total_ne = 0;
    DevConst *K = nullptr;
    int32_t *nbr = nullptr;
    double *eta = nullptr, *alpha = nullptr;
    unsigned long long *lam = nullptr;
    unsigned int *err = nullptr, *counters = nullptr;  // one tile counter per launch slot
    int *d_order = nullptr;
    int2 *tiles = nullptr;
    int ntiles = 0;
    std::vector<int2> tiles_by_order, tiles_by_case;
    int tile_order = 0;          // 0: highest order first, 1: case by case
    KParams *params = nullptr;   // [4][ncases]: stages 0, 1, 2 and the plain RHS
    std::vector<KParams> hstage, hrhs;
    double *stage_a = nullptr, *stage_b = nullptr;
    const double *params_x = nullptr;
    bool params_dirty = true;
    int wpb = 4, grid = 0, chunk = 2, variant = 0;
    size_t smem = 0;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    float tuned_ms = -1.0f;
    std::string last_error;
};

namespace {

int bfail(pdg_batch *b, int code, const char *fmt, ...)
{
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        b->last_error = buf;
    }
    return code;
}

#define BCK(call, what)                                                                                        \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return bfail(b, PDG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e_));          \
    } while (0)

void drop_graph(pdg_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int configure(pdg_batch *b, int wpb, int chunk, int variant)
{
    const void *fn = BATCH_VARIANTS[variant].fn;
    if (wpb > BATCH_VARIANTS[variant].max_wpb) return bfail(b, PDG_ERR_UNSUPPORTED, "block too large for the variant");
    const size_t smem = (size_t)wpb * BATCH_WARP_DOUBLES * sizeof(double);
    int max_smem = 0;
    BCK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device), "device attribute");
    if (smem > (size_t)max_smem) return bfail(b, PDG_ERR_UNSUPPORTED, "batch block does not fit in shared memory");
    BCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
    int per_sm = 0;
    BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wpb, smem), "occupancy");
    if (per_sm < 1) return bfail(b, PDG_ERR_UNSUPPORTED, "batch kernel cannot be resident");
    if (wpb != b->wpb || chunk != b->chunk || variant != b->variant) drop_graph(b);
    b->wpb = wpb;
    b->chunk = chunk;
    b->variant = variant;
    b->smem = smem;
    b->grid = b->sms * per_sm;
    return PDG_OK;
}

int upload_tiles(pdg_batch *b, int tile_order, cudaStream_t s)
{
    const std::vector<int2> &t = tile_order == 0 ? b->tiles_by_order : b->tiles_by_case;
    BCK(cudaMemcpyAsync(b->tiles, t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice, s), "upload tiles");
    b->tile_order = tile_order;
    return PDG_OK;
}

KParams case_params(const pdg_batch *b, int c)
{
    KParams P;
    std::memset(&P, 0, sizeof(P));
    const int Np = b->order[c] + 1;
    P.nbr = b->nbr + b->eoff[c] * 4;
    P.K = b->K + c;
    P.eta_out = b->eta + b->eoff[c];
    P.alpha_out = b->alpha + b->eoff[c];
    P.lam_bits = b->lam + c;
    P.err = b->err;
    P.ne = b->ne[c];
    P.nnodes = b->ne[c] * Np * Np;
    P.nwt = 0;
    P.gamma = b->p.gamma;
    P.gm1 = b->p.gamma - 1.0;
    P.gm1inv = 1.0 / P.gm1;
    P.alpha_max = b->p.alpha_max;
    P.alpha_min = b->p.alpha_min;
    P.modal_threshold = b->modal_threshold[c];
    P.diss_scale = b->p.face_dissipation;
    P.blending = b->p.blending;
    P.compat = b->p.compat;
    P.dt = b->dt[c];
    return P;
}

int upload_stage_params(pdg_batch *b, double *x, cudaStream_t s)
{
    const int nc = b->ncases;
    b->hstage.resize(3 * (size_t)nc);
    for (int st = 0; st < 3; st++)
        for (int c = 0; c < nc; c++) {
            KParams P = case_params(b, c);
            double *in = st == 0 ? x : (st == 1 ? b->stage_a : b->stage_b);
            double *out = st == 0 ? b->stage_a : (st == 1 ? b->stage_b : x);
            P.u = in + b->off[c];
            P.un = x + b->off[c];
            P.out = out + b->off[c];
            P.stage = st;
            b->hstage[(size_t)st * nc + c] = P;
        }
    BCK(cudaMemcpyAsync(b->params, b->hstage.data(), sizeof(KParams) * b->hstage.size(), cudaMemcpyHostToDevice, s),
        "upload stage parameters");
    b->params_x = x;
    b->params_dirty = false;
    return PDG_OK;
}

int launch_stage(pdg_batch *b, int slot, cudaStream_t s)
{
    BCK(cudaMemsetAsync(b->counters + slot, 0, sizeof(unsigned int), s), "reset tile counter");
    BatchArgs A;
    A.params = b->params + (size_t)slot * b->ncases;
    A.tiles = b->tiles;
    A.order = b->d_order;
    A.counter = b->counters + slot;
    A.err = b->err;
    A.ntiles = b->ntiles;
    A.chunk = b->chunk;
    void *args[] = {&A};
    BCK(cudaLaunchKernel(BATCH_VARIANTS[b->variant].fn, dim3(b->grid), dim3(32 * b->wpb), args, b->smem, s),
        "batch kernel launch");
    b->launches++;
    return PDG_OK;
}

int rhs_launch(pdg_batch *b, const double *u, double *dudt, cudaStream_t s)
{
    const int nc = b->ncases;
    b->hrhs.resize(nc);
    for (int c = 0; c < nc; c++) {
        KParams P = case_params(b, c);
        P.u = u + b->off[c];
        P.out = dudt + b->off[c];
        P.stage = -1;
        b->hrhs[c] = P;
    }
    BCK(cudaMemcpyAsync(b->params + 3 * (size_t)nc, b->hrhs.data(), sizeof(KParams) * nc, cudaMemcpyHostToDevice, s),
        "upload parameters");
    return launch_stage(b, 3, s);
}

}  // namespace

extern "C" {

int pdg_batch_create(int ncases, const pdg_mesh *meshes, const pdg_params *params, pdg_batch **out)
{
    if (!out) return PDG_ERR_ARG;
    *out = nullptr;
    if (ncases < 1 || !meshes || !params) return PDG_ERR_ARG;
    if (params->parabolic || params->filter || !(params->gamma > 1.0)) return PDG_ERR_UNSUPPORTED;
    pdg_batch *b = new pdg_batch();
    b->p = *params;
    b->ncases = ncases;
    auto cleanup = [&](int code) {
        pdg_batch_destroy(b);
        return code;
    };
    std::vector<DevConst> hK(ncases);
    std::vector<int32_t> hnbr;
    for (int c = 0; c < ncases; c++) {
        const pdg_mesh &m = meshes[c];
        if (m.dim != 2 || m.order < 1 || m.order > PDG_BATCH_MAX_N || m.num_elements < 1 || !m.nbr || !(m.h[0] > 0.0) ||
            !(m.h[1] > 0.0))
            return cleanup(PDG_ERR_ARG);
        const int Np = m.order + 1;
        for (int64_t i = 0; i < m.num_elements * 4; i++)
            if (m.nbr[i] < 0 || m.nbr[i] >= m.num_elements) return cleanup(PDG_ERR_ARG);
        b->order.push_back(m.order);
        b->ne.push_back(m.num_elements);
        b->off.push_back(b->total);
        b->eoff.push_back(b->total_ne);
        b->hmin.push_back(std::min(m.h[0], m.h[1]));
        b->dt.push_back(0.0);
        const double h[3] = {m.h[0], m.h[1], 1.0};
        double thr = 0.0;
        fill_constants(2, m.order, h, hK[c], thr);
        b->modal_threshold.push_back(thr);
        b->total += m.num_elements * Np * Np * 4;
        b->total_ne += m.num_elements;
        hnbr.insert(hnbr.end(), m.nbr, m.nbr + m.num_elements * 4);
        const int epw = 32 / (Np <= 2 ? 2 : (Np <= 4 ? 4 : 8));
        for (int64_t e = 0; e < m.num_elements; e += epw) {
            if (e > 0x7fffffff) return cleanup(PDG_ERR_ARG);
            b->tiles_by_case.push_back(make_int2(c, (int)e));
        }
    }
    b->ntiles = (int)b->tiles_by_case.size();
    b->tiles_by_order = b->tiles_by_case;
    std::stable_sort(b->tiles_by_order.begin(), b->tiles_by_order.end(),
                     [&](const int2 &x, const int2 &y) { return b->order[x.x] > b->order[y.x]; });
    if (cudaGetDevice(&b->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
        return cleanup(PDG_ERR_CUDA);
    const size_t fbytes = sizeof(double) * (size_t)b->total;
    if (cudaMalloc(&b->K, sizeof(DevConst) * ncases) || cudaMalloc(&b->nbr, sizeof(int32_t) * hnbr.size()) ||
        cudaMalloc(&b->eta, sizeof(double) * b->total_ne) || cudaMalloc(&b->alpha, sizeof(double) * b->total_ne) ||
        cudaMalloc(&b->lam, sizeof(unsigned long long) * ncases) || cudaMalloc(&b->err, sizeof(unsigned int)) ||
        cudaMalloc(&b->counters, 4 * sizeof(unsigned int)) || cudaMalloc(&b->d_order, sizeof(int) * ncases) ||
        cudaMalloc(&b->tiles, sizeof(int2) * b->ntiles) || cudaMalloc(&b->params, sizeof(KParams) * 4 * ncases) ||
        cudaMalloc(&b->stage_a, fbytes) || cudaMalloc(&b->stage_b, fbytes))
        return cleanup(PDG_ERR_NOMEM);
    if (cudaMemcpy(b->K, hK.data(), sizeof(DevConst) * ncases, cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->nbr, hnbr.data(), sizeof(int32_t) * hnbr.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->d_order, b->order.data(), sizeof(int) * ncases, cudaMemcpyHostToDevice) ||
        cudaMemcpy(b->tiles, b->tiles_by_order.data(), sizeof(int2) * b->ntiles, cudaMemcpyHostToDevice) ||
        cudaMemset(b->lam, 0, sizeof(unsigned long long) * ncases) || cudaMemset(b->err, 0, sizeof(unsigned int)) ||
        cudaMemset(b->eta, 0, sizeof(double) * b->total_ne) || cudaMemset(b->alpha, 0, sizeof(double) * b->total_ne))
        return cleanup(PDG_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) return cleanup(PDG_ERR_CUDA);
    const int r = configure(b, 4, 2, 0);
    if (r) return cleanup(r);
    *out = b;
    return PDG_OK;
}

int pdg_batch_destroy(pdg_batch *b)
{
    if (!b) return PDG_OK;
    drop_graph(b);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->K);
    cudaFree(b->nbr);
    cudaFree(b->eta);
    cudaFree(b->alpha);
    cudaFree(b->lam);
    cudaFree(b->err);
    cudaFree(b->counters);
    cudaFree(b->d_order);
    cudaFree(b->tiles);
    cudaFree(b->params);
    cudaFree(b->stage_a);
    cudaFree(b->stage_b);
    delete b;
    return PDG_OK;
}

int64_t pdg_batch_offset(const pdg_batch *b, int case_index)
{
    if (!b || case_index < 0 || case_index > b->ncases) return -1;
    return case_index == b->ncases ? b->total : b->off[case_index];
}

int pdg_batch_set_dt(pdg_batch *b, const double *dt)
{
    if (!b || !dt) return PDG_ERR_ARG;
    for (int c = 0; c < b->ncases; c++) {
        if (!(dt[c] >= 0.0)) return bfail(b, PDG_ERR_ARG, "pdg_batch_set_dt: case %d has dt %g", c, dt[c]);
        b->dt[c] = dt[c];
    }
    b->params_dirty = true;
    return PDG_OK;
}

int pdg_batch_rhs(pdg_batch *b, const double *u, double *dudt, void *stream)
{
    if (!b) return PDG_ERR_ARG;
    if (!u || !dudt || u == dudt) return bfail(b, PDG_ERR_ARG, "pdg_batch_rhs: null or aliased buffers");
    return rhs_launch(b, u, dudt, (cudaStream_t)stream);
}

int pdg_batch_rk3_step(pdg_batch *b, double *u, int nsteps, int use_graph, void *stream)
{
    if (!b) return PDG_ERR_ARG;
    if (!u || nsteps < 0) return bfail(b, PDG_ERR_ARG, "pdg_batch_rk3_step: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    int r;
    if (u != b->params_x || b->params_dirty)
        if ((r = upload_stage_params(b, u, s))) return r;
    if (!use_graph) {
        for (int i = 0; i < nsteps; i++)
            for (int st = 0; st < 3; st++)
                if ((r = launch_stage(b, st, s))) return r;
        return PDG_OK;
    }
    if (!b->exec) {
        // the graph reads its per-case parameters (state pointers, dt) from
        // device memory, so it only depends on the launch configuration
        BCK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        int rc = PDG_OK;
        for (int st = 0; st < 3 && rc == PDG_OK; st++) rc = launch_stage(b, st, b->cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return bfail(b, PDG_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
        b->graph = g;
        BCK(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
        b->launches -= 3;  // counted per replay below
    }
    for (int i = 0; i < nsteps; i++) {
        BCK(cudaGraphLaunch(b->exec, s), "graph launch");
        b->launches += 3;
    }
    return PDG_OK;
}

int pdg_batch_tune(pdg_batch *b, const double *u, void *stream, float *best_ms)
{
    if (!b || !u) return PDG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCK(cudaEventCreate(&e0), "event");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return bfail(b, PDG_ERR_CUDA, "event");
    }
    const int wpbs[] = {1, 2, 4, 8}, chunks[] = {1, 2, 4, 8};
    float best = 1e30f;
    int bw = b->wpb, bc = b->chunk, bo = b->tile_order, bv = b->variant;
    int r = PDG_OK;
    for (int order = 0; order < 2 && r == PDG_OK; order++) {
        if ((r = upload_tiles(b, order, s))) break;
        for (int variant = 0; variant < BATCH_NVARIANTS && r == PDG_OK; variant++)
        for (int wpb : wpbs) {
            for (int chunk : chunks) {
                if (configure(b, wpb, chunk, variant) != PDG_OK) continue;  // does not fit: skip the candidate
                if ((r = rhs_launch(b, u, b->stage_a, s))) break;  // warm-up
                if (cudaEventRecord(e0, s) != cudaSuccess) { r = PDG_ERR_CUDA; break; }
                for (int k = 0; k < 3 && r == PDG_OK; k++) r = rhs_launch(b, u, b->stage_a, s);
                if (r || cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
                    r = r ? r : PDG_ERR_CUDA;
                    break;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= 3.0f;
                if (ms < best) {
                    best = ms;
                    bw = wpb;
                    bc = chunk;
                    bo = order;
                    bv = variant;
                }
            }
            if (r) break;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r) return r;
    if ((r = upload_tiles(b, bo, s))) return r;
    if ((r = configure(b, bw, bc, bv))) return r;
    drop_graph(b);
    b->tuned_ms = best;
    if (best_ms) *best_ms = best;
    BCK(cudaStreamSynchronize(s), "synchronize");
    return PDG_OK;
}

int pdg_batch_config(const pdg_batch *b, int *warps_per_block, int *blocks, int *chunk, int *tile_order,
                     int *register_variant)
{
    if (!b) return PDG_ERR_ARG;
    if (register_variant) *register_variant = b->variant;
    if (warps_per_block) *warps_per_block = b->wpb;
    if (blocks) *blocks = b->grid;
    if (chunk) *chunk = b->chunk;
    if (tile_order) *tile_order = b->tile_order;
    return PDG_OK;
}

int pdg_batch_max_char_speed(pdg_batch *b, double *lam)
{
    if (!b || !lam) return PDG_ERR_ARG;
    std::vector<unsigned long long> bits(b->ncases);
    BCK(cudaDeviceSynchronize(), "synchronize");
    BCK(cudaMemcpy(bits.data(), b->lam, sizeof(unsigned long long) * b->ncases, cudaMemcpyDeviceToHost), "read");
    for (int c = 0; c < b->ncases; c++) std::memcpy(&lam[c], &bits[c], sizeof(double));
    return PDG_OK;
}

int pdg_batch_check(pdg_batch *b, uint32_t *flags)
{
    if (!b || !flags) return PDG_ERR_ARG;
    unsigned int f = 0;
    BCK(cudaDeviceSynchronize(), "synchronize");
    BCK(cudaMemcpy(&f, b->err, sizeof(f), cudaMemcpyDeviceToHost), "read error word");
    BCK(cudaMemset(b->err, 0, sizeof(f)), "clear error word");
    *flags = f;
    if (f & PDG_FLAG_NONFINITE) return bfail(b, PDG_ERR_NONFINITE, "non-finite value in a state");
    if (f & PDG_FLAG_NONPHYSICAL) return bfail(b, PDG_ERR_NONPHYSICAL, "non-positive density or pressure");
    return PDG_OK;
}

int64_t pdg_batch_launch_count(const pdg_batch *b) { return b ? b->launches : -1; }

const char *pdg_batch_last_error(const pdg_batch *b) { return b ? b->last_error.c_str() : "null batch"; }

}  // extern "C"
