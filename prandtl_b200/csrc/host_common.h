// host_common.h — host helpers shared by the context-based entry points
// (capi.cu) and the allocation-free entry point (noalloc.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernel_table.h"
#include "line_kernels.cuh"

namespace pdg_host {

using pdg::DevConst;
using pdg::KernelInfo;
using pdg::KParams;

struct LaunchCfg {
    KernelInfo ki;
    int wpb;      // warps per block
    int grid;     // blocks
    size_t smem;  // dynamic shared memory bytes
};

// LGL operators, subcell normals and modal transform of an affine element
// of extents h (DGSEMIntegrator ctor, DGSEMIntegrator.cpp:41-149).
void fill_constants(int dim, int N, const double *h, DevConst &K, double &modal_threshold);

// Kernel, block and grid for one kernel kind on `device` (sets the kernel's
// dynamic shared-memory limit).  No allocation.
int kernel_config(int dim, int N, int kind, int64_t ne, int device, LaunchCfg *cfg, const char **why);

// Whether a kernel kind takes part in the (dim, parabolic, filter) operator.
bool kind_used(int kind, int dim, bool parabolic, int filter);  // filter: params.filter bits

int launch_kernel(const LaunchCfg &cfg, KParams P, int64_t ne, cudaStream_t s);

}  // namespace pdg_host
