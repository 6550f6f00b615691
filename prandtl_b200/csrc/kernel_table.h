// kernel_table.h — host-side view of the templated element kernels.
#pragma once

namespace pdg {

enum KernelKind { KIND_EULER = 0, KIND_LIFT = 1, KIND_NS = 2, KIND_NSFACE = 3, KIND_COUNT = 4 };

struct KernelInfo {
    const void *fn;   // __global__ function, argument: const KParams
    int el_doubles;   // shared doubles per element slot (0: thread-per-face-node kernel)
    int epw;          // elements per warp
};

bool kernel_info_2d(int N, int kind, KernelInfo *out);
bool kernel_info_3d(int N, int kind, KernelInfo *out);

}  // namespace pdg
