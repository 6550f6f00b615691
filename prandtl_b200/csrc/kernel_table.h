// kernel_table.h — host-side view of the templated kernels.
#pragma once

namespace pdg {

enum KernelKind {
    KIND_EULER = 0,     // rhs_kernel<dim, N, false>
    KIND_LIFT = 1,      // lift_kernel<dim, N>
    KIND_NS = 2,        // rhs_kernel<dim, N, true>
    KIND_FACE_NS = 3,   // face_kernel<dim, N, true>
    KIND_FACE_EULER = 4,// face_kernel<dim, N, false>
    KIND_LIFT_FACE = 5, // lift_face_kernel<dim, N>
    KIND_COUNT = 6
};

struct KernelInfo {
    const void *fn;   // __global__ function, argument: const KParams
    int el_doubles;   // shared doubles per element slot (0: thread-per-face-node kernel)
    int epw;          // elements per warp
};

bool kernel_info_2d(int N, int kind, KernelInfo *out);
bool kernel_info_3d(int N, int kind, KernelInfo *out);

}  // namespace pdg
