// adjoint_3d.cu — instantiations of the 3D adjoint kernels for N = 1..5.
#include "adjoint_kernels.cuh"
#include "kernel_table.h"

namespace pdg {

template <int N> static bool adj_info_n(int kind, KernelInfo *out)
{
    using S = Shape<3, N>;
    out->epw = S::EPW;
    out->el_doubles = 0;
    switch (kind) {
    case KIND_ADJ_RHS:
        out->fn = (const void *)&adj_rhs_kernel<3, N>;
        out->el_doubles = AdjShape<3, N>::EL;
        break;
    case KIND_ADJ_LIFT:
        out->fn = (const void *)&adj_lift_kernel<3, N>;
        out->el_doubles = S::EL_LIFT;
        out->wpb = AdjLiftLaunch<3, N>::wpb;
        break;
    case KIND_ADJ_FACE_E0: out->fn = (const void *)&adj_faces_kernel<3, N, false>; break;
    case KIND_ADJ_FACE_NS0: out->fn = (const void *)&adj_faces_kernel<3, N, true>; break;
    case KIND_ADJ_GATHER: out->fn = (const void *)&adj_gather_kernel<3, N>; break;
    case KIND_ADJ_BOUNDARY: out->fn = (const void *)&adj_boundary_kernel<3, N>; break;
    default: return false;
    }
    return true;
}

bool adj_kernel_info_3d(int N, int kind, KernelInfo *out)
{
    switch (N) {
    case 1: return adj_info_n<1>(kind, out);
    case 2: return adj_info_n<2>(kind, out);
    case 3: return adj_info_n<3>(kind, out);
    case 4: return adj_info_n<4>(kind, out);
    case 5: return adj_info_n<5>(kind, out);
    default: return false;
    }
}

}  // namespace pdg
