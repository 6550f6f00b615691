// kernels_2d.cu — instantiations of the 2D element kernels for N = 1..5
// and the table the host dispatches through.
#include "dgsem_kernels.cuh"
#include "kernel_table.h"

namespace pdg {

template <int N> static bool info_n(int kind, KernelInfo *out)
{
    using S = Shape<2, N>;
    out->epw = S::EPW;
    if (kind == KIND_EULER) { out->fn = (const void *)&euler_rhs_kernel<2, N>; out->el_doubles = S::EL_EULER; }
    else if (kind == KIND_LIFT) { out->fn = (const void *)&lift_kernel<2, N>; out->el_doubles = S::EL_LIFT; }
    else if (kind == KIND_NS) { out->fn = (const void *)&ns_rhs_kernel<2, N>; out->el_doubles = S::EL_NS; }
    else if (kind == KIND_NSFACE) { out->fn = (const void *)&ns_face_kernel<2, N>; out->el_doubles = 0; }
    else return false;
    return true;
}

bool kernel_info_2d(int N, int kind, KernelInfo *out)
{
    switch (N) {
    case 1: return info_n<1>(kind, out);
    case 2: return info_n<2>(kind, out);
    case 3: return info_n<3>(kind, out);
    case 4: return info_n<4>(kind, out);
    case 5: return info_n<5>(kind, out);
    default: return false;
    }
}

}  // namespace pdg
