// kernels_2d.cu — instantiations of the 2D kernels for N = 1..5 and the
// table the host dispatches through.
#include "kernel_table.h"
#include "line_kernels.cuh"
#include "filter_kernels.cuh"
#include "geo_kernels.cuh"

namespace pdg {

template <int N> static bool info_n(int kind, KernelInfo *out)
{
    using S = Shape<2, N>;
    out->epw = S::EPW;
    out->el_doubles = 0;
    switch (kind) {
    case KIND_EULER: out->fn = (const void *)&rhs_kernel<2, N, false>; out->el_doubles = S::EL_RHS; break;
    case KIND_NS: out->fn = (const void *)&rhs_kernel<2, N, true>; out->el_doubles = S::EL_RHS; break;
    case KIND_EULER_FACES: out->fn = (const void *)&rhs_kernel<2, N, false, true>; out->el_doubles = S::EL_RHS; break;
    case KIND_NS_FACES: out->fn = (const void *)&rhs_kernel<2, N, true, true>; out->el_doubles = S::EL_RHS; break;
    case KIND_BOUNDARY: out->fn = (const void *)&boundary_kernel<2, N>; break;
    case KIND_BOUNDARY_NS: out->fn = (const void *)&boundary_kernel<2, N, true>; break;
    case KIND_EULER_FACES_BDR:
        out->fn = (const void *)&rhs_kernel<2, N, false, true, true>;
        out->el_doubles = S::EL_RHS;
        break;
    case KIND_NS_FACES_BDR:
        out->fn = (const void *)&rhs_kernel<2, N, true, true, true>;
        out->el_doubles = S::EL_RHS;
        break;
    case KIND_LIFT_FACE_BDR: out->fn = (const void *)&lift_face_kernel<2, N, true>; break;
    case KIND_LIFT_BDR: out->fn = (const void *)&lift_kernel<2, N, true>; out->el_doubles = S::EL_LIFTF; break;
    case KIND_LIFT_BDR_PTTT: out->fn = (const void *)&lift_kernel<2, N, true, true>; out->el_doubles = S::EL_LIFTF; break;
    case KIND_LIFT: out->fn = (const void *)&lift_kernel<2, N>; out->el_doubles = S::EL_LIFTF; break;
    case KIND_LIFT_FACE: out->fn = (const void *)&lift_face_kernel<2, N>; break;
    case KIND_LIFT_FACE_FLUX: out->fn = (const void *)&lift_face_kernel<2, N, false, FACE_JUMP | FACE_FLUX>; break;
    case KIND_FACE_FLUX: out->fn = (const void *)&lift_face_kernel<2, N, false, FACE_FLUX>; break;
    case KIND_NS_FACES_FB:
        out->fn = (const void *)&rhs_kernel<2, N, true, true, false, true>;
        out->el_doubles = S::EL_RHS_FB;
        break;
    case KIND_EULER_FACES_FB:
        out->fn = (const void *)&rhs_kernel<2, N, false, true, false, true>;
        out->el_doubles = S::EL_RHS_FB;
        break;
    case KIND_FACE_E0: out->fn = (const void *)&face_kernel<2, N, 0, false>; break;
    case KIND_FACE_E1: out->fn = (const void *)&face_kernel<2, N, 1, false>; break;
    
    case KIND_FACE_NS0: out->fn = (const void *)&face_kernel<2, N, 0, true>; break;
    case KIND_FACE_NS1: out->fn = (const void *)&face_kernel<2, N, 1, true>; break;
    
    case KIND_FILTER_BOUNDS: out->fn = (const void *)&filter_bounds_kernel<2, N>; out->epw = 1; break;
    case KIND_POSITIVITY: out->fn = (const void *)&positivity_kernel<2, N>; out->epw = 1; break;
    case KIND_GEO: out->fn = (const void *)&geo_rhs_kernel<2, N>; out->el_doubles = GeoShape<2, N, false>::EL; break;
    case KIND_GEO_NS: out->fn = (const void *)&geo_rhs_kernel<2, N, true>; out->el_doubles = GeoShape<2, N, true>::EL; break;
    case KIND_GEO_LIFT: out->fn = (const void *)&geo_lift_kernel<2, N>; out->el_doubles = GeoLiftShape<2, N>::EL; break;
    case KIND_FILTER:
        out->fn = (const void *)&filter_kernel<2, N>;
        out->el_doubles = FilterShape<2, N>::EL;
        out->epw = 1;
        break;
    default: return adj_kernel_info_2d(N, kind, out);
    }
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
