// kernel_table.h — host-side view of the templated kernels.
#pragma once

namespace pdg {

enum KernelKind {
    KIND_EULER = 0,      // rhs_kernel<dim, N, false>: Euler volume terms (+ stage)
    KIND_LIFT = 1,       // lift_kernel<dim, N>: BR1 gradients, viscous volume term, face columns
    KIND_NS = 2,         // rhs_kernel<dim, N, true>: NS inviscid volume terms (+ stage)
    KIND_LIFT_FACE = 3,  // lift_face_kernel<dim, N>
    KIND_FACE_E0 = 4,    // face_kernel<dim, N, d, false>, d = 0, 1, 2
    KIND_FACE_E1 = 5,
    KIND_FACE_E2 = 6,
    KIND_FACE_NS0 = 7,   // face_kernel<dim, N, d, true>, d = 0, 1, 2
    KIND_FACE_NS1 = 8,
    KIND_FACE_NS2 = 9,
    KIND_FILTER_BOUNDS = 10,  // filter_bounds_kernel<dim, N>: per-element entropy minimum
    KIND_FILTER = 11,         // filter_kernel<dim, N>: entropy/positivity filter of the stage output
    KIND_ADJ_RHS = 12,        // adj_rhs_kernel<dim, N>: adjoint of the inviscid volume terms and blending
    KIND_ADJ_LIFT = 13,       // adj_lift_kernel<dim, N>: adjoint of the viscous terms
    KIND_ADJ_FACE_E0 = 14,    // adj_faces_kernel<dim, N, false>: every direction's adjoint face terms (Euler)
    KIND_ADJ_GATHER = 15,     // adj_gather_kernel<dim, N>: adds the face terms to ubar (+ an RK stage's adjoint)
    KIND_ADJ_FACE_E2 = 16,    // (unused)
    KIND_ADJ_FACE_NS0 = 17,   // adj_faces_kernel<dim, N, true>: the same with the BR1 jumps (NS)
    KIND_ADJ_FACE_NS1 = 18,   // (unused)
    KIND_ADJ_FACE_NS2 = 19,   // (unused)
    KIND_EULER_FACES = 20,    // rhs_kernel<dim, N, false, true>: Euler volume + face terms (+ stage)
    KIND_NS_FACES = 21,       // rhs_kernel<dim, N, true, true>: NS inviscid volume + all face terms (+ stage)
    KIND_BOUNDARY = 22,       // boundary_kernel<dim, N>: boundary faces of the separate-face path (Euler)
    KIND_ADJ_BOUNDARY = 23,   // adj_boundary_kernel<dim, N>: adjoint of the boundary faces (Euler)
    KIND_EULER_FACES_BDR = 24,  // rhs_kernel<dim, N, false, true, true>: KIND_EULER_FACES for meshes with boundaries
    KIND_LIFT_FACE_BDR = 25,    // lift_face_kernel<dim, N, true>: NS meshes with boundary faces
    KIND_LIFT_BDR = 26,         // lift_kernel<dim, N, true>
    KIND_NS_FACES_BDR = 27,     // rhs_kernel<dim, N, true, true, true>
    KIND_BOUNDARY_NS = 28,      // boundary_kernel<dim, N, true>: NS boundary faces of the separate-face path
    KIND_LIFT_BDR_PTTT = 29,    // lift_kernel<2, N, true, true>: a mesh with a total-pressure inflow (2D)
    KIND_NS_FACES_FB = 30,      // rhs_kernel<dim, N, true, true, false, true>: KIND_NS_FACES reading the face-flux buffer
    KIND_EULER_FACES_FB = 31,   // rhs_kernel<dim, N, false, true, false, true>: KIND_EULER_FACES reading it
    KIND_LIFT_FACE_FLUX = 32,   // lift_face_kernel<dim, N, false, FACE_JUMP | FACE_FLUX>: jumps + face fluxes (NS)
    KIND_FACE_FLUX = 33,        // lift_face_kernel<dim, N, false, FACE_FLUX>: face fluxes (Euler)
    KIND_POSITIVITY = 34,       // positivity_kernel<dim, N>: positivity limiter of the stage output
    KIND_GEO = 35,              // geo_rhs_kernel<dim, N>: Euler right-hand side (+ stage) on a general-geometry mesh
    KIND_GEO_LIFT = 36,         // geo_lift_kernel<dim, N>: BR1 primitive gradients on a general-geometry mesh
    KIND_GEO_NS = 37,           // geo_rhs_kernel<dim, N, true>: Navier-Stokes right-hand side (+ stage), general geometry
    KIND_COUNT = 38
};

struct KernelInfo {
    const void *fn;   // __global__ function, argument: const KParams
    int el_doubles;   // shared doubles per element slot (0: thread-per-face-node kernel)
    int epw;          // elements per warp
    int wpb = 4;      // warps per block of an element kernel (fewer when shared memory is short)
};

bool kernel_info_2d(int N, int kind, KernelInfo *out);
bool adj_kernel_info_2d(int N, int kind, KernelInfo *out);
bool adj_kernel_info_3d(int N, int kind, KernelInfo *out);
bool kernel_info_3d(int N, int kind, KernelInfo *out);

}  // namespace pdg
