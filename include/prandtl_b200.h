/*
 * prandtl_b200.h — C ABI of the B200-native DGSEM right-hand side and SSP-RK
 * stage update.
 *
 * This ABI stands in for Prandtl's `DGSEMOperator : mfem::TimeDependentOperator`
 * (src/Operators/DGSEMOperator.hpp:15).  Every entry point names the reference
 * interface it replaces.  Plain C types only: device pointers are `double*`,
 * CUDA streams are passed as `void*` (a `cudaStream_t`), sizes are int64.
 *
 * State layout (identical to the reference's MFEM `Ordering::byNODES` vector,
 * src/Simulation/Simulation.hpp:64, with DG element-contiguous numbering):
 *
 *     u[v * num_nodes + e * Np^dim + lex(i, j, k)],   lex = (k*Np + j)*Np + i
 *
 * with v = 0..dim+1 (rho, rho*u, rho*v[, rho*w], E), Np = order + 1 and
 * num_nodes = num_elements * Np^dim.  Gradient fields (BR1 lifting output) use
 * the same layout and hold primitive-variable gradients (rho, u, v[, w], p).
 *
 * Mesh: affine, axis-aligned quads/hexes of extent h[0..dim-1] with a face
 * neighbour table nbr[e*2*dim + f], f = (-x, +x, -y, +y, -z, +z); an entry
 * -1 - b marks a boundary face with boundary condition b (pdg_set_boundary,
 * Euler only).  Element
 * numbering is free; the face orientation rule is: the face between element a's
 * +d face and element b's -d face has element 1 = a when a <= b (normal +d),
 * else element 1 = b (normal -d) — MFEM gives element 1 to the lower-numbered
 * element of a face.
 *
 * Errors: every call returns a pdg_status; pdg_last_error() returns text for
 * the last failing call on a context.  Nothing aborts the process.  Kernels
 * record non-finite or non-physical states in a device error word that
 * pdg_check() reads and clears.
 *
 * Threading: one context per stream; a context is not reentrant (the reference
 * operator's Mult mutates `mutable` members the same way,
 * src/Integrators/DGSEMIntegrator/DGSEMIntegrator.hpp:26-58).
 */
#ifndef PRANDTL_B200_H
#define PRANDTL_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pdg_status {
    PDG_OK = 0,
    PDG_ERR_ARG = 1,          /* bad argument / size */
    PDG_ERR_CUDA = 2,         /* CUDA runtime error */
    PDG_ERR_NONFINITE = 3,    /* NaN/Inf met in a state (device error word) */
    PDG_ERR_NONPHYSICAL = 4,  /* rho <= 0 or p <= 0 met (device error word) */
    PDG_ERR_UNSUPPORTED = 5,  /* (dim, order, flags) combination not compiled */
    PDG_ERR_NOMEM = 6,        /* device allocation failed */
    PDG_ERR_CAPACITY = 7      /* mesh too large for pdg_rhs_noalloc's fixed scratch */
} pdg_status;

/* Device error-word bits (pdg_check). */
#define PDG_FLAG_NONFINITE   1u
#define PDG_FLAG_NONPHYSICAL 2u

/* Physics + scheme options.  Mirrors the reference's compile-time macros
 * (parse_compile_config.py:15-34) and runtime JSON keys
 * (src/Simulation/Simulation.cpp:99-157, 477-488) as runtime fields. */
typedef struct pdg_params {
    int32_t parabolic;        /* PARABOLIC: Navier-Stokes with BR1 lifting */
    int32_t blending;         /* SUBCELL_FV_BLENDING: Persson-Peraire + subcell FV */
    int32_t compat;           /* 1: reproduce the reference's value-changing quirks
                                 (stale viscous state, z-flux fill, 3D face
                                 dissipation term, running max wave speed) */
    int32_t filter;           /* after every RK stage: bit 1 the entropy filter, bit 2 the positivity limiter */
    double gamma;             /* ratio of specific heats */
    double Pr;                /* Prandtl number */
    double mu;                /* constant dynamic viscosity */
    double R_gas;             /* gas constant (only used by diagnostics) */
    double alpha_max;         /* blending cap, reference default 0.5 */
    double alpha_min;         /* blending snap threshold, reference default 0.001 */
    double face_dissipation;  /* 1.0 = reference LLF term; 0.0 switches it off
                                 (used by the discrete entropy-conservation test) */
} pdg_params;

typedef struct pdg_mesh {
    int32_t dim;              /* 2 or 3 */
    int32_t order;            /* polynomial order N (Np = N + 1 LGL nodes) */
    int64_t num_elements;
    double h[3];              /* element extents */
    const int32_t *nbr;       /* HOST pointer, num_elements * 2*dim entries */
} pdg_mesh;

typedef struct pdg_ctx pdg_ctx;

/* Fill *p with the reference defaults (gamma 1.4, Pr 0.72, mu 0, R 287,
 * alpha_max 0.5, alpha_min 0.001, blending on, compat on). */
void pdg_default_params(pdg_params *p);

/* DGSEMOperator ctor + DGSEMIntegrator ctor + PerssonPeraireIndicator ctor
 * (src/Operators/DGSEMOperator.cpp:5-50; src/Integrators/DGSEMIntegrator/
 * DGSEMIntegrator.cpp:8-149; src/Simulation/Simulation.cpp:486-488).
 * Builds LGL D / D-hat / D-hat2, subcell normals, the modal Vandermonde and
 * uploads the neighbour table.  Allocates its scratch (alpha, eta, gradient
 * fields, error word) on the current device.  Two environment switches,
 * read here, exist for measurements: PDG_ELEMENT_FACES=0 makes the fixed
 * operator use the separate face kernels instead of face terms inside the
 * volume kernel (same results to rounding), PDG_FACE_BUFFER=0 has each
 * element evaluate its own faces' inviscid fluxes instead of reading the
 * face buffer that the face-node kernel fills once per face (same results to
 * rounding), PDG_PREFETCH=0 turns off the lifting kernel's L2 prefetch of
 * the next element, PDG_HOST_PIPELINE=0 makes pdg_rk3_step_host copy the
 * whole state in, step and copy it out one after the other (same results). */
int pdg_create(const pdg_mesh *mesh, const pdg_params *params, pdg_ctx **out);
int pdg_destroy(pdg_ctx *ctx);

/* General geometry: skewed, graded, curved or unstructured quadrilaterals and
 * hexahedra (the reference's meshes as MFEM reads them, src/Simulation/
 * Simulation.cpp:271-336; DGSEMIntegrator evaluates MFEM's element
 * transformation at every node, DGSEMIntegrator.cpp:252-266, forms the
 * subcell metrics from it, :1199-1304, and the face normals with CalcOrtho,
 * :186).  x: HOST pointer, dim * num_nodes physical coordinates of the DG
 * nodes in the byNODES layout (x[k * num_nodes + e * Np^dim + lex]: the
 * images of the LGL nodes under the element's map; the element's geometry
 * is their degree-N interpolant).  Faces are taken in each element's own
 * frame: nbr[e*2*dim + f] with f = 2 d + side along the element's local
 * axis d.  face_orient: HOST pointer, num_elements * 2*dim codes, or NULL
 * when every neighbour meets a face with its opposite face (f ^ 1) and
 * aligned axes.  For an interior face the code is f2 + 8 o: the
 * neighbour's face f2 that meets face f, and the map o of face-node indices:
 * with (a, b) this element's node indices along the face's two tangential
 * axes (ascending axis order; b = 0 in 2D) the neighbour's are (b, a) if
 * o & 1 else (a, b), then a -> N - a if o & 2, b -> N - b if o & 4 (2D: o
 * is 0 or 2).  The library forms J and the adjugate at every node, each face
 * node's normal out of the face's element 1 (the lower-numbered element)
 * and the CFL length, the smallest singular value of the Jacobian at an
 * element centre (MFEM's GetElementSize(e, 1), Simulation.cpp:896-906),
 * which replaces mesh->h.  Call once, before the first evaluation.  The
 * entropy filter and the positivity limiter run as on box meshes (the
 * limiter contracts towards J-weighted element means).  Euler: both operators (compat changes the 3D face dissipation
 * term, the running maximum wave speed and the subsonic conditions' in-place
 * divisions, as on box meshes), every boundary condition type, one kernel
 * per right-hand side or RK stage (PDG_KERNEL_GEO).  Navier-Stokes: the
 * fixed operator (compat = 0) with every condition the box path takes with
 * Navier-Stokes (slip wall and symmetry: PDG_ERR_UNSUPPORTED at the first
 * evaluation, as there); the BR1 lifting kernel (PDG_KERNEL_GEO_LIFT, the adjugate at
 * every node; pdg_gradients runs it alone) and the right-hand-side kernel
 * with the contravariant viscous fluxes (PDG_KERNEL_GEO_NS).  pdg_rhs_vjp, pdg_rk_stage_vjp and pdg_rk_stage_part
 * return PDG_ERR_UNSUPPORTED on such a context; pdg_rk3_step_host copies
 * the state whole.  PDG_ERR_ARG: a call after the first evaluation, a
 * non-positive Jacobian at a node, a code
 * whose neighbour face does not point back, or a neighbour whose normal at
 * the matching node is not the opposite of this element's (a non-conforming
 * face or a wrong code); PDG_ERR_UNSUPPORTED: the reference-value
 * Navier-Stokes operator. */
int pdg_set_geometry(pdg_ctx *ctx, const double *x, const int32_t *face_orient);

/* Boundary conditions (the integrators of src/Integrators/BoundaryConditions/, attached to
 * boundary attributes by DGSEMOperator::AddBdrFaceIntegrator,
 * src/Operators/DGSEMOperator.cpp:593 and src/Simulation/Simulation.cpp:
 * 490-798).  A neighbour entry -1 - b (0 <= b < PDG_MAX_BOUNDARIES) marks a
 * boundary face with condition b; every condition the mesh uses must be set
 * before the first evaluation (else PDG_ERR_ARG).  Navier-Stokes boundary
 * faces: types 1, 2, 3, 6, 7, 8 (2D), 10 and 11, and 9 with compat = 0 (others:
 * PDG_ERR_UNSUPPORTED at the first evaluation; the reference has no viscous
 * flux for 4 and 5); pdg_rhs_vjp differentiates every condition of an Euler
 * mesh and none of a Navier-Stokes one.  `state` holds the condition's
 * data as listed beside each type (conserved, dim + 2 values, for the two
 * prescribed-state types) and may be NULL for types without data.  With
 * compat = 1 the subsonic and Riemann-invariant conditions keep the
 * reference's in-place division of the interior momenta before the face flux
 * reads them; compat = 0 uses the interior state as it is.  The total-
 * pressure inflow is 2D only (the reference's 3D branch writes past its
 * direction vector): PDG_ERR_UNSUPPORTED in 3D. */
#define PDG_MAX_BOUNDARIES 16
#define PDG_BC_SUPERSONIC_INFLOW  1  /* SupersonicInflowBdrFaceIntegrator: prescribed outer state */
#define PDG_BC_SUPERSONIC_OUTFLOW 2  /* SupersonicOutflowBdrFaceIntegrator: outer state = interior */
#define PDG_BC_SPECIFIED_STATE    3  /* SpecifiedStateBdrFaceIntegrator: prescribed outer state */
#define PDG_BC_SLIP_WALL          4  /* SlipWallBdrFaceIntegrator: pressure flux from the wall Riemann problem */
#define PDG_BC_SYMMETRY           5  /* SymmetryBdrFaceIntegrator: normal momentum mirrored */
#define PDG_BC_SUBSONIC_OUTFLOW_P 6  /* SubsonicOutflowPBdrFaceIntegrator: state = {p} */
#define PDG_BC_SUBSONIC_INFLOW_RV 7  /* SubsonicInflowRVBdrFaceIntegrator: state = {rho, V[dim]} */
#define PDG_BC_SUBSONIC_INFLOW_PTTT 8  /* SubsonicInflowPtTtAngBdrFaceIntegrator, 2D: state = {cp, pt, Tt, theta, phi} (degrees) */
#define PDG_BC_RIEMANN_INVARIANT  9  /* RiemannInvariantBdrFaceIntegrator: state = primitive {rho, v[dim], p} */
#define PDG_BC_NOSLIP_ADIABATIC  10  /* NoSlipAdiabWallBdrFaceIntegrator, zero heat flux: state = wall velocity {V[dim]} */
#define PDG_BC_NOSLIP_ISOTHERMAL 11  /* NoSlipIsothWallBdrFaceIntegrator: state = {T_wall, V[dim]}, with params.R_gas */
int pdg_set_boundary(pdg_ctx *ctx, int index, int type, const double *state);

/* TimeDependentOperator::Height (DGSEMOperator.cpp:18): number of vdofs. */
int64_t pdg_size(const pdg_ctx *ctx);

/* DGSEMOperator::Mult(u, dudt) (src/Operators/DGSEMOperator.cpp:537-591):
 * blending coefficient, [entropy variables, BR1 lifting, primitive gradients],
 * volume + subcell FV + face terms.  u, dudt: DEVICE pointers, byNODES. */
int pdg_rhs(pdg_ctx *ctx, const double *u, double *dudt, void *stream);

/* Allocation-free right-hand side.  No counterpart in the reference: it is
 * for callers that cannot allocate device memory when they need the operator
 * — code running where another allocator owns the device's memory, or an
 * integrator that must keep its footprint fixed — so it takes no context and
 * calls no cudaMalloc, cudaFree or allocating library routine.  It computes
 * the same dudt = L(u) as pdg_rhs for the given mesh and parameters, except
 * that the wave-speed maximum starts from zero on every call; the mesh must
 * be periodic (boundary faces need pdg_set_boundary on a context, so a
 * negative neighbour entry returns PDG_ERR_ARG).  u, dudt: DEVICE pointers,
 * byNODES, not aliased.
 *
 * All device scratch (constants, neighbour table, blending outputs, the
 * Navier-Stokes lifting jumps and face columns) lives in one file-scope
 * device array of PDG_NOALLOC_SCRATCH_DOUBLES doubles (24 MiB) that every GPU
 * loading this library holds until the process exits.  A mesh that needs
 * more returns PDG_ERR_CAPACITY: at order 3 that is above about 5,000
 * elements for Navier-Stokes in 3D and above about 600,000 for Euler.
 * The first call on a device looks up the array's device address on that
 * device (the current device) and keeps it for the process; make that first
 * call before any stream capture.  The kept address does not survive
 * cudaDeviceReset.  Every call on a device shares the array and leaves its
 * contents behind: calls that overlap on the GPU race.
 * Every call copies the constants and the neighbour table from (pageable)
 * host memory with cudaMemcpyAsync on `stream`; CUDA may perform such copies
 * synchronously with respect to the host.
 * The kernels are the separate-face sequence (volume kernel, then one face
 * pass per direction) for both operators; for compat = 0 pdg_rhs evaluates
 * the faces inside the volume kernel instead, and the two agree to rounding
 * (1e-14 relative), not bit for bit.
 * The device error word is cleared on entry and not reported: a caller that
 * needs to detect a non-finite or non-physical state checks dudt itself. */
#define PDG_NOALLOC_SCRATCH_DOUBLES (3 * 1024 * 1024)
int pdg_rhs_noalloc(const pdg_mesh *mesh, const pdg_params *params, const double *u, double *dudt,
                    void *stream);

/* Same with HOST pointers (the MFEM adapter path: Mult on host Vectors).
 * Copies in, computes, copies out, synchronises. */
int pdg_rhs_host(pdg_ctx *ctx, const double *u_host, double *dudt_host);

/* One SSP-RK3 stage with the RHS fused into the axpy (the stage bodies of
 * MFEM's RK3SSPSolver::Step as called at src/Simulation/Simulation.cpp:1010):
 *   stage 0: uout = us + dt*L(us)                       (us = un)
 *   stage 1: uout = 3/4 un + 1/4 (us + dt*L(us))
 *   stage 2: uout = 1/3 un + 2/3 (us + dt*L(us))
 * followed by the entropy filter and/or the positivity limiter that
 * params.filter selects.  DEVICE pointers;
 * uout may alias neither un nor us. */
int pdg_rk_stage(pdg_ctx *ctx, int stage, double dt, const double *un,
                 const double *us, double *uout, void *stream);

/* ODESolver::Step for RK3SSPSolver (Simulation.cpp:1010): advances u (DEVICE)
 * in place by one step of size dt using context-owned stage buffers. */
int pdg_rk3_step(pdg_ctx *ctx, double dt, double *u, void *stream);

/* nsteps of pdg_rk3_step replayed from a CUDA graph: the first call for a
 * (u, dt) pair captures one step (all its stage kernels) on an internal
 * stream; later calls with the same pair only launch the graph.  Same values
 * as pdg_rk3_step.  For small meshes, whose steps are bound by launch cost. */
int pdg_rk3_steps(pdg_ctx *ctx, double dt, double *u, int nsteps, void *stream);

/* Same step with a HOST state (the path an MFEM adapter would take for
 * ODESolver::Step on host Vectors): copies u in, runs the three fused stages,
 * copies the result back and synchronises.  u_host may be pinned or pageable
 * (pinned memory lets the copies overlap the kernels).  For the fixed
 * operator on a periodic mesh of at least 4096 elements without the filter
 * or limiter the step is pipelined: the state crosses PCIe in 32 element
 * chunks, stage 0 works on the runs of chunks whose reads (radius three in
 * face neighbours for Navier-Stokes) have landed while the rest are still
 * copying, and stage 2's volume kernel runs in four runs with each finished
 * run copied back behind it; the result equals pdg_rk3_step's bit for bit.
 * Work already queued on the legacy default stream comes first. */
int pdg_rk3_step_host(pdg_ctx *ctx, double dt, double *u_host);

/* DGSEMOperator::GetMaxCharSpeed (DGSEMOperator.hpp:106-109).  With compat=1
 * this is the running maximum over every RHS evaluated so far (the
 * reference never resets it); with compat=0 it is the maximum of the last
 * RHS.  Synchronises the stream of the last call. */
int pdg_max_char_speed(pdg_ctx *ctx, double *out);

/* dt rule of Simulation::Run (Simulation.cpp:893-907,1013-1018):
 * dt = cfl * hmin / (max_char_speed * (N+1)^2). */
int pdg_cfl_dt(pdg_ctx *ctx, double cfl, double *dt_out);

/* Per-element Persson-Peraire indicator and blending coefficient of the last
 * RHS (DGSEMOperator::ComputeBlendingCoefficient, DGSEMOperator.cpp:60-80),
 * copied to HOST arrays of num_elements doubles (either may be NULL). */
int pdg_get_blending(pdg_ctx *ctx, double *eta_host, double *alpha_host);

/* BR1 primitive-variable gradients of a DEVICE state u (the reference's
 * MultLifting + ComputeGlobalPrimitiveGradVector, DGSEMNonlinearForm.cpp:
 * 424-645 and DGSEMOperator.cpp:134-159): grads (DEVICE, dim*size doubles)
 * receives d/dx_d of (rho, u, v[, w], p) in the byNODES layout, direction d
 * slowest.  The right-hand side computes the same gradients internally and
 * only keeps the viscous fluxes derived from them. */
int pdg_gradients(pdg_ctx *ctx, const double *u, double *grads, void *stream);

/* Adjoint (vector-Jacobian product) of the right-hand side: ubar =
 * (dL/du)^T cot, with L = DGSEMOperator::Mult (DGSEMOperator.cpp:537-591) in
 * its fixed form; the reference has no adjoint.  Requires params.compat = 0
 * (PDG_ERR_UNSUPPORTED otherwise).  The blending coefficient is
 * differentiated where its sigmoid is active and is constant where it is
 * snapped or capped.  u, cot, ubar: DEVICE pointers, byNODES; ubar is
 * overwritten and aliases neither input.  The first call allocates the
 * adjoint scratch. */
int pdg_rhs_vjp(pdg_ctx *ctx, const double *u, const double *cot, double *ubar, void *stream);

/* Adjoint of one SSP-RK3 stage (pdg_rk_stage, the stage bodies of MFEM's
 * RK3SSPSolver::Step as called at src/Simulation/Simulation.cpp:1010) with the
 * stage algebra fused into the vector-Jacobian product's last kernel.  For
 * stage s, out = a_s un + b_s (us + dt L(us)), and the cotangent lam of out,
 * with g = (dL/dus)^T lam:
 *   stage 2: out = 2/3 (lam + dt g),  bx = 1/3 lam
 *   stage 1: out = 1/4 (lam + dt g),  bx = bx + 3/4 lam
 *   stage 0: bx = bx + lam + dt g     (us = un; out is scratch)
 * so that a step's adjoint is stages 2, 1, 0 with lam = the previous stage's
 * out, leaving the cotangent of the step's input in bx.  The reference has
 * no adjoint.  Fixed operator, meshes without boundary faces
 * (PDG_ERR_UNSUPPORTED otherwise; use pdg_rhs_vjp).  DEVICE pointers; out and
 * bx alias no other argument. */
int pdg_rk_stage_vjp(pdg_ctx *ctx, int stage, double dt, const double *us, const double *lam, double *out,
                     double *bx, void *stream);

/* Entropy filter (params.filter & 1): EntropyFilter::FilterSolution
 * (src/Filters/EntropyFilter.cpp:171-242) after every RK stage, with the
 * element bounds of GetEntropyConstraints (:81-158) taken at the stage input.
 * Applies to pdg_rk_stage / pdg_rk3_step*; pdg_rhs is never filtered.
 * pdg_filter_count returns the number of element filterings since creation
 * (synchronises). */
int pdg_filter_count(pdg_ctx *ctx, int64_t *filtered);

/* Positivity limiter (params.filter & 2), after the entropy filter when both
 * are set.  The reference's MinmodLimiter (src/Limiters/MinmodLimiter.cpp:
 * 22-77) limits nothing and it has no positivity limiter; this is the
 * conservative limiter of Zhang & Shu (2010) with the pressure step of Zhang,
 * Xia & Shu (2012): each element's nodes are contracted towards its LGL mean
 * until density and pressure are at least min(1e-13, mean density, mean
 * pressure).  pdg_limiter_count returns the number of element limitings
 * since creation (synchronises). */
int pdg_limiter_count(pdg_ctx *ctx, int64_t *limited);

/* One kernel of a fused RK stage (pdg_rk_stage) over the elements
 * [e_begin, e_end), for a caller that interleaves a stage with its own work:
 * the multi-rank driver runs the elements that need no neighbour rank's data
 * while face data is in flight, as the reference's shared-face exchange
 * (ExchangeFaceNbrData, src/Operators/NonlinearForm/DGSEMNonlinearForm.cpp:
 * 748; Navier-Stokes also :533, :1426-1429) separates its face loops.  A
 * stage is PDG_PART_START (resets the wave-speed maximum), then over every
 * element PDG_PART_FACES (face-node kernel: BR1 jumps and the inviscid flux
 * of each element's +d faces, reading the state of the element and its +d
 * neighbours), PDG_PART_LIFT (Navier-Stokes: lifting kernel, reading the
 * face-node results of the element's faces and writing its viscous face
 * columns) and PDG_PART_VOLUME (volume kernel: the element's stage output,
 * reading the face-node results of its faces and its neighbours' viscous
 * face columns), each part of an element after the parts it reads.  Fixed
 * operator on a mesh without boundary faces, no filter or limiter
 * (PDG_ERR_UNSUPPORTED otherwise).  DEVICE pointers as pdg_rk_stage; uout is
 * only read by PDG_PART_VOLUME. */
#define PDG_PART_START  0
#define PDG_PART_FACES  1
#define PDG_PART_LIFT   2
#define PDG_PART_VOLUME 3
int pdg_rk_stage_part(pdg_ctx *ctx, int part, int stage, double dt, const double *un, const double *us, double *uout,
                      int64_t e_begin, int64_t e_end, void *stream);

/* The context's viscous face columns (Navier-Stokes): *cols = device buffer
 * of *count doubles, fcol[d][side][e][face node][i] (side 1: the element's +d
 * face, i over the dim + 1 momentum and energy rows of the normal viscous
 * flux), written by PDG_PART_LIFT.  A multi-rank driver copies the columns of
 * its slab's boundary elements to the neighbour ranks, which write them into
 * their ghost elements' slots before their PDG_PART_VOLUME.  No reference
 * counterpart (the reference exchanges gradients, DGSEMNonlinearForm.cpp:
 * 1426-1429). */
int pdg_face_columns(pdg_ctx *ctx, double **cols, int64_t *count);

/* Reads and clears the device error word (PDG_FLAG_*).  Synchronises. */
int pdg_check(pdg_ctx *ctx, uint32_t *flags);

/* Text of the last error on this context ("" if none). */
const char *pdg_last_error(const pdg_ctx *ctx);

/* Number of kernels this context has launched since creation. */
int64_t pdg_launch_count(const pdg_ctx *ctx);

/* Kernel timing (no reference counterpart: the reference only times the
 * whole run, Simulation.cpp:910-914).  When enabled, every kernel launch is
 * bracketed by CUDA events on its own stream.  pdg_profile_read synchronises,
 * returns the summed device time (ms) and launch count of one kernel kind
 * (PDG_KERNEL_*) since the last read, and clears that kind's records. */
#define PDG_KERNEL_EULER     0  /* Euler volume (+ stage) kernel */
#define PDG_KERNEL_LIFT      1  /* BR1 lifting + viscous volume term kernel */
#define PDG_KERNEL_NS        2  /* Navier-Stokes inviscid volume (+ stage) kernel */
#define PDG_KERNEL_LIFT_FACE 3  /* BR1 lifting face-jump kernel */
#define PDG_KERNEL_FACE_E0   4  /* Euler face kernels, x / y / z */
#define PDG_KERNEL_FACE_NS0  7  /* Navier-Stokes face kernels, x / y / z (7, 8, 9) */
#define PDG_KERNEL_FILTER_BOUNDS 10  /* entropy filter: per-element entropy minimum */
#define PDG_KERNEL_FILTER    11  /* entropy filter of a stage output */
#define PDG_KERNEL_ADJ_RHS   12  /* adjoint: inviscid volume terms and blending */
#define PDG_KERNEL_ADJ_LIFT  13  /* adjoint: viscous terms */
#define PDG_KERNEL_ADJ_FACE_E0  14  /* adjoint Euler face terms, every direction */
#define PDG_KERNEL_ADJ_GATHER   15  /* adjoint: face terms added to the output (+ the RK stage's adjoint) */
#define PDG_KERNEL_ADJ_FACE_NS0 17  /* adjoint Navier-Stokes face terms, every direction */
#define PDG_KERNEL_EULER_FACES 20   /* Euler volume + face terms (+ stage), fixed operator */
#define PDG_KERNEL_NS_FACES  21     /* Navier-Stokes inviscid volume + all face terms (+ stage), fixed operator */
#define PDG_KERNEL_BOUNDARY  22     /* boundary faces of the separate-face path (Euler) */
#define PDG_KERNEL_ADJ_BOUNDARY 23  /* adjoint of the boundary faces (Euler) */
#define PDG_KERNEL_EULER_FACES_BDR 24  /* PDG_KERNEL_EULER_FACES for meshes with boundary faces */
#define PDG_KERNEL_LIFT_FACE_BDR 25  /* Navier-Stokes meshes with boundary faces: face jumps, */
#define PDG_KERNEL_LIFT_BDR  26      /* lifting kernel, */
#define PDG_KERNEL_NS_FACES_BDR 27   /* volume kernel with element-side faces */
#define PDG_KERNEL_BOUNDARY_NS 28    /* boundary faces of the separate-face path (Navier-Stokes) */
#define PDG_KERNEL_LIFT_BDR_PTTT 29  /* lifting kernel of a 2D mesh with a total-pressure inflow */
#define PDG_KERNEL_NS_FACES_FB 30    /* Navier-Stokes volume + face terms reading the face buffer (periodic, fixed) */
#define PDG_KERNEL_EULER_FACES_FB 31 /* Euler volume + face terms reading the face buffer (periodic, fixed) */
#define PDG_KERNEL_LIFT_FACE_FLUX 32 /* face-node kernel: BR1 jumps + inviscid face fluxes into the buffer */
#define PDG_KERNEL_FACE_FLUX 33      /* face-node kernel: inviscid face fluxes into the buffer (Euler) */
#define PDG_KERNEL_POSITIVITY 34     /* positivity limiter of a stage output */
#define PDG_KERNEL_GEO 35            /* Euler right-hand side on a general-geometry mesh (pdg_set_geometry) */
#define PDG_KERNEL_GEO_LIFT 36       /* BR1 lifting on a general-geometry mesh */
#define PDG_KERNEL_GEO_NS 37         /* Navier-Stokes right-hand side on a general-geometry mesh */
int pdg_profile_enable(pdg_ctx *ctx, int on);
int pdg_profile_read(pdg_ctx *ctx, int kind, double *total_ms, int64_t *launches);

/* ---- Batched sweep: many independent cases in one launch per RK stage ----
 *
 * No single reference counterpart: the reference runs one case per process
 * (Simulation::Run, src/Simulation/Simulation.cpp:800-1020) and a sweep is a
 * loop over runs.  A batch holds periodic 2D Euler cases (params.parabolic =
 * params.filter = 0) of any size and order 1..5 that share pdg_params; their
 * states are concatenated, case c occupying pdg_batch_offset(c) ..
 * pdg_batch_offset(c + 1) - 1 in the usual byNODES layout of its own mesh.
 * Every case has its own time step (pdg_batch_set_dt) and running wave-speed
 * maximum.  Results per case equal the per-case context's pdg_rhs /
 * pdg_rk3_step to rounding. */
typedef struct pdg_batch pdg_batch;
int pdg_batch_create(int ncases, const pdg_mesh *meshes, const pdg_params *params, pdg_batch **out);
int pdg_batch_destroy(pdg_batch *batch);
/* Offset (in doubles) of case c's state; c = ncases gives the total size. */
int64_t pdg_batch_offset(const pdg_batch *batch, int case_index);
/* Per-case time steps (host array of ncases doubles). */
int pdg_batch_set_dt(pdg_batch *batch, const double *dt);
/* DGSEMOperator::Mult of every case in one launch.  DEVICE pointers. */
int pdg_batch_rhs(pdg_batch *batch, const double *u, double *dudt, void *stream);
/* nsteps SSP-RK3 steps of every case in place (RK3SSPSolver::Step,
 * Simulation.cpp:1010), three launches per step; with use_graph the step is
 * captured once in a CUDA graph and replayed. */
int pdg_batch_rk3_step(pdg_batch *batch, double *u, int nsteps, int use_graph, void *stream);
/* Autotuner: times the batch kernel on u for each register budget (255, 170
 * or 128 registers per thread: variant 0, 1, 2) x warps per block x tiles per
 * fetch x tile order candidate and keeps the fastest (synchronises).
 * best_ms (may be null) receives the fastest launch time. */
int pdg_batch_tune(pdg_batch *batch, const double *u, void *stream, float *best_ms);
int pdg_batch_config(const pdg_batch *batch, int *warps_per_block, int *blocks, int *tiles_per_fetch,
                     int *tile_order, int *register_variant);
/* Per-case running maximum wave speed (host array of ncases; synchronises). */
int pdg_batch_max_char_speed(pdg_batch *batch, double *lam);
int pdg_batch_check(pdg_batch *batch, uint32_t *flags);
int64_t pdg_batch_launch_count(const pdg_batch *batch);
const char *pdg_batch_last_error(const pdg_batch *batch);

#ifdef __cplusplus
}
#endif

#endif /* PRANDTL_B200_H */
