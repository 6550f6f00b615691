"""prandtl_b200 — B200-native DGSEM right-hand side and SSP-RK stage update.

Host-side mirror of the reference's operator interface for the hot path:

* ``DGSEMOperator`` stands in for ``Prandtl::DGSEMOperator :
  mfem::TimeDependentOperator`` (src/Operators/DGSEMOperator.hpp:15):
  ``Mult(u, dudt)``, ``GetMaxCharSpeed()``, ``Height()``.
* ``RK3SSPSolver`` stands in for MFEM's ``RK3SSPSolver`` as the reference
  drives it (``Init(op)``, ``Step(x, t, dt)``, src/Simulation/Simulation.cpp:
  807, 1010), with each stage's right-hand side fused into the stage axpy.
* ``cfl_dt`` is the time-step rule of ``Simulation::Run``
  (Simulation.cpp:893-907, 1013-1018).

All compute runs in the CUDA library ``_lib/libprandtl_b200.so`` through the C
ABI of ``include/prandtl_b200.h``; there is no CPU fallback.  State vectors use
the reference's byNODES layout.  Device arrays are torch CUDA tensors (float64,
contiguous); host arrays are numpy float64 arrays (``Mult`` then copies through
the host entry point).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mesh import CartesianMesh, periodic_box  # noqa: F401
from .meshio import read_mesh  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libprandtl_b200.so")

PDG_OK = 0
KERNEL_EULER, KERNEL_LIFT, KERNEL_NS, KERNEL_LIFT_FACE = 0, 1, 2, 3
KERNEL_FACE_EULER = (4, 5, 6)
KERNEL_FACE_NS = (7, 8, 9)
KERNEL_FILTER_BOUNDS, KERNEL_FILTER = 10, 11
KERNEL_ADJ_RHS, KERNEL_ADJ_LIFT = 12, 13
KERNEL_ADJ_FACE_EULER = (14,)   # adj_faces_kernel: every direction in one launch
KERNEL_ADJ_FACE_NS = (17,)
KERNEL_ADJ_GATHER = 15
KERNEL_EULER_FACES, KERNEL_NS_FACES, KERNEL_BOUNDARY, KERNEL_ADJ_BOUNDARY, KERNEL_EULER_FACES_BDR = 20, 21, 22, 23, 24
KERNEL_LIFT_FACE_BDR, KERNEL_LIFT_BDR, KERNEL_NS_FACES_BDR, KERNEL_BOUNDARY_NS = 25, 26, 27, 28
KERNEL_LIFT_BDR_PTTT = 29
KERNEL_NS_FACES_FB, KERNEL_EULER_FACES_FB, KERNEL_LIFT_FACE_FLUX, KERNEL_FACE_FLUX = 30, 31, 32, 33
KERNEL_POSITIVITY = 34
KERNEL_GEO = 35
KERNEL_GEO_LIFT = 36
KERNEL_GEO_NS = 37
# params.filter bits
FILTER_ENTROPY, FILTER_POSITIVITY = 1, 2
# boundary condition types (pdg_set_boundary)
BC_SUPERSONIC_INFLOW, BC_SUPERSONIC_OUTFLOW, BC_SPECIFIED_STATE, BC_SLIP_WALL, BC_SYMMETRY = 1, 2, 3, 4, 5
BC_SUBSONIC_OUTFLOW_P, BC_SUBSONIC_INFLOW_RV, BC_SUBSONIC_INFLOW_PTTT, BC_RIEMANN_INVARIANT = 6, 7, 8, 9
BC_NOSLIP_ADIABATIC, BC_NOSLIP_ISOTHERMAL = 10, 11
MAX_BOUNDARIES = 16
# pdg_rk_stage_part parts
PART_START, PART_FACES, PART_LIFT, PART_VOLUME = 0, 1, 2, 3
PDG_FLAG_NONFINITE = 1
PDG_FLAG_NONPHYSICAL = 2
_STATUS = {1: "bad argument", 2: "CUDA error", 3: "non-finite state", 4: "non-physical state",
           5: "unsupported configuration", 6: "out of device memory",
           7: "mesh exceeds the allocation-free scratch"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class PdgParams(C.Structure):
    _fields_ = [("parabolic", C.c_int32), ("blending", C.c_int32), ("compat", C.c_int32),
                ("filter", C.c_int32), ("gamma", C.c_double), ("Pr", C.c_double),
                ("mu", C.c_double), ("R_gas", C.c_double), ("alpha_max", C.c_double),
                ("alpha_min", C.c_double), ("face_dissipation", C.c_double)]


class PdgMesh(C.Structure):
    _fields_ = [("dim", C.c_int32), ("order", C.c_int32), ("num_elements", C.c_int64),
                ("h", C.c_double * 3), ("nbr", _ip)]


class PdgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS.get(code, 'error')} ({code}): {msg}")
        self.code = code


_lib = None


def library():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m prandtl_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.pdg_default_params.argtypes = [C.POINTER(PdgParams)]
    L.pdg_create.argtypes = [C.POINTER(PdgMesh), C.POINTER(PdgParams), C.POINTER(C.c_void_p)]
    L.pdg_destroy.argtypes = [C.c_void_p]
    L.pdg_size.restype = C.c_int64
    L.pdg_size.argtypes = [C.c_void_p]
    L.pdg_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pdg_rhs_host.argtypes = [C.c_void_p, _dp, _dp]
    L.pdg_rk_stage.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pdg_rk3_step.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    L.pdg_rk3_steps.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    L.pdg_max_char_speed.argtypes = [C.c_void_p, _dp]
    L.pdg_cfl_dt.argtypes = [C.c_void_p, C.c_double, _dp]
    L.pdg_get_blending.argtypes = [C.c_void_p, _dp, _dp]
    L.pdg_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pdg_check.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.pdg_last_error.restype = C.c_char_p
    L.pdg_last_error.argtypes = [C.c_void_p]
    L.pdg_launch_count.restype = C.c_int64
    L.pdg_launch_count.argtypes = [C.c_void_p]
    L.pdg_rk3_step_host.argtypes = [C.c_void_p, C.c_double, _dp]
    L.pdg_profile_enable.argtypes = [C.c_void_p, C.c_int]
    L.pdg_profile_read.argtypes = [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_int64)]
    vp = C.c_void_p
    L.pdg_batch_create.argtypes = [C.c_int, C.POINTER(PdgMesh), C.POINTER(PdgParams), C.POINTER(vp)]
    L.pdg_batch_destroy.argtypes = [vp]
    L.pdg_batch_offset.restype = C.c_int64
    L.pdg_batch_offset.argtypes = [vp, C.c_int]
    L.pdg_batch_set_dt.argtypes = [vp, _dp]
    L.pdg_batch_rhs.argtypes = [vp, vp, vp, vp]
    L.pdg_batch_rk3_step.argtypes = [vp, vp, C.c_int, C.c_int, vp]
    L.pdg_batch_tune.argtypes = [vp, vp, vp, C.POINTER(C.c_float)]
    L.pdg_batch_config.argtypes = [vp] + [C.POINTER(C.c_int)] * 5
    L.pdg_batch_max_char_speed.argtypes = [vp, _dp]
    L.pdg_batch_check.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.pdg_batch_launch_count.restype = C.c_int64
    L.pdg_batch_launch_count.argtypes = [vp]
    L.pdg_batch_last_error.restype = C.c_char_p
    L.pdg_batch_last_error.argtypes = [vp]
    L.pdg_filter_count.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.pdg_limiter_count.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.pdg_rhs_vjp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pdg_rk_stage_vjp.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
    L.pdg_rhs_noalloc.argtypes = [C.POINTER(PdgMesh), C.POINTER(PdgParams), C.c_void_p, C.c_void_p, C.c_void_p]
    L.pdg_set_boundary.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    L.pdg_set_geometry.argtypes = [C.c_void_p, _dp, _ip]
    L.pdg_rk_stage_part.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int64, C.c_int64, C.c_void_p]
    L.pdg_face_columns.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
    _lib = L
    return L


def default_params(**overrides) -> PdgParams:
    p = PdgParams()
    library().pdg_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


class DGSEMOperator:
    """DGSEMOperator::Mult on the GPU for one periodic Cartesian mesh.

    Parameters mirror the reference's compile-time flags and runtime keys:
    ``parabolic`` (PARABOLIC), ``blending`` (SUBCELL_FV_BLENDING), ``compat``
    (reproduce the reference's value-changing quirks), ``filter`` (after
    each RK stage: 1 the entropy filter, 2 the positivity limiter, 3 both),
    ``gamma``, ``Pr``, ``mu``, ``alpha_max``,
    ``alpha_min``, ``face_dissipation``.
    """

    def __init__(self, mesh: CartesianMesh, **params):
        self.mesh = mesh
        self.params = default_params(**params)
        self._nbr = np.ascontiguousarray(mesh.nbr, dtype=np.int32)
        h = list(mesh.h) + [1.0] * (3 - mesh.dim)
        self._m = PdgMesh(mesh.dim, mesh.order, mesh.num_elements, (C.c_double * 3)(*h),
                          self._nbr.ctypes.data_as(_ip))
        self._ctx = C.c_void_p()
        self._call(library().pdg_create(C.byref(self._m), C.byref(self.params), C.byref(self._ctx)), "pdg_create")
        for b, spec in (getattr(mesh, "boundaries", None) or {}).items():
            self.set_boundary(b, *spec)
        if getattr(mesh, "coords", None) is not None:
            self._set_geometry(mesh)

    def _set_geometry(self, mesh):
        """Node coordinates and face orientation codes of a general-geometry
        mesh (pdg_set_geometry: skewed, graded, curved or unstructured elements)."""
        self._coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        if self._coords.shape != (mesh.dim, mesh.num_nodes):
            raise ValueError(f"mesh.coords has shape {self._coords.shape}, expected {(mesh.dim, mesh.num_nodes)}")
        fo = getattr(mesh, "face_orient", None)
        self._face_orient = None if fo is None else np.ascontiguousarray(fo, dtype=np.int32)
        ptr = None if self._face_orient is None else self._face_orient.ctypes.data_as(_ip)
        self._call(library().pdg_set_geometry(self._ctx, self._coords.ctypes.data_as(_dp), ptr), "pdg_set_geometry")

    def set_boundary(self, index: int, type: int, state=None):
        """Boundary condition ``index`` of the mesh's negative neighbour
        entries (pdg_set_boundary; the reference's BdrFaceIntegrators)."""
        st = None
        if state is not None:
            st = np.ascontiguousarray(state, dtype=np.float64)
            self._bc_state = getattr(self, "_bc_state", {})
            self._bc_state[index] = st
        ptr = st.ctypes.data_as(_dp) if st is not None else None
        self._call(library().pdg_set_boundary(self._ctx, int(index), int(type), ptr), "pdg_set_boundary")

    def _call(self, code: int, what: str):
        if code != PDG_OK:
            msg = ""
            if self._ctx:
                msg = library().pdg_last_error(self._ctx).decode()
            raise PdgError(code, f"{what}: {msg}")

    def close(self):
        if getattr(self, "_ctx", None):
            library().pdg_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- TimeDependentOperator interface ---
    def Height(self) -> int:
        return int(library().pdg_size(self._ctx))

    @property
    def size(self) -> int:
        return self.Height()

    def _check_dev(self, *ts):
        for t in ts:
            if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()):
                raise ValueError("device arrays must be contiguous float64 CUDA tensors")
            if t.numel() != self.size:
                raise ValueError(f"array has {t.numel()} entries, operator size is {self.size}")

    def Mult(self, u, dudt, stream=None):
        """dudt = L(u).  torch CUDA tensors (device path) or numpy arrays (host path)."""
        if _is_torch(u):
            self._check_dev(u, dudt)
            self._call(library().pdg_rhs(self._ctx, C.c_void_p(u.data_ptr()), C.c_void_p(dudt.data_ptr()),
                                         C.c_void_p(_stream_handle(stream))), "pdg_rhs")
        else:
            if u.dtype != np.float64 or dudt.dtype != np.float64 or not u.flags.c_contiguous or not dudt.flags.c_contiguous:
                raise ValueError("host arrays must be contiguous float64")
            if u.size != self.size or dudt.size != self.size:
                raise ValueError("host array size does not match the operator")
            self._call(library().pdg_rhs_host(self._ctx, u.ctypes.data_as(_dp), dudt.ctypes.data_as(_dp)),
                       "pdg_rhs_host")
        return dudt

    def GetMaxCharSpeed(self) -> float:
        v = C.c_double()
        self._call(library().pdg_max_char_speed(self._ctx, C.byref(v)), "pdg_max_char_speed")
        return v.value

    # --- fused stage update ---
    def rk_stage(self, stage: int, dt: float, un, us, uout, stream=None):
        self._check_dev(us, uout)
        if un is not None:
            self._check_dev(un)
        self._call(library().pdg_rk_stage(self._ctx, stage, dt, C.c_void_p(un.data_ptr() if un is not None else 0),
                                          C.c_void_p(us.data_ptr()), C.c_void_p(uout.data_ptr()),
                                          C.c_void_p(_stream_handle(stream))), "pdg_rk_stage")
        return uout

    def rk3_step(self, u, dt: float, stream=None, nsteps: int = 1, graph: bool = False):
        """nsteps SSP-RK3 steps of a device state in place; with graph=True
        they are replayed from a CUDA graph captured for (u, dt)."""
        self._check_dev(u)
        if graph:
            self._call(library().pdg_rk3_steps(self._ctx, dt, C.c_void_p(u.data_ptr()), int(nsteps),
                                               C.c_void_p(_stream_handle(stream))), "pdg_rk3_steps")
            return u
        for _ in range(nsteps):
            self._call(library().pdg_rk3_step(self._ctx, dt, C.c_void_p(u.data_ptr()),
                                              C.c_void_p(_stream_handle(stream))), "pdg_rk3_step")
        return u

    def rk3_step_host(self, u: np.ndarray, dt: float):
        """One step on a HOST state (copy in, three fused stages, copy out)."""
        if u.dtype != np.float64 or not u.flags.c_contiguous or u.size != self.size:
            raise ValueError("host state must be a contiguous float64 array of the operator size")
        self._call(library().pdg_rk3_step_host(self._ctx, dt, u.ctypes.data_as(_dp)), "pdg_rk3_step_host")
        return u

    def profile(self, on: bool = True):
        self._call(library().pdg_profile_enable(self._ctx, int(on)), "pdg_profile_enable")

    def profile_read(self, kind: int):
        """(total device ms, launches) of one kernel kind since the last read."""
        ms, n = C.c_double(), C.c_int64()
        self._call(library().pdg_profile_read(self._ctx, kind, C.byref(ms), C.byref(n)), "pdg_profile_read")
        return ms.value, n.value

    def cfl_dt(self, cfl: float) -> float:
        v = C.c_double()
        self._call(library().pdg_cfl_dt(self._ctx, cfl, C.byref(v)), "pdg_cfl_dt")
        return v.value

    def blending(self):
        ne = self.mesh.num_elements
        eta, alpha = np.empty(ne), np.empty(ne)
        self._call(library().pdg_get_blending(self._ctx, eta.ctypes.data_as(_dp), alpha.ctypes.data_as(_dp)),
                   "pdg_get_blending")
        return eta, alpha

    def gradients(self, u, stream=None):
        """BR1 primitive gradients of a device state u: tensor of dim*size doubles."""
        import torch
        self._check_dev(u)
        g = torch.empty(self.mesh.dim * self.size, dtype=u.dtype, device=u.device)
        self._call(library().pdg_gradients(self._ctx, C.c_void_p(u.data_ptr()), C.c_void_p(g.data_ptr()),
                                           C.c_void_p(_stream_handle(stream))), "pdg_gradients")
        return g

    def check(self) -> int:
        """Reads and clears the device error word; raises PdgError on a flag."""
        f = C.c_uint32()
        self._call(library().pdg_check(self._ctx, C.byref(f)), "pdg_check")
        return f.value

    def vjp(self, u, cot, out=None, stream=None):
        """(dL/du)^T cot for device tensors u, cot (fixed operator, compat=0)."""
        import torch
        self._check_dev(u, cot)
        ubar = out if out is not None else torch.empty_like(u)
        self._check_dev(ubar)
        self._call(library().pdg_rhs_vjp(self._ctx, C.c_void_p(u.data_ptr()), C.c_void_p(cot.data_ptr()),
                                         C.c_void_p(ubar.data_ptr()), C.c_void_p(_stream_handle(stream))),
                   "pdg_rhs_vjp")
        return ubar

    def rk_stage_vjp(self, stage: int, dt: float, us, lam, out, bx, stream=None):
        """Adjoint of rk_stage(stage, dt, un, us, .) for the cotangent lam of its
        output (pdg_rk_stage_vjp): stage 2 sets out and bx, stage 1 sets out and
        adds to bx, stage 0 adds to bx (out is scratch).  Fixed operator,
        meshes without boundary faces."""
        self._check_dev(us, lam, out, bx)
        self._call(library().pdg_rk_stage_vjp(self._ctx, int(stage), float(dt), C.c_void_p(us.data_ptr()),
                                              C.c_void_p(lam.data_ptr()), C.c_void_p(out.data_ptr()),
                                              C.c_void_p(bx.data_ptr()), C.c_void_p(_stream_handle(stream))),
                   "pdg_rk_stage_vjp")
        return out

    def filter_count(self) -> int:
        """Element filterings by the entropy filter since creation (synchronises)."""
        n = C.c_int64()
        self._call(library().pdg_filter_count(self._ctx, C.byref(n)), "pdg_filter_count")
        return n.value

    def rk_stage_part(self, part: int, stage: int, dt: float, un, us, uout, e_begin: int, e_end: int, stream=None):
        """One kernel of a fused stage over elements [e_begin, e_end)
        (pdg_rk_stage_part): PART_START, then PART_FACES, PART_LIFT and
        PART_VOLUME over every element, each after the parts it reads."""
        for t in (un, us, uout):
            if t is not None:
                self._check_dev(t)
        ptr = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)  # noqa: E731
        self._call(library().pdg_rk_stage_part(self._ctx, int(part), int(stage), float(dt), ptr(un), ptr(us), ptr(uout),
                                               int(e_begin), int(e_end), C.c_void_p(_stream_handle(stream))),
                   "pdg_rk_stage_part")

    def face_columns(self):
        """The context's viscous face columns as a float64 CUDA tensor (a view,
        shape [dim, 2, num_elements, face nodes, dim + 1]); Navier-Stokes only."""
        import torch
        ptr, n = C.c_void_p(), C.c_int64()
        self._call(library().pdg_face_columns(self._ctx, C.byref(ptr), C.byref(n)), "pdg_face_columns")
        m = self.mesh
        shape = (m.dim, 2, m.num_elements, m.Np ** (m.dim - 1), m.dim + 1)
        assert int(np.prod(shape)) == n.value

        class _View:  # a CUDA array interface over the context's buffer
            __cuda_array_interface__ = {"shape": shape, "typestr": "<f8", "data": (ptr.value, False), "version": 3,
                                        "strides": None}
        dev = torch.device("cuda", torch.cuda.current_device())
        return torch.as_tensor(_View(), device=dev)

    def limiter_count(self) -> int:
        """Element limitings by the positivity limiter since creation (synchronises)."""
        n = C.c_int64()
        self._call(library().pdg_limiter_count(self._ctx, C.byref(n)), "pdg_limiter_count")
        return n.value

    def launch_count(self) -> int:
        return int(library().pdg_launch_count(self._ctx))


class DGSEMBatch:
    """Many independent periodic 2D Euler cases advanced together: one
    persistent launch per SSP-RK3 stage over all cases, replayed from a CUDA
    graph.  The state is one device tensor; case c is
    ``u[offsets[c]:offsets[c + 1]]`` in its own mesh's byNODES layout."""

    def __init__(self, meshes, **params):
        self.meshes = list(meshes)
        self.params = default_params(**params)
        self._nbrs = [np.ascontiguousarray(m.nbr, dtype=np.int32) for m in self.meshes]
        arr = (PdgMesh * len(self.meshes))()
        for i, (m, nb) in enumerate(zip(self.meshes, self._nbrs)):
            h = list(m.h) + [1.0] * (3 - m.dim)
            arr[i] = PdgMesh(m.dim, m.order, m.num_elements, (C.c_double * 3)(*h), nb.ctypes.data_as(_ip))
        self._arr = arr
        self._b = C.c_void_p()
        code = library().pdg_batch_create(len(self.meshes), arr, C.byref(self.params), C.byref(self._b))
        if code != PDG_OK:
            raise PdgError(code, "pdg_batch_create")
        L = library()
        self.offsets = np.array([L.pdg_batch_offset(self._b, c) for c in range(len(self.meshes) + 1)],
                                dtype=np.int64)

    def _call(self, code, what):
        if code != PDG_OK:
            raise PdgError(code, f"{what}: {library().pdg_batch_last_error(self._b).decode()}")

    def close(self):
        if getattr(self, "_b", None):
            library().pdg_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def size(self) -> int:
        return int(self.offsets[-1])

    def _check_dev(self, *ts):
        for t in ts:
            if not (t.is_cuda and t.element_size() == 8 and t.dtype.is_floating_point and t.is_contiguous()):
                raise ValueError("device arrays must be contiguous float64 CUDA tensors")
            if t.numel() != self.size:
                raise ValueError(f"array has {t.numel()} entries, batch size is {self.size}")

    def set_dt(self, dt):
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        if dt.size != len(self.meshes):
            raise ValueError("one dt per case")
        self._call(library().pdg_batch_set_dt(self._b, dt.ctypes.data_as(_dp)), "pdg_batch_set_dt")

    def Mult(self, u, dudt, stream=None):
        self._check_dev(u, dudt)
        self._call(library().pdg_batch_rhs(self._b, C.c_void_p(u.data_ptr()), C.c_void_p(dudt.data_ptr()),
                                           C.c_void_p(_stream_handle(stream))), "pdg_batch_rhs")
        return dudt

    def rk3_step(self, u, nsteps: int = 1, graph: bool = True, stream=None):
        self._check_dev(u)
        self._call(library().pdg_batch_rk3_step(self._b, C.c_void_p(u.data_ptr()), int(nsteps), int(bool(graph)),
                                                C.c_void_p(_stream_handle(stream))), "pdg_batch_rk3_step")
        return u

    def tune(self, u, stream=None) -> float:
        self._check_dev(u)
        ms = C.c_float()
        self._call(library().pdg_batch_tune(self._b, C.c_void_p(u.data_ptr()), C.c_void_p(_stream_handle(stream)),
                                            C.byref(ms)), "pdg_batch_tune")
        return ms.value

    def config(self) -> dict:
        v = [C.c_int() for _ in range(5)]
        self._call(library().pdg_batch_config(self._b, *[C.byref(x) for x in v]), "pdg_batch_config")
        return dict(zip(("warps_per_block", "blocks", "tiles_per_fetch", "tile_order", "register_variant"),
                        (x.value for x in v)))

    def max_char_speed(self) -> np.ndarray:
        lam = np.empty(len(self.meshes))
        self._call(library().pdg_batch_max_char_speed(self._b, lam.ctypes.data_as(_dp)), "pdg_batch_max_char_speed")
        return lam

    def cfl_dt(self, cfl: float) -> np.ndarray:
        """Per-case dt = cfl h_min / (lambda_max (N+1)^2) from the running maxima."""
        lam = self.max_char_speed()
        return np.array([cfl * min(m.h) / (l * (m.order + 1) ** 2) for m, l in zip(self.meshes, lam)])

    def check(self) -> int:
        f = C.c_uint32()
        self._call(library().pdg_batch_check(self._b, C.byref(f)), "pdg_batch_check")
        return f.value

    def launch_count(self) -> int:
        return int(library().pdg_batch_launch_count(self._b))


class RK3SSPSolver:
    """Shu-Osher SSP-RK3 with the operator's RHS fused into each stage."""

    def Init(self, op: DGSEMOperator):
        self.op = op

    def Step(self, x, t: float, dt: float, stream=None) -> float:
        self.op.rk3_step(x, dt, stream=stream)
        return t + dt
