"""ctypes bindings of the CPU oracle (liboracle.so) and of the reference's own
hot-path sources built against the stand-in MFEM header (_ref/libref_*.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the reference result.  The product package
(prandtl_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
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


def make_params(parabolic=0, blending=1, compat=1, filter=0, gamma=1.4, Pr=0.72, mu=0.0,
                R_gas=287.0, alpha_max=0.5, alpha_min=0.001, face_dissipation=1.0) -> PdgParams:
    return PdgParams(int(parabolic), int(blending), int(compat), int(filter), gamma, Pr, mu,
                     R_gas, alpha_max, alpha_min, face_dissipation)


def make_mesh(mesh) -> tuple[PdgMesh, np.ndarray]:
    nbr = np.ascontiguousarray(mesh.nbr, dtype=np.int32)
    h = list(mesh.h) + [1.0] * (3 - mesh.dim)
    m = PdgMesh(mesh.dim, mesh.order, mesh.num_elements, (C.c_double * 3)(*h),
                nbr.ctypes.data_as(_ip))
    return m, nbr


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


_lib = None
_lib_fma = None


def lib(fma: bool = False):
    """The oracle library; fma=True: the same source compiled with fused
    multiply-adds (liboracle_fma.so), whose spread from the plain build is
    the rounding floor of a state."""
    global _lib, _lib_fma
    if (_lib_fma if fma else _lib) is None:
        path = os.path.join(HERE, "liboracle_fma.so" if fma else "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run oracle/build_oracle.sh")
        L = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(PdgMesh), C.POINTER(PdgParams)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_boundary.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_rhs.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_rk3_step.argtypes = [C.c_void_p, C.c_double, _dp]
        L.orc_rk_stage.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp]
        L.orc_max_char_speed.restype = C.c_double
        L.orc_max_char_speed.argtypes = [C.c_void_p]
        L.orc_get_blending.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_get_gradients.argtypes = [C.c_void_p, _dp]
        L.orc_filtered_elements.restype = C.c_int64
        L.orc_filtered_elements.argtypes = [C.c_void_p]
        L.orc_limited_elements.restype = C.c_int64
        L.orc_limited_elements.argtypes = [C.c_void_p]
        L.orc_positivity_apply.argtypes = [C.c_void_p, _dp]
        L.orc_set_geometry.restype = C.c_int
        L.orc_set_geometry.argtypes = [C.c_void_p, _dp, _ip]
        L.orc_gll.argtypes = [C.c_int, _dp, _dp]
        L.orc_derivative_matrices.argtypes = [C.c_int, _dp, _dp, _dp]
        L.orc_logmean.restype = C.c_double
        L.orc_logmean.argtypes = [C.c_double, C.c_double]
        L.orc_volume_flux.restype = C.c_double
        L.orc_volume_flux.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp]
        L.orc_face_flux.restype = C.c_double
        L.orc_face_flux.argtypes = [C.c_int, C.c_double, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_viscous_flux.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        L.orc_conserv2entropy.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.orc_entgrad2primgrad.argtypes = [C.c_int, C.c_double, C.c_int, _dp, _dp]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        if fma:
            _lib_fma = L
        else:
            _lib = L
    return _lib_fma if fma else _lib


class Oracle:
    """CPU restatement of DGSEMOperator (+ RK3SSPSolver) on one mesh."""

    def __init__(self, mesh, fma=False, **params):
        self.mesh = mesh
        self.params = make_params(**params)
        self._m, self._nbr = make_mesh(mesh)
        self._L = lib(fma)
        self.h = self._L.orc_create(C.byref(self._m), C.byref(self.params))
        if not self.h:
            raise ValueError("orc_create rejected the mesh/params")
        for b, (typ, state) in (getattr(mesh, "boundaries", None) or {}).items():
            self.set_boundary(b, typ, state)
        if getattr(mesh, "coords", None) is not None:
            self._x = np.ascontiguousarray(mesh.coords, dtype=np.float64)
            fo = getattr(mesh, "face_orient", None)
            self._fo = None if fo is None else np.ascontiguousarray(fo, dtype=np.int32)
            if self._L.orc_set_geometry(self.h, _ptr(self._x), None if self._fo is None else self._fo.ctypes.data_as(_ip)):
                raise ValueError("orc_set_geometry rejected the geometry")

    def set_boundary(self, index: int, typ: int, state=None):
        st = None if state is None else np.ascontiguousarray(state, dtype=np.float64)
        self._L.orc_set_boundary(self.h, int(index), int(typ), None if st is None else _ptr(st))

    def __del__(self):
        try:
            if getattr(self, "h", None) and getattr(self, "_L", None) is not None:
                self._L.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass  # interpreter shutdown

    def rhs(self, u: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self._L.orc_rhs(self.h, _ptr(u), _ptr(out))
        return out

    def rk_stage(self, stage, dt, un, us):
        un = np.ascontiguousarray(un, dtype=np.float64)
        us = np.ascontiguousarray(us, dtype=np.float64)
        out = np.empty_like(un)
        self._L.orc_rk_stage(self.h, stage, dt, _ptr(un), _ptr(us), _ptr(out))
        return out

    def rk3_step(self, u: np.ndarray, dt: float) -> np.ndarray:
        x = np.array(u, dtype=np.float64, copy=True)
        self._L.orc_rk3_step(self.h, dt, _ptr(x))
        return x

    def max_char_speed(self) -> float:
        return self._L.orc_max_char_speed(self.h)

    def blending(self):
        ne = self.mesh.num_elements
        eta, alpha = np.empty(ne), np.empty(ne)
        self._L.orc_get_blending(self.h, _ptr(eta), _ptr(alpha))
        return eta, alpha

    def gradients(self):
        g = np.empty(self.mesh.dim * self.mesh.size)
        self._L.orc_get_gradients(self.h, _ptr(g))
        return g

    def filtered_elements(self) -> int:
        return self._L.orc_filtered_elements(self.h)

    def limited_elements(self) -> int:
        """Positivity-limiter applications (params filter & 2) so far."""
        return self._L.orc_limited_elements(self.h)

    def positivity(self, u: np.ndarray) -> np.ndarray:
        """The positivity limiter alone applied to a copy of u."""
        x = np.array(u, dtype=np.float64, copy=True)
        self._L.orc_positivity_apply(self.h, _ptr(x))
        return x


_ref_libs = {}


def ref_available(parabolic: bool) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_ns.so" if parabolic else "libref_euler.so"))


def ref_lib(parabolic: bool):
    key = bool(parabolic)
    if key not in _ref_libs:
        path = os.path.join(HERE, "_ref", "libref_ns.so" if key else "libref_euler.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run oracle/build_ref.sh")
        L = C.CDLL(path)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _ip, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double]
        L.ref_create_geo.restype = C.c_void_p
        L.ref_create_geo.argtypes = [C.c_int, C.c_int, C.c_int, _ip, _dp, _ip, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_boundary.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.ref_rhs.restype = C.c_double
        L.ref_rhs.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_get_blending.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_get_gradients.argtypes = [C.c_void_p, _dp]
        L.ref_logmean.restype = C.c_double
        L.ref_logmean.argtypes = [C.c_double, C.c_double]
        L.ref_volume_flux.restype = C.c_double
        L.ref_volume_flux.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.ref_face_flux.restype = C.c_double
        L.ref_face_flux.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.ref_viscous_flux.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ref_conserv2entropy.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_entgrad2primgrad.argtypes = [C.c_void_p, _dp, _dp]
        _ref_libs[key] = L
    return _ref_libs[key]


class Reference:
    """The reference's DGSEMIntegrator & co., compiled against the stand-in MFEM."""

    def __init__(self, mesh, parabolic=False, gamma=1.4, Pr=0.72, mu=0.0, alpha_max=0.5, alpha_min=0.001):
        self.mesh = mesh
        self.L = ref_lib(parabolic)
        self._nbr = np.ascontiguousarray(mesh.nbr, dtype=np.int32)
        h = np.array(list(mesh.h) + [1.0] * (3 - mesh.dim))
        self._h = h
        if getattr(mesh, "coords", None) is not None:
            self._x = np.ascontiguousarray(mesh.coords, dtype=np.float64)
            fo = getattr(mesh, "face_orient", None)
            self._fo = None if fo is None else np.ascontiguousarray(fo, dtype=np.int32)
            self.h = self.L.ref_create_geo(mesh.dim, mesh.order, mesh.num_elements, self._nbr.ctypes.data_as(_ip),
                                           _ptr(self._x), None if self._fo is None else self._fo.ctypes.data_as(_ip),
                                           gamma, Pr, mu, alpha_max, alpha_min)
        else:
            self.h = self.L.ref_create(mesh.dim, mesh.order, mesh.num_elements, _ptr(h),
                                       self._nbr.ctypes.data_as(_ip), gamma, Pr, mu, alpha_max, alpha_min)
        for b, (typ, state) in (getattr(mesh, "boundaries", None) or {}).items():
            st = None if state is None else np.ascontiguousarray(state, dtype=np.float64)
            if self.L.ref_set_boundary(self.h, int(b), int(typ), None if st is None else _ptr(st)):
                raise ValueError(f"boundary condition {b}: type {typ} rejected")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def rhs(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self.lam = self.L.ref_rhs(self.h, _ptr(u), _ptr(out))
        return out

    def blending(self):
        ne = self.mesh.num_elements
        eta, alpha = np.empty(ne), np.empty(ne)
        self.L.ref_get_blending(self.h, _ptr(eta), _ptr(alpha))
        return eta, alpha

    def gradients(self):
        g = np.empty(self.mesh.dim * self.mesh.size)
        self.L.ref_get_gradients(self.h, _ptr(g))
        return g
