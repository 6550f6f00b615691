"""pdg_rhs_noalloc (the allocation-free right-hand side) against pdg_rhs.

Called through the C ABI twice in a row on different states, so the second
call runs on the scratch array the first one left behind.  Tolerance: the
parity bar of the other GPU tests, 1e-12 relative in max norm.
"""
import ctypes as C

import numpy as np
import pytest

import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import rel_maxnorm, rough

TOL = 1e-12


def _abi_mesh(mesh):
    nbr = np.ascontiguousarray(mesh.nbr, dtype=np.int32)
    h = list(mesh.h) + [1.0] * (3 - mesh.dim)
    m = pb.PdgMesh(mesh.dim, mesh.order, mesh.num_elements, (C.c_double * 3)(*h),
                   nbr.ctypes.data_as(C.POINTER(C.c_int32)))
    return m, nbr


def _tgv(order, n=4):
    m = periodic_box(3, order, (n, n - 1, n + 1), 0.0, 2 * np.pi)
    u = cases.taylor_green(m)
    return m, [u, rough(u, m, 5)]


def _kh(order, n=6):
    m = periodic_box(2, order, (n, n + 1), -1.0, 1.0)
    u = cases.kelvin_helmholtz(m)
    return m, [rough(u, m, 3), u]


CASES = [
    ("tgv_ns_n3", _tgv, 3, dict(parabolic=1, mu=0.01, Pr=0.71, compat=1)),
    ("tgv_ns_n2_fixed", _tgv, 2, dict(parabolic=1, mu=0.01, Pr=0.71, compat=0)),
    ("kh_euler_n4", _kh, 4, dict(parabolic=0, compat=1)),
    ("kh_euler_n3_fixed", _kh, 3, dict(parabolic=0, compat=0)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,order,params", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_pdg_rhs(name, make, order, params, cuda_device):
    import torch
    mesh, states = make(order)
    op = pb.DGSEMOperator(mesh, **params)
    m, nbr = _abi_mesh(mesh)
    p = pb.default_params(**params)
    L = pb.library()
    stream = torch.cuda.current_stream().cuda_stream
    for u in states:  # two calls in a row
        ud = torch.from_numpy(u).to(cuda_device)
        want = torch.empty_like(ud)
        got = torch.full_like(ud, float("nan"))
        op.Mult(ud, want)
        rc = L.pdg_rhs_noalloc(C.byref(m), C.byref(p), C.c_void_p(ud.data_ptr()), C.c_void_p(got.data_ptr()),
                               C.c_void_p(stream))
        assert rc == pb.PDG_OK
        torch.cuda.synchronize()
        assert rel_maxnorm(got.cpu().numpy(), want.cpu().numpy()) < TOL
    del nbr
    op.close()


@pytest.mark.gpu
def test_noalloc_rejects_oversized_mesh(cuda_device):
    """A mesh beyond the fixed scratch returns PDG_ERR_CAPACITY.  The state
    and output are real device buffers of the mesh's size, so the call is
    safe whatever order its checks run in."""
    import torch
    mesh = periodic_box(3, 3, (18, 18, 18), 0.0, 1.0)  # 5832 elements of NS scratch
    m, nbr = _abi_mesh(mesh)
    p = pb.default_params(parabolic=1, mu=0.01)
    u = torch.from_numpy(cases.taylor_green(periodic_box(3, 3, (18, 18, 18), 0.0, 2 * np.pi))).to(cuda_device)
    out = torch.zeros_like(u)
    rc = pb.library().pdg_rhs_noalloc(C.byref(m), C.byref(p), C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                                      None)
    torch.cuda.synchronize()
    assert rc == 7
    assert not out.any()  # nothing was written
    del nbr


@pytest.mark.gpu
def test_noalloc_rejects_bad_arguments(cuda_device):
    import torch
    mesh = periodic_box(2, 3, (4, 4), 0.0, 1.0)
    m, nbr = _abi_mesh(mesh)
    p = pb.default_params()
    L = pb.library()
    u = torch.from_numpy(cases.kelvin_helmholtz(mesh)).to(cuda_device)
    out = torch.zeros_like(u)
    pu, po = C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr())
    assert L.pdg_rhs_noalloc(None, C.byref(p), pu, po, None) == 1
    assert L.pdg_rhs_noalloc(C.byref(m), C.byref(p), pu, pu, None) == 1   # aliased
    assert L.pdg_rhs_noalloc(C.byref(m), C.byref(p), pu, None, None) == 1  # no output
    nbr[0] = 99  # a neighbour outside the mesh
    assert L.pdg_rhs_noalloc(C.byref(m), C.byref(p), pu, po, None) == 1
    torch.cuda.synchronize()
    assert not out.any()
