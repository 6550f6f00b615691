"""Reverse-mode pointwise physics (adjoint_physics.cuh) against torch autograd.

The device functions are compiled for the host (they are __host__
__device__) into a small test library and run on the CPU; each reverse-mode
function must reproduce autograd's vector-Jacobian product of the same
forward formula in oracle/torch_rhs.py to 1e-12 relative.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle.torch_rhs import TorchDGSEM
from prandtl_b200.mesh import periodic_box

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "adjoint_host.cu")
LIB = os.path.join(HERE, "native", "_build", "libadjhost.so")
TOL = 1e-12
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    deps = [SRC, os.path.join(HERE, "..", "prandtl_b200", "csrc", "adjoint_physics.cuh"),
            os.path.join(HERE, "..", "prandtl_b200", "csrc", "physics.cuh")]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(d) for d in deps):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
                        "-Xcompiler", "-fPIC", "-o", LIB, SRC], check=True)
    return C.CDLL(LIB)


def p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def state(rng, dim, near=None):
    rho = rng.uniform(0.5, 2.0)
    v = rng.uniform(-1.0, 1.0, dim)
    pr = rng.uniform(0.5, 3.0)
    if near is not None:  # a nearby state (the log-mean series branch)
        rho, v, pr = near[0] * (1 + 1e-4 * rng.standard_normal()), near[1] + 1e-4, near[2] * (1 + 1e-4)
    E = pr / 0.4 + 0.5 * rho * float(v @ v)
    return np.concatenate([[rho], rho * v, [E]]), (rho, v, pr)


def tdgsem(dim):
    return TorchDGSEM(periodic_box(dim, 1, 2, 0.0, 1.0), parabolic=True, mu=0.013, Pr=0.71)


def grads(fn, inputs, cot):
    ts = [torch.tensor(x, requires_grad=True) for x in inputs]
    out = fn(*ts)
    loss = sum((o * float(c)) for o, c in zip(out, cot))
    g = torch.autograd.grad(loss, ts, allow_unused=True)
    return [gi.numpy() if gi is not None else np.zeros_like(x) for gi, x in zip(g, inputs)], \
        np.array([float(o.detach()) for o in out])


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("near", [False, True])
def test_volume_flux_vjp(lib, dim, near):
    rng = np.random.default_rng(10 + dim + 5 * near)
    T = tdgsem(dim)
    for trial in range(6):
        sa, prim_a = state(rng, dim)
        sb, _ = state(rng, dim, prim_a if near else None)
        d = trial % dim
        metric = rng.uniform(0.3, 2.0)
        cot = rng.standard_normal(dim + 2)

        def f(a, b):
            return T.volume_flux([a[v] for v in range(dim + 2)], [b[v] for v in range(dim + 2)], d, metric)
        (ga_t, gb_t), F_t = grads(f, [sa, sb], cot)
        F = np.zeros(dim + 2)
        lib.h_volume_flux(dim, C.c_double(1.4), p(sa), p(sb), d, C.c_double(metric), p(F))
        assert rel(F, F_t) < TOL
        ga, gb = np.zeros(dim + 2), np.zeros(dim + 2)
        lib.h_volume_flux_vjp(dim, C.c_double(1.4), p(sa), p(sb), d, C.c_double(metric), p(cot), p(ga), p(gb))
        assert rel(ga, ga_t) < TOL and rel(gb, gb_t) < TOL


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("near", [False, True])
def test_face_flux_vjp(lib, dim, near):
    rng = np.random.default_rng(20 + dim + 5 * near)
    T = tdgsem(dim)
    for trial in range(6):
        sa, prim_a = state(rng, dim)
        sb, _ = state(rng, dim, prim_a if near else None)
        d = trial % dim
        nrm = rng.uniform(0.3, 2.0) * (1 if trial % 2 else -1)
        cot = rng.standard_normal(dim + 2)

        def f(a, b):
            return T.face_flux([a[v] for v in range(dim + 2)], [b[v] for v in range(dim + 2)], d, nrm)
        (ga_t, gb_t), F_t = grads(f, [sa, sb], cot)
        F = np.zeros(dim + 2)
        lib.h_face_flux(dim, C.c_double(1.4), C.c_double(1.0), p(sa), p(sb), d, C.c_double(nrm), p(F))
        assert rel(F, F_t) < TOL
        ga, gb = np.zeros(dim + 2), np.zeros(dim + 2)
        lib.h_face_flux_vjp(dim, C.c_double(1.4), C.c_double(1.0), p(sa), p(sb), d, C.c_double(nrm), p(cot),
                            p(ga), p(gb))
        assert rel(ga, ga_t) < TOL and rel(gb, gb_t) < TOL


@pytest.mark.parametrize("dim", [2, 3])
def test_entropy_vars_vjp(lib, dim):
    rng = np.random.default_rng(30 + dim)
    T = tdgsem(dim)
    for _ in range(6):
        s, _ = state(rng, dim)
        cot = rng.standard_normal(dim + 2)
        (g_t,), w_t = grads(lambda x: T.entropy_vars([x[v] for v in range(dim + 2)]), [s], cot)
        w = np.zeros(dim + 2)
        lib.h_entropy_vars(dim, C.c_double(1.4), p(s), p(w))
        assert rel(w, w_t) < TOL
        g = np.zeros(dim + 2)
        lib.h_entropy_vars_vjp(dim, C.c_double(1.4), p(s), p(cot), p(g))
        assert rel(g, g_t) < TOL


@pytest.mark.parametrize("dim", [2, 3])
def test_entgrad_vjp(lib, dim):
    rng = np.random.default_rng(40 + dim)
    T = tdgsem(dim)
    for _ in range(6):
        s, _ = state(rng, dim)
        gin = rng.standard_normal(dim + 2)
        cot = rng.standard_normal(dim + 2)
        (sb_t, gb_t), o_t = grads(lambda x, g: T.entgrad_to_primgrad([x[v] for v in range(dim + 2)],
                                                                   [g[v] for v in range(dim + 2)]), [s, gin], cot)
        o = gin.copy()
        lib.h_entgrad(dim, C.c_double(1.4), p(s), p(o))
        assert rel(o, o_t) < TOL
        gb, sb = np.zeros(dim + 2), np.zeros(dim + 2)
        lib.h_entgrad_vjp(dim, C.c_double(1.4), p(s), p(gin), p(cot), p(gb), p(sb))
        assert rel(gb, gb_t) < TOL and rel(sb, sb_t) < TOL


@pytest.mark.parametrize("dim", [2, 3])
def test_viscous_cols_vjp(lib, dim):
    rng = np.random.default_rng(50 + dim)
    T = tdgsem(dim)
    nv = dim + 2
    lk = T.mu * T.gamma / T.Pr
    for _ in range(6):
        s, _ = state(rng, dim)
        dq = rng.standard_normal(dim * nv)
        cot = rng.standard_normal(dim * (dim + 1))

        def f(x, g):
            cols = T.viscous_cols([x[v] for v in range(nv)], [[g[d * nv + v] for v in range(nv)] for d in range(dim)])
            return [c for col in cols for c in col]
        (sb_t, dqb_t), c_t = grads(f, [s, dq], cot)
        cols = np.zeros(dim * (dim + 1))
        lib.h_viscous_cols(dim, C.c_double(1.4), C.c_double(T.mu), C.c_double(lk), p(s), p(dq), p(cols))
        assert rel(cols, c_t) < TOL
        sb, dqb = np.zeros(nv), np.zeros(dim * nv)
        lib.h_viscous_cols_vjp(dim, C.c_double(1.4), C.c_double(T.mu), C.c_double(lk), p(s), p(dq), p(cot), p(sb),
                               p(dqb))
        assert rel(sb, sb_t) < TOL and rel(dqb, dqb_t) < TOL
