"""Synthetic initial states for the benchmark workloads.

The reference's own initial conditions differ from the benchmark definitions
(its vortex and Kelvin-Helmholtz parameters differ, and its Taylor-Green
initial condition writes the energy into the z-momentum slot), so every state
here is generated from the workload definition: seeded, deterministic, and
identical for the CPU and GPU paths.
"""
from __future__ import annotations

import numpy as np

from .mesh import CartesianMesh, periodic_box

GAMMA = 1.4

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output for counters x (uint64 array), wrapping arithmetic."""
    with np.errstate(over="ignore"):
        z = (x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counters: np.ndarray) -> np.ndarray:
    """Counter-based uniform [0,1) doubles: top 53 bits of splitmix64(seed*2^32 + i)."""
    base = np.uint64(seed) << np.uint64(32)
    with np.errstate(over="ignore"):
        z = splitmix64(base + counters.astype(np.uint64))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def prim_to_cons(dim: int, rho, vel, p, gamma=GAMMA) -> np.ndarray:
    ke = 0.5 * rho * sum(v * v for v in vel)
    out = [rho] + [rho * v for v in vel] + [p / (gamma - 1.0) + ke]
    return np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1) for a in out])


def isentropic_vortex(mesh: CartesianMesh, strength: float = 5.0, gamma=GAMMA) -> np.ndarray:
    """Shu-Yee isentropic vortex on free stream rho=u=v=p=1 centred at the origin."""
    x, y = mesh.node_coords()
    r2 = x * x + y * y
    eps = strength
    du = eps / (2 * np.pi) * np.exp(0.5 * (1 - r2))
    T = 1.0 - (gamma - 1.0) * eps ** 2 / (8 * gamma * np.pi ** 2) * np.exp(1 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    return prim_to_cons(2, rho, [1.0 - du * y, 1.0 + du * x], p, gamma)


def taylor_green(mesh: CartesianMesh, Ma: float = 0.1, gamma=GAMMA) -> np.ndarray:
    """Taylor-Green vortex, rho = 1, p0 = 1/(gamma Ma^2), on [0, 2pi]^3."""
    x, y, z = mesh.node_coords()
    p0 = 1.0 / (gamma * Ma * Ma)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    return prim_to_cons(3, np.ones_like(x), [u, v, w], p, gamma)


def kelvin_helmholtz(mesh: CartesianMesh, seed: int = 0, gamma=GAMMA) -> np.ndarray:
    """Kelvin-Helmholtz shear layer: rho = 2 (|y| < 0.5) else 1, u = +-0.5 joined
    by tanh profiles of width 0.05, p = 2.5, v = uniform(-1e-2, 1e-2) noise per
    node from splitmix64(seed, global node id)."""
    x, y = mesh.node_coords()
    width = 0.05
    # s = 1 inside the band |y| < 0.5, 0 outside, smoothed over `width`
    s = 0.5 * (np.tanh((y + 0.5) / width) - np.tanh((y - 0.5) / width))
    rho = 1.0 + s
    u = -0.5 + s
    noise = uniform01(seed, np.arange(x.size))
    v = 1e-2 * (2.0 * noise - 1.0)
    p = np.full_like(x, 2.5)
    return prim_to_cons(2, rho, [u, v], p, gamma)


def vortex_mesh(n: int = 32, order: int = 3) -> CartesianMesh:
    return periodic_box(2, order, n, -5.0, 5.0)


def tgv_mesh(n: int = 32, order: int = 3) -> CartesianMesh:
    return periodic_box(3, order, n, 0.0, 2 * np.pi)


def kh_mesh(n: int = 64, order: int = 4) -> CartesianMesh:
    return periodic_box(2, order, n, -1.0, 1.0)


def sweep_cases(num: int = 256, seed: int = 3):
    """The batched vortex sweep: n ~ U{8..64}, N ~ U{2,3,4,5}, strength ~ U[1,5]."""
    u = uniform01(seed, np.arange(3 * num)).reshape(num, 3)
    ns = 8 + np.minimum((u[:, 0] * 57).astype(int), 56)
    Ns = 2 + np.minimum((u[:, 1] * 4).astype(int), 3)
    eps = 1.0 + 4.0 * u[:, 2]
    return [(int(a), int(b), float(c)) for a, b, c in zip(ns, Ns, eps)]
