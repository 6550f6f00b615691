"""Synthetic initial states for the benchmark workloads.

The reference's own initial conditions differ from the benchmark definitions
(its vortex and Kelvin-Helmholtz parameters differ, and its Taylor-Green
initial condition writes the energy into the z-momentum slot), so every state
here is generated from the workload definition: seeded, deterministic, and
identical for the CPU and GPU paths.
"""
from __future__ import annotations

import numpy as np

from .mesh import CartesianMesh, box, periodic_box

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


# Boundary-condition types as pdg_set_boundary numbers them.
_INFLOW, _OUTFLOW, _SLIP, _NOSLIP = 1, 2, 4, 10


def forward_facing_step(order: int = 3, cells_per_unit: int = 10, mach: float = 3.0, gamma=GAMMA):
    """Mach-3 wind tunnel with a forward-facing step (the classic Euler
    setup: a 3 x 1 channel, a step of height 0.2 from x = 0.6): mesh and
    uniform initial state.  Supersonic inflow on the left, outflow on the
    right, slip walls elsewhere (the step's faces included)."""
    h = 1.0 / cells_per_unit
    nx, ny = 3 * cells_per_unit, cells_per_unit
    keep = np.ones((nx, ny), dtype=bool)
    keep[int(round(0.6 / h)):, :int(round(0.2 / h))] = False
    rho, p = gamma, 1.0
    fs = prim_to_cons(2, np.array([rho]), [np.array([mach]), np.array([0.0])], np.array([p]), gamma).reshape(-1)
    mesh = box(2, order, (nx, ny), (0.0, 0.0), (3.0, 1.0), bdr=[(0, 1), (2, 2)], keep=keep, cut=2,
               boundaries={0: (_INFLOW, fs), 1: (_OUTFLOW, None), 2: (_SLIP, None)})
    u = np.repeat(fs[:, None], mesh.num_nodes, axis=1).reshape(-1)
    return mesh, u


def lid_driven_cavity(n: int = 16, order: int = 3, lid_speed: float = 1.0, mach: float = 0.1, gamma=GAMMA):
    """Lid-driven cavity on [0,1]^2 (Navier-Stokes): no-slip adiabatic walls,
    the top one moving at lid_speed; fluid at rest with p = 1/(gamma Ma^2).
    Returns the mesh and the initial state; viscosity is the caller's."""
    mesh = box(2, order, (n, n), 0.0, 1.0, bdr=[(0, 0), (0, 1)],
               boundaries={0: (_NOSLIP, [0.0, 0.0]), 1: (_NOSLIP, [lid_speed, 0.0])})
    p = 1.0 / (gamma * mach * mach)
    nn = mesh.num_nodes
    u = prim_to_cons(2, np.ones(nn), [np.zeros(nn), np.zeros(nn)], np.full(nn, p), gamma)
    return mesh, u.reshape(-1)
