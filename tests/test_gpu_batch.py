"""Batched sweep (one persistent launch per RK stage over many cases) against
per-case contexts and the oracle.

Cases mix orders 1-5 and sizes; the batch's right-hand side and its graph
replayed SSP-RK3 steps must equal, case by case, what a per-case
DGSEMOperator computes (same kernels' arithmetic: 1e-12 relative in max norm)
and the oracle (1e-12 for the right-hand side).
"""
import numpy as np
import pytest

import oracle
import prandtl_b200 as pb
from prandtl_b200 import cases
from prandtl_b200.mesh import periodic_box

from helpers import rel_maxnorm, rough

TOL = 1e-12
pytestmark = pytest.mark.gpu


def _mixed_cases(num=12, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(num):
        n = int(rng.integers(2, 9))
        N = int(rng.integers(1, 6))
        m = periodic_box(2, N, (n, n + int(rng.integers(0, 3))), -5.0, 5.0)
        eps = float(rng.uniform(1, 5))
        u = cases.isentropic_vortex(m, strength=eps)
        if i % 3 == 0:
            u = rough(u, m, seed + i)  # exercises the subcell blending
        out.append((m, u))
    return out


def _pack(batch, states):
    u = np.empty(batch.size)
    for c, s in enumerate(states):
        u[batch.offsets[c]:batch.offsets[c + 1]] = s
    return u


@pytest.mark.parametrize("compat", [1, 0])
def test_batch_rhs_matches_per_case_and_oracle(compat, cuda_device):
    import torch
    cs = _mixed_cases()
    batch = pb.DGSEMBatch([m for m, _ in cs], compat=compat)
    u = torch.from_numpy(_pack(batch, [s for _, s in cs])).to(cuda_device)
    out = torch.full_like(u, float("nan"))
    batch.Mult(u, out)
    got = out.cpu().numpy()
    lam = batch.max_char_speed()
    for c, (m, s) in enumerate(cs):
        op = pb.DGSEMOperator(m, compat=compat)
        ud = torch.from_numpy(s).to(cuda_device)
        want = torch.empty_like(ud)
        op.Mult(ud, want)
        g = got[batch.offsets[c]:batch.offsets[c + 1]]
        assert rel_maxnorm(g, want.cpu().numpy()) < TOL, f"case {c}"
        assert rel_maxnorm(g, oracle.Oracle(m, compat=compat).rhs(s)) < TOL, f"case {c} vs oracle"
        assert abs(lam[c] - op.GetMaxCharSpeed()) <= 1e-14 * lam[c]
    assert batch.check() == 0


@pytest.mark.parametrize("graph", [True, False])
def test_batch_steps_match_per_case(graph, cuda_device):
    import torch
    cs = _mixed_cases(num=10, seed=3)
    batch = pb.DGSEMBatch([m for m, _ in cs])
    u = torch.from_numpy(_pack(batch, [s for _, s in cs])).to(cuda_device)
    tmp = torch.empty_like(u)
    batch.Mult(u, tmp)
    dt = batch.cfl_dt(0.5)
    batch.set_dt(dt)
    batch.rk3_step(u, nsteps=5, graph=graph)
    got = u.cpu().numpy()
    for c, (m, s) in enumerate(cs):
        op = pb.DGSEMOperator(m)
        x = torch.from_numpy(s).to(cuda_device)
        for _ in range(5):
            op.rk3_step(x, float(dt[c]))
        assert rel_maxnorm(got[batch.offsets[c]:batch.offsets[c + 1]], x.cpu().numpy()) < TOL, f"case {c}"
    assert batch.check() == 0
    assert batch.launch_count() == 1 + 15


def test_batch_tuner_keeps_results(cuda_device):
    """The autotuner picks a configuration; results do not depend on it beyond rounding."""
    import torch
    cs = _mixed_cases(num=8, seed=5)
    batch = pb.DGSEMBatch([m for m, _ in cs])
    u = torch.from_numpy(_pack(batch, [s for _, s in cs])).to(cuda_device)
    a, b = torch.empty_like(u), torch.empty_like(u)
    batch.Mult(u, a)
    ms = batch.tune(u)
    cfg = batch.config()
    assert ms > 0 and cfg["warps_per_block"] in (1, 2, 4, 8) and cfg["tiles_per_fetch"] in (1, 2, 4, 8)
    assert cfg["blocks"] >= 148
    batch.Mult(u, b)
    # warps per block, tiles per fetch and tile order leave the arithmetic
    # unchanged; the register-budget variants are separate compilations whose
    # instruction selection may differ in the last bit
    assert rel_maxnorm(b.cpu().numpy(), a.cpu().numpy()) < 1e-14
