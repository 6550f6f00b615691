"""Generates tests/golden/*.npz from the reference's own hot-path sources.

The reference cannot run here as a program (its MFEM and hypre submodules are
empty), so oracle/build_ref.sh compiles its DGSEMIntegrator, fluxes, lifting,
indicator and modal basis unmodified against a stand-in MFEM header and this
script drives them through the restated assembly loops (oracle/ref_shim).
Each fixture stores the input state, the reference right-hand side, the
blending coefficients, the running wave speed and (parabolic) the primitive
gradients.  Inputs are seeded and small so the CPU suite stays fast.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref/libref_*.so)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from prandtl_b200 import cases  # noqa: E402
from prandtl_b200.mesh import periodic_box  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rough(u, mesh, seed, amp_rho=0.15, amp_e=0.03):
    rng = np.random.default_rng(seed)
    nn = mesh.num_nodes
    u = u.copy()
    u[:nn] *= 1 + amp_rho * rng.standard_normal(nn)
    u[(mesh.nv - 1) * nn:] *= 1 + amp_e * rng.standard_normal(nn)
    return u


def fixtures():
    m = cases.vortex_mesh(6, 3)
    yield "vortex_2d_n3", m, cases.isentropic_vortex(m), dict(parabolic=False)
    m = cases.kh_mesh(6, 4)
    yield "kh_2d_n4", m, cases.kelvin_helmholtz(m), dict(parabolic=False)
    m = periodic_box(2, 2, (5, 4), -1.0, 1.0)
    yield "rough_2d_n2_euler", m, rough(cases.kelvin_helmholtz(m), m, 11), dict(parabolic=False)
    m = cases.tgv_mesh(3, 3)
    yield "tgv_3d_n3_ns", m, cases.taylor_green(m), dict(parabolic=True, mu=1 / 1600, Pr=0.71)
    m = cases.tgv_mesh(3, 2)
    yield "rough_3d_n2_ns", m, rough(cases.taylor_green(m), m, 12), dict(parabolic=True, mu=0.02, Pr=0.71)
    m = cases.tgv_mesh(3, 3)
    yield "rough_3d_n3_euler", m, rough(cases.taylor_green(m), m, 13), dict(parabolic=False)
    m = periodic_box(2, 3, 4, -1.0, 1.0)
    yield "rough_2d_n3_ns", m, rough(cases.kelvin_helmholtz(m), m, 14), dict(parabolic=True, mu=5e-3, Pr=0.72)


def main():
    for name, mesh, u, kw in fixtures():
        ref = oracle.Reference(mesh, **kw)
        dudt = ref.rhs(u)
        eta, alpha = ref.blending()
        data = dict(dim=mesh.dim, order=mesh.order, n=np.array(mesh.n), lo=np.array(mesh.lo), hi=np.array(mesh.hi),
                    parabolic=int(kw.get("parabolic", False)), mu=kw.get("mu", 0.0), Pr=kw.get("Pr", 0.72),
                    u=u, dudt=dudt, eta=eta, alpha=alpha, lam=ref.lam)
        if kw.get("parabolic"):
            data["grads"] = ref.gradients()
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
        print(f"{name}: size {u.size}, blended {int((alpha > 0).sum())}/{mesh.num_elements}, lam {ref.lam:.6f}")


if __name__ == "__main__":
    main()
