"""Generates tests/golden/*.npz from the reference's own hot-path sources.

The reference cannot run here as a program (its MFEM and hypre submodules are
empty), so oracle/build_ref.sh compiles its DGSEMIntegrator, fluxes, lifting,
indicator and modal basis unmodified against a stand-in MFEM header and this
script drives them through the restated assembly loops (oracle/ref_shim).
Each fixture stores the input state, the reference right-hand side, the
blending coefficients, the running wave speed and (parabolic) the primitive
gradients.  Inputs are seeded and small so the CPU suite stays fast.

Usage: python tests/golden/make_golden.py [name prefix]   (needs oracle/_ref/libref_*.so)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from prandtl_b200 import cases  # noqa: E402
from prandtl_b200.mesh import box, periodic_box  # noqa: E402

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
    # boundary faces (Euler): the reference's BdrFaceIntegrator and condition
    # files; types as pdg_set_boundary numbers them
    fs2 = [1.2, 0.3, -0.2, 2.6]
    m = box(2, 3, (4, 3), -1.0, 1.0, bdr=[(0, 1), (2, 2)],
            boundaries={0: (1, fs2), 1: (2, None), 2: (4, None)})
    u = rough(cases.kelvin_helmholtz(periodic_box(2, 3, (4, 3), -1.0, 1.0)), m, 15, 0.05, 0.02)
    yield "bdr_2d_n3_inflow_outflow_walls", m, u, dict(parabolic=False)
    m = box(2, 2, (3, 4), -1.0, 1.0, bdr=[(0, 1), (2, 3)],
            boundaries={0: (8, [3.5, 3.0, 2.0, 10.0, 0.0]), 1: (6, [2.2]), 2: (9, [1.0, 0.3, -0.1, 2.0]),
                        3: (7, [1.3, 0.2, 0.05])})
    u = rough(cases.kelvin_helmholtz(periodic_box(2, 2, (3, 4), -1.0, 1.0)), m, 16, 0.05, 0.02)
    yield "bdr_2d_n2_subsonic", m, u, dict(parabolic=False)
    fs3 = [1.1, 0.2, -0.1, 0.15, 2.8]
    m = box(3, 2, (3, 2, 3), 0.0, 2 * np.pi, bdr=[(0, 0), (1, 2), (3, 4)],
            boundaries={0: (4, None), 1: (5, None), 2: (2, None), 3: (3, fs3), 4: (1, fs3)})
    u = rough(cases.taylor_green(periodic_box(3, 2, (3, 2, 3), 0.0, 2 * np.pi), Ma=0.4), m, 17, 0.05, 0.02)
    yield "bdr_3d_n2_all", m, u, dict(parabolic=False)


def main(prefix: str = ""):
    for name, mesh, u, kw in fixtures():
        if not name.startswith(prefix):
            continue
        ref = oracle.Reference(mesh, **kw)
        dudt = ref.rhs(u)
        eta, alpha = ref.blending()
        data = dict(dim=mesh.dim, order=mesh.order, n=np.array(mesh.n), lo=np.array(mesh.lo), hi=np.array(mesh.hi),
                    parabolic=int(kw.get("parabolic", False)), mu=kw.get("mu", 0.0), Pr=kw.get("Pr", 0.72),
                    u=u, dudt=dudt, eta=eta, alpha=alpha, lam=ref.lam)
        if kw.get("parabolic"):
            data["grads"] = ref.gradients()
        if mesh.boundaries:
            idx = sorted(mesh.boundaries)
            bdata = np.zeros((len(idx), 7))
            bn = np.zeros(len(idx), dtype=np.int64)
            for r, b in enumerate(idx):
                d = mesh.boundaries[b][1]
                if d is not None:
                    bn[r] = len(d)
                    bdata[r, :len(d)] = d
            data.update(nbr=np.asarray(mesh.nbr, dtype=np.int32), bc_index=np.array(idx),
                        bc_type=np.array([mesh.boundaries[b][0] for b in idx]), bc_n=bn, bc_data=bdata)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
        print(f"{name}: size {u.size}, blended {int((alpha > 0).sum())}/{mesh.num_elements}, lam {ref.lam:.6f}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "")
