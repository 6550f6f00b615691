"""Shared helpers for the parity tests."""
from __future__ import annotations

import glob
import os

import numpy as np

from prandtl_b200.mesh import periodic_box

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    mesh = periodic_box(int(z["dim"]), int(z["order"]), tuple(int(v) for v in z["n"]),
                        tuple(float(v) for v in z["lo"]), tuple(float(v) for v in z["hi"]))
    params = dict(parabolic=int(z["parabolic"]), mu=float(z["mu"]), Pr=float(z["Pr"]))
    if "nbr" in z.files:  # boundary faces and their conditions
        mesh.nbr = z["nbr"].reshape(mesh.num_elements, 2 * mesh.dim)
        mesh.boundaries = {int(b): (int(t), (z["bc_data"][r, :int(n)] if int(n) else None))
                           for r, (b, t, n) in enumerate(zip(z["bc_index"], z["bc_type"], z["bc_n"]))}
    return mesh, params, {k: z[k] for k in z.files}


def rel_maxnorm(a, b):
    """max|a - b| / max|b| (the parity measure: relative error in max norm)."""
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def rough(u, mesh, seed, amp_rho=0.15, amp_e=0.03):
    rng = np.random.default_rng(seed)
    nn = mesh.num_nodes
    u = u.copy()
    u[:nn] *= 1 + amp_rho * rng.standard_normal(nn)
    u[(mesh.nv - 1) * nn:] *= 1 + amp_e * rng.standard_normal(nn)
    return u
