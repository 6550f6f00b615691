"""Writes tests/golden/mesh_{ffs,ramp,ramjet}.npz: the element corners, corner
coordinates and boundary elements parsed from three of the reference's Gmsh
files (TestCases/Euler/2D/ForwardFacingStep/ForwardFacingStep.msh,
Ramp/Ramp15deg_v2.msh, Nagashima_Ramjet/TR0/Nagashima_TR0_11kQuad_v2.msh),
so that the GPU tests can build those meshes where the reference tree is
absent.  Run where the tree is:  python tests/golden/make_mesh_fixtures.py
[reference tree] (else PRANDTL_REFERENCE, else where oracle/build_ref.sh found
the tree, recorded in oracle/_ref/REFERENCE_TREE).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from prandtl_b200 import meshio  # noqa: E402

FILES = {
    "ffs": "TestCases/Euler/2D/ForwardFacingStep/ForwardFacingStep.msh",
    "ramp": "TestCases/Euler/2D/Ramp/Ramp15deg_v2.msh",
    "ramjet": "TestCases/Euler/2D/Nagashima_Ramjet/TR0/Nagashima_TR0_11kQuad_v2.msh",
}


def main():
    rec = os.path.join(HERE, "..", "..", "oracle", "_ref", "REFERENCE_TREE")
    ref = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PRANDTL_REFERENCE")
           or (open(rec).read().strip() if os.path.exists(rec) else ""))
    if not ref or not os.path.isdir(ref):
        sys.exit("reference tree not found (pass it, or set PRANDTL_REFERENCE)")
    for name, rel in FILES.items():
        with open(os.path.join(ref, rel)) as f:
            p = meshio._parse_gmsh(f.read())
        keys = sorted(p["bdr"].items(), key=lambda kv: sorted(kv[0]))
        bverts = np.array([sorted(k) for k, _ in keys], dtype=np.int32)
        battr = np.array([a for _, a in keys], dtype=np.int32)
        names = sorted(p["names"].items(), key=lambda kv: kv[1])
        np.savez_compressed(os.path.join(HERE, f"mesh_{name}.npz"), dim=p["dim"], verts=p["verts"].astype(np.int32),
                            coords=p["coords"], attrs=p["attrs"].astype(np.int32), bverts=bverts, battr=battr,
                            name_keys=np.array([k for k, _ in names]), name_vals=np.array([v for _, v in names]),
                            source=rel)
        print(name, p["verts"].shape[0], "elements")


if __name__ == "__main__":
    main()
