"""The MFEM adapter header (include/prandtl_b200_mfem.hpp) compiles against
the MFEM interface, links to the library, and reports a failed context
creation (no GPU here) as an exception instead of aborting."""
import os
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
NATIVE = os.path.join(ROOT, "tests", "native")
LIBDIR = os.path.join(ROOT, "prandtl_b200", "_lib")


def test_adapter_compiles_links_and_reports_errors(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libprandtl_b200.so")):
        pytest.skip("library not built")
    exe = tmp_path / "adapter_check"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", NATIVE, "-I", os.path.join(ROOT, "include"),
                    os.path.join(NATIVE, "mfem_adapter_check.cpp"), "-L", LIBDIR, "-lprandtl_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0
    assert out.stdout.startswith("error: pdg_create failed") or out.stdout.startswith("constructed 128")


def _build(tmp_path, src, name):
    exe = tmp_path / name
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-O2", "-I", NATIVE, "-I", os.path.join(ROOT, "include"),
                    os.path.join(NATIVE, src), "-L", LIBDIR, "-lprandtl_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return exe


@pytest.mark.gpu
@pytest.mark.parametrize("case,compat", [("tgv_ns", 1), ("tgv_ns", 0), ("vortex", 1), ("vortex", 0)])
def test_adapter_on_gpu_matches_oracle(case, compat, tmp_path, cuda_device):
    """GpuDGSEMOperator::Mult and two GpuRK3SSPSolver::Step calls on host
    vectors, in a C++ program of their own, against the oracle: 1e-12
    relative in max norm (the parity bar of the other GPU tests)."""
    import numpy as np

    import oracle
    from prandtl_b200 import cases
    from prandtl_b200.mesh import periodic_box

    from helpers import rel_maxnorm, rough
    if not os.path.exists(os.path.join(LIBDIR, "libprandtl_b200.so")):
        pytest.skip("library not built")
    if case == "tgv_ns":
        mesh = periodic_box(3, 3, (6, 5, 7), 0.0, 2 * np.pi)
        u = rough(cases.taylor_green(mesh), mesh, 23, 0.02, 0.002)
        par = dict(parabolic=1, mu=0.01, Pr=0.71)
    else:
        mesh = cases.vortex_mesh(12, 3)
        u = cases.isentropic_vortex(mesh)
        par = dict(parabolic=0, mu=0.0, Pr=0.72)
    orc = oracle.Oracle(mesh, compat=compat, **par)
    ref = orc.rhs(u)
    lam = orc.max_char_speed()
    dt = 0.5 * min(mesh.h) / (lam * (mesh.order + 1) ** 2)
    h = list(mesh.h) + [1.0] * (3 - mesh.dim)
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(np.array([mesh.dim, mesh.order, par["parabolic"], compat], dtype=np.int32).tobytes())
        f.write(np.array([mesh.num_elements], dtype=np.int64).tobytes())
        f.write(np.array(h + [par["mu"], par["Pr"], dt], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(mesh.nbr, dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(u, dtype=np.float64).tobytes())
    exe = _build(tmp_path, "mfem_adapter_run.cpp", "adapter_run")
    r = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = np.fromfile(outp, dtype=np.float64)
    n = u.size
    dudt, lam_gpu, t, x = res[:n], res[n], res[n + 1], res[n + 2:]
    assert rel_maxnorm(dudt, ref) < 1e-12
    assert abs(lam_gpu - lam) <= 1e-12 * lam
    assert abs(t - 2 * dt) <= 1e-15 * t
    want = orc.rk3_step(orc.rk3_step(u, dt), dt)
    assert rel_maxnorm(x, want) < 1e-12
