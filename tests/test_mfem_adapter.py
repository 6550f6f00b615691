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
