"""The reference-tree adapter (pcr_b200/csrc/adapter/CudaRenderer.h, the
file a maintainer copies to code/Gpu/Cuda/CudaRenderer.h) compiles against
the reference's own headers, used the way code/Cli/Main.cpp:445-473 uses a
GpuRenderer (tests/cpp/adapter_usage.cpp).  This keeps the field names it
reads (Material, Plane, Triangle, Sphere, AreaLight, Bvh::Node, SceneData)
matching the reference.  Needs the reference tree (PCR_REFERENCE_ROOT, or a
`reference` directory beside this repository); skips where it is absent."""
import os
import subprocess

import pytest

from conftest import REFERENCE_ROOT, REPO, have_reference


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_adapter_compiles_against_reference_headers():
    code = os.path.join(REFERENCE_ROOT, "code")
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror=return-type",
           "-I", code, "-I", os.path.join(code, "Includes"), "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(REPO, "pcr_b200", "csrc"), "-I", os.path.join(REPO, "pcr_b200", "csrc", "adapter"),
           "-I", "/usr/local/cuda/include", os.path.join(REPO, "tests", "cpp", "adapter_usage.cpp")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-4000:]
