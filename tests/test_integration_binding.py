"""The C++ drop-in (peridem_b200/host/gpu_dem_model.h: model::GpuDEMModel,
a subclass of the reference's model::DEMModel) compiles against the
reference's unmodified headers and links with the reference's own objects
and libpdgpu.so into pdgpu_peridem (peridem_b200/host/Makefile).  No GPU is
needed to build it; tests/test_gpu_dropin.py runs it.  Skipped where the
reference sources or its compiled objects are absent."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from __graft_entry__ import REF  # noqa: E402

OBJ = os.path.join(ROOT, "oracle", "_ref", "obj")
LIB = os.path.join(ROOT, "peridem_b200", "_lib", "libpdgpu.so")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference sources absent")
@pytest.mark.skipif(not os.path.isdir(OBJ), reason="reference objects absent (make -C oracle ref)")
@pytest.mark.skipif(not os.path.exists(LIB), reason="libpdgpu.so not built")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_dropin_program_builds_against_the_unmodified_reference(tmp_path):
    out = tmp_path / "pdgpu_peridem"
    host = os.path.join(ROOT, "peridem_b200", "host")
    objs = sorted(os.path.join(d, f) for d, _, fs in os.walk(OBJ) for f in fs
                  if f.endswith(".o") and f != "ref_driver.o")
    shim = os.path.join(ROOT, "oracle", "shim")
    cmd = ["g++", "-std=c++23", "-O1", "-DFMT_HEADER_ONLY", "-w", "-I", host, "-I", os.path.join(ROOT, "include"),
           "-I", shim, "-I", os.path.join(shim, "vtk"), "-I", os.path.join(REF, "src"),
           "-I", os.path.join(REF, "external"), "-I", os.path.join(REF, "external", "fmt", "include"),
           "-o", str(out), os.path.join(host, "pdgpu_peridem.cpp"), *objs,
           "-L", os.path.dirname(LIB), "-lpdgpu", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    assert out.exists()
    # the header asks nothing private of the reference: no friend declaration
    # and no access-specifier override
    text = open(os.path.join(host, "gpu_dem_model.h")).read()
    assert "friend" not in text and "#define private" not in text
