"""The reference-side binding shown in INTEGRATION.md (a model::DEMModel
subclass that drives libpdgpu) compiles against the reference's own headers
and include/pdgpu.h: every C++ block of the document is extracted and
syntax-checked with the include paths and shims the oracle build of the
reference uses.  The binding asks the maintainer to make it a friend of the
four bond-law classes (their constants are private); the test applies that
same one-line change to a temporary copy of the material header, which it
puts first on the include path.  Skipped where the reference sources are
absent."""
import os
import re
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from __graft_entry__ import REF  # noqa: E402


def _friend_material_header(dst):
    """A copy of the reference's material header with `friend class
    model::GpuDEMModel;` in each bond-law class, as INTEGRATION.md asks."""
    src = os.path.join(REF, "src", "material", "mparticle", "material.h")
    text = open(src).read()
    text = text.replace('#include "influenceFn.h"', '#include "material/mparticle/influenceFn.h"', 1)
    text = text.replace("namespace material {", "namespace model {\nclass GpuDEMModel;\n}\n\nnamespace material {", 1)
    for cls in ("RnpMaterial", "PmbMaterial", "PdElastic", "PdState"):
        head = f"class {cls} : public Material {{"
        assert head in text, head
        text = text.replace(head, head + "\n  friend class model::GpuDEMModel;", 1)
    out = dst / "material" / "mparticle"
    out.mkdir(parents=True)
    (out / "material.h").write_text(text)
    return str(dst)


def _blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, flags=re.S)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference sources absent")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_integration_binding_compiles(tmp_path):
    blocks = _blocks()
    assert blocks, "INTEGRATION.md holds no C++ block"
    shim = os.path.join(ROOT, "oracle", "shim")
    friend = _friend_material_header(tmp_path / "friend")
    for k, code in enumerate(blocks):
        src = tmp_path / f"block{k}.cpp"
        src.write_text(code)
        cmd = ["g++", "-std=c++23", "-fsyntax-only", "-DFMT_HEADER_ONLY", "-w", "-I", friend,
               "-I", shim, "-I", os.path.join(shim, "vtk"), "-I", os.path.join(REF, "src"),
               "-I", os.path.join(REF, "external"), "-I", os.path.join(REF, "external", "fmt", "include"),
               "-I", os.path.join(ROOT, "include"), "-x", "c++", str(src)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
