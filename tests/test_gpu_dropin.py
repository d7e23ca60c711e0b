"""The C++ drop-in end to end: pdgpu_peridem (PeriDEM's command-line
program with model::GpuDEMModel, peridem_b200/host/gpu_dem_model.h, in
place of model::DEMModel) reads the same YAML deck as the reference, runs
the reference's own DEMModel::init, steps on the GPU through libpdgpu, and
runs the reference's own post-processing on the downloaded state.  Its final
state (written with pdgpu_write_vtu) and post-processing key data must match
the reference binary's dump at the same step within the FP64 parity
tolerances of tests/parity.py (u, v, x to 1e-10; compressive-test reaction
to 1e-12 relative; two-particle penetration and max y to 1e-10 of the
particle size).

The drop-in reads no private member of the reference: bond-law constants
come from the decks (pdgpu_material_constants) and are checked against each
material's public critical stretch.
"""
import json
import os
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import parity
import refrun
import scenarios
from peridem_b200 import scene as scn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "peridem_b200", "_lib", "pdgpu_peridem")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refrun.have_reference(), reason="reference binary not built"),
              pytest.mark.skipif(not os.path.exists(DROPIN), reason="pdgpu_peridem not built")]


def _read_vtu(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">')
    root = ET.fromstring(head.decode() + "</VTKFile>")
    base = rest.index(b"_") + 1
    arrays = {}
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        nb = int(np.frombuffer(rest[base + off:base + off + 8], dtype=np.uint64)[0])
        dt = {"Float64": np.float64, "Float32": np.float32, "Int64": np.int64, "UInt64": np.uint64,
              "UInt8": np.uint8}[da.get("type")]
        a = np.frombuffer(rest[base + off + 8:base + off + 8 + nb], dtype=dt)
        arrays[da.get("Name")] = a.reshape(-1, int(da.get("NumberOfComponents", "1")))
    return arrays


@pytest.mark.parametrize("case", ["compressive_small", "two_particle_rnp", "compressive_force_bc"])
def test_dropin_program_matches_reference(case, tmp_path):
    factory, steps, _ = scenarios.CASES[case]
    spec = factory()
    scn.write_deck(spec, str(tmp_path))
    init, dumps = refrun.run_reference(str(tmp_path), steps, [steps])
    ref = dumps[steps]
    vtu = str(tmp_path / "final.vtu")
    r = subprocess.run([DROPIN, "-i", "deck.yaml", "-nThreads", "1", "-finalVtu", vtu, "-steps", str(steps)],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    out = json.loads(line)
    assert out["n"] == steps
    assert out["time"] == pytest.approx(float(ref["time"][0]), rel=1e-14)
    N = int(init["N"][0])
    a = _read_vtu(vtu)
    x = a["Points"].reshape(N, 3)
    u = a["Displacement"].reshape(N, 3)
    v = a["Velocity"].reshape(N, 3)
    xr = init["xRef"].reshape(N, 3)
    eu = refrun.rel_err(u, ref["u"].reshape(N, 3), floor=1e-30)
    ev = refrun.rel_err(v, ref["v"].reshape(N, 3), floor=1e-30)
    ex = refrun.rel_err(x - xr, ref["x"].reshape(N, 3) - xr, floor=1e-30)
    print(f"{case}: u {eu:.2e} v {ev:.2e} x {ex:.2e}; {out}")
    assert eu <= parity.KIN_TOL and ev <= parity.KIN_TOL and ex <= parity.KIN_TOL
    if int(init["test"][0]) == 2:
        rr = float(ref["reaction"][0])
        assert abs(out["reaction"] - rr) <= 1e-12 * max(1.0, abs(rr)), (out["reaction"], rr)
        pr = float(ref["wall_penetration"][0])
        assert abs(out["wall_penetration"] - pr) <= 1e-12 * max(1e-12, abs(pr))
    if int(init["test"][0]) == 1:
        scale = float(np.max(init["p_boundR"]))
        for key in ("pen_dist", "max_y"):
            rk = float(ref[key][0])
            assert abs(out[key] - rk) <= parity.PP_TOL * max(abs(rk), scale), (key, out[key], rk)
