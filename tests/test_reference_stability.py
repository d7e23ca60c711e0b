"""Why the benchmark scene keeps the configured step but not the configured
contact stiffness: the reference itself, compiled here
(oracle/_ref/peridem_ref), blows up with the configuration's contact
stiffness at the configuration's step, and runs through the same impact
when the contact spring is softened to omega dt = 0.3 (scene.stable_kn).

Two discs of the compressive test's smallest size (R = 1 mm, h = R/15,
horizon 3h, RNPBond E = 2 GPa, rho = 1200), the top one approaching at
0.1 m/s, dt = 5e-8 s (the compressive test's configured step):
  * with Kn = 10 x 18 K / (pi horizon^5) (the configuration's "contact
    stiffness 10x bulk"), velocities grow to ~1e5 m/s as soon as the discs
    touch: the node-pair penalty spring has omega dt >> 2;
  * with scene.stable_kn the same run stays bounded through the impact
    (the bonds themselves are stable at this step);
  * the smaller step of scene.stable_dt (0.2 h / c) is stable too.
CPU only; skipped where the reference binary is not built.
"""
import math

import numpy as np
import pytest

import refrun
from peridem_b200 import scene as scn

pytestmark = pytest.mark.skipif(not refrun.have_reference(), reason="reference binary not built")

R = 1e-3


def _run(tmp_path, dt, kn, steps):
    spec = scn.two_particle(h_div=15, radius=R, material="RNPBond", v0=-0.1, gap=0.02 * R / 15, nt=steps,
                            dt=dt)
    for c in spec.contact.values():
        c.kn = kn
        c.kn_factor = 1.0
    scn.write_deck(spec, str(tmp_path))
    dumps = list(range(20, steps + 1, 20))
    _, d = refrun.run_reference(str(tmp_path), steps, dumps)
    return [float(np.max(np.abs(d[k]["v"]))) for k in dumps]


def test_configured_step_blows_up_in_the_reference(tmp_path):
    E, nu = 2.0e9, 0.25
    K = E / (3 * (1 - 2 * nu))
    h = R / 15
    eps = 3 * h
    kn_cfg = 10 * 18 * K / (math.pi * eps ** 5)
    vmax = _run(tmp_path, 5e-8, kn_cfg, 300)
    print("dt 5e-8:", ["%.2e" % v for v in vmax])
    assert max(vmax) > 1e3, "expected the reference to blow up at the configured step"


@pytest.mark.parametrize("dt", [5e-8, None])
def test_softened_contact_stays_bounded_in_the_reference(tmp_path, dt):
    h = R / 15
    dt = scn.stable_dt(2.0e9, 1200.0, h) if dt is None else dt
    kn = scn.stable_kn(1200.0, h * h, dt)
    vmax = _run(tmp_path, dt, kn, int(round(3.0e-5 / dt / 20)) * 20)  # 30 us: through the impact
    print(f"dt {dt:.3e}:", ["%.2e" % v for v in vmax])
    assert max(vmax) < 1.0


def test_config0_step_blows_up_in_the_reference_even_with_softened_contact(tmp_path):
    """Config 0 (two discs, h = R/10) at its configured dt = 1e-7 s: even with
    the softened contact spring the reference blows up within a few hundred
    steps of contact, so config 0 runs at scene.stable_dt."""
    h = R / 10
    dt = 1e-7
    spec = scn.two_particle(h_div=10, radius=R, material="RNPBond", v0=-0.1, gap=0.02 * h, nt=600, dt=dt)
    for c in spec.contact.values():
        c.kn = scn.stable_kn(1200.0, h * h, dt)
        c.kn_factor = 1.0
    scn.write_deck(spec, str(tmp_path))
    dumps = list(range(100, 601, 100))
    _, d = refrun.run_reference(str(tmp_path), 600, dumps)
    vmax = [float(np.max(np.abs(d[k]["v"]))) for k in dumps]
    print("config 0 step:", ["%.2e" % v for v in vmax])
    assert max(vmax) > 1e3
