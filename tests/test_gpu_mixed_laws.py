"""The mixed-precision bond loop against the FP64 form, law by law, on
identical states: one DEMModel::computePeridynamicForces evaluation
(pdgpu_compute_pd_forces) of each precision on the same displacement field
and the same broken-bond state.

Two families of states:
  * taken from FP64 trajectories of the parity scenes (after contact and, for
    the PMB impact, after fracture), so pre-broken bonds are exercised;
  * a smooth synthetic deformation (peak strain 2e-3, and 3e-2 to break
    bonds where the law has a critical stretch) on 2-D discs and 3-D spheres
    for RNP, PMB, PD elastic and PD state.

(Whole trajectories are not compared here: the contact laws switch on
discontinuously — damping on entry, friction by the sign of the slip — so two
runs that differ at FP32 rounding part ways after the first contact.)

Tolerances (FP32 bond arithmetic, FP64 per-node sums):
  force   max |f_mixed - f_fp64| <= 1e-3 max |f_fp64| over nodes none of whose
          bonds ended in a different state
  damage  max |Z_mixed - Z_fp64| <= 1e-3 max(1, max Z_fp64)
  bonds   bonds whose final state differs <= max(2, 1e-3 x broken)
"""
import numpy as np
import pytest

from peridem_b200 import scene as scn
from scenarios import CASES, R

pytestmark = pytest.mark.gpu

LAW_NAMES = ("RNPBond", "PMBBond", "PDElasticBond", "PDState")


def _model(sc, prec):
    from peridem_b200.model import GpuDEMModel
    return GpuDEMModel(sc, precision=prec, build_neighbors=True, compute_mx=True)


def _evaluate(sc, prec, u, bonds):
    m = _model(sc, prec)
    try:
        m.set_field("u", u)
        m.set_field("bonds", bonds)
        m.compute_pd_forces()
        return m.field("f"), m.field("Z"), m.field("bonds"), m.pd_neighbors()
    finally:
        m.close()


def _compare(name, sc, u, bonds):
    from peridem_b200.model import PREC_FP64, PREC_MIXED
    fa, za, ba, (rp, _) = _evaluate(sc, PREC_FP64, u, bonds)
    fb, zb, bb, _ = _evaluate(sc, PREC_MIXED, u, bonds)
    active = np.zeros(sc.n_nodes, dtype=bool)
    for p in range(sc.n_particles):
        if sc.p_compute_force[p]:
            active[sc.p_start[p]:sc.p_end[p]] = True
    rp = rp.astype(np.int64)
    diff_bonds = np.nonzero(ba != bb)[0]
    owner = np.repeat(np.arange(sc.n_nodes), np.diff(rp))
    ok = active.copy()
    ok[owner[diff_bonds]] = False
    fmax = max(float(np.max(np.abs(fa[active]))), 1e-300)
    df = float(np.max(np.abs(fa[ok] - fb[ok]))) / fmax if ok.any() else 0.0
    zmax = max(1.0, float(np.max(za[active])))
    dz = float(np.max(np.abs(za[active] - zb[active]))) / zmax
    nbroken = int(np.sum(ba))
    print(f"{name}: nodes {int(active.sum())} bonds {len(ba)} broken {nbroken} "
          f"(pre-broken {int(np.sum(bonds))}) | f {df:.2e}  Z {dz:.2e}  bond states differ "
          f"{len(diff_bonds)}")
    assert fmax > 0, "no force to compare"
    assert df <= 1e-3, df
    assert dz <= 1e-3, dz
    assert len(diff_bonds) <= max(2, 1e-3 * nbroken), len(diff_bonds)


@pytest.mark.parametrize("case", sorted(CASES))
def test_mixed_force_on_fp64_trajectory_state(case):
    from peridem_b200.model import PREC_FP64
    fac, steps, _ = CASES[case]
    sc = scn.build_scene(fac())
    m = _model(sc, PREC_FP64)
    try:
        m.integrate_begin()
        m.integrate_step(steps)
        m.sync()
        u, bonds = m.field("u"), m.field("bonds")
    finally:
        m.close()
    _compare(case, sc, u, bonds)


def _smooth_u(sc, strain=2e-3, seed=0):
    rng = np.random.default_rng(seed)
    x = sc.xref
    span = float(np.max(np.ptp(x[:, :sc.dim], axis=0)))
    k = 2 * np.pi / span
    u = np.zeros_like(x)
    for q in range(sc.dim):
        ph = rng.uniform(0, 2 * np.pi, size=3)
        u[:, q] = strain / k * (np.sin(k * x[:, 0] + ph[0]) * np.cos(k * x[:, 1] + ph[1])
                                * (np.cos(k * x[:, 2] + ph[2]) if sc.dim == 3 else 1.0))
    return u


@pytest.mark.parametrize("strain", [2e-3, 3e-2])
@pytest.mark.parametrize("law", LAW_NAMES)
@pytest.mark.parametrize("dim", [2, 3])
def test_mixed_force_on_smooth_deformation(law, dim, strain):
    if dim == 2:
        spec = scn.two_particle(h_div=8, radius=R, material=law, v0=-1.0, gap=0.02 * R / 8, nt=10)
    else:
        spec = scn.column_3d(n_spheres=2, median_r=R, sigma=0.0, h_div=4, box=(3e-3, 3e-3, 6e-3),
                             seed=1, material=law, piston_speed=-2.0, nt=10)
    sc = scn.build_scene(spec)
    u = _smooth_u(sc, strain)
    from peridem_b200.model import PREC_FP64
    m = _model(sc, PREC_FP64)
    try:
        bonds = np.zeros(len(m.pd_neighbors()[1]), dtype=np.uint8)
    finally:
        m.close()
    # pre-break every 50th bond to exercise the broken-bond branch
    bonds[::50] = 1
    _compare(f"{law} {dim}-D strain {strain:g}", sc, u, bonds)
