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
    bonds = _prebroken(sc)
    _compare(f"{law} {dim}-D strain {strain:g}", sc, u, bonds)


def _prebroken(sc, every=50):
    """Every `every`-th bond broken, in both directions (as the reference's
    bonds break), to exercise the broken-bond branch."""
    from peridem_b200.model import PREC_FP64
    m = _model(sc, PREC_FP64)
    try:
        rp, col = m.pd_neighbors()
    finally:
        m.close()
    rp = rp.astype(np.int64)
    col = col.astype(np.int64)
    bonds = np.zeros(len(col), dtype=np.uint8)
    owner = np.repeat(np.arange(sc.n_nodes), np.diff(rp))
    for k in range(0, len(col), every):
        i, j = owner[k], col[k]
        bonds[k] = 1
        row = col[rp[j]:rp[j + 1]]
        bonds[rp[j] + int(np.nonzero(row == i)[0][0])] = 1
    return bonds


@pytest.mark.parametrize("law", LAW_NAMES)
def test_symmetric_bond_visits_match_per_node_visits(law):
    """The mixed 2-D loop's two schemes on the same state: bond states and
    damage identical (the same FP32 stretch from either end), forces equal
    up to FP32 rounding of the sums (1e-5 of the largest)."""
    from peridem_b200.model import GpuDEMModel, PREC_MIXED
    sc = scn.build_scene(scn.compressive_2d(n_particles=12, r_range=(R, 1.3 * R), h_div=10, width=10e-3,
                                            seed=4, material=law, nt=10))
    u = _smooth_u(sc, 2e-2, seed=3)
    bonds = _prebroken(sc, 37)
    out = []
    for scheme in (0, 1):
        m = GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True, bond_scheme=scheme)
        try:
            m.set_field("u", u)
            m.set_field("bonds", bonds)
            m.compute_pd_forces()
            out.append((m.bond_scheme(), m.field("f"), m.field("Z"), m.field("bonds")))
        finally:
            m.close()
    (s0, f0, z0, b0), (s1, f1, z1, b1) = out
    assert (s0, s1) == (0, 1), "the symmetric scheme should apply to this 2-D scene when asked"
    assert np.array_equal(b0, b1), int(np.sum(b0 != b1))
    assert np.array_equal(z0, z1), float(np.max(np.abs(z0 - z1)))
    fmax = float(np.max(np.abs(f1)))
    df = float(np.max(np.abs(f0 - f1))) / fmax
    print(f"{law}: broken {int(b0.sum())} (pre-broken {int(bonds.sum())}), f {df:.2e}")
    assert df <= 1e-5, df


def test_row_length_order_leaves_results_unchanged():
    """The per-node loop in node order (scheme 0, the default) against the
    row-length order (scheme 2): each node sums its own row in the same order
    either way, so 300 steps of a compression agree to the bit."""
    from peridem_b200.model import GpuDEMModel, PREC_MIXED
    sc = scn.build_scene(scn.compressive_2d(n_particles=12, r_range=(R, 1.3 * R), h_div=10, width=10e-3,
                                            seed=4, nt=10, wall_speed=-2.0))
    out = []
    for scheme in (0, 2):
        m = GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True, bond_scheme=scheme)
        try:
            m.integrate_begin()
            m.integrate_step(300, graph_steps=50)
            m.sync()
            out.append((m.bond_scheme(), m.field("f"), m.field("u"), m.field("Z"), m.field("bonds")))
        finally:
            m.close()
    assert (out[0][0], out[1][0]) == (0, 2)
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)
