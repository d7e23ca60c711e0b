"""Comparison of the FP64 CUDA path with the reference's own state dumps
(live runs of oracle/_ref/peridem_ref or the golden fixtures it wrote).

Tolerances, each stated where it is asserted:

* forces f: max|f_gpu - f_ref| <= F_TOL_STEP * max|f_ref| after the
  integrate() prelude and the first step (same state on both sides; the only
  differences are the order of the per-node sums and RNP's exp()), and
  <= F_TOL * max|f_ref| at later steps, where those last-bit differences
  have fed back through hundreds of contact steps (largest seen: 1.4e-11,
  PD state with the Gaussian influence function after 300 steps);
* u, v, x to KIN_TOL normwise;
* bond-broken flags and contact candidate sets: identical;
* contact-search control (update interval, counter, radius): identical;
* damage Z to Z_TOL relative (the reference's running max uses its own
  relative-epsilon comparison, so it can stop up to 1e-5 below the maximum);
* compressive-test reaction to 1e-12 relative; two-particle test penetration
  and max y to PP_TOL relative to the particle size.
"""
import numpy as np

import refrun

F_TOL_STEP = 1e-12
F_TOL = 1e-10
KIN_TOL = 1e-10
Z_TOL = 2e-5
PP_TOL = 1e-10


def model(init, **kw):
    from peridem_b200.model import GpuDEMModel, PREC_FP64
    sc = refrun.scene_from_dump(init)
    kw.setdefault("precision", PREC_FP64)
    return sc, GpuDEMModel(sc, **kw)


def searching_nodes(init):
    """Nodes whose candidate lists the contact pass reads: those of non-wall,
    force-computing particles that are not fully constrained."""
    N = int(init["N"][0])
    out = []
    for p in range(int(init["Np"][0])):
        if init["p_type"][p] == 0 and init["p_computeForce"][p] and not init["p_allDofsConstrained"][p]:
            out.extend(range(int(init["p_globStart"][p]), int(init["p_globEnd"][p])))
    return [i for i in out if i < N]


def compare(tag, m, ref, init, n, f_tol=None):
    """Assert the GPU model's state equals the reference dump `ref` of step n."""
    N = int(init["N"][0])
    if f_tol is None:
        f_tol = F_TOL_STEP if n <= 1 else F_TOL
    f = m.field("f")
    fr = ref["f"].reshape(N, 3)
    ef = refrun.rel_err(f, fr)
    eu = refrun.rel_err(m.field("u"), ref["u"].reshape(N, 3), floor=1e-30)
    ev = refrun.rel_err(m.field("v"), ref["v"].reshape(N, 3), floor=1e-30)
    ex = refrun.rel_err(m.field("x") - init["xRef"].reshape(N, 3),
                        ref["x"].reshape(N, 3) - init["xRef"].reshape(N, 3), floor=1e-30)
    bonds = m.field("bonds")
    nb = int(np.sum(bonds != ref["bond_state"]))
    z = m.field("Z")
    zr = ref["Z"]
    ez = float(np.max(np.abs(z - zr) / np.maximum(np.abs(zr), 1e-6))) if zr.size else 0.0
    msg = f"{tag}: f {ef:.2e} (tol {f_tol:.0e}) u {eu:.2e} v {ev:.2e} x {ex:.2e} bonds-diff {nb} Z {ez:.2e}"
    print(msg)
    assert nb == 0, msg
    assert ef <= f_tol, msg
    assert eu <= KIN_TOL and ev <= KIN_TOL and ex <= KIN_TOL, msg
    assert ez <= Z_TOL, msg
    sc = m.scalars()
    if int(init["is_multi"][0]):
        assert sc["contact_update_interval"] == int(ref["contNeighUpdateInterval"][0]), (tag, sc)
        assert sc["contact_counter"] == int(ref["contNeighTimestepCounter"][0]), (tag, sc)
        assert sc["contact_search_radius"] == float(ref["contNeighSearchRadius"][0]), (tag, sc)
        rp, col = m.contact_lists()
        nodes = searching_nodes(init)
        got = refrun.csr_sets(rp, col, nodes)
        exp = refrun.csr_sets(ref["c_rowptr"], ref["c_col"], nodes)
        bad = [i for i in nodes if got[i] != exp[i]]
        assert not bad, f"{tag}: contact candidate sets differ at {len(bad)} nodes, e.g. {bad[:5]}"
    test, every = int(init["test"][0]), int(init["dtTestOut"][0])
    if test == 2 and n % every == 0:
        r = float(ref["reaction"][0])
        assert abs(sc["reaction"] - r) <= 1e-12 * max(1.0, abs(r)), (tag, sc["reaction"], r)
    if test == 1 and n >= every:
        # ppTwoParticleTest keeps the values of its last test-output step
        scale = float(np.max(init["p_boundR"]))
        for key in ("pen_dist", "max_y"):
            r = float(ref[key][0])
            assert abs(sc[key] - r) <= PP_TOL * max(abs(r), scale), (tag, key, sc[key], r)
