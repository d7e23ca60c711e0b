"""The learned surrogate.

* gradients: one forward/backward pass of the trainer (tensor-core GEMMs and
  the pdgpu_sur_* kernels) against a NumPy FP64 oracle that applies the same
  BF16 roundings to the GEMM operands; max |g - g_oracle| <= 1e-2 max |g|.
* training: on held-out bond-loop samples, the network's force error is
  below that of the same reduced model without it (the bond loop's tangent
  on the modes alone): what the network gains.
* in the step, on deformed particles: the device chain judged against the
  bond loop on the first check step, with and without the network; the
  CUDA-core chain the step runs against the tensor-core GEMM chain.
* in the step, over a run: under load (repeated impacts on the moving
  wall) the wall's contact impulse of perturbed surrogate runs matches that
  of perturbed FP64 runs as an ensemble (impacts amplify any difference, a
  1e-9 one included, to O(1) within ~150 steps, so single runs are not
  comparable pointwise); on a loose packing the surrogate carries most
  particle-steps without changing the result.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(x):
    import torch
    return torch.as_tensor(np.asarray(x, dtype=np.float64)).to(torch.bfloat16).to(torch.float64).numpy()


def test_trainer_gradients_match_cpu_oracle():
    import torch
    from peridem_b200.surrogate import Trainer, RANK
    B = 64
    rng = np.random.default_rng(3)
    X = rng.standard_normal((B, RANK)).astype(np.float32)
    T = rng.standard_normal((B, RANK)).astype(np.float32)
    tr = Trainer(seed=5)
    Xd = torch.as_tensor(X, device="cuda").to(torch.bfloat16)
    Td = torch.as_tensor(T, device="cuda")
    Y, cache = tr.forward(Xd)
    loss, grads = tr.backward(Y, Td, cache)
    torch.cuda.synchronize()
    g = [x.cpu().numpy().astype(np.float64) for x in grads]
    W = [w.cpu().numpy().astype(np.float64) for w in tr.W]
    b = [x.cpu().numpy().astype(np.float64) for x in tr.b]
    # oracle
    Xb = _bf16(X)
    Wb = [_bf16(w) for w in W]
    H1 = np.tanh(Xb @ Wb[0].T + b[0]); H1b = _bf16(H1)
    H2 = np.tanh(H1b @ Wb[1].T + b[1]); H2b = _bf16(H2)
    Yo = H2b @ Wb[2].T + b[2]
    n = Yo.size
    dY = 2.0 / n * (Yo - T); dYb = _bf16(dY)
    dW3 = dYb.T @ H2b; db3 = dY.sum(0)
    dH2 = dYb @ Wb[2]; dZ2 = dH2 * (1 - H2 ** 2); dZ2b = _bf16(dZ2)
    dW2 = dZ2b.T @ H1b; db2 = dZ2.sum(0)
    dH1 = dZ2b @ Wb[1]; dZ1 = dH1 * (1 - H1 ** 2); dZ1b = _bf16(dZ1)
    dW1 = dZ1b.T @ Xb; db1 = dZ1.sum(0)
    ref = [dW1, dW2, dW3, db1, db2, db3]
    assert abs(float(loss.item()) - float(((Yo - T) ** 2).sum())) <= 1e-3 * float(((Yo - T) ** 2).sum())
    for name, a, r in zip(["dW1", "dW2", "dW3", "db1", "db2", "db3"], g, ref):
        e = np.max(np.abs(a - r)) / max(np.max(np.abs(r)), 1e-30)
        print(f"{name}: rel err {e:.2e}")
        assert a.shape == r.shape
        assert e <= 1e-2, name


def _scene(seed, n, gapf, sf=5.0, wall=-2.0):
    from peridem_b200 import scene as scn
    h = 1e-3 / 8
    return scn.build_scene(scn.compressive_2d(n_particles=n, r_range=(1e-3, 1.3e-3), h_div=8, width=10e-3,
                                              seed=seed, gap=gapf * h, wall_speed=wall, nt=40000,
                                              search_factor=sf))


_MODEL = {}


def _trained():
    """Trained on snapshots of a 16-particle compression (wall at 1 m/s)."""
    from peridem_b200 import surrogate as sg
    if "s" not in _MODEL:
        _MODEL["s"] = sg.build(_scene(4, 16, 1.02, wall=-1.0), steps=12000, every=40, iters=6000,
                               samples_per_particle=1200)
    return _MODEL["s"]


def test_training_beats_linear_reduced_model():
    s = _trained()
    for S in s.shapes:
        r = S.report
        print(S.zone, {k: round(v, 5) for k, v in r.items()})
        assert r["n_test_loaded"] > 0
        assert r["force_err_mlp"] < 0.05
        assert r["force_err_mlp"] < r["force_err_linear"]


def _run(sc, prec, steps, sur=None, near=True, chk=50):
    from peridem_b200.model import GpuDEMModel
    m = GpuDEMModel(sc, precision=prec, build_neighbors=True, compute_mx=True)
    try:
        if sur is not None:
            sur.attach(m, check_interval=chk, near_gate=near)
        m.integrate_begin()
        m.integrate_step(steps, graph_steps=1)
        m.sync()
        return m.history(), m.field("u"), (m.surrogate_stats() if sur is not None else None)
    finally:
        m.close()


def _deformed_packing(s):
    """A held-out packing whose every particle gets a deformation in its
    shape's modes with an RMS nodal displacement of 2e-7 of the reference
    mesh (peak bond stretch a few tenths of the critical stretch)."""
    from peridem_b200 import surrogate as sg
    sc = _scene(9, 12, 1.02)
    rng = np.random.default_rng(11)
    u = np.zeros((sc.n_nodes, 3))
    for S in s.shapes:
        for p in sg._zone_particles(sc, S.zone):
            c = rng.standard_normal(sg.RANK)
            c *= 2e-7 / np.linalg.norm(c)
            sg._place(sc, u, p, (S.phi @ c) * np.sqrt(S.n_nodes))
    return sc, u


def _check_step_errors(sc, u, model, chain="cuda"):
    """The first check step's comparison per particle (err2 rows of the
    particles the surrogate covers) and the largest damage Z."""
    from peridem_b200.model import GpuDEMModel, PREC_MIXED
    m = GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True)
    try:
        model.attach(m, check_interval=50, near_gate=False, chain=chain)
        # after integrate_begin (forces of the undeformed state): the first
        # step moves u by gravity alone, a rigid translation
        m.integrate_begin()
        m.set_field("u", u)
        m.integrate_step(1)
        m.sync()
        e = m.surrogate_errors()
        zmax = float(np.max(m.field("Z")))
    finally:
        m.close()
    return e[e[:, 1] > 0], zmax


def test_surrogate_chain_on_deformed_particles():
    """On the first step the bond loop runs for all particles and the
    surrogate's force is compared with it, per particle: the network beats
    the tangent part alone, inside the stretch gate."""
    import copy
    s = _trained()
    sc, u = _deformed_packing(s)
    linear = copy.deepcopy(s)
    for S in linear.shapes:   # the network's output is zero: the tangent part alone
        S.W[2] = np.zeros_like(S.W[2])
        S.b[2] = np.zeros_like(S.b[2])

    def errors(model):
        e, zmax = _check_step_errors(sc, u, model)
        assert zmax < 0.5, zmax   # inside the stretch gate
        return np.sqrt(e[:, 0] / e[:, 1])

    e_mlp, e_lin = errors(s), errors(linear)
    print(f"in-step relative force error per particle: network median {np.median(e_mlp):.4f} max "
          f"{e_mlp.max():.4f}; tangent alone median {np.median(e_lin):.4f} max {e_lin.max():.4f}")
    assert len(e_mlp) == len(e_lin) > 0
    assert e_mlp.max() < 0.05
    assert np.median(e_mlp) < np.median(e_lin)


def test_cuda_core_chain_matches_tensor_core_chain():
    """The step's CUDA-core chain (gather with projection, fused layers, lift
    with the scatter) against the tcgen05 GEMM chain the training uses, on
    the same deformed packing: both take BF16 operands with FP32
    accumulation and differ in summation order only.  Per particle, the
    difference of the two surrogate forces is bounded by the triangle
    inequality through their errors against the same bond-loop force:
    | |f_a - f| - |f_b - f| | <= 2e-3 |f|."""
    s = _trained()
    sc, u = _deformed_packing(s)
    ea, _ = _check_step_errors(sc, u, s, chain="cuda")
    eb, _ = _check_step_errors(sc, u, s, chain="tensor")
    assert len(ea) == len(eb) > 0
    np.testing.assert_array_equal(ea[:, 1], eb[:, 1])   # the same bond loop
    da, db, nf = np.sqrt(ea[:, 0]), np.sqrt(eb[:, 0]), np.sqrt(ea[:, 1])
    print(f"chain difference per particle, max |e_a - e_b| / |f| = {np.max(np.abs(da - db) / nf):.2e}; "
          f"errors against the bond loop {np.median(da / nf):.4f} / {np.median(db / nf):.4f}")
    assert np.all(np.abs(da - db) <= 2e-3 * nf)


def _impulse_ensemble(sc, prec, seeds, sur=None, steps=3000, at=1000):
    """Per seed: the run with v scaled by (1 + 1e-6 noise) at step `at`
    (seed 0: unperturbed); returns the wall's contact impulse (sum of the
    contact-reaction records), the number of non-zero records and, with the
    surrogate, its statistics of the unperturbed run."""
    from peridem_b200.model import GpuDEMModel
    imp, loaded, stats = [], [], None
    for seed in seeds:
        m = GpuDEMModel(sc, precision=prec, build_neighbors=True, compute_mx=True)
        try:
            if sur is not None:
                sur.attach(m, check_interval=50, near_gate=True)
            m.integrate_begin()
            m.integrate_step(at, graph_steps=50)
            m.sync()
            if seed:
                v = m.field("v")
                rng = np.random.default_rng(seed)
                m.set_field("v", v * (1.0 + 1e-6 * rng.standard_normal(v.shape)))
            m.integrate_step(steps - at, graph_steps=50)
            m.sync()
            h = m.history()
            imp.append(float(np.sum(h[:, 3])))
            loaded.append(int(np.sum(h[:, 3] != 0)))
            if sur is not None and seed == 0:
                stats = m.surrogate_stats()
        finally:
            m.close()
    return np.array(imp), loaded, stats


def test_gated_surrogate_keeps_the_wall_impulse():
    """Compression under load with the surrogate carrying part of it: 24
    particles (a column of about eight layers, lattice gaps 1.02 h), the
    wall at 2 m/s for 3000 steps, contact search radius equal to the contact
    radius (skin 1).  The particles fall onto the wall from step ~1270 on and
    keep striking it; particles with contact candidates stay on the bond
    loop, the rest on the surrogate.  Four runs each of FP64 and of
    mixed+surrogate, three of them with the velocities perturbed by 1e-6
    (relative) before the first impact: the mean contact impulse on the wall
    agrees within three standard errors (plus 5 % of the FP64 mean), and the
    surrogate carries at least a fifth of all particle-steps."""
    from peridem_b200.model import PREC_FP64, PREC_MIXED
    sc = _scene(7, 24, 1.02, sf=1.0)
    seeds = (0, 1, 2, 3)
    i64, l64, _ = _impulse_ensemble(sc, PREC_FP64, seeds)
    isur, lsur, st = _impulse_ensemble(sc, PREC_MIXED, seeds, sur=_trained())
    frac = st[2] / st[3]
    m64, msur = float(np.mean(i64)), float(np.mean(isur))
    se = float(np.sqrt((np.var(i64, ddof=1) + np.var(isur, ddof=1)) / len(seeds)))
    print(f"FP64 impulses {np.round(i64, 1)} (records with contact {l64}); surrogate {np.round(isur, 1)} "
          f"({lsur}); mean {m64:.4e} vs {msur:.4e}, standard error {se:.3e}; "
          f"particle-steps on the surrogate {st[2]}/{st[3]} ({frac:.3f})")
    assert min(l64) > 0 and min(lsur) > 0, "the wall never touched the packing"
    assert abs(msur - m64) <= 3.0 * se + 0.05 * abs(m64)
    assert st[3] == 3000 * st[1]
    assert frac >= 0.2, "the surrogate should carry the particles the load has not reached"


def test_surrogate_carries_a_loose_packing():
    """Loose packing (gaps 3 h, search radius 1.9 h, 8000 steps): most
    particle-steps run on the surrogate and the displacements stay within
    1e-3 of the mixed form without it."""
    from peridem_b200.model import PREC_MIXED
    sc = _scene(7, 12, 3.0, sf=2.0)
    _, ua, _ = _run(sc, PREC_MIXED, 8000)
    _, ub, st = _run(sc, PREC_MIXED, 8000, sur=_trained())
    frac = st[2] / st[3]
    du = float(np.max(np.abs(ua - ub))) / max(float(np.max(np.abs(ua))), 1e-300)
    print(f"particle-steps on the surrogate {st[2]}/{st[3]} ({frac:.3f}); displacement rel err {du:.2e}")
    assert frac > 0.9
    assert du <= 1e-3
