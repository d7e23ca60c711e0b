"""The learned surrogate of the bond loop (2-D, mixed-precision form).

Per zone whose particles share a reference mesh ("shape"), a particle's
displacement in its body frame, u_b = R(-orient) (u_i - u_centre) / scale, is
projected on 32 displacement modes, a = phi^T u_b.  Its body-frame force
density is the bond loop's tangent on the modes applied to a (exact for
small deformations in the span, and free of rigid rotation to first order)
plus the nonlinear residual that an MLP 32-256-256-32 (tanh) predicts from a,
in 32 residual force modes; the node force density is
f_i = fscale R(orient) f_b.  The per-particle force scale is the bond loop's
response to one fixed body-frame strain relative to that of the particle the
model was trained on, so particles of one shape but different sizes share
the network.

Training data come from the GPU solver itself: trajectory snapshots of a
running simulation give the displacement modes (leading singular vectors,
computed with torch on the GPU: data preparation), and bond-loop evaluations
on a probe context (pdgpu_compute_pd_forces) give the tangent (central
differences) and the forces of deformations sampled in the modes' span.  The
network is trained by the library's own kernels: forward and backward passes
on the tensor-core GEMM (pdgpu_tc_gemm), MSE gradient, tanh backward, bias
gradients, transposes and Adam (pdgpu_sur_*).  The same model with the
network left out (the tangent part alone) is the linear reduced model the
network is measured against.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import api

RANK = 32
HIDDEN = 256


# ---------------------------------------------------------------------------
# body frame
# ---------------------------------------------------------------------------
def surrogate_zones(sc) -> List[int]:
    """Zones of non-wall, force-computing particles that share one mesh size."""
    zones = []
    for z in sorted(set(int(v) for v in sc.p_zone)):
        sel = _zone_particles(sc, z)
        if sel and len({int(sc.p_end[p] - sc.p_start[p]) for p in sel}) == 1:
            zones.append(z)
    return zones


def _zone_particles(sc, z):
    return [p for p in range(sc.n_particles)
            if sc.p_zone[p] == z and sc.p_type[p] == 0 and sc.p_compute_force[p]]


def body_frame(sc, field_xyz: np.ndarray, p: int, relative: bool) -> np.ndarray:
    """R(-orient) (v_i - v_centre) / scale (relative) or R(-orient) v_i
    (forces) for the nodes of particle p, flattened as (x0, y0, x1, y1, ...)."""
    a, b = int(sc.p_start[p]), int(sc.p_end[p])
    v = field_xyz[a:b, :2].astype(np.float64)
    if relative:
        v = (v - field_xyz[int(sc.p_center[p]), :2]) / sc.p_scale[p]
    c, s = np.cos(sc.p_orient[p]), np.sin(sc.p_orient[p])
    out = np.empty_like(v)
    out[:, 0] = c * v[:, 0] + s * v[:, 1]
    out[:, 1] = -s * v[:, 0] + c * v[:, 1]
    return out.reshape(-1)


def _place(sc, u: np.ndarray, p: int, ub: np.ndarray) -> None:
    """u of particle p's nodes from body-frame rows: R(orient) ub scale."""
    a, b = int(sc.p_start[p]), int(sc.p_end[p])
    v = ub.reshape(-1, 2) * sc.p_scale[p]
    cs, sn = np.cos(sc.p_orient[p]), np.sin(sc.p_orient[p])
    u[a:b, 0] = cs * v[:, 0] - sn * v[:, 1]
    u[a:b, 1] = sn * v[:, 0] + cs * v[:, 1]


def reference_coords(sc, p: int) -> np.ndarray:
    """Body-frame reference coordinates of particle p's nodes (n x 2)."""
    return body_frame(sc, sc.xref, p, relative=True).reshape(-1, 2)


# ---------------------------------------------------------------------------
# bond-loop probes
# ---------------------------------------------------------------------------
def _probe(sc):
    from .model import GpuDEMModel, PREC_MIXED
    return GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True)


def calibration_norms(sc, zones: List[int], strain=(1e-4, -5e-5)) -> np.ndarray:
    """Per particle, the norm of the bond loop's body-frame force for one
    fixed body-frame strain (zero outside the zones).  A particle's force
    scale is its norm over the norm of the particle that defined the shape
    model (the first of its zone in the training scene)."""
    u = np.zeros((sc.n_nodes, 3))
    eps = np.diag(strain)
    for z in zones:
        for p in _zone_particles(sc, z):
            a, b = int(sc.p_start[p]), int(sc.p_end[p])
            d = sc.xref[a:b, :2] - sc.xref[int(sc.p_center[p]), :2]
            c, s = np.cos(sc.p_orient[p]), np.sin(sc.p_orient[p])
            R = np.array([[c, -s], [s, c]])
            u[a:b, :2] = d @ (R @ eps @ R.T).T
    m = _probe(sc)
    try:
        m.set_field("u", u)
        m.compute_pd_forces()
        f = m.field("f")
    finally:
        m.close()
    out = np.zeros(sc.n_particles)
    for z in zones:
        for p in _zone_particles(sc, z):
            out[p] = np.linalg.norm(body_frame(sc, f, p, relative=False))
    return out


def force_floor(sc, zones: List[int], strain: float = 1e-6) -> np.ndarray:
    """Per particle, the force norm of a uniform body-frame strain of
    ``strain``: the run-time gate compares the surrogate's error with
    max(|f|, floor)."""
    u = np.zeros((sc.n_nodes, 3))
    for z in zones:
        for p in _zone_particles(sc, z):
            a, b = int(sc.p_start[p]), int(sc.p_end[p])
            u[a:b, :2] = strain * (sc.xref[a:b, :2] - sc.xref[int(sc.p_center[p]), :2])
    m = _probe(sc)
    try:
        m.set_field("u", u)
        m.compute_pd_forces()
        f = m.field("f")
    finally:
        m.close()
    floor = np.zeros(sc.n_particles)
    for z in zones:
        for p in _zone_particles(sc, z):
            floor[p] = np.linalg.norm(body_frame(sc, f, p, relative=False))
    return floor


def tangent_modes(sc, z: int, phi: np.ndarray, fscale: np.ndarray, rms: float = 1e-9) -> np.ndarray:
    """The bond loop's tangent at zero deformation on the displacement modes:
    column k is the body-frame force (over fscale) of mode k per unit
    coefficient, by central differences of amplitude ``rms`` (RMS nodal
    displacement, in units of the reference mesh) on the zone's first
    particle.  Rigid rotation has zero tangent force, so this linear part is
    rotation-free to first order."""
    p0 = _zone_particles(sc, z)[0]
    n = phi.shape[0] // 2
    eps = rms * np.sqrt(n)
    m = _probe(sc)
    out = np.zeros_like(phi)
    try:
        intact = np.zeros(len(m.pd_neighbors()[1]), dtype=np.uint8)
        for k in range(phi.shape[1]):
            fk = []
            for sgn in (1.0, -1.0):
                u = np.zeros((sc.n_nodes, 3))
                _place(sc, u, p0, sgn * eps * phi[:, k])
                m.set_field("u", u)
                m.set_field("bonds", intact)
                m.compute_pd_forces()
                fk.append(body_frame(sc, m.field("f"), p0, relative=False) / fscale[p0])
            out[:, k] = (fk[0] - fk[1]) / (2.0 * eps)
    finally:
        m.close()
    return out


# ---------------------------------------------------------------------------
# snapshots and samples
# ---------------------------------------------------------------------------
@dataclass
class Snapshots:
    u: Dict[int, List[np.ndarray]] = field(default_factory=dict)  # zone -> body-frame u_b rows
    f: Dict[int, List[np.ndarray]] = field(default_factory=dict)  # zone -> body-frame f_b / fscale rows


def collect_snapshots(sc, steps: int, every: int, fscale: np.ndarray, zones: List[int],
                      z_max: float = 0.5) -> Snapshots:
    """Run the mixed-precision solver on ``sc`` for ``steps`` steps and, every
    ``every`` steps, record (u_b, f_b) of every particle whose damage is
    below z_max; f is the bond loop's force for that displacement and bond
    state, evaluated on a probe context.  The run stops early once a
    snapshot finds no particle below z_max: nothing later can be recorded,
    and a packing that far gone (broken bonds pressed together) is usually
    one whose step has become unstable, with a contact-list rebuild every
    step."""
    from .model import GpuDEMModel, PREC_MIXED
    run = GpuDEMModel(sc, precision=PREC_MIXED, build_neighbors=True, compute_mx=True)
    probe = _probe(sc)
    snap = Snapshots({z: [] for z in zones}, {z: [] for z in zones})
    try:
        run.integrate_begin()
        done = 0
        while done < steps:
            k = min(every, steps - done)
            run.integrate_step(k, graph_steps=1)
            done += k
            u = run.field("u")
            probe.set_field("u", u)
            probe.set_field("bonds", run.field("bonds"))
            probe.compute_pd_forces()
            f = probe.field("f")
            Z = probe.field("Z")
            kept = 0
            for z in zones:
                for p in _zone_particles(sc, z):
                    a, b = int(sc.p_start[p]), int(sc.p_end[p])
                    if float(Z[a:b].max()) >= z_max:
                        continue
                    snap.u[z].append(body_frame(sc, u, p, relative=True))
                    snap.f[z].append(body_frame(sc, f, p, relative=False) / fscale[p])
                    kept += 1
            if kept == 0:
                break
    finally:
        run.close()
        probe.close()
    return snap


def sample_in_span(sc, phi: Dict[int, np.ndarray], fscale: np.ndarray, zones: List[int], rounds: int,
                   seed: int = 0, z_max: float = 0.5, amp=(-7.0, -5.0)) -> Snapshots:
    """Bond-loop forces for deformations sampled in the span of each zone's
    displacement modes: every particle of the zones gets its own random
    direction and a log-uniform RMS nodal displacement 10^amp (in units of
    the reference mesh, ~1 mm across; the top of the band reaches a few
    tenths of the critical stretch), all evaluated by one probe call per
    round; samples whose damage reaches z_max are dropped."""
    rng = np.random.default_rng(seed)
    snap = Snapshots({z: [] for z in zones}, {z: [] for z in zones})
    m = _probe(sc)
    try:
        intact = np.zeros(len(m.pd_neighbors()[1]), dtype=np.uint8)
        for _ in range(rounds):
            u = np.zeros((sc.n_nodes, 3))
            rows = {}
            for z in zones:
                P = phi[z]
                for p in _zone_particles(sc, z):
                    c = rng.standard_normal(P.shape[1])
                    c *= 10.0 ** rng.uniform(*amp) / np.linalg.norm(c)
                    ub = (P @ c) * np.sqrt(P.shape[0] / 2)  # RMS node displacement ~ amplitude
                    rows[p] = ub
                    _place(sc, u, p, ub)
            m.set_field("u", u)
            m.set_field("bonds", intact)
            m.compute_pd_forces()
            f = m.field("f")
            Z = m.field("Z")
            for z in zones:
                for p in _zone_particles(sc, z):
                    a, b = int(sc.p_start[p]), int(sc.p_end[p])
                    if float(Z[a:b].max()) >= z_max:
                        continue
                    # body frame relative to the centre node, as at run time
                    ub = rows[p].reshape(-1, 2)
                    snap.u[z].append((ub - ub[int(sc.p_center[p]) - a]).reshape(-1))
                    snap.f[z].append(body_frame(sc, f, p, relative=False) / fscale[p])
    finally:
        m.close()
    return snap


def complete_basis(traj: Optional[np.ndarray], X: np.ndarray, rank: int = RANK) -> np.ndarray:
    """The trajectory modes first, then smooth polynomial displacement fields
    (x^i y^j e_k, i + j <= 6, lowest degree first) orthonormalised against
    them, up to ``rank`` columns."""
    cols = [] if traj is None else [traj[:, k] for k in range(traj.shape[1])]
    xs = X / max(np.abs(X).max(), 1e-300)
    cand = []
    for deg in range(0, 7):
        for i in range(deg + 1):
            mono = xs[:, 0] ** (deg - i) * xs[:, 1] ** i
            for comp in range(2):
                v = np.zeros((len(X), 2))
                v[:, comp] = mono
                cand.append(v.reshape(-1))
    basis = []
    for v in cols + cand:
        w = np.array(v, dtype=np.float64)
        for b in basis:
            w -= (b @ w) * b
        n = np.linalg.norm(w)
        if n > 1e-8 * max(np.linalg.norm(v), 1e-300):
            basis.append(w / n)
        if len(basis) == rank:
            break
    if len(basis) < rank:
        raise ValueError(f"cannot complete a rank-{rank} basis on {2 * len(X)} values")
    return np.stack(basis, axis=1)


def pod_basis(rows: np.ndarray, rank: int = RANK) -> np.ndarray:
    """Leading right singular vectors of the snapshot rows (K x rank)."""
    import torch
    X = torch.as_tensor(rows, dtype=torch.float64, device="cuda")
    _, _, Vh = torch.linalg.svd(X, full_matrices=False)
    return Vh[:rank].T.contiguous().cpu().numpy()


# ---------------------------------------------------------------------------
# training with the library's kernels
# ---------------------------------------------------------------------------
class Trainer:
    """MLP 32-256-256-32 (tanh, tanh, linear) trained with pdgpu_tc_gemm and
    the pdgpu_sur_* kernels; master weights FP32, GEMM operands BF16."""

    def __init__(self, seed: int = 0):
        import torch
        self.t = torch
        self.L = api.lib()
        g = torch.Generator(device="cpu").manual_seed(seed)
        dev = "cuda"

        def xavier(o, i):
            lim = (6.0 / (i + o)) ** 0.5
            return ((torch.rand(o, i, generator=g) * 2 - 1) * lim).to(dev)

        self.W = [xavier(HIDDEN, RANK), xavier(HIDDEN, HIDDEN), xavier(RANK, HIDDEN)]
        self.b = [torch.zeros(HIDDEN, device=dev), torch.zeros(HIDDEN, device=dev),
                  torch.zeros(RANK, device=dev)]
        self.params = self.W + self.b
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)

    def gemm(self, A, B, bias=None, act=0, out_f=True, out_b=False):
        """act(A B^T + bias) on the tensor cores (BF16 operands)."""
        t = self.t
        M, K = A.shape
        N = B.shape[0]
        Cf = t.empty(M, N, device="cuda") if out_f else None
        Cb = t.empty(M, N, device="cuda", dtype=t.bfloat16) if out_b else None
        rc = self.L.pdgpu_tc_gemm(A.data_ptr(), K, B.data_ptr(), K, M, N, K,
                                  bias.data_ptr() if bias is not None else None, act,
                                  Cf.data_ptr() if Cf is not None else None,
                                  Cb.data_ptr() if Cb is not None else None, N, self.err.data_ptr(), None)
        if rc != 0:
            raise RuntimeError(f"pdgpu_tc_gemm failed ({rc})")
        return Cf, Cb

    def transpose(self, X):
        out = self.t.empty(X.shape[1], X.shape[0], device="cuda", dtype=self.t.bfloat16)
        if self.L.pdgpu_sur_transpose(X.data_ptr(), X.shape[0], X.shape[1], out.data_ptr(), None):
            raise RuntimeError("pdgpu_sur_transpose failed")
        return out

    def forward(self, Xb):
        H1f, H1b = self.gemm(Xb, self.Wb[0], self.b[0], act=1, out_b=True)
        H2f, H2b = self.gemm(H1b, self.Wb[1], self.b[1], act=1, out_b=True)
        Y, _ = self.gemm(H2b, self.Wb[2], self.b[2], act=0)
        return Y, (Xb, H1f, H1b, H2f, H2b)

    def backward(self, Y, T, cache):
        """Gradients of mean((Y - T)^2); returns (sum of squares, [dW1, dW2,
        dW3, db1, db2, db3])."""
        t, L = self.t, self.L
        Xb, H1f, H1b, H2f, H2b = cache
        B = Y.shape[0]
        n = Y.numel()
        dY = t.empty_like(Y)
        dYb = t.empty(Y.shape, device="cuda", dtype=t.bfloat16)
        loss = t.zeros(1, dtype=t.float64, device="cuda")
        L.pdgpu_sur_mse_grad(Y.data_ptr(), T.data_ptr(), n, ctypes.c_float(2.0 / n), dY.data_ptr(),
                             dYb.data_ptr(), loss.data_ptr(), None)
        dW3, _ = self.gemm(self.transpose(dYb), self.transpose(H2b))      # 32 x 256
        db3 = t.empty(RANK, device="cuda")
        L.pdgpu_sur_colsum(dY.data_ptr(), B, RANK, db3.data_ptr(), None)
        dH2, _ = self.gemm(dYb, self.transpose(self.Wb[2]))               # B x 256
        dZ2 = t.empty_like(dH2)
        dZ2b = t.empty(dH2.shape, device="cuda", dtype=t.bfloat16)
        L.pdgpu_sur_tanh_back(dH2.data_ptr(), H2f.data_ptr(), dH2.numel(), dZ2.data_ptr(), dZ2b.data_ptr(), None)
        dW2, _ = self.gemm(self.transpose(dZ2b), self.transpose(H1b))     # 256 x 256
        db2 = t.empty(HIDDEN, device="cuda")
        L.pdgpu_sur_colsum(dZ2.data_ptr(), B, HIDDEN, db2.data_ptr(), None)
        dH1, _ = self.gemm(dZ2b, self.transpose(self.Wb[1]))              # B x 256
        dZ1 = t.empty_like(dH1)
        dZ1b = t.empty(dH1.shape, device="cuda", dtype=t.bfloat16)
        L.pdgpu_sur_tanh_back(dH1.data_ptr(), H1f.data_ptr(), dH1.numel(), dZ1.data_ptr(), dZ1b.data_ptr(), None)
        dW1, _ = self.gemm(self.transpose(dZ1b), self.transpose(Xb))      # 256 x 32
        db1 = t.empty(HIDDEN, device="cuda")
        L.pdgpu_sur_colsum(dZ1.data_ptr(), B, HIDDEN, db1.data_ptr(), None)
        return loss, [dW1, dW2, dW3, db1, db2, db3]

    def adam(self, grads, lr):
        self.step += 1
        for k, (p, m, v, g) in enumerate(zip(self.params, self.m, self.v, grads)):
            wb = self.Wb[k] if k < 3 else None
            self.L.pdgpu_sur_adam(p.data_ptr(), m.data_ptr(), v.data_ptr(), g.data_ptr(), p.numel(),
                                  ctypes.c_float(lr), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                  ctypes.c_float(1e-8), self.step,
                                  wb.data_ptr() if wb is not None else None, None)

    def fit(self, X: np.ndarray, T: np.ndarray, iters: int = 3000, batch: int = 4096, lr: float = 2e-3,
            seed: int = 0) -> List[float]:
        """Minibatch Adam with a cosine learning-rate schedule; returns the
        mean squared error every 200 iterations."""
        t = self.t
        Xd = t.as_tensor(X, dtype=t.float32, device="cuda").to(t.bfloat16)
        Td = t.as_tensor(T, dtype=t.float32, device="cuda")
        n = Xd.shape[0]
        batch = min(batch, n // 16 * 16)
        if batch < 16:
            raise ValueError(f"{n} training rows: too few to train")
        rng = t.Generator(device="cuda").manual_seed(seed)
        hist = []
        for it in range(iters):
            idx = t.randint(0, n, (batch,), device="cuda", generator=rng)
            Y, cache = self.forward(Xd[idx].contiguous())
            loss, grads = self.backward(Y, Td[idx].contiguous(), cache)
            self.adam(grads, lr * (0.5 * (1 + np.cos(np.pi * it / iters)) * 0.95 + 0.05))
            if it % 200 == 0 or it == iters - 1:
                hist.append(float(loss.item()) / (batch * RANK))
        if int(self.err.item()):
            raise RuntimeError("a tensor-core wait timed out during training")
        return hist

    def weights(self):
        return ([w.cpu().numpy().astype(np.float32) for w in self.W],
                [b.cpu().numpy().astype(np.float32) for b in self.b])


# ---------------------------------------------------------------------------
# the model of one shape
# ---------------------------------------------------------------------------
@dataclass
class ShapeModel:
    zone: int
    n_nodes: int
    phi: np.ndarray       # K x 32 displacement modes
    psi: np.ndarray       # K x 32 force modes of the nonlinear residual
    kphi: np.ndarray      # K x 32 tangent force of each displacement mode
    sx: np.ndarray        # 32: input coefficient scales
    sy: np.ndarray        # 32: output coefficient scales (folded into W[2], b[2])
    W: List[np.ndarray]
    b: List[np.ndarray]
    fref: float           # calibration norm of the particle with force scale 1
    report: Dict[str, float] = field(default_factory=dict)


def _bf(x):
    import torch
    return torch.as_tensor(np.asarray(x, dtype=np.float64)).to(torch.bfloat16).to(torch.float64).numpy()


def network(S: ShapeModel, X: np.ndarray) -> np.ndarray:
    """The network on scaled coefficients X, in FP64 on the BF16-rounded
    operands the device uses, minus its output at zero (as the device
    subtracts it)."""
    def run(x):
        h = np.tanh(_bf(x) @ _bf(S.W[0]).T + S.b[0])
        h = np.tanh(_bf(h) @ _bf(S.W[1]).T + S.b[1])
        return _bf(h) @ _bf(S.W[2]).T + S.b[2]
    return run(X) - run(np.zeros((1, X.shape[1])))


def predict_forces(S: ShapeModel, U: np.ndarray, with_network: bool = True) -> np.ndarray:
    """Body-frame forces (over fscale) of rows U: the tangent part
    kphi (phi^T u) plus, with the network, the lifted nonlinear residual."""
    a = U @ S.phi
    F = a @ S.kphi.T
    if with_network:
        F = F + network(S, a / S.sx) @ S.psi.T
    return F


def train_shape(z: int, U: np.ndarray, F: np.ndarray, phi: np.ndarray, kphi: np.ndarray, fref: float,
                iters: int = 3000, seed: int = 0, holdout: float = 0.1) -> ShapeModel:
    """Residual force modes, coefficient scales and network of one zone from
    sample rows U (displacements in the span of ``phi``) and F (forces over
    fscale).  The network learns what the tangent part misses (the material
    and geometric nonlinearity); the report gives held-out relative force
    errors with and without the network, and of the projection alone."""
    rng = np.random.default_rng(seed)
    n = len(U)
    perm = rng.permutation(n)
    n_test = max(1, int(holdout * n))
    test, train = perm[:n_test], perm[n_test:]
    a = U @ phi
    Rf = F - a @ kphi.T                       # nonlinear residual
    psi = pod_basis(Rf[train])
    bcoef = Rf @ psi
    sx = a[train].std(axis=0) + 1e-30
    sy = bcoef[train].std(axis=0) + 1e-30
    tr = Trainer(seed)
    hist = tr.fit(a[train] / sx, bcoef[train] / sy, iters=iters, seed=seed)
    W, b = tr.weights()
    W[2] = (W[2] * sy[:, None]).astype(np.float32)   # output in residual coefficients
    b[2] = (b[2] * sy).astype(np.float32)
    S = ShapeModel(z, U.shape[1] // 2, phi, psi, kphi, sx, sy, W, b, float(fref))
    loaded = test[np.linalg.norm(F[test], axis=1) > 0]

    def rel(Fp):
        return float(np.linalg.norm(Fp - F[loaded]) / np.linalg.norm(F[loaded])) if len(loaded) else 0.0

    S.report = {"n_train": float(len(train)), "n_test": float(n_test), "n_test_loaded": float(len(loaded)),
                "loss_first": hist[0], "loss_last": hist[-1],
                "force_err_mlp": rel(predict_forces(S, U[loaded])),
                "force_err_linear": rel(predict_forces(S, U[loaded], with_network=False)),
                "force_err_projection": rel(a[loaded] @ kphi.T + (Rf[loaded] @ psi) @ psi.T)}
    return S


@dataclass
class Surrogate:
    shapes: List[ShapeModel]

    def scales(self, sc):
        """Per-particle force scale and gate floor of the scene ``sc``."""
        zones = [S.zone for S in self.shapes]
        norms = calibration_norms(sc, zones)
        fscale = np.ones(sc.n_particles)
        for S in self.shapes:
            for p in _zone_particles(sc, S.zone):
                fscale[p] = norms[p] / S.fref
        return fscale, force_floor(sc, zones)

    def attach(self, model, check_interval: int = 50, z_gate: float = 0.5, err_gate: float = 0.05,
               near_gate: bool = True, chain: str = "cuda") -> None:
        """Install on a GpuDEMModel (mixed precision, before integrate_begin):
        per shape the projection phi^T / sx, the three layers and the lift
        [psi, kphi sx] of [network output, scaled coefficients].  With
        ``near_gate`` particles with contact candidates stay on the bond loop.
        ``chain``: "cuda" runs the chain on CUDA cores (four launches per
        step), "tensor" on the tcgen05 GEMMs (the training kernels)."""
        if chain not in ("cuda", "tensor"):
            raise ValueError(f"chain {chain!r}: 'cuda' or 'tensor'")
        model._check(model.lib.pdgpu_set_surrogate_chain(model.ctx, 0 if chain == "cuda" else 1))
        sc = model.scene
        fscale, floor = self.scales(sc)
        keep = []
        arr = (api.SurShape * len(self.shapes))()
        fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        for k, S in enumerate(self.shapes):
            phi_t = np.ascontiguousarray((S.phi / S.sx).T, dtype=np.float32)                        # 32 x K
            lift = np.ascontiguousarray(np.hstack([S.psi, S.kphi * S.sx[None, :]]), dtype=np.float32)  # K x 64
            mats = [phi_t, lift] + [np.ascontiguousarray(w, dtype=np.float32) for w in S.W] + \
                   [np.ascontiguousarray(v, dtype=np.float32) for v in S.b]
            keep += mats
            arr[k].zone, arr[k].n_nodes = S.zone, S.n_nodes
            arr[k].phi_t, arr[k].psi = fp(mats[0]), fp(mats[1])
            arr[k].w1, arr[k].w2, arr[k].w3 = fp(mats[2]), fp(mats[3]), fp(mats[4])
            arr[k].b1, arr[k].b2, arr[k].b3 = fp(mats[5]), fp(mats[6]), fp(mats[7])
        vals = [np.ascontiguousarray(v, dtype=np.float64) for v in (fscale, floor, sc.p_orient, sc.p_scale)]
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        model._check(model.lib.pdgpu_set_surrogate(model.ctx, len(self.shapes), ctypes.cast(arr, ctypes.c_void_p),
                                                   *(dp(v) for v in vals), check_interval, z_gate, err_gate,
                                                   1 if near_gate else 0))
        model._sur_keep = keep + vals

    def save(self, path: str) -> None:
        d = {}
        for k, S in enumerate(self.shapes):
            d[f"s{k}_meta"] = np.array([S.zone, S.n_nodes])
            d[f"s{k}_fref"] = np.array([S.fref])
            for name in ("phi", "psi", "kphi", "sx", "sy"):
                d[f"s{k}_{name}"] = getattr(S, name)
            for i in range(3):
                d[f"s{k}_W{i}"] = S.W[i]
                d[f"s{k}_b{i}"] = S.b[i]
        np.savez_compressed(path, **d)


def build(sc, steps: int = 20000, every: int = 100, iters: int = 3000, seed: int = 0,
          samples_per_particle: int = 40) -> Surrogate:
    """Train on the scene ``sc``: collect trajectory snapshots of the mixed
    solver, learn the displacement modes from them (unit-normalised rows,
    completed by polynomial fields), take the bond loop's tangent on the
    modes, sample bond-loop forces in their span and fit the residual force
    modes and networks.  Each model's report also gives the errors on the
    trajectory snapshots themselves (full space, not only the span)."""
    zones = surrogate_zones(sc)
    norms = calibration_norms(sc, zones)
    fref = {z: norms[_zone_particles(sc, z)[0]] for z in zones}
    fscale = np.ones(sc.n_particles)
    for z in zones:
        for p in _zone_particles(sc, z):
            fscale[p] = norms[p] / fref[z]
    snap = collect_snapshots(sc, steps, every, fscale, zones)
    phi, kphi = {}, {}
    for z in zones:
        U = np.array(snap.u[z])
        nrm = np.linalg.norm(U, axis=1) if len(U) else np.zeros(0)
        traj = pod_basis(U[nrm > 0] / nrm[nrm > 0, None]) if (nrm > 0).sum() >= 1 else None
        phi[z] = complete_basis(traj, reference_coords(sc, _zone_particles(sc, z)[0]))
        kphi[z] = tangent_modes(sc, z, phi[z], fscale)
    aug = sample_in_span(sc, phi, fscale, zones, rounds=samples_per_particle, seed=seed)
    shapes = []
    for z in zones:
        if len(aug.u[z]) < 32:
            raise ValueError(f"zone {z}: {len(aug.u[z])} samples below the damage gate "
                             f"(trajectory rows {len(snap.u[z])})")
        S = train_shape(z, np.array(aug.u[z]), np.array(aug.f[z]), phi[z], kphi[z], fref[z], iters=iters,
                        seed=seed)
        U = np.array(snap.u[z])
        F = np.array(snap.f[z])
        loaded = np.linalg.norm(F, axis=1) > 0 if len(F) else np.zeros(0, dtype=bool)
        if loaded.any():
            S.report["traj_loaded_rows"] = float(loaded.sum())
            for key, net in (("traj_force_err_mlp", True), ("traj_force_err_linear", False)):
                Fp = predict_forces(S, U[loaded], with_network=net)
                S.report[key] = float(np.linalg.norm(Fp - F[loaded]) / np.linalg.norm(F[loaded]))
        shapes.append(S)
    return Surrogate(shapes)


def load(path: str) -> Surrogate:
    d = np.load(path)
    shapes = []
    k = 0
    while f"s{k}_meta" in d:
        z, nn = (int(v) for v in d[f"s{k}_meta"])
        shapes.append(ShapeModel(z, nn, d[f"s{k}_phi"], d[f"s{k}_psi"], d[f"s{k}_kphi"], d[f"s{k}_sx"],
                                 d[f"s{k}_sy"], [d[f"s{k}_W{i}"] for i in range(3)],
                                 [d[f"s{k}_b{i}"] for i in range(3)], float(d[f"s{k}_fref"][0])))
        k += 1
    return Surrogate(shapes)
