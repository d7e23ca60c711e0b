"""ORACLE TEST INFRASTRUCTURE ONLY: NumPy restatement of the reference's
quadrature-point strain and stress for linear triangles, checked against the
reference itself (oracle/_ref/ref_strain, fixtures in tests/golden).

Follows fe::getCurrentQuadPoints and fe::getStrainStress
(src/fe/meshUtil.cpp:170-420) with fe::TriElem::getQuadDatas
(src/fe/triElem.cpp:60-95) in their evaluation order:

* per element, J = [[x1 - x0, y1 - y0], [x2 - x0, y2 - y0]],
  detJ = J00 J11 - J01 J10, shape derivatives
  dN/dx = (r0 J11 - r1 J01) / detJ, dN/dy = (-r0 J10 + r1 J00) / detJ with the
  reference derivatives r = (-1, -1), (1, 0), (0, 1);
* the quadrature point's current position (N0 x0 + N1 x1 + N2 x2) + sum u_i N_i;
* strain and stress are util::SymMatrix3, whose six entries are 32-bit
  floats: every accumulation adds in double and rounds to float
  (e_xx += u_x + dN/dx and e_yy += u_y + dN/dy, as the reference writes
  them; e_xy += 0.5 u_x dN/dy + 0.5 u_y dN/dx); plane strain sets
  e_zz = -nu (e_xx + e_yy) / (1 - nu) (the sum in float); stress
  s_ii = lambda tr + 2 mu e_ii, s_ij = 2 mu e_ij with the trace summed in
  float; plane stress sets s_zz = nu (s_xx + s_yy).
Components are stored (xx, yy, zz, yz, xz, xy).  The reference keeps three
entries per triangle whatever the rule (fe::BaseElem::getNumQuadPoints is
the node count), so a one-point rule leaves entries 1 and 2 zero.
"""
import numpy as np

F32 = np.float32


def _f(v):
    return np.asarray(v, dtype=np.float64).astype(F32)


def strain_stress_tri(xref, u, conn, points, nu, lam, mu, plane_strain):
    """xref, u [n, 3]; conn [m, 3]; points [nq <= 3, 2]; returns xq [3 m, 3],
    strain, stress [3 m, 6] (float64 holding float32 values)."""
    xref = np.asarray(xref, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    conn = np.asarray(conn, dtype=np.int64)
    m, nq = len(conn), len(points)
    x0, x1, x2 = (xref[conn[:, k]] for k in range(3))
    J00, J01 = x1[:, 0] - x0[:, 0], x1[:, 1] - x0[:, 1]
    J10, J11 = x2[:, 0] - x0[:, 0], x2[:, 1] - x0[:, 1]
    det = J00 * J11 - J01 * J10
    r = [(-1.0, -1.0), (1.0, 0.0), (0.0, 1.0)]
    d = [((r0 * J11 - r1 * J01) / det, (-r0 * J10 + r1 * J00) / det) for r0, r1 in r]
    assert nq <= 3
    xq = np.zeros((m, 3, 3))
    strain = np.zeros((m, 3, 6))
    stress = np.zeros((m, 3, 6))
    uu = [u[conn[:, k]] for k in range(3)]
    for q, (px, py) in enumerate(points):
        s = (1.0 - px - py, px, py)
        for c in range(3):
            # the reference maps x and y only; z stays the reference point's 0
            pos = s[0] * x0[:, c] + s[1] * x1[:, c] + s[2] * x2[:, c] if c < 2 else np.zeros(m)
            for k in range(3):
                pos = pos + uu[k][:, c] * s[k]
            xq[:, q, c] = pos
        e = np.zeros((m, 6), dtype=F32)
        for k in range(3):
            e[:, 0] = _f(e[:, 0].astype(np.float64) + (uu[k][:, 0] + d[k][0]))
            e[:, 1] = _f(e[:, 1].astype(np.float64) + (uu[k][:, 1] + d[k][1]))
            e[:, 5] = _f(e[:, 5].astype(np.float64) + (0.5 * uu[k][:, 0] * d[k][1] + 0.5 * uu[k][:, 1] * d[k][0]))
        nu_ = np.asarray(nu, dtype=np.float64)
        ps = np.asarray(plane_strain, dtype=bool)
        ezz = _f(-nu_ * (e[:, 0] + e[:, 1]).astype(np.float64) / (1.0 - nu_))
        e[:, 2] = np.where(ps, ezz, e[:, 2])
        tr = ((e[:, 0] + e[:, 1]) + e[:, 2]).astype(np.float64)   # float sums
        lam_ = np.asarray(lam, dtype=np.float64)
        mu2 = 2.0 * np.asarray(mu, dtype=np.float64)
        t = np.zeros((m, 6), dtype=F32)
        t[:, 0] = _f(lam_ * tr + mu2 * e[:, 0].astype(np.float64))
        t[:, 5] = _f(mu2 * e[:, 5].astype(np.float64))
        t[:, 4] = _f(mu2 * e[:, 4].astype(np.float64))
        t[:, 1] = _f(lam_ * tr + mu2 * e[:, 1].astype(np.float64))
        t[:, 3] = _f(mu2 * e[:, 3].astype(np.float64))
        t[:, 2] = _f(lam_ * tr + mu2 * e[:, 2].astype(np.float64))
        szz = _f(nu_ * (t[:, 0] + t[:, 1]).astype(np.float64))
        t[:, 2] = np.where(ps, t[:, 2], szz)
        strain[:, q] = e
        stress[:, q] = t
    return xq.reshape(m * 3, 3), strain.reshape(m * 3, 6), stress.reshape(m * 3, 6)


def strain_stress_tet(xref, u, conn, lam, mu):
    """Linear tetrahedra, one-point rule (fe::TetElem, src/fe/tetElem.cpp:
    J rows x_k - x_0, util::det by cofactors along the first row, util::inv
    as the adjugate times 1/det, util::dot for the derivatives; the position
    (((0 + N0 x0) + N1 x1) + N2 x2) + N3 x3 plus u_i N_i); strain terms per
    node xx, yy, xy, zz, yz, xz; three entries per element.  Returns xq
    [3 m, 3], strain, stress [3 m, 6]."""
    xref = np.asarray(xref, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    conn = np.asarray(conn, dtype=np.int64)
    m = len(conn)
    X = [xref[conn[:, k]] for k in range(4)]
    U = [u[conn[:, k]] for k in range(4)]
    M = [[X[r + 1][:, c] - X[0][:, c] for c in range(3)] for r in range(3)]
    det = (M[0][0] * (M[1][1] * M[2][2] - M[2][1] * M[1][2])
           - M[0][1] * (M[1][0] * M[2][2] - M[2][0] * M[1][2])
           + M[0][2] * (M[1][0] * M[2][1] - M[2][0] * M[1][1]))
    di = 1. / det
    n = [[None] * 3 for _ in range(3)]
    n[0][0] = di * (M[1][1] * M[2][2] - M[2][1] * M[1][2])
    n[0][1] = -di * (M[0][1] * M[2][2] - M[2][1] * M[0][2])
    n[0][2] = di * (M[0][1] * M[1][2] - M[1][1] * M[0][2])
    n[1][0] = -di * (M[1][0] * M[2][2] - M[2][0] * M[1][2])
    n[1][1] = di * (M[0][0] * M[2][2] - M[2][0] * M[0][2])
    n[1][2] = -di * (M[0][0] * M[1][2] - M[1][0] * M[0][2])
    n[2][0] = di * (M[1][0] * M[2][1] - M[2][0] * M[1][1])
    n[2][1] = -di * (M[0][0] * M[2][1] - M[2][0] * M[0][1])
    n[2][2] = di * (M[0][0] * M[1][1] - M[1][0] * M[0][1])
    r = [(-1.0, -1.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)]
    d = []
    for k in range(4):
        row = []
        for a in range(3):
            v = np.zeros(m)
            for b in range(3):
                v = v + n[a][b] * r[k][b]
            row.append(v)
        d.append(row)
    e = np.zeros((m, 6), dtype=F32)
    for k in range(4):
        ux, uy, uz = U[k][:, 0], U[k][:, 1], U[k][:, 2]
        e[:, 0] = _f(e[:, 0].astype(np.float64) + (ux + d[k][0]))
        e[:, 1] = _f(e[:, 1].astype(np.float64) + (uy + d[k][1]))
        e[:, 5] = _f(e[:, 5].astype(np.float64) + (0.5 * ux * d[k][1] + 0.5 * uy * d[k][0]))
        e[:, 2] = _f(e[:, 2].astype(np.float64) + (uz + d[k][2]))
        e[:, 3] = _f(e[:, 3].astype(np.float64) + (0.5 * uy * d[k][2] + 0.5 * uz * d[k][1]))
        e[:, 4] = _f(e[:, 4].astype(np.float64) + (0.5 * ux * d[k][2] + 0.5 * uz * d[k][0]))
    tr = ((e[:, 0] + e[:, 1]) + e[:, 2]).astype(np.float64)
    lam_ = np.asarray(lam, dtype=np.float64)
    mu2 = 2.0 * np.asarray(mu, dtype=np.float64)
    t = np.zeros((m, 6), dtype=F32)
    for a in (0, 1, 2):
        t[:, a] = _f(lam_ * tr + mu2 * e[:, a].astype(np.float64))
    for a in (3, 4, 5):
        t[:, a] = _f(mu2 * e[:, a].astype(np.float64))
    N = (1. - 0.25 - 0.25 - 0.25, 0.25, 0.25, 0.25)
    xq = np.zeros((m, 3, 3))
    strain = np.zeros((m, 3, 6))
    stress = np.zeros((m, 3, 6))
    for c in range(3):
        p = np.zeros(m)
        for k in range(4):
            p = p + N[k] * X[k][:, c]
        for k in range(4):
            p = p + U[k][:, c] * N[k]
        xq[:, 0, c] = p
    strain[:, 0] = e
    stress[:, 0] = t
    return xq.reshape(m * 3, 3), strain.reshape(m * 3, 6), stress.reshape(m * 3, 6)
