// Strain and stress at the quadrature points of linear triangles: the
// Strain_Stress output of DEMModel::output (demModel.cpp:2026-2072), which
// calls fe::getCurrentQuadPoints and fe::getStrainStress (fe/meshUtil.cpp)
// on every particle's finite-element mesh.  One thread per element.
//
// The arithmetic follows the reference in its order (compiled without FMA
// contraction, as the reference's x86-64 build):
//   * J = [[x1 - x0, y1 - y0], [x2 - x0, y2 - y0]], detJ = J00 J11 - J01 J10,
//     dN/dx = (r0 J11 - r1 J01) / detJ, dN/dy = (-r0 J10 + r1 J00) / detJ for
//     the reference derivatives r = (-1, -1), (1, 0), (0, 1)
//     (fe::TriElem::getQuadDatas);
//   * the quadrature point's current position: (N0 x0 + N1 x1) + N2 x2 in x
//     and y, 0 in z, plus u_i N_i node by node;
//   * util::SymMatrix3 keeps 32-bit floats: each accumulation adds in double
//     and rounds to float; e_xx += u_x + dN/dx and e_yy += u_y + dN/dy as the
//     reference writes them, e_xy += 0.5 u_x dN/dy + 0.5 u_y dN/dx; plane
//     strain: e_zz = -nu (e_xx + e_yy) / (1 - nu) with the sum in float;
//     s_ii = lambda tr + 2 mu e_ii (tr summed in float), s_ij = 2 mu e_ij;
//     plane stress: s_zz = nu (s_xx + s_yy).
// The reference stores three entries per triangle whatever the rule
// (fe::BaseElem::getNumQuadPoints is the node count), so the entries past a
// rule's points are zero.

#include "pdgpu_internal.h"

namespace pdgpu {

namespace {

constexpr int kStrainBlock = 128;

__device__ __forceinline__ float acc(float s, double x) { return (float)((double)s + x); }

__global__ void __launch_bounds__(kStrainBlock)
    k_strain_tri(const double *__restrict__ xref, const double *__restrict__ u, int64_t n_elem,
                 const int64_t *__restrict__ conn, int nq, double p0x, double p0y, double p1x, double p1y,
                 double p2x, double p2y, const double *__restrict__ nu, const double *__restrict__ lam,
                 const double *__restrict__ mu, const uint8_t *__restrict__ plane_strain, double *__restrict__ xq,
                 double *__restrict__ strain, double *__restrict__ stress) {
  const int64_t e = (int64_t)blockIdx.x * kStrainBlock + threadIdx.x;
  if (e >= n_elem) return;
  double x[3][2], uu[3][2];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int64_t i = conn[3 * e + k];
    x[k][0] = xref[2 * i];
    x[k][1] = xref[2 * i + 1];
    uu[k][0] = u[2 * i];
    uu[k][1] = u[2 * i + 1];
  }
  const double J00 = x[1][0] - x[0][0], J01 = x[1][1] - x[0][1];
  const double J10 = x[2][0] - x[0][0], J11 = x[2][1] - x[0][1];
  const double det = J00 * J11 - J01 * J10;
  const double r[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
  double dn[3][2];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    dn[k][0] = (r[k][0] * J11 - r[k][1] * J01) / det;
    dn[k][1] = (-r[k][0] * J10 + r[k][1] * J00) / det;
  }
  // strain and stress are the same at every point of a linear triangle
  float s[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // xx, yy, zz, yz, xz, xy
#pragma unroll
  for (int k = 0; k < 3; k++) {
    s[0] = acc(s[0], uu[k][0] + dn[k][0]);
    s[1] = acc(s[1], uu[k][1] + dn[k][1]);
    s[5] = acc(s[5], 0.5 * uu[k][0] * dn[k][1] + 0.5 * uu[k][1] * dn[k][0]);
  }
  const double nu_e = nu[e], lam_e = lam[e], mu2 = 2.0 * mu[e];
  const bool ps = plane_strain[e] != 0;
  if (ps) s[2] = (float)(-nu_e * (double)(s[0] + s[1]) / (1.0 - nu_e));
  const double tr = (double)((s[0] + s[1]) + s[2]);
  float t[6];
  t[0] = (float)(lam_e * tr + mu2 * (double)s[0]);
  t[5] = (float)(mu2 * (double)s[5]);
  t[4] = (float)(mu2 * (double)s[4]);
  t[1] = (float)(lam_e * tr + mu2 * (double)s[1]);
  t[3] = (float)(mu2 * (double)s[3]);
  t[2] = (float)(lam_e * tr + mu2 * (double)s[2]);
  if (!ps) t[2] = (float)(nu_e * (double)(t[0] + t[1]));
  const double pts[3][2] = {{p0x, p0y}, {p1x, p1y}, {p2x, p2y}};
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int64_t o = 3 * e + q;
    double c[3] = {0.0, 0.0, 0.0};
    float sq[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, tq[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (q < nq) {
      const double px = pts[q][0], py = pts[q][1];
      const double N[3] = {1.0 - px - py, px, py};
      c[0] = N[0] * x[0][0] + N[1] * x[1][0] + N[2] * x[2][0];
      c[1] = N[0] * x[0][1] + N[1] * x[1][1] + N[2] * x[2][1];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        c[0] += uu[k][0] * N[k];
        c[1] += uu[k][1] * N[k];
        c[2] += 0.0 * N[k];  // u_z is zero in 2-D
      }
#pragma unroll
      for (int a = 0; a < 6; a++) {
        sq[a] = s[a];
        tq[a] = t[a];
      }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) xq[3 * o + a] = c[a];
#pragma unroll
    for (int a = 0; a < 6; a++) {
      strain[6 * o + a] = (double)sq[a];
      stress[6 * o + a] = (double)tq[a];
    }
  }
}

// Linear tetrahedra (3-D), the one-point rule (the centroid; the
// reference's only tetrahedron rule that fits the three entries it stores
// per element): J rows x_k - x_0 (k = 1..3), detJ by cofactors along the
// first row, J^-1 as the adjugate times 1/detJ (util::inv), dN/dx = J^-1 r
// (util::dot) for r = (-1, -1, -1), (1, 0, 0), (0, 1, 0), (0, 0, 1)
// (fe::TetElem::getQuadDatas); the position (((0 + N0 x0) + N1 x1) + N2 x2) +
// N3 x3 per component plus u_i N_i; strain per node i: xx, yy, xy, then zz,
// yz, xz; no plane-strain or plane-stress rule in 3-D.
__global__ void __launch_bounds__(kStrainBlock)
    k_strain_tet(const double *__restrict__ xref, const double *__restrict__ u, int64_t n_elem,
                 const int64_t *__restrict__ conn, const double *__restrict__ nu, const double *__restrict__ lam,
                 const double *__restrict__ mu, double *__restrict__ xq, double *__restrict__ strain,
                 double *__restrict__ stress) {
  const int64_t e = (int64_t)blockIdx.x * kStrainBlock + threadIdx.x;
  if (e >= n_elem) return;
  double x[4][3], uu[4][3];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int64_t i = conn[4 * e + k];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x[k][c] = xref[4 * i + c];
      uu[k][c] = u[4 * i + c];
    }
  }
  double m[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) m[r][c] = x[r + 1][c] - x[0][c];
  const double det = m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                     m[0][1] * (m[1][0] * m[2][2] - m[2][0] * m[1][2]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[2][0] * m[1][1]);
  const double di = 1. / det;
  double n[3][3];
  n[0][0] = di * (m[1][1] * m[2][2] - m[2][1] * m[1][2]);
  n[0][1] = -di * (m[0][1] * m[2][2] - m[2][1] * m[0][2]);
  n[0][2] = di * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
  n[1][0] = -di * (m[1][0] * m[2][2] - m[2][0] * m[1][2]);
  n[1][1] = di * (m[0][0] * m[2][2] - m[2][0] * m[0][2]);
  n[1][2] = -di * (m[0][0] * m[1][2] - m[1][0] * m[0][2]);
  n[2][0] = di * (m[1][0] * m[2][1] - m[2][0] * m[1][1]);
  n[2][1] = -di * (m[0][0] * m[2][1] - m[2][0] * m[0][1]);
  n[2][2] = di * (m[0][0] * m[1][1] - m[1][0] * m[0][1]);
  const double r[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  double dn[4][3];
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double v = 0.0;
#pragma unroll
      for (int b = 0; b < 3; b++) v += n[a][b] * r[k][b];
      dn[k][a] = v;
    }
  float s[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // xx, yy, zz, yz, xz, xy
#pragma unroll
  for (int k = 0; k < 4; k++) {
    s[0] = acc(s[0], uu[k][0] + dn[k][0]);
    s[1] = acc(s[1], uu[k][1] + dn[k][1]);
    s[5] = acc(s[5], 0.5 * uu[k][0] * dn[k][1] + 0.5 * uu[k][1] * dn[k][0]);
    s[2] = acc(s[2], uu[k][2] + dn[k][2]);
    s[3] = acc(s[3], 0.5 * uu[k][1] * dn[k][2] + 0.5 * uu[k][2] * dn[k][1]);
    s[4] = acc(s[4], 0.5 * uu[k][0] * dn[k][2] + 0.5 * uu[k][2] * dn[k][0]);
  }
  const double lam_e = lam[e], mu2 = 2.0 * mu[e];
  (void)nu;
  const double tr = (double)((s[0] + s[1]) + s[2]);
  float t[6];
  t[0] = (float)(lam_e * tr + mu2 * (double)s[0]);
  t[5] = (float)(mu2 * (double)s[5]);
  t[4] = (float)(mu2 * (double)s[4]);
  t[1] = (float)(lam_e * tr + mu2 * (double)s[1]);
  t[3] = (float)(mu2 * (double)s[3]);
  t[2] = (float)(lam_e * tr + mu2 * (double)s[2]);
  const double N[4] = {1. - 0.25 - 0.25 - 0.25, 0.25, 0.25, 0.25};
  double c[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double p = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) p += N[k] * x[k][a];
#pragma unroll
    for (int k = 0; k < 4; k++) p += uu[k][a] * N[k];
    c[a] = p;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int64_t o = 3 * e + q;
#pragma unroll
    for (int a = 0; a < 3; a++) xq[3 * o + a] = q == 0 ? c[a] : 0.0;
#pragma unroll
    for (int a = 0; a < 6; a++) {
      strain[6 * o + a] = q == 0 ? (double)s[a] : 0.0;
      stress[6 * o + a] = q == 0 ? (double)t[a] : 0.0;
    }
  }
}

}  // namespace

cudaError_t launch_strain_tet(const DevData &d, int64_t n_elem, const int64_t *conn, const double *nu,
                              const double *lam, const double *mu, double *xq, double *strain, double *stress,
                              cudaStream_t s) {
  if (n_elem <= 0) return cudaSuccess;
  const unsigned g = (unsigned)((n_elem + kStrainBlock - 1) / kStrainBlock);
  k_strain_tet<<<g, kStrainBlock, 0, s>>>(d.xref, d.u, n_elem, conn, nu, lam, mu, xq, strain, stress);
  return cudaGetLastError();
}

cudaError_t launch_strain_tri(const DevData &d, int64_t n_elem, const int64_t *conn, int nq, const double *pts,
                              const double *nu, const double *lam, const double *mu, const uint8_t *plane_strain,
                              double *xq, double *strain, double *stress, cudaStream_t s) {
  if (n_elem <= 0) return cudaSuccess;
  double p[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < nq && q < 3; q++) {
    p[2 * q] = pts[2 * q];
    p[2 * q + 1] = pts[2 * q + 1];
  }
  const unsigned g = (unsigned)((n_elem + kStrainBlock - 1) / kStrainBlock);
  k_strain_tri<<<g, kStrainBlock, 0, s>>>(d.xref, d.u, n_elem, conn, nq, p[0], p[1], p[2], p[3], p[4], p[5], nu, lam,
                                          mu, plane_strain, xq, strain, stress);
  return cudaGetLastError();
}

}  // namespace pdgpu
