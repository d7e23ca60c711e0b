// ORACLE TEST INFRASTRUCTURE ONLY: the reference's own quadrature-point
// strain and stress (fe::getCurrentQuadPoints and fe::getStrainStress,
// src/fe/meshUtil.cpp, as DEMModel::output calls them for the Strain_Stress
// tag, src/model/dem/demModel.cpp:2026-2072) on one finite-element mesh read
// from a binary file, so that tests can compare the GPU kernel with it.
//
//   ref_strain IN OUT
//
// IN  (little-endian): int64 dim, n_nodes, n_elem, n_vertex, vtk element
//     type, quadrature order, plane strain (0/1); double nu, lambda, mu;
//     double xref[n_nodes][3], u[n_nodes][3]; int64 conn[n_elem][n_vertex].
// OUT: int64 n_quad; double xq[n_quad][3], strain[n_quad][6],
//      stress[n_quad][6] (components xx, yy, zz, yz, xz, xy).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <utility>
#include <vector>
#include <fmt/format.h>

#include "inp/decks/meshDeck.h"
#include "util/matrix.h"
#include "util/point.h"

// fe::Mesh keeps its arrays private; the mesh is filled here directly
// instead of from a file (only this header is opened up)
#define private public
#define protected public
#include "fe/mesh.h"
#undef private
#undef protected
#include "fe/meshUtil.h"
#include "fe/tetElem.h"
#include "fe/triElem.h"
#include "util/feElementDefs.h"
#include "util/matrix.h"
#include "util/parallelUtil.h"
#include "util/point.h"

namespace {

template <class T>
bool get(FILE *f, T *v, size_t n) {
  return std::fread(v, sizeof(T), n, f) == n;
}

template <class T>
bool put(FILE *f, const T *v, size_t n) {
  return std::fwrite(v, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: ref_strain IN OUT\n");
    return 2;
  }
  FILE *in = std::fopen(argv[1], "rb");
  if (!in) return 3;
  int64_t hdr[7];
  double mat[3];
  if (!get(in, hdr, 7) || !get(in, mat, 3)) return 4;
  const int64_t dim = hdr[0], nn = hdr[1], ne = hdr[2], nv = hdr[3], etype = hdr[4], order = hdr[5];
  const bool plane_strain = hdr[6] != 0;
  std::vector<double> xr((size_t)nn * 3), uu((size_t)nn * 3);
  std::vector<int64_t> conn((size_t)(ne * nv));
  if (!get(in, xr.data(), xr.size()) || !get(in, uu.data(), uu.size()) || !get(in, conn.data(), conn.size()))
    return 5;
  std::fclose(in);

  util::parallel::initNThreads(1);  // the reference's loops run on its taskflow executor
  fe::Mesh mesh((size_t)dim);
  mesh.d_numNodes = (size_t)nn;
  mesh.d_numElems = (size_t)ne;
  mesh.d_eType = (size_t)etype;
  mesh.d_eNumVertex = (size_t)nv;
  mesh.d_nodes.resize((size_t)nn);
  std::vector<util::Point> xref((size_t)nn), u((size_t)nn);
  for (int64_t i = 0; i < nn; i++) {
    xref[i] = util::Point(xr[3 * i], xr[3 * i + 1], xr[3 * i + 2]);
    u[i] = util::Point(uu[3 * i], uu[3 * i + 1], uu[3 * i + 2]);
    mesh.d_nodes[i] = xref[i];
  }
  mesh.d_enc.assign(conn.begin(), conn.end());

  size_t per = 0;
  if (etype == util::vtk_type_triangle) per = fe::TriElem(order).getNumQuadPoints();
  else if (etype == util::vtk_type_tetra) per = fe::TetElem(order).getNumQuadPoints();
  else return 6;
  const size_t nq = per * (size_t)ne;
  std::vector<util::Point> xq(nq);
  std::vector<util::SymMatrix3> strain(nq), stress(nq);
  fe::getCurrentQuadPoints(&mesh, xref, u, xq, 0, 0, (size_t)order);
  fe::getStrainStress(&mesh, xref, u, plane_strain, strain, stress, 0, 0, mat[0], mat[1], mat[2], true,
                      (size_t)order);

  FILE *out = std::fopen(argv[2], "wb");
  if (!out) return 7;
  const int64_t n = (int64_t)nq;
  bool ok = put(out, &n, 1);
  for (size_t q = 0; q < nq && ok; q++) {
    const double p[3] = {xq[q].d_x, xq[q].d_y, xq[q].d_z};
    ok = put(out, p, 3);
  }
  for (auto *v : {&strain, &stress})
    for (size_t q = 0; q < nq && ok; q++) {
      double m[6];
      (*v)[q].copy(m);
      ok = put(out, m, 6);
    }
  std::fclose(out);
  return ok ? 0 : 8;
}
