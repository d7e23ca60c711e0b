// Mesh size of every particle on the device: util::computeMeshSize
// (src/util/geom.cpp:578-604), which BaseParticle calls once per particle
// (baseParticle.cpp:146) and whose value sets the particle's horizon, its
// contact radius and the internal contact of broken bonds.
//
// The reference scans all ordered node pairs (i, j) of the particle, i-major,
// starting from guess = |x_start - x_start+1|, and takes a pair's distance
// as the new guess when util::isLess(distance, guess) (relative epsilon
// 1e-5).  The result is the last such record, which is not always the exact
// minimum distance.  Here the same chain is followed record by record: each
// pass finds, for every particle at once, the first pair in scan order after
// the particle's last record whose distance isLess than its guess (a
// minimum over scan keys, found in parallel over a cell list of the nodes);
// that pair is the next record.  Passes repeat until no particle finds one.
// Only pairs closer than a particle's current guess can be records, so the
// cell list needs cells no smaller than the largest starting guess.
//
// Compiled with --fmad=false: distances round as the reference's do.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pdgpu_internal.h"

namespace {

constexpr double kCompareEps = 1.0e-5;  // util::isLess (function.cpp:15-23)
constexpr int64_t kMaxCells = int64_t(1) << 26;

__host__ __device__ inline bool less_rel(double a, double b) {
  const double aa = a < 0 ? -a : a, bb = b < 0 ? -b : b;
  return (b - a) > ((aa < bb ? bb : aa) * kCompareEps);
}

__host__ __device__ inline double dist3(const double *x, int64_t i, int64_t j) {
  const double a = x[3 * i] - x[3 * j], b = x[3 * i + 1] - x[3 * j + 1], c = x[3 * i + 2] - x[3 * j + 2];
  return sqrt(a * a + b * b + c * c);
}

struct MsGrid {
  double lo[3];
  double inv_cell;
  int64_t dims[3];
};

__device__ inline int64_t cell_c(double v, const MsGrid &g, int q) {
  double c = floor((v - g.lo[q]) * g.inv_cell);
  if (c < 0.0) c = 0.0;
  if (c > (double)(g.dims[q] - 1)) c = (double)(g.dims[q] - 1);
  return (int64_t)c;
}

__global__ void k_ms_cells(const double *x, int64_t n, MsGrid g, int32_t *cell_of, int32_t *cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cell_c(x[3 * i], g, 0) + g.dims[0] * (cell_c(x[3 * i + 1], g, 1) + g.dims[1] * cell_c(x[3 * i + 2], g, 2));
  cell_of[i] = (int32_t)c;
  atomicAdd(cnt + c, 1);
}

__global__ void k_ms_scatter(int64_t n, const int32_t *cell_of, const int32_t *start, int32_t *fill, int32_t *nodes) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t c = cell_of[i];
  nodes[start[c] + atomicAdd(fill + c, 1)] = (int32_t)i;
}

// One pass: for node i of particle p, the smallest scan key (i - s) * n_p +
// (j - s) beyond the particle's last record whose distance isLess than the
// particle's guess.
__global__ void k_ms_pass(const double *x, const int32_t *pt, int64_t n, MsGrid g, const int32_t *cstart,
                          const int32_t *cnodes, const int64_t *pstart, const int64_t *pend, const double *guess,
                          const long long *pos, unsigned long long *best) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t p = pt[i];
  if (p < 0) return;
  const int64_t s = pstart[p], np = pend[p] - s;
  const double gp = guess[p];
  const long long last = pos[p];
  const int64_t row = (i - s) * np;
  if (row + np - 1 <= last) return;  // the whole row lies before the last record
  const int64_t cx = cell_c(x[3 * i], g, 0), cy = cell_c(x[3 * i + 1], g, 1), cz = cell_c(x[3 * i + 2], g, 2);
  unsigned long long mine = ~0ull;
  for (int64_t z = cz > 0 ? cz - 1 : 0; z <= cz + 1 && z < g.dims[2]; z++)
    for (int64_t y = cy > 0 ? cy - 1 : 0; y <= cy + 1 && y < g.dims[1]; y++)
      for (int64_t xx = cx > 0 ? cx - 1 : 0; xx <= cx + 1 && xx < g.dims[0]; xx++) {
        const int64_t c = xx + g.dims[0] * (y + g.dims[1] * z);
        for (int32_t a = cstart[c]; a < cstart[c + 1]; a++) {
          const int64_t j = cnodes[a];
          if (j == i || pt[j] != p) continue;
          const long long key = (long long)(row + (j - s));
          if (key <= last || (unsigned long long)key >= mine) continue;
          if (less_rel(dist3(x, i, j), gp)) mine = (unsigned long long)key;
        }
      }
  if (mine != ~0ull) atomicMin(best + p, mine);
}

}  // namespace

extern "C" PDGPU_API int pdgpu_mesh_size(int32_t device, const double *x, int64_t n_nodes,
                                         const int64_t *particle_start, const int64_t *particle_end,
                                         int64_t n_particles, double *h) {
  if (!x || !particle_start || !particle_end || !h || n_nodes <= 0 || n_particles <= 0) return PDGPU_ERR_ARG;
  if (n_nodes > INT32_MAX) return PDGPU_ERR_ARG;
  for (int64_t p = 0; p < n_particles; p++)
    if (particle_start[p] < 0 || particle_end[p] > n_nodes || particle_end[p] < particle_start[p])
      return PDGPU_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return PDGPU_ERR_NODEVICE;
  // starting guesses and the particle of every node (-1: a particle of
  // fewer than two nodes, whose mesh size is 0)
  std::vector<double> guess(n_particles, 0.0);
  std::vector<long long> pos(n_particles, -1);
  std::vector<int32_t> pt(n_nodes, -1);
  double gmax = 0.0;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t p = 0; p < n_particles; p++) {
    const int64_t s = particle_start[p], e = particle_end[p];
    if (e - s < 2) continue;
    guess[p] = dist3(x, s, s + 1);
    gmax = std::max(gmax, guess[p]);
    for (int64_t i = s; i < e; i++) {
      pt[i] = (int32_t)p;
      for (int q = 0; q < 3; q++) {
        lo[q] = std::min(lo[q], x[3 * i + q]);
        hi[q] = std::max(hi[q], x[3 * i + q]);
      }
    }
  }
  for (int64_t p = 0; p < n_particles; p++) h[p] = guess[p];
  if (!(gmax > 0.0)) return PDGPU_OK;
  if (!(std::isfinite(lo[0]) && std::isfinite(hi[0]))) return PDGPU_ERR_ARG;
  MsGrid g{};
  double cell = gmax * (1.0 + 1e-9);
  for (;;) {
    double cells = 1.0;
    for (int q = 0; q < 3; q++) cells *= std::floor((hi[q] - lo[q]) / cell) + 1.0;
    if (cells <= (double)kMaxCells) break;
    cell *= 1.25;
  }
  int64_t ncells = 1;
  for (int q = 0; q < 3; q++) {
    g.lo[q] = lo[q];
    g.dims[q] = (int64_t)std::floor((hi[q] - lo[q]) / cell) + 1;
    ncells *= g.dims[q];
  }
  g.inv_cell = 1.0 / cell;

  double *dx = nullptr, *dguess = nullptr;
  int32_t *dpt = nullptr, *cell_of = nullptr, *cnt = nullptr, *cstart = nullptr, *fill = nullptr, *cnodes = nullptr;
  int64_t *dps = nullptr, *dpe = nullptr;
  long long *dpos = nullptr;
  unsigned long long *dbest = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  int rc = PDGPU_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == PDGPU_OK) rc = (e == cudaErrorMemoryAllocation) ? PDGPU_ERR_NOMEM : PDGPU_ERR_CUDA;
    return rc == PDGPU_OK;
  };
  const unsigned gb = (unsigned)((n_nodes + 255) / 256);
  if (ok(cudaMalloc(&dx, 24 * (size_t)n_nodes)) && ok(cudaMalloc(&dpt, 4 * (size_t)n_nodes)) &&
      ok(cudaMalloc(&cell_of, 4 * (size_t)n_nodes)) && ok(cudaMalloc(&cnodes, 4 * (size_t)n_nodes)) &&
      ok(cudaMalloc(&cnt, 4 * (size_t)(ncells + 1))) && ok(cudaMalloc(&cstart, 4 * (size_t)(ncells + 1))) &&
      ok(cudaMalloc(&fill, 4 * (size_t)ncells)) && ok(cudaMalloc(&dps, 8 * (size_t)n_particles)) &&
      ok(cudaMalloc(&dpe, 8 * (size_t)n_particles)) && ok(cudaMalloc(&dguess, 8 * (size_t)n_particles)) &&
      ok(cudaMalloc(&dpos, 8 * (size_t)n_particles)) && ok(cudaMalloc(&dbest, 8 * (size_t)n_particles)) &&
      ok(cudaMemcpy(dx, x, 24 * (size_t)n_nodes, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(dpt, pt.data(), 4 * (size_t)n_nodes, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(dps, particle_start, 8 * (size_t)n_particles, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(dpe, particle_end, 8 * (size_t)n_particles, cudaMemcpyHostToDevice)) &&
      ok(cudaMemset(cnt, 0, 4 * (size_t)(ncells + 1))) && ok(cudaMemset(fill, 0, 4 * (size_t)ncells))) {
    // cell list (counting sort of the nodes by cell)
    k_ms_cells<<<gb, 256>>>(dx, n_nodes, g, cell_of, cnt);
    if (ok(cudaGetLastError()) &&
        ok(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, cstart, (int)(ncells + 1))) &&
        ok(cudaMalloc(&tmp, tmp_bytes)) &&
        ok(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, cstart, (int)(ncells + 1)))) {
      k_ms_scatter<<<gb, 256>>>(n_nodes, cell_of, cstart, fill, cnodes);
      ok(cudaGetLastError());
    }
    // record by record
    std::vector<unsigned long long> best(n_particles);
    for (int pass = 0; rc == PDGPU_OK; pass++) {
      if (!ok(cudaMemcpy(dguess, guess.data(), 8 * (size_t)n_particles, cudaMemcpyHostToDevice)) ||
          !ok(cudaMemcpy(dpos, pos.data(), 8 * (size_t)n_particles, cudaMemcpyHostToDevice)) ||
          !ok(cudaMemset(dbest, 0xff, 8 * (size_t)n_particles)))
        break;
      k_ms_pass<<<gb, 256>>>(dx, dpt, n_nodes, g, cstart, cnodes, dps, dpe, dguess, dpos, dbest);
      if (!ok(cudaGetLastError()) ||
          !ok(cudaMemcpy(best.data(), dbest, 8 * (size_t)n_particles, cudaMemcpyDeviceToHost)))
        break;
      bool changed = false;
      for (int64_t p = 0; p < n_particles; p++) {
        if (best[p] == ~0ull) continue;
        const int64_t s = particle_start[p], np = particle_end[p] - s;
        const int64_t i = s + (int64_t)(best[p] / (unsigned long long)np), j = s + (int64_t)(best[p] % (unsigned long long)np);
        guess[p] = dist3(x, i, j);
        pos[p] = (long long)best[p];
        changed = true;
      }
      if (!changed) break;
    }
  }
  cudaFree(dx);
  cudaFree(dpt);
  cudaFree(cell_of);
  cudaFree(cnodes);
  cudaFree(cnt);
  cudaFree(cstart);
  cudaFree(fill);
  cudaFree(dps);
  cudaFree(dpe);
  cudaFree(dguess);
  cudaFree(dpos);
  cudaFree(dbest);
  cudaFree(tmp);
  if (rc != PDGPU_OK) return rc;
  for (int64_t p = 0; p < n_particles; p++) h[p] = guess[p];
  return PDGPU_OK;
}
