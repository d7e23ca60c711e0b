// Set-up kernels of the tiled bond loop: the neighbour window of every tile
// and the 16-bit particle-local neighbour offsets of the mixed form.
#include <climits>
#include <cstdint>

#include "pdgpu_internal.h"

namespace pdgpu {

namespace {

// window [min j, max j + 1) over the bonds of the tile's nodes, widened to
// include the tile's own nodes
__global__ void k_tile_windows(DevData d, BondTile *tiles) {
  __shared__ long long lo_s[32], hi_s[32];
  BondTile &T = tiles[blockIdx.x];
  long long lo = T.node_begin, hi = T.node_end - 1;
  for (int64_t i = T.node_begin; i < T.node_end; i++)
    for (int64_t k = d.pd_row[i] + threadIdx.x; k < d.pd_row[i + 1]; k += blockDim.x) {
      const long long j = d.pd_col[k];
      lo = j < lo ? j : lo;
      hi = j > hi ? j : hi;
    }
  for (int o = 16; o > 0; o >>= 1) {
    const long long a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    lo_s[threadIdx.x >> 5] = lo;
    hi_s[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      lo = lo_s[w] < lo ? lo_s[w] : lo;
      hi = hi_s[w] > hi ? hi_s[w] : hi;
    }
    T.win_begin = lo;
    T.win_end = hi + 1;
    T.bond_begin = d.pd_row[T.node_begin];
    T.bond_end = d.pd_row[T.node_end];
  }
}

__global__ void k_mixed_setup(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  const DevParticle &P = d.particles[d.ptid[i]];
  const int st = d.dim == 2 ? 2 : 4;
  float r[3] = {0.f, 0.f, 0.f};
  for (int q = 0; q < d.dim; q++) r[q] = (float)(d.xref[st * i + q] - d.xref[st * P.center + q]);
  d.xv_mixed[i] = make_float4(r[0], r[1], r[2], (float)d.vol[i]);
  if (!d.use16) return;
  for (int64_t k = d.pd_row[i]; k < d.pd_row[i + 1]; k++)
    d.pd_col16[k] = (uint16_t)(d.pd_col[k] - P.start);
}

}  // namespace

void launch_tile_windows(const DevData &d, BondTile *tiles, int n_tiles, cudaStream_t s) {
  if (n_tiles > 0) k_tile_windows<<<n_tiles, 256, 0, s>>>(d, tiles);
}

void launch_mixed_setup(const DevData &d, cudaStream_t s) {
  k_mixed_setup<<<(unsigned)((d.n_nodes + 255) / 256), 256, 0, s>>>(d);
}

}  // namespace pdgpu
