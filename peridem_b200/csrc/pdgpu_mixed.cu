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

// Symmetric layout, pass 1: per node of a tile, how many of its bonds go to
// later nodes of the same tile (n_up) and how many leave the tile.
__global__ void k_sym_count(DevData d, const BondTile *tiles, const int32_t *node_tile, int64_t *n_up) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  const int32_t t = node_tile[i];
  if (t < 0) {
    n_up[i] = 0;
    d.sym_meta[i] = make_uint2(0u, 0u);
    return;
  }
  const int64_t nb = tiles[t].node_begin, ne = tiles[t].node_end;
  uint32_t up = 0, out = 0;
  for (int64_t k = d.pd_row[i]; k < d.pd_row[i + 1]; k++) {
    const int64_t j = d.pd_col[k];
    if (j >= nb && j < ne) up += j > i;
    else out++;
  }
  n_up[i] = up;
  d.sym_meta[i] = make_uint2(0u, up | ((up + out) << 16));
}

// Pass 2: slot bases (exclusive scan of n_up, relative to the tile's first
// node) and the reordered rows.  The slots of node i's bonds to later nodes
// follow its row order; the bond (j, i) of a later node j finds its slot as
// slot_base[i] + the rank of j among i's bonds to later nodes.
__global__ void k_sym_fill(DevData d, BondTile *tiles, const int32_t *node_tile, const int64_t *scan) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  const int32_t t = node_tile[i];
  if (t < 0) return;
  BondTile &T = tiles[t];
  const int64_t nb = T.node_begin, ne = T.node_end;
  const int64_t start = d.particles[T.particle].start;
  const uint2 m = d.sym_meta[i];
  const uint32_t n_up = m.y & 0xffffu, n_uo = m.y >> 16;
  const int64_t r0 = d.pd_row[i], r1 = d.pd_row[i + 1];
  int64_t e_up = r0, e_out = r0 + n_up, e_low = r0 + n_uo;
  for (int64_t k = r0; k < r1; k++) {
    const int64_t j = d.pd_col[k];
    const uint16_t pos = (uint16_t)(k - r0);
    if (j >= nb && j < ne && j > i) {
      d.sym_col[e_up] = (uint16_t)(j - start);
      d.sym_pos[e_up++] = pos;
    } else if (j < nb || j >= ne) {
      d.sym_col[e_out] = (uint16_t)(j - start);
      d.sym_pos[e_out++] = pos;
    } else {
      // rank of i among j's bonds to later nodes of the tile, in row order
      uint32_t rank = 0;
      for (int64_t q = d.pd_row[j]; q < d.pd_row[j + 1]; q++) {
        const int64_t c = d.pd_col[q];
        if (c == i) break;
        rank += (c > j && c < ne);
      }
      d.sym_col[e_low] = (uint16_t)(scan[j] - scan[nb] + rank);
      d.sym_pos[e_low++] = pos;
    }
  }
  d.sym_meta[i].x = (uint32_t)(scan[i] - scan[nb]);
  if (i == nb) {
    // the tile's slot count (written once per tile, by its first node)
    T.slots = (int32_t)(scan[ne] - scan[nb]);
  }
}

// The symmetric loop reads one broken bit per pair of tile nodes (node i's,
// for i < j); both directions must agree, as in every state the reference
// produces (a bond breaks from both ends at the same step).  Where a host
// uploaded only one direction as broken, the pair is made broken both ways.
__global__ void k_sym_bits(DevData d, const BondTile *tiles, const int32_t *node_tile) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  const int32_t t = node_tile[i];
  if (t < 0) return;
  const int64_t ne = tiles[t].node_end;
  for (int64_t k = d.pd_row[i]; k < d.pd_row[i + 1]; k++) {
    const int64_t j = d.pd_col[k];
    if (j <= i || j >= ne) continue;
    for (int64_t m = d.pd_row[j]; m < d.pd_row[j + 1]; m++)
      if (d.pd_col[m] == (int32_t)i) {
        const bool a = (d.bond_bits[k >> 5] >> (k & 31)) & 1u, b = (d.bond_bits[m >> 5] >> (m & 31)) & 1u;
        if (a != b) {
          atomicOr(d.bond_bits + (k >> 5), 1u << (k & 31));
          atomicOr(d.bond_bits + (m >> 5), 1u << (m & 31));
        }
        break;
      }
  }
}

__global__ void k_node_tiles(const BondTile *tiles, int n_tiles, int32_t *node_tile) {
  const int t = blockIdx.x;
  if (t >= n_tiles) return;
  for (int64_t i = tiles[t].node_begin + threadIdx.x; i < tiles[t].node_end; i += blockDim.x) node_tile[i] = t;
}

}  // namespace

void launch_sym_count(const DevData &d, const BondTile *tiles, const int32_t *node_tile, int64_t *n_up,
                      cudaStream_t s) {
  k_sym_count<<<(unsigned)((d.n_nodes + 255) / 256), 256, 0, s>>>(d, tiles, node_tile, n_up);
}

void launch_sym_fill(const DevData &d, BondTile *tiles, int n_tiles, const int32_t *node_tile,
                     const int64_t *scan, cudaStream_t s) {
  (void)n_tiles;
  k_sym_fill<<<(unsigned)((d.n_nodes + 255) / 256), 256, 0, s>>>(d, tiles, node_tile, scan);
}

void launch_sym_bits(const DevData &d, const BondTile *tiles, const int32_t *node_tile, cudaStream_t s) {
  k_sym_bits<<<(unsigned)((d.n_nodes + 255) / 256), 256, 0, s>>>(d, tiles, node_tile);
}

void launch_node_tiles(const BondTile *tiles, int n_tiles, int32_t *node_tile, cudaStream_t s) {
  if (n_tiles > 0) k_node_tiles<<<n_tiles, 256, 0, s>>>(tiles, n_tiles, node_tile);
}

void launch_tile_windows(const DevData &d, BondTile *tiles, int n_tiles, cudaStream_t s) {
  if (n_tiles > 0) k_tile_windows<<<n_tiles, 256, 0, s>>>(d, tiles);
}

void launch_mixed_setup(const DevData &d, cudaStream_t s) {
  k_mixed_setup<<<(unsigned)((d.n_nodes + 255) / 256), 256, 0, s>>>(d);
}

}  // namespace pdgpu
