// Peridynamic neighbour-list build that allocates nothing.
//
// Same sets as pdgpu_build_pd_neighbors (same particle, j != i, strict
// squared distance against horizon^2 in the kd-tree's arithmetic order; rows
// sorted by node index), for callers that cannot allocate device memory:
// hosts whose device memory is owned by another allocator (for example a
// framework's caching allocator that has reserved the GPU), or code paths in
// which cudaMalloc is not allowed.
//
// The call blocks the host: it waits for its stream three times (bounding
// box, grid-cell occupancy, neighbour count) and copies small results to
// host memory.  It therefore cannot run inside a stream capture; it checks
// for one on entry and returns PDGPU_ERR_STATE.  A host with a capture in
// progress on another stream must pass a non-default stream of its own
// (work on the legacy default stream would break that capture).
//
// All scratch lives in one file-scope device array (kScratchBytes, 16 MiB),
// which every GPU that loads this library keeps until the process exits.
// Its host-side name is only a stand-in: the device address is fetched once
// per device with cudaGetSymbolAddress (first call on that device, with it
// current) and passed to the kernels.  A cudaDeviceReset of that device can
// move the array, so the call must not be used on a device after it was
// reset in the same process.  Every call shares the array and overwrites
// what the last call left there; calls that overlap on the GPU (two streams,
// or two host threads on one device) race on it.
//
// This file is compiled with --fmad=false (the distance test must round like
// the reference's).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "pdgpu_internal.h"

namespace {

constexpr int64_t kMaxNodes = int64_t(1) << 18;   // 262 144 nodes
constexpr int64_t kMaxCells = int64_t(1) << 20;   // 1 048 576 grid cells
constexpr int kMaxRow = 1024;                     // neighbours of one node
constexpr int kMaxCellNodes = 8192;               // nodes of one grid cell
constexpr int kScanBlock = 1024;
constexpr int64_t kMaxScanBlocks = (kMaxCells + 1 + kScanBlock - 1) / kScanBlock + 1;

// scratch layout (bytes)
constexpr size_t kOffCellOf = 0;
constexpr size_t kOffCellTmp = kOffCellOf + 4 * kMaxNodes;
constexpr size_t kOffCellNodes = kOffCellTmp + 4 * kMaxNodes;
constexpr size_t kOffCellCnt = kOffCellNodes + 4 * kMaxNodes;
constexpr size_t kOffCellStart = kOffCellCnt + 4 * (kMaxCells + 1);
constexpr size_t kOffCellFill = kOffCellStart + 4 * (kMaxCells + 1);
constexpr size_t kOffBlock = ((kOffCellFill + 4 * kMaxCells + 255) / 256) * 256;
constexpr size_t kOffBox = kOffBlock + 8 * kMaxScanBlocks;
constexpr size_t kOffFlag = kOffBox + 8 * 8;     // int32: row overflow, largest cell, largest row
constexpr size_t kScratchUsed = kOffFlag + 64;
constexpr size_t kScratchBytes = size_t(16) << 20;
static_assert(kScratchUsed <= kScratchBytes, "scratch layout exceeds the static array");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct Scratch {
  int32_t *cell_of, *cell_tmp, *cell_nodes, *cell_cnt, *cell_start, *cell_fill;
  long long *block_sums;
  unsigned long long *box;  // 3 mins, 3 maxes (order-preserving encodings), horizon max
  int32_t *flag;            // [0] row-overflow flag, [1] largest cell count, [2] largest row
};

Scratch carve(unsigned char *base) {
  Scratch s;
  s.cell_of = reinterpret_cast<int32_t *>(base + kOffCellOf);
  s.cell_tmp = reinterpret_cast<int32_t *>(base + kOffCellTmp);
  s.cell_nodes = reinterpret_cast<int32_t *>(base + kOffCellNodes);
  s.cell_cnt = reinterpret_cast<int32_t *>(base + kOffCellCnt);
  s.cell_start = reinterpret_cast<int32_t *>(base + kOffCellStart);
  s.cell_fill = reinterpret_cast<int32_t *>(base + kOffCellFill);
  s.block_sums = reinterpret_cast<long long *>(base + kOffBlock);
  s.box = reinterpret_cast<unsigned long long *>(base + kOffBox);
  s.flag = reinterpret_cast<int32_t *>(base + kOffFlag);
  return s;
}

// doubles as unsigned integers that order like the doubles
__device__ __forceinline__ unsigned long long ord(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double unord(unsigned long long b) {
  const unsigned long long r = (b >> 63) ? (b & 0x7fffffffffffffffull) : ~b;
  double v;
  memcpy(&v, &r, 8);
  return v;
}

struct Grid3 {
  double lo[3];
  double inv_cell;
  int dims[3];
};

__global__ void k_box(const double *x, const uint32_t *pt, const double *hz, int64_t n, int dim,
                      Scratch s) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int q = 0; q < dim; q++) {
      atomicMin(s.box + q, ord(x[3 * i + q]));
      atomicMax(s.box + 3 + q, ord(x[3 * i + q]));
    }
    atomicMax(s.box + 6, ord(hz[pt[i]]));
  }
}

__device__ __forceinline__ int coord(double v, const Grid3 &g, int q) {
  double c = floor((v - g.lo[q]) * g.inv_cell);
  if (c < 0.0) c = 0.0;
  if (c > (double)(g.dims[q] - 1)) c = (double)(g.dims[q] - 1);
  return (int)c;
}

__global__ void k_count_cells(const double *x, int64_t n, int dim, Grid3 g, Scratch s) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = coord(x[3 * i], g, 0) + g.dims[0] * coord(x[3 * i + 1], g, 1);
  if (dim == 3) c += g.dims[0] * g.dims[1] * coord(x[3 * i + 2], g, 2);
  s.cell_of[i] = c;
  const int had = atomicAdd(s.cell_cnt + c, 1);
  atomicMax(s.flag + 1, had + 1);
}

// exclusive scan in three launches; block sums live in the scratch array
template <class T>
__global__ void k_scan_blocks(const T *in, int64_t n, long long *bsum) {
  __shared__ long long sh[32];
  const int64_t base = (int64_t)blockIdx.x * kScanBlock;
  long long v = 0;
  for (int64_t k = base + threadIdx.x; k < base + kScanBlock && k < n; k += blockDim.x) v += in[k];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    bsum[blockIdx.x] = t;
  }
}

__global__ void k_scan_sums(long long *bsum, int64_t nb) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    long long run = 0;
    for (int64_t b = 0; b < nb; b++) {
      const long long t = bsum[b];
      bsum[b] = run;
      run += t;
    }
    bsum[nb] = run;
  }
}

// out[k] = sum_{m<k} in[m] for k < n, out[n] = total (in may alias out)
template <class Tin, class Tout>
__global__ void k_scan_apply(const Tin *in, Tout *out, int64_t n, const long long *bsum) {
  __shared__ long long wsum[kScanBlock / 32];
  const int64_t k = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const long long v = k < n ? (long long)in[k] : 0;
  long long incl = v;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  long long woff = 0;
  for (int w = 0; w < warp; w++) woff += wsum[w];
  __syncthreads();
  if (k < n) out[k] = (Tout)(bsum[blockIdx.x] + woff + incl - v);
  if (k == n - 1) out[n] = (Tout)(bsum[blockIdx.x] + woff + incl);
}

__global__ void k_scatter(int64_t n, Scratch s) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = s.cell_of[i];
  s.cell_tmp[s.cell_start[c] + atomicAdd(s.cell_fill + c, 1)] = (int32_t)i;
}

__global__ void k_sort_cells(int64_t ncells, Scratch s) {
  const int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncells) return;
  const int b0 = s.cell_start[c], b1 = s.cell_start[c + 1];
  for (int a = b0 + lane; a < b1; a += 32) {
    const int32_t va = s.cell_tmp[a];
    int rank = 0;
    for (int b = b0; b < b1; b++) rank += s.cell_tmp[b] < va;
    s.cell_nodes[b0 + rank] = va;
  }
}

// one warp per node; COUNT writes row counts into rowptr[i], FILL writes
// the columns (in cell order; rows are sorted afterwards)
template <bool FILL>
__global__ void k_cand(const double *x, const uint32_t *pt, const double *hz, int64_t n, int dim,
                       Grid3 g, Scratch s, uint64_t *rowptr, uint32_t *col, int64_t cap) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const double q0 = x[3 * i], q1 = x[3 * i + 1], q2 = x[3 * i + 2];
  const uint32_t pi = pt[i];
  const double r = hz[pi];
  const double r2 = r * r;
  const int c0 = coord(q0, g, 0), c1 = coord(q1, g, 1), c2 = dim == 3 ? coord(q2, g, 2) : 0;
  int64_t out = FILL ? (int64_t)rowptr[i] : 0;
  const int64_t end = FILL ? (int64_t)rowptr[i + 1] : 0;
  long long count = 0;
  for (int cz = dim == 3 ? max(c2 - 1, 0) : 0; cz <= (dim == 3 ? min(c2 + 1, g.dims[2] - 1) : 0); cz++)
    for (int cy = max(c1 - 1, 0); cy <= min(c1 + 1, g.dims[1] - 1); cy++)
      for (int cx = max(c0 - 1, 0); cx <= min(c0 + 1, g.dims[0] - 1); cx++) {
        const int cell = cx + g.dims[0] * (cy + g.dims[1] * cz);
        const int b0 = s.cell_start[cell], b1 = s.cell_start[cell + 1];
        for (int base = b0; base < b1; base += 32) {
          const int a = base + lane;
          bool hit = false;
          int32_t j = -1;
          if (a < b1) {
            j = s.cell_nodes[a];
            if (j != i && pt[j] == pi) {
              // nanoflann's L2 order: query minus point, dims 0, 1, 2
              double dd = 0.0, df;
              df = q0 - x[3 * j];
              dd += df * df;
              df = q1 - x[3 * j + 1];
              dd += df * df;
              if (dim == 3) {
                df = q2 - x[3 * j + 2];
                dd += df * df;
              }
              hit = dd < r2;
            }
          }
          const unsigned bal = __ballot_sync(0xffffffffu, hit);
          if (FILL) {
            if (hit) {
              const int64_t at = out + __popc(bal & ((1u << lane) - 1u));
              if (at < end && at < cap) col[at] = (uint32_t)j;
            }
            out += __popc(bal);
          } else {
            count += __popc(bal);
          }
        }
      }
  if (!FILL && lane == 0) {
    rowptr[i] = (uint64_t)count;
    atomicMax(s.flag + 2, (int)(count < 0x7fffffff ? count : 0x7fffffff));
  }
}

// order each row by node index inside a per-warp shared-memory slice
__global__ void k_sort_rows(int64_t n, const uint64_t *rowptr, uint32_t *col, Scratch s) {
  __shared__ uint32_t buf[8][kMaxRow];
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (i >= n) return;
  const int64_t b0 = (int64_t)rowptr[i], len = (int64_t)rowptr[i + 1] - b0;
  if (len > kMaxRow) {
    if (lane == 0) atomicExch(s.flag, 1);
    return;
  }
  for (int a = lane; a < len; a += 32) buf[warp][a] = col[b0 + a];
  __syncwarp();
  for (int a = lane; a < len; a += 32) {
    const uint32_t va = buf[warp][a];
    int rank = 0;
    for (int b = 0; b < len; b++) rank += buf[warp][b] < va;
    col[b0 + rank] = va;
  }
}

// device address of the scratch array, fetched once per device
constexpr int kMaxDevices = 64;
unsigned char *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int say(char *err, size_t len, int code, const char *msg) {
  if (err && len) snprintf(err, len, "%s", msg);
  return code;
}

}  // namespace

extern "C" PDGPU_API int pdgpu_build_neighbors_noalloc(const double *x, const uint32_t *particle,
                                                      const double *horizon, int64_t n_nodes,
                                                      int32_t dim, uint64_t *rowptr,
                                                      uint32_t *col, int64_t col_capacity,
                                                      int64_t *n_bonds, void *stream, char *err,
                                                      size_t err_len) {
  char msg[256];
  if (!x || !particle || !horizon || !rowptr || !n_bonds || (dim != 2 && dim != 3) || n_nodes <= 0 ||
      col_capacity < 0)
    return say(err, err_len, PDGPU_ERR_ARG, "bad argument");
  if (n_nodes > kMaxNodes) {
    snprintf(msg, sizeof msg, "%lld nodes exceed the maximum of %lld for the allocation-free build",
             (long long)n_nodes, (long long)kMaxNodes);
    return say(err, err_len, PDGPU_ERR_ARG, msg);
  }
  cudaStream_t s = (cudaStream_t)stream;
  {
    // the call synchronises its stream, which no capture allows; on the
    // legacy default stream the query itself fails while another stream
    // captures in global mode
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      if (e != cudaSuccess) cudaGetLastError();
      return say(err, err_len, PDGPU_ERR_STATE,
                 "a stream capture is in progress: this call blocks the host and cannot be captured "
                 "(pass a non-default stream that is not capturing)");
    }
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return say(err, err_len, PDGPU_ERR_CUDA, "cudaGetDevice failed");
  unsigned char *base;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p) {
        snprintf(msg, sizeof msg, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return say(err, err_len, PDGPU_ERR_CUDA, msg);
      }
      g_scratch_ptr[dev] = (unsigned char *)p;
    }
    base = g_scratch_ptr[dev];
  }
  const Scratch sc = carve(base);
  auto ck = [&](cudaError_t e, const char *what) -> int {
    if (e == cudaSuccess) return PDGPU_OK;
    snprintf(msg, sizeof msg, "%s failed: %s", what, cudaGetErrorString(e));
    return say(err, err_len, PDGPU_ERR_CUDA, msg);
  };
  int rc;
  // bounding box and largest horizon (the previous call's values are reset)
  unsigned long long init[8] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
  if ((rc = ck(cudaMemcpyAsync(sc.box, init, sizeof init, cudaMemcpyHostToDevice, s), "box reset")))
    return rc;
  k_box<<<296, 256, 0, s>>>(x, particle, horizon, n_nodes, dim, sc);
  unsigned long long box[8];
  if ((rc = ck(cudaMemcpyAsync(box, sc.box, sizeof box, cudaMemcpyDeviceToHost, s), "box read")))
    return rc;
  if ((rc = ck(cudaStreamSynchronize(s), "box"))) return rc;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int q = 0; q < dim; q++) {
    lo[q] = unord(box[q]);
    hi[q] = unord(box[3 + q]);
  }
  for (int q = 0; q < dim; q++)
    if (!(hi[q] - lo[q] < 1e300)) return say(err, err_len, PDGPU_ERR_ARG, "coordinates must be finite");
  // cells a little wider than the largest horizon: a neighbour is never more
  // than one cell away, whatever the rounding of the cell index
  double cell = unord(box[6]) * (1.0 + 1e-6);
  if (!(cell > 0) || !(cell < 1e300)) return say(err, err_len, PDGPU_ERR_ARG, "horizons must be positive");
  Grid3 g{};
  int64_t ncells = 1;
  for (;;) {
    double cells = 1.0;
    for (int q = 0; q < dim; q++) cells *= std::floor((hi[q] - lo[q] + 2 * cell) / cell) + 1.0;
    if (cells <= (double)kMaxCells) break;
    cell *= 1.25;  // coarser cells keep the grid inside the scratch array
  }
  for (int q = 0; q < 3; q++) {
    g.lo[q] = q < dim ? lo[q] - cell : 0.0;
    g.dims[q] = q < dim ? (int)std::floor((hi[q] - lo[q] + 2 * cell) / cell) + 1 : 1;
    ncells *= g.dims[q];
  }
  g.inv_cell = 1.0 / cell;
  // cell list
  if ((rc = ck(cudaMemsetAsync(sc.cell_cnt, 0, 4 * (ncells + 1), s), "memset"))) return rc;
  if ((rc = ck(cudaMemsetAsync(sc.cell_fill, 0, 4 * ncells, s), "memset"))) return rc;
  if ((rc = ck(cudaMemsetAsync(sc.flag, 0, 16, s), "memset"))) return rc;
  const unsigned gn = (unsigned)((n_nodes + 255) / 256);
  k_count_cells<<<gn, 256, 0, s>>>(x, n_nodes, dim, g, sc);
  {
    // a grid made coarse to fit the scratch array can put most nodes in one
    // cell; the per-cell sort and the candidate scan are quadratic in a
    // cell's count, so such inputs are refused before those passes run
    int32_t big = 0;
    if ((rc = ck(cudaMemcpyAsync(&big, sc.flag + 1, 4, cudaMemcpyDeviceToHost, s), "cell read")))
      return rc;
    if ((rc = ck(cudaStreamSynchronize(s), "cells"))) return rc;
    if (big > kMaxCellNodes) {
      snprintf(msg, sizeof msg,
               "domain too large for the allocation-free grid: one cell holds %d nodes (at most %d)",
               big, kMaxCellNodes);
      return say(err, err_len, PDGPU_ERR_ARG, msg);
    }
  }
  // cell_start[c] = sum of counts below c; cell_start[ncells] = n_nodes
  const int64_t nb_c = (ncells + kScanBlock - 1) / kScanBlock;
  k_scan_blocks<int32_t><<<(unsigned)nb_c, 256, 0, s>>>(sc.cell_cnt, ncells, sc.block_sums);
  k_scan_sums<<<1, 32, 0, s>>>(sc.block_sums, nb_c);
  k_scan_apply<int32_t, int32_t><<<(unsigned)nb_c, kScanBlock, 0, s>>>(sc.cell_cnt, sc.cell_start,
                                                                      ncells, sc.block_sums);
  k_scatter<<<gn, 256, 0, s>>>(n_nodes, sc);
  k_sort_cells<<<(unsigned)((ncells * 32 + 255) / 256), 256, 0, s>>>(ncells, sc);
  // neighbour counts, offsets, columns
  const unsigned gw = (unsigned)((n_nodes * 32 + 255) / 256);
  k_cand<false><<<gw, 256, 0, s>>>(x, particle, horizon, n_nodes, dim, g, sc, rowptr, col,
                                   col_capacity);
  const int64_t nb_r = (n_nodes + kScanBlock - 1) / kScanBlock;
  k_scan_blocks<uint64_t><<<(unsigned)nb_r, 256, 0, s>>>(rowptr, n_nodes, sc.block_sums);
  k_scan_sums<<<1, 32, 0, s>>>(sc.block_sums, nb_r);
  k_scan_apply<uint64_t, uint64_t><<<(unsigned)nb_r, kScanBlock, 0, s>>>(rowptr, rowptr, n_nodes,
                                                                        sc.block_sums);
  uint64_t total = 0;
  int32_t longest = 0;
  if ((rc = ck(cudaMemcpyAsync(&total, rowptr + n_nodes, 8, cudaMemcpyDeviceToHost, s), "count read")))
    return rc;
  if ((rc = ck(cudaMemcpyAsync(&longest, sc.flag + 2, 4, cudaMemcpyDeviceToHost, s), "row read")))
    return rc;
  if ((rc = ck(cudaStreamSynchronize(s), "count"))) return rc;
  *n_bonds = (int64_t)total;
  if (longest > kMaxRow) {
    // rows are sorted in a per-warp shared-memory slice of kMaxRow entries;
    // the size query already refuses what the build could not sort
    snprintf(msg, sizeof msg, "a node has %d neighbours, more than the %d the allocation-free build sorts",
             longest, kMaxRow);
    return say(err, err_len, PDGPU_ERR_OVERFLOW, msg);
  }
  if (!col) return say(err, err_len, PDGPU_OK, "");  // size query
  if ((int64_t)total > col_capacity) {
    snprintf(msg, sizeof msg, "need room for %llu neighbours, col holds %lld",
             (unsigned long long)total, (long long)col_capacity);
    return say(err, err_len, PDGPU_ERR_OVERFLOW, msg);
  }
  k_cand<true><<<gw, 256, 0, s>>>(x, particle, horizon, n_nodes, dim, g, sc, rowptr, col,
                                  col_capacity);
  k_sort_rows<<<gw, 256, 0, s>>>(n_nodes, rowptr, col, sc);
  int32_t flag = 0;
  if ((rc = ck(cudaMemcpyAsync(&flag, sc.flag, 4, cudaMemcpyDeviceToHost, s), "flag read"))) return rc;
  if ((rc = ck(cudaStreamSynchronize(s), "build"))) return rc;
  if ((rc = ck(cudaGetLastError(), "kernel launch"))) return rc;
  if (flag) {
    snprintf(msg, sizeof msg, "a node has more than %d neighbours", kMaxRow);
    return say(err, err_len, PDGPU_ERR_OVERFLOW, msg);
  }
  return say(err, err_len, PDGPU_OK, "");
}
