// Tiled bond loop, FP64 form (compiled with --fmad=false: the reference's arithmetic).
#define PDGPU_BONDS_FP64 1
#include "pdgpu_bonds.cuh"

namespace pdgpu {

namespace {
template <int DIM>
void pd_dim(const DevData &d, const BondTile *t, int n, int lanes, size_t smem, cudaStream_t s) {
  using namespace PDGPU_BONDS_NS;
  switch (lanes) {
    case 4: k_pd_tiled<DIM, 4><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 8: k_pd_tiled<DIM, 8><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 16: k_pd_tiled<DIM, 16><<<n, kTileThreads, smem, s>>>(d, t); break;
    default: k_pd_tiled<DIM, 32><<<n, kTileThreads, smem, s>>>(d, t); break;
  }
}
template <int DIM>
void pre_dim(const DevData &d, const BondTile *t, int n, int lanes, size_t smem, cudaStream_t s) {
  using namespace PDGPU_BONDS_NS;
  switch (lanes) {
    case 4: k_prepass_tiled<DIM, 4><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 8: k_prepass_tiled<DIM, 8><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 16: k_prepass_tiled<DIM, 16><<<n, kTileThreads, smem, s>>>(d, t); break;
    default: k_prepass_tiled<DIM, 32><<<n, kTileThreads, smem, s>>>(d, t); break;
  }
}
template <int DIM>
int set_limit(size_t bytes) {
  using namespace PDGPU_BONDS_NS;
  const void *fs[] = {(const void *)k_pd_tiled<DIM, 4>, (const void *)k_pd_tiled<DIM, 8>,
                      (const void *)k_pd_tiled<DIM, 16>, (const void *)k_pd_tiled<DIM, 32>,
                      (const void *)k_prepass_tiled<DIM, 4>, (const void *)k_prepass_tiled<DIM, 8>,
                      (const void *)k_prepass_tiled<DIM, 16>, (const void *)k_prepass_tiled<DIM, 32>};
  for (auto f : fs)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
      return -1;
  return 0;
}
}  // namespace

void launch_pd_tiled_fp64(const DevData &d, const BondTile *t, int n, int lanes, size_t smem,
                          cudaStream_t s) {
  if (n <= 0) return;
  if (d.dim == 2) pd_dim<2>(d, t, n, lanes, smem, s);
  else pd_dim<3>(d, t, n, lanes, smem, s);
}

void launch_prepass_tiled_fp64(const DevData &d, const BondTile *t, int n, int lanes, size_t smem,
                               cudaStream_t s) {
  if (n <= 0) return;
  if (d.dim == 2) pre_dim<2>(d, t, n, lanes, smem, s);
  else pre_dim<3>(d, t, n, lanes, smem, s);
}

size_t tile_smem_fp64(int dim, bool state, int64_t window) {
  return PDGPU_BONDS_NS::tile_smem_bytes(dim, state, (int)window);
}

int set_tile_smem_limit_fp64(int dim, size_t bytes) {
  return dim == 2 ? set_limit<2>(bytes) : set_limit<3>(bytes);
}

}  // namespace pdgpu
