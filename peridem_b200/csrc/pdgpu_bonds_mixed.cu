// Tiled bond loop, mixed-precision form: FP32 bond arithmetic on
// particle-local coordinates, FP64 per-node reductions.
//
// One CTA per tile of one particle's nodes (the tiles of the FP64 form).
// At the start of a tile:
//   * one thread hands the tile's neighbour columns (16- or 32-bit) and the
//     words of the broken-bond bitmap to the bulk-copy engine
//     (cp.async.bulk, completion counted on an mbarrier);
//   * all threads stage the neighbour window as packed FP32 node records
//     (2-D: {x, y, ux, uy} + volume; 3-D: {x, y, z, volume} + {ux, uy, uz}),
//     coordinates relative to the particle centre.
// The bond loop then reads only shared memory.  Each material law is its own
// instantiation, so the per-bond path carries no material dispatch; every
// index inside a tile is 32-bit.
//
// The arithmetic follows DEMModel::computePeridynamicForces
// (demModel.cpp:685-788) and the material laws of material.h, restated in
// FP32 with a cancellation-free stretch and fast intrinsics; the relative
// comparisons util::isGreater (a - b > 1e-5 max(|a|, |b|)) become
// comparisons against thresholds precomputed per particle.
//
// The state-based pre-pass (dilatation) keeps the generic tiled kernel.

#include "pdgpu_bonds.cuh"

namespace pdgpu {

namespace mixed_loop {

using bonds_mixed::gmask;
using bonds_mixed::gsum;
using bonds_mixed::gmax;

constexpr int kThreads = 256;
constexpr unsigned kWaitTries = 1u << 22;  // bounded mbarrier wait

// ---- bulk copy + mbarrier (PTX) ----
__device__ __forceinline__ uint32_t sa(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          sa(dst)),
      "l"(src), "r"(bytes), "r"(sa(bar))
      : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// true once phase 0 completed; false after kWaitTries attempts
__device__ __forceinline__ bool bar_wait(uint64_t *bar) {
  for (unsigned t = 0; t < kWaitTries; t++)
    if (bar_try(bar, 0)) return true;
  return false;
}

// Shared-memory plan of one tile (byte offsets into the dynamic stage);
// identical on host and device.
struct Plan {
  int64_t col0;      // first column entry copied (16-byte aligned)
  int64_t word0;     // first bitmap word copied (16-byte aligned)
  uint32_t col_bytes, bit_bytes;
  uint32_t off_a, off_b, off_m, total;
};

__host__ __device__ inline Plan plan(int dim, bool state, int col_size, int64_t kb, int64_t ke,
                                     int64_t w) {
  Plan p;
  const int64_t per16 = 16 / col_size;
  p.col0 = kb / per16 * per16;
  const int64_t col1 = (ke + per16 - 1) / per16 * per16;
  p.word0 = (kb >> 5) / 4 * 4;
  const int64_t word1 = (((ke + 31) >> 5) + 3) / 4 * 4;
  p.col_bytes = (uint32_t)((col1 - p.col0) * col_size);
  p.bit_bytes = (uint32_t)((word1 - p.word0) * 4);
  p.off_a = p.col_bytes + p.bit_bytes;                       // float4 records
  p.off_b = p.off_a + (uint32_t)(16 * w);                    // 2-D: float vol | 3-D: float4 u
  p.off_m = p.off_b + (uint32_t)((dim == 2 ? 4 : 16) * w);   // state: float2 per node
  p.off_m = (p.off_m + 15) / 16 * 16;
  p.total = p.off_m + (state ? (uint32_t)(8 * w) : 0u);
  p.total = (p.total + 15) / 16 * 16;
  return p;
}

enum { LAW_RNP = 0, LAW_PMB = 1, LAW_ELASTIC = 2, LAW_STATE = 3 };

// node-side view of the stage
template <int DIM>
struct View {
  const float4 *a;   // 2-D {x, y, ux, uy} | 3-D {x, y, z, vol}
  const float *vol;  // 2-D volumes
  const float4 *b;   // 3-D {ux, uy, uz, 0}
  const float2 *m;   // state: {theta (3K - 5G) / m_x, 15 G / m_x}

  __device__ __forceinline__ void node(int l, float (&x)[3], float (&u)[3], float &v) const {
    const float4 p = a[l];
    if constexpr (DIM == 2) {
      x[0] = p.x, x[1] = p.y, x[2] = 0.f;
      u[0] = p.z, u[1] = p.w, u[2] = 0.f;
      v = vol[l];
    } else {
      const float4 q = b[l];
      x[0] = p.x, x[1] = p.y, x[2] = p.z;
      u[0] = q.x, u[1] = q.y, u[2] = q.z;
      v = p.w;
    }
  }
};

template <int DIM>
__device__ __forceinline__ float dot(const float (&a)[3], const float (&b)[3]) {
  float s = a[0] * b[0] + a[1] * b[1];
  if constexpr (DIM == 3) s += a[2] * b[2];
  return s;
}

// the bond loop of one node for one material law; returns the force sum of
// this lane's bonds and their largest |stretch / critical stretch|
template <int DIM, int LPN, int LAW, typename CT>
__device__ __forceinline__ void node_bonds(const DevData &d, const MixParticle &M, const View<DIM> &V,
                                           const CT *s_col, const uint32_t *s_bits, int k0, int k1,
                                           int col_off, int bit_off, int shift, int64_t kb, int li,
                                           float (&F)[3], float &zmax) {
  const int lane = threadIdx.x % LPN;
  float xi[3], ui[3], vi;
  V.node(li, xi, ui, vi);
  float2 mi = make_float2(0.f, 0.f);
  if constexpr (LAW == LAW_STATE) mi = V.m[li];
  const bool gauss = d.inf.type == PDGPU_INF_GAUSSIAN;
#pragma unroll 2
  for (int k = k0 + lane; k < k1; k += LPN) {
    const int lj = (int)s_col[k + col_off] + shift;
    const int b = k + bit_off;
    const bool broken = (s_bits[b >> 5] >> (b & 31)) & 1u;
    float xj[3], uj[3], volj;
    V.node(lj, xj, uj, volj);
    float dx[3], du[3], y[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      dx[q] = xj[q] - xi[q];
      du[q] = uj[q] - ui[q];
      y[q] = dx[q] + du[q];
    }
    const float r2 = dot<DIM>(dx, dx);
    const float inv_r = rsqrtf(r2);
    const float rji = r2 * inv_r;
    const float dxdu = dot<DIM>(dx, du);
    float S, z, inv_ly = 0.f;
    if constexpr (LAW == LAW_RNP) {
      // linearised stretch; critical stretch rbar / sqrt(r)
      S = dxdu * inv_r * inv_r;
      z = fabsf(S) * rsqrtf(inv_r) * M.inv_rbar;
    } else {
      const float y2 = dot<DIM>(y, y);
      inv_ly = rsqrtf(y2);
      const float ly = y2 * inv_ly;
      // (|y| - r) / r without cancellation
      S = __fdividef(2.f * dxdu + dot<DIM>(du, du), rji * (ly + rji));
      z = fabsf(S) * M.inv_s0;
    }
    zmax = fmaxf(zmax, z);
    if (!broken) {
      const float vol = rji > M.low_thr ? volj * (M.check_up - rji) * M.inv_h : volj;
      const float J = gauss ? M.j0 * __expf(rji * rji * M.j1) : M.j0 + M.j1 * rji;
      float sf = 0.f;
      if constexpr (LAW == LAW_RNP) {
        if (M.irreversible && z > M.fsc_thr) {
          atomicOr(d.bond_bits + ((kb + k) >> 5), 1u << ((kb + k) & 31));
        } else {
          sf = J * M.k_force * S * __expf(-M.beta * rji * S * S) * vol * inv_r;
        }
      } else if constexpr (LAW == LAW_PMB) {
        if (fabsf(S) > M.s0_thr) {
          atomicOr(d.bond_bits + ((kb + k) >> 5), 1u << ((kb + k) & 31));
        } else {
          sf = J * M.k_force * S * vol * inv_ly;
        }
      } else if constexpr (LAW == LAW_ELASTIC) {
        sf = J * M.k_force * S * vol * inv_ly;
      } else {
        const float2 mj = V.m[lj];
        sf = J * rji * ((mi.x + mj.x) + S * (mi.y + mj.y)) * vol * inv_ly;
      }
      // bond-based RNP acts along the reference bond, the others along y
#pragma unroll
      for (int q = 0; q < DIM; q++) F[q] += sf * (LAW == LAW_RNP ? dx[q] : y[q]);
    } else {
      // broken bond: short-range repulsion between the two nodes
      const float inv_R = rsqrtf(dot<DIM>(y, y));
      const float sf = fminf(M.kn * volj * (1.f - M.rc * inv_R), 0.f);
#pragma unroll
      for (int q = 0; q < DIM; q++) F[q] += sf * y[q];
    }
  }
}

template <int DIM, int LPN, int LAW, typename CT>
__device__ __forceinline__ void tile_nodes(const DevData &d, const BondTile &T, const MixParticle &M,
                                           const View<DIM> &V, const CT *s_col, const uint32_t *s_bits,
                                           const Plan &p) {
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const int st = DIM == 2 ? 2 : 4;
  const int64_t kb = T.bond_begin;
  const int col_off = (int)(kb - p.col0);
  const int bit_off = (int)(kb - 32 * p.word0);
  const int shift = sizeof(CT) == 2 ? (int)(M.start - T.win_begin) : (int)(-T.win_begin);
  for (int64_t i = T.node_begin + threadIdx.x / LPN; i < T.node_end; i += kThreads / LPN) {
    if (!(d.flags[i] & NODE_ACTIVE)) {
      if (lane == 0)
        for (int q = 0; q < DIM; q++) d.f[st * i + q] = 0.0;
      continue;
    }
    const int k0 = (int)(d.pd_row[i] - kb), k1 = (int)(d.pd_row[i + 1] - kb);
    float F[3] = {0.f, 0.f, 0.f};
    float zmax = 0.f;
    node_bonds<DIM, LPN, LAW, CT>(d, M, V, s_col, s_bits, k0, k1, col_off, bit_off, shift, kb,
                                  (int)(i - T.win_begin), F, zmax);
    const double Fx = gsum<LPN>((double)F[0], gm);
    const double Fy = gsum<LPN>((double)F[1], gm);
    const double Fz = DIM == 3 ? gsum<LPN>((double)F[2], gm) : 0.0;
    const float Z = gmax<LPN>(zmax, gm);
    if (lane == 0) {
      d.f[st * i] = Fx;
      d.f[st * i + 1] = Fy;
      if constexpr (DIM == 3) d.f[st * i + 2] = Fz;
      d.Z[i] = Z;
    }
  }
}

template <int DIM, int LPN, typename CT>
__global__ void __launch_bounds__(kThreads) k_bonds_mixed(DevData d, const BondTile *tiles, const CT *col) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  if (d.ctrl->error) return;
  const BondTile T = tiles[blockIdx.x];
  const MixParticle M = d.mixp[T.particle];
  const bool state = M.material == PDGPU_MAT_PDSTATE;
  const int w = (int)(T.win_end - T.win_begin);
  const Plan p = plan(DIM, state, (int)sizeof(CT), T.bond_begin, T.bond_end, w);
  CT *s_col = reinterpret_cast<CT *>(smem);
  uint32_t *s_bits = reinterpret_cast<uint32_t *>(smem + p.col_bytes);

  // columns and bitmap words of the tile's bonds: bulk copies
  if (threadIdx.x == 0) {
    bar_init(&bar);
    bar_arrive_tx(&bar, p.col_bytes + p.bit_bytes);
    if (p.col_bytes) bulk_load(s_col, col + p.col0, p.col_bytes, &bar);
    if (p.bit_bytes) bulk_load(s_bits, d.bond_bits + p.word0, p.bit_bytes, &bar);
  }

  // neighbour window: packed FP32 records relative to the particle centre
  float4 *sa4 = reinterpret_cast<float4 *>(smem + p.off_a);
  float *svol = reinterpret_cast<float *>(smem + p.off_b);
  float4 *sb4 = reinterpret_cast<float4 *>(smem + p.off_b);
  float2 *sm2 = reinterpret_cast<float2 *>(smem + p.off_m);
  {
    const int st = DIM == 2 ? 2 : 4;
    const DevParticle &P = d.particles[T.particle];
    double xc[DIM], uc[DIM];
#pragma unroll
    for (int q = 0; q < DIM; q++) {
      xc[q] = d.xref[st * P.center + q];
      uc[q] = d.u[st * P.center + q];
    }
    for (int a = threadIdx.x; a < w; a += kThreads) {
      const int64_t j = T.win_begin + a;
      float xr[DIM], ur[DIM];
#pragma unroll
      for (int q = 0; q < DIM; q++) {
        xr[q] = (float)(__ldg(d.xref + st * j + q) - xc[q]);
        ur[q] = (float)(d.u[st * j + q] - uc[q]);
      }
      const float vj = (float)__ldg(d.vol + j);
      if constexpr (DIM == 2) {
        sa4[a] = make_float4(xr[0], xr[1], ur[0], ur[1]);
        svol[a] = vj;
      } else {
        sa4[a] = make_float4(xr[0], xr[1], xr[2], vj);
        sb4[a] = make_float4(ur[0], ur[1], ur[2], 0.f);
      }
      if (state) {
        const double inv_m = 1.0 / d.mx[j];
        sm2[a] = make_float2((float)(d.theta[j] * M.tf_coef * inv_m), (float)(M.am_coef * inv_m));
      }
    }
  }
  __syncthreads();
  if (!bar_wait(&bar)) {
    // the copies did not land: record it, give them one more bounded wait so
    // that none is left writing into this CTA's shared memory, and stop
    if (threadIdx.x == 0 && atomicCAS(&d.ctrl->error, 0, DEV_ERR_STAGE_TIMEOUT) == 0)
      d.ctrl->error_info = blockIdx.x;
    bar_wait(&bar);
    return;
  }

  View<DIM> V{sa4, svol, sb4, sm2};
  switch (M.material) {
    case PDGPU_MAT_RNP: tile_nodes<DIM, LPN, LAW_RNP, CT>(d, T, M, V, s_col, s_bits, p); break;
    case PDGPU_MAT_PMB: tile_nodes<DIM, LPN, LAW_PMB, CT>(d, T, M, V, s_col, s_bits, p); break;
    case PDGPU_MAT_PDELASTIC: tile_nodes<DIM, LPN, LAW_ELASTIC, CT>(d, T, M, V, s_col, s_bits, p); break;
    default: tile_nodes<DIM, LPN, LAW_STATE, CT>(d, T, M, V, s_col, s_bits, p); break;
  }
}

template <int DIM, typename CT>
void launch_dim(const DevData &d, const CT *col, const BondTile *t, int n, int lanes, size_t smem,
                cudaStream_t s) {
  switch (lanes) {
    case 4: k_bonds_mixed<DIM, 4, CT><<<n, kThreads, smem, s>>>(d, t, col); break;
    case 8: k_bonds_mixed<DIM, 8, CT><<<n, kThreads, smem, s>>>(d, t, col); break;
    case 16: k_bonds_mixed<DIM, 16, CT><<<n, kThreads, smem, s>>>(d, t, col); break;
    default: k_bonds_mixed<DIM, 32, CT><<<n, kThreads, smem, s>>>(d, t, col); break;
  }
}

template <int DIM>
void launch_pre(const DevData &d, const BondTile *t, int n, int lanes, size_t smem, cudaStream_t s) {
  using namespace bonds_mixed;
  switch (lanes) {
    case 4: k_prepass_tiled<DIM, 4><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 8: k_prepass_tiled<DIM, 8><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 16: k_prepass_tiled<DIM, 16><<<n, kTileThreads, smem, s>>>(d, t); break;
    default: k_prepass_tiled<DIM, 32><<<n, kTileThreads, smem, s>>>(d, t); break;
  }
}

template <int DIM>
int set_limit(size_t bytes) {
  using bonds_mixed::k_prepass_tiled;
  const void *fs[] = {
      (const void *)k_bonds_mixed<DIM, 4, uint16_t>,  (const void *)k_bonds_mixed<DIM, 8, uint16_t>,
      (const void *)k_bonds_mixed<DIM, 16, uint16_t>, (const void *)k_bonds_mixed<DIM, 32, uint16_t>,
      (const void *)k_bonds_mixed<DIM, 4, int32_t>,   (const void *)k_bonds_mixed<DIM, 8, int32_t>,
      (const void *)k_bonds_mixed<DIM, 16, int32_t>,  (const void *)k_bonds_mixed<DIM, 32, int32_t>,
      (const void *)k_prepass_tiled<DIM, 4>,          (const void *)k_prepass_tiled<DIM, 8>,
      (const void *)k_prepass_tiled<DIM, 16>,         (const void *)k_prepass_tiled<DIM, 32>};
  for (auto f : fs)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
      return -1;
  return 0;
}

}  // namespace mixed_loop

void launch_pd_tiled_mixed(const DevData &d, const BondTile *t, int n, int lanes, size_t smem,
                           cudaStream_t s) {
  using namespace mixed_loop;
  if (n <= 0) return;
  if (d.use16) {
    if (d.dim == 2) launch_dim<2>(d, d.pd_col16, t, n, lanes, smem, s);
    else launch_dim<3>(d, d.pd_col16, t, n, lanes, smem, s);
  } else {
    if (d.dim == 2) launch_dim<2>(d, (const int32_t *)d.pd_col, t, n, lanes, smem, s);
    else launch_dim<3>(d, (const int32_t *)d.pd_col, t, n, lanes, smem, s);
  }
}

void launch_prepass_tiled_mixed(const DevData &d, const BondTile *t, int n, int lanes, size_t smem,
                                cudaStream_t s) {
  if (n <= 0) return;
  if (d.dim == 2) mixed_loop::launch_pre<2>(d, t, n, lanes, smem, s);
  else mixed_loop::launch_pre<3>(d, t, n, lanes, smem, s);
}

size_t tile_smem_mixed(int dim, bool state, int64_t window) {
  return bonds_mixed::tile_smem_bytes(dim, state, (int)window);
}

size_t tile_smem_mixed_main(int dim, bool state, bool col16, const BondTile &t) {
  return mixed_loop::plan(dim, state, col16 ? 2 : 4, t.bond_begin, t.bond_end,
                          t.win_end - t.win_begin)
      .total;
}

int set_tile_smem_limit_mixed(int dim, size_t bytes) {
  return dim == 2 ? mixed_loop::set_limit<2>(bytes) : mixed_loop::set_limit<3>(bytes);
}

}  // namespace pdgpu
