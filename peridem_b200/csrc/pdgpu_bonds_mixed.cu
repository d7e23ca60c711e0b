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

// threads per CTA: 256 in 2-D; in 3-D, where a tile's neighbour window is
// large (~100 KB of stage) and only two CTAs fit an SM, up to 512, so that
// two CTAs per SM (one computing while the other waits at a tile barrier)
// fit the register file
template <int DIM, int LPN>
constexpr int kThreadsFor = DIM == 3 ? (256 * LPN < 512 ? 256 * LPN : 512) : 256;
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
// orders this CTA's earlier shared-memory accesses before later bulk-copy writes
__device__ __forceinline__ void fence_async_smem() {
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
// true once the phase of the given parity completed; false after kWaitTries attempts
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  for (unsigned t = 0; t < kWaitTries; t++)
    if (bar_try(bar, parity)) return true;
  return false;
}

// Shared-memory plan of one tile (byte offsets into the dynamic stage);
// identical on host and device.  Bulk-copied regions start and end on 16-byte
// boundaries of the global arrays, which carry tail padding for that.
struct Plan {
  int64_t col0;   // first column entry copied
  int64_t word0;  // first bitmap word copied
  int64_t row0;   // first row offset copied (pd_row)
  uint32_t col_bytes, bit_bytes, row_bytes;
  uint32_t off_row, off_xv, off_u, off_m, total;
};

__host__ __device__ inline Plan plan(int dim, bool state, int col_size, int64_t kb, int64_t ke,
                                     int64_t nb, int64_t ne, int64_t w) {
  Plan p;
  const int64_t per16 = 16 / col_size;
  p.col0 = kb / per16 * per16;
  const int64_t col1 = (ke + per16 - 1) / per16 * per16;
  p.word0 = (kb >> 5) / 4 * 4;
  const int64_t word1 = (((ke + 31) >> 5) + 3) / 4 * 4;
  p.row0 = nb / 2 * 2;
  const int64_t row1 = (ne + 1 + 1) / 2 * 2;  // rows nb .. ne inclusive
  p.col_bytes = (uint32_t)((col1 - p.col0) * col_size);
  p.bit_bytes = (uint32_t)((word1 - p.word0) * 4);
  p.row_bytes = (uint32_t)((row1 - p.row0) * 8);
  p.off_row = p.col_bytes + p.bit_bytes;
  p.off_xv = p.off_row + p.row_bytes;                        // float4 {x, y, z, vol}
  p.off_u = p.off_xv + (uint32_t)(16 * w);                   // 2-D float2 | 3-D float4 u
  p.off_m = p.off_u + (uint32_t)((dim == 2 ? 8 : 16) * w);   // state: float2 per node
  p.total = p.off_m + (state ? (uint32_t)(8 * w) : 0u);
  p.total = (p.total + 15) / 16 * 16;
  return p;
}

enum { LAW_RNP = 0, LAW_PMB = 1, LAW_ELASTIC = 2, LAW_STATE = 3 };

// node-side view of the stage
template <int DIM>
struct View {
  const float4 *xv;  // {x, y, z, vol}, reference coordinates relative to the particle centre
  const float2 *u2;  // 2-D displacement relative to the centre's
  const float4 *u4;  // 3-D displacement relative to the centre's
  const float2 *m;   // state: {theta (3K - 5G) / m_x, 15 G / m_x}

  __device__ __forceinline__ void node(int l, float (&x)[3], float (&u)[3], float &v) const {
    const float4 p = xv[l];
    x[0] = p.x, x[1] = p.y, x[2] = p.z;
    v = p.w;
    if constexpr (DIM == 2) {
      const float2 q = u2[l];
      u[0] = q.x, u[1] = q.y, u[2] = 0.f;
    } else {
      const float4 q = u4[l];
      u[0] = q.x, u[1] = q.y, u[2] = q.z;
    }
  }
};

template <int DIM>
__device__ __forceinline__ float dot(const float (&a)[3], const float (&b)[3]) {
  float s = a[0] * b[0] + a[1] * b[1];
  if constexpr (DIM == 3) s += a[2] * b[2];
  return s;
}

__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One bond (i, j) of node i for one material law.  zq tracks the damage
// measure in a monotone form: RNP S^2 r (Z = sqrt(zq) / rbar), the others
// |S| (Z = zq / s0).  `broken` is the bond's state before this step.
template <int DIM, int LAW, bool BROKEN_KNOWN_CLEAR>
__device__ __forceinline__ void bond(const DevData &d, const MixParticle &M, const View<DIM> &V,
                                     const float (&xi)[3], const float (&ui)[3], float2 mi, int lj,
                                     bool broken, bool gauss, int64_t kglob, float (&F)[3],
                                     float &zmax) {
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
  float S, zq, inv_ly = 0.f;
  if constexpr (LAW == LAW_RNP) {
    S = dxdu * (inv_r * inv_r);  // linearised stretch
    zq = S * S * rji;
  } else {
    const float y2 = dot<DIM>(y, y);
    inv_ly = rsqrtf(y2);
    const float ly = y2 * inv_ly;
    S = __fdividef(2.f * dxdu + dot<DIM>(du, du), rji * (ly + rji));  // (|y| - r) / r
    zq = fabsf(S);
  }
  zmax = fmaxf(zmax, zq);
  if (BROKEN_KNOWN_CLEAR || !broken) {
    const float vol = volj * (rji > M.low_thr ? fmaf(-rji, M.inv_h, M.cu_h) : 1.f);
    // influence times the law's constant
    const float kJ = gauss ? M.kj0 * ex2(rji * rji * M.j1) : fmaf(M.kj1, rji, M.kj0);
    float sf = 0.f;
    if constexpr (LAW == LAW_RNP) {
      if (M.irreversible && zq > M.fsc_q)
        atomicOr(d.bond_bits + (kglob >> 5), 1u << (kglob & 31));
      else
        sf = kJ * S * ex2(M.nbeta_l2e * zq) * vol * inv_r;
    } else if constexpr (LAW == LAW_PMB) {
      if (zq > M.s0_thr)
        atomicOr(d.bond_bits + (kglob >> 5), 1u << (kglob & 31));
      else
        sf = kJ * S * vol * inv_ly;
    } else if constexpr (LAW == LAW_ELASTIC) {
      sf = kJ * S * vol * inv_ly;
    } else {
      const float2 mj = V.m[lj];
      sf = kJ * rji * ((mi.x + mj.x) + S * (mi.y + mj.y)) * vol * inv_ly;
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

// does any bond of [b0, b1) (bit positions in the staged bitmap) start broken?
template <int LPN>
__device__ __forceinline__ bool any_broken(const uint32_t *s_bits, int b0, int b1, unsigned gm) {
  const int lane = threadIdx.x % LPN;
  const int w0 = b0 >> 5, w1 = (b1 - 1) >> 5;
  bool hit = false;
  for (int w = w0 + lane; w <= w1; w += LPN) {
    uint32_t m = s_bits[w];
    if (w == w0) m &= ~0u << (b0 & 31);
    if (w == w1) m &= ~0u >> (31 - ((b1 - 1) & 31));
    hit |= m != 0u;
  }
  return __any_sync(gm, hit);
}

template <int DIM, int LPN, int LAW, typename CT>
__device__ __forceinline__ void tile_nodes(const DevData &d, const BondTile &T, const MixParticle &M,
                                           const View<DIM> &V, const CT *s_col, const uint32_t *s_bits,
                                           const int64_t *s_row, const Plan &p) {
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const int st = DIM == 2 ? 2 : 4;
  const int64_t kb = T.bond_begin;
  const int col_off = (int)(kb - p.col0);
  const int bit_off = (int)(kb - 32 * p.word0);
  const int shift = sizeof(CT) == 2 ? (int)(M.start - T.win_begin) : (int)(-T.win_begin);
  const bool gauss = d.inf.type == PDGPU_INF_GAUSSIAN;
  // every node of a tile computes forces (tiles cover force-computing particles only)
  for (int64_t pos = T.node_begin + threadIdx.x / LPN; pos < T.node_end; pos += kThreadsFor<DIM, LPN> / LPN) {
    // bond scheme 2: the tile's nodes longest row first
    const int64_t i = d.node_order ? (int64_t)d.node_order[pos] : pos;
    const int k0 = (int)(s_row[i - p.row0] - kb), k1 = (int)(s_row[i + 1 - p.row0] - kb);
    const int li = (int)(i - T.win_begin);
    float xi[3], ui[3], vi;
    V.node(li, xi, ui, vi);
    float2 mi = make_float2(0.f, 0.f);
    if constexpr (LAW == LAW_STATE) mi = V.m[li];
    float F[3] = {0.f, 0.f, 0.f};
    float zmax = 0.f;
    if (!any_broken<LPN>(s_bits, k0 + bit_off, k1 + bit_off, gm)) {
      // no bond of this node starts broken: no per-bond state test; four
      // bonds in flight per thread (measured: 17 % faster than two on a
      // bond loop beyond L2, 9 % on config 1; packed FP32x2 pairs of bonds
      // measured 12 % slower on the 2-D compressive test)
#pragma unroll 4
      for (int k = k0 + lane; k < k1; k += LPN)
        bond<DIM, LAW, true>(d, M, V, xi, ui, mi, (int)s_col[k + col_off] + shift, false, gauss,
                             kb + k, F, zmax);
    } else {
      for (int k = k0 + lane; k < k1; k += LPN) {
        const int b = k + bit_off;
        const bool broken = (s_bits[b >> 5] >> (b & 31)) & 1u;
        bond<DIM, LAW, false>(d, M, V, xi, ui, mi, (int)s_col[k + col_off] + shift, broken, gauss,
                              kb + k, F, zmax);
      }
    }
    const double Fx = gsum<LPN>((double)F[0], gm);
    const double Fy = gsum<LPN>((double)F[1], gm);
    const double Fz = DIM == 3 ? gsum<LPN>((double)F[2], gm) : 0.0;
    const float zq = gmax<LPN>(zmax, gm);
    if (lane == 0) {
      d.f[st * i] = Fx;
      d.f[st * i + 1] = Fy;
      if constexpr (DIM == 3) d.f[st * i + 2] = Fz;
      d.Z[i] = LAW == LAW_RNP ? sqrtf(zq) * M.inv_rbar : zq * M.inv_s0;
    }
  }
}

// PD state pre-pass, one bond (demModel.cpp:610-679): the extension
// e = |y| - r (cancellation-free) and, for a bond that is not broken, its
// term r e J(r) vol_j of the dilatation sum; a bond whose stretch exceeds
// the critical stretch breaks here (the main loop then sees it broken).
template <int DIM, bool BROKEN_KNOWN_CLEAR>
__device__ __forceinline__ void pre_bond(const DevData &d, const MixParticle &M, const View<DIM> &V,
                                         const float (&xi)[3], const float (&ui)[3], int lj, bool broken,
                                         bool gauss, int64_t kglob, float &th) {
  float xj[3], uj[3], volj;
  V.node(lj, xj, uj, volj);
  float dx[3], eta[3], y[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    dx[q] = xj[q] - xi[q];
    eta[q] = uj[q] - ui[q];
    y[q] = dx[q] + eta[q];
  }
  const float r2 = dot<DIM>(dx, dx);
  const float inv_r = rsqrtf(r2);
  const float rji = r2 * inv_r;
  const float y2 = dot<DIM>(y, y);
  const float l = y2 * rsqrtf(y2);
  const float cl = __fdividef(2.f * dot<DIM>(dx, eta) + dot<DIM>(eta, eta), l + rji);
  if (BROKEN_KNOWN_CLEAR || !broken) {
    if (fabsf(cl * inv_r) > M.s0_thr) {
      atomicOr(d.bond_bits + (kglob >> 5), 1u << (kglob & 31));
    } else {
      const float vol = volj * (rji > M.low_thr ? fmaf(-rji, M.inv_h, M.cu_h) : 1.f);
      const float J = gauss ? M.j0 * ex2(r2 * M.j1) : fmaf(M.j1, rji, M.j0);
      th = fmaf(rji * cl, J * vol, th);
    }
  }
}

// the pre-pass over one staged tile: theta_i = 3 sum / m_x,i
template <int DIM, int LPN, typename CT>
__device__ __forceinline__ void tile_theta(const DevData &d, const BondTile &T, const MixParticle &M,
                                           const View<DIM> &V, const CT *s_col, const uint32_t *s_bits,
                                           const int64_t *s_row, const Plan &p) {
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const int64_t kb = T.bond_begin;
  const int col_off = (int)(kb - p.col0);
  const int bit_off = (int)(kb - 32 * p.word0);
  const int shift = sizeof(CT) == 2 ? (int)(M.start - T.win_begin) : (int)(-T.win_begin);
  const bool gauss = d.inf.type == PDGPU_INF_GAUSSIAN;
  for (int64_t pos = T.node_begin + threadIdx.x / LPN; pos < T.node_end; pos += kThreadsFor<DIM, LPN> / LPN) {
    // bond scheme 2: the tile's nodes longest row first
    const int64_t i = d.node_order ? (int64_t)d.node_order[pos] : pos;
    const int k0 = (int)(s_row[i - p.row0] - kb), k1 = (int)(s_row[i + 1 - p.row0] - kb);
    const int li = (int)(i - T.win_begin);
    float xi[3], ui[3], vi;
    V.node(li, xi, ui, vi);
    float th = 0.f;
    if (!any_broken<LPN>(s_bits, k0 + bit_off, k1 + bit_off, gm)) {
#pragma unroll 2
      for (int k = k0 + lane; k < k1; k += LPN)
        pre_bond<DIM, true>(d, M, V, xi, ui, (int)s_col[k + col_off] + shift, false, gauss, kb + k, th);
    } else {
      for (int k = k0 + lane; k < k1; k += LPN) {
        const int b = k + bit_off;
        const bool broken = (s_bits[b >> 5] >> (b & 31)) & 1u;
        pre_bond<DIM, false>(d, M, V, xi, ui, (int)s_col[k + col_off] + shift, broken, gauss, kb + k, th);
      }
    }
    const double t = gsum<LPN>((double)th, gm);
    if (lane == 0) d.theta[i] = 3.0 * t / d.mx[i];
  }
}

// ---------------------------------------------------------------------------
// Symmetric form (2-D): a bond (i, j) whose nodes both lie in the tile is
// evaluated once, by node i's thread when i < j.  Stretch, influence, volume
// correction and law factor are symmetric in (i, j); only the neighbour's
// volume differs, so the thread adds c vol_j dir to node i and leaves
// -c vol_i dir and the bond's damage measure in a tile-local slot for node j.
// After a barrier, node j's thread adds the slots of its bonds to earlier
// nodes.  Bonds that leave the tile are evaluated from both ends, as before.
// A row is ordered [to later tile nodes | leaving the tile | to earlier tile
// nodes] (sym_col; sym_pos maps an entry back to its place in pd_col), so the
// evaluated entries come first and the slot reads last.  Deterministic: every
// sum has a fixed order.
// ---------------------------------------------------------------------------
struct SymPlan {
  int64_t meta0;        // first node metadata entry copied
  uint32_t meta_bytes;  // bulk-copied node metadata
  uint32_t off_meta, off_part_f, off_part_z, off_fj, off_zq, total;
};

__host__ __device__ inline SymPlan sym_plan(const Plan &p, int64_t nb, int64_t ne, int slots) {
  SymPlan q;
  q.meta0 = nb / 2 * 2;
  const int64_t meta1 = (ne + 1) / 2 * 2;
  q.meta_bytes = (uint32_t)((meta1 - q.meta0) * 8);
  const uint32_t nodes = (uint32_t)(ne - nb);
  q.off_meta = p.total;                                          // 16-byte aligned
  q.off_part_f = q.off_meta + (q.meta_bytes + 15u) / 16u * 16u;  // double2 per tile node
  q.off_part_z = q.off_part_f + 16u * nodes;                     // float per tile node
  q.off_fj = (q.off_part_z + 4u * nodes + 15u) / 16u * 16u;      // float2 per slot
  q.off_zq = q.off_fj + 8u * (uint32_t)slots;                    // float per slot
  q.total = (q.off_zq + 4u * (uint32_t)slots + 15u) / 16u * 16u;
  return q;
}

// one bond of phase A: force on i added to F; with slot >= 0 (j a later node
// of the tile) j's share and the damage measure go to the slot.  e is the
// bond's index in the symmetric order; row_i node i's first entry in pd_col.
template <int LAW, bool BROKEN_KNOWN_CLEAR>
__device__ __forceinline__ void bond_sym(const DevData &d, const MixParticle &M, const View<2> &V,
                                         const float (&xi)[3], const float (&ui)[3], float vi, float2 mi,
                                         int lj, bool broken, bool gauss, int64_t e, int64_t row_i,
                                         int64_t i, int64_t win_begin, int slot, float2 *s_fj, float *s_zq,
                                         float (&F)[3], float &zmax) {
  float xj[3], uj[3], volj;
  V.node(lj, xj, uj, volj);
  float dx[2], du[2], y[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    dx[q] = xj[q] - xi[q];
    du[q] = uj[q] - ui[q];
    y[q] = dx[q] + du[q];
  }
  const float r2 = dx[0] * dx[0] + dx[1] * dx[1];
  const float inv_r = rsqrtf(r2);
  const float rji = r2 * inv_r;
  const float dxdu = dx[0] * du[0] + dx[1] * du[1];
  float S, zq, inv_ly = 0.f;
  if constexpr (LAW == LAW_RNP) {
    S = dxdu * (inv_r * inv_r);
    zq = S * S * rji;
  } else {
    const float y2 = y[0] * y[0] + y[1] * y[1];
    inv_ly = rsqrtf(y2);
    const float ly = y2 * inv_ly;
    S = __fdividef(2.f * dxdu + (du[0] * du[0] + du[1] * du[1]), rji * (ly + rji));
    zq = fabsf(S);
  }
  zmax = fmaxf(zmax, zq);
  float c = 0.f;  // force per unit neighbour volume, along dir
  bool along_ref = LAW == LAW_RNP;
  if (BROKEN_KNOWN_CLEAR || !broken) {
    const float corr = rji > M.low_thr ? fmaf(-rji, M.inv_h, M.cu_h) : 1.f;
    const float kJ = gauss ? M.kj0 * ex2(rji * rji * M.j1) : fmaf(M.kj1, rji, M.kj0);
    bool breaks = false;
    if constexpr (LAW == LAW_RNP) {
      breaks = M.irreversible && zq > M.fsc_q;
      if (!breaks) c = kJ * S * ex2(M.nbeta_l2e * zq) * corr * inv_r;
    } else if constexpr (LAW == LAW_PMB) {
      breaks = zq > M.s0_thr;
      if (!breaks) c = kJ * S * corr * inv_ly;
    } else if constexpr (LAW == LAW_ELASTIC) {
      c = kJ * S * corr * inv_ly;
    } else {
      const float2 mj = V.m[lj];
      c = kJ * rji * ((mi.x + mj.x) + S * (mi.y + mj.y)) * corr * inv_ly;
    }
    if (breaks) {
      // both directed bonds break together (the same stretch from either end)
      const int64_t g = row_i + d.sym_pos[e];
      atomicOr(d.bond_bits + (g >> 5), 1u << (g & 31));
      if (slot >= 0) {
        const int64_t j = win_begin + lj;
        for (int64_t m = d.pd_row[j]; m < d.pd_row[j + 1]; m++)
          if (d.pd_col[m] == (int32_t)i) {
            atomicOr(d.bond_bits + (m >> 5), 1u << (m & 31));
            break;
          }
      }
    }
  } else {
    // broken bond: short-range repulsion between the two nodes
    const float inv_R = rsqrtf(y[0] * y[0] + y[1] * y[1]);
    c = fminf(M.kn * (1.f - M.rc * inv_R), 0.f);
    along_ref = false;
  }
  const float d0 = along_ref ? dx[0] : y[0], d1 = along_ref ? dx[1] : y[1];
  const float ci = c * volj;
  F[0] = fmaf(ci, d0, F[0]);
  F[1] = fmaf(ci, d1, F[1]);
  if (slot >= 0) {
    const float cj = -c * vi;
    s_fj[slot] = make_float2(cj * d0, cj * d1);
    s_zq[slot] = zq;
  }
}

template <int LPN, int LAW, typename CT>
__device__ __forceinline__ void tile_sym(const DevData &d, const BondTile &T, const MixParticle &M,
                                         const View<2> &V, const CT *s_col, const uint32_t *s_bits,
                                         const int64_t *s_row, const Plan &p, const SymPlan &q,
                                         unsigned char *smem) {
  constexpr int kT = kThreadsFor<2, LPN>;
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const int64_t kb = T.bond_begin;
  const int col_off = (int)(kb - p.col0);
  const int bit_off = (int)(kb - 32 * p.word0);
  const int shift = (int)(M.start - T.win_begin);
  const bool gauss = d.inf.type == PDGPU_INF_GAUSSIAN;
  const uint2 *s_meta = reinterpret_cast<const uint2 *>(smem + q.off_meta);
  double2 *s_pf = reinterpret_cast<double2 *>(smem + q.off_part_f);
  float *s_pz = reinterpret_cast<float *>(smem + q.off_part_z);
  float2 *s_fj = reinterpret_cast<float2 *>(smem + q.off_fj);
  float *s_zq = reinterpret_cast<float *>(smem + q.off_zq);
  // phase A: bonds to later tile nodes and bonds leaving the tile
  for (int64_t i = T.node_begin + threadIdx.x / LPN; i < T.node_end; i += kT / LPN) {
    const int64_t row_i = s_row[i - p.row0];
    const int k0 = (int)(row_i - kb), k1 = (int)(s_row[i + 1 - p.row0] - kb);
    const uint2 meta = s_meta[i - q.meta0];
    const int base = (int)meta.x, n_up = (int)(meta.y & 0xffffu), n_uo = (int)(meta.y >> 16);
    const int li = (int)(i - T.win_begin);
    float xi[3], ui[3], vi;
    V.node(li, xi, ui, vi);
    float2 mi = make_float2(0.f, 0.f);
    if constexpr (LAW == LAW_STATE) mi = V.m[li];
    float F[3] = {0.f, 0.f, 0.f};
    float zmax = 0.f;
    if (!any_broken<LPN>(s_bits, k0 + bit_off, k1 + bit_off, gm)) {
#pragma unroll 4
      for (int k = k0 + lane; k < k0 + n_uo; k += LPN)
        bond_sym<LAW, true>(d, M, V, xi, ui, vi, mi, (int)s_col[k + col_off] + shift, false, gauss, kb + k,
                            row_i, i, T.win_begin, k - k0 < n_up ? base + k - k0 : -1, s_fj, s_zq, F, zmax);
    } else {
      for (int k = k0 + lane; k < k0 + n_uo; k += LPN) {
        const int b = (int)(row_i - 32 * p.word0) + (int)d.sym_pos[kb + k];
        const bool broken = (s_bits[b >> 5] >> (b & 31)) & 1u;
        bond_sym<LAW, false>(d, M, V, xi, ui, vi, mi, (int)s_col[k + col_off] + shift, broken, gauss, kb + k,
                             row_i, i, T.win_begin, k - k0 < n_up ? base + k - k0 : -1, s_fj, s_zq, F, zmax);
      }
    }
    const double Fx = gsum<LPN>((double)F[0], gm);
    const double Fy = gsum<LPN>((double)F[1], gm);
    const float zq = gmax<LPN>(zmax, gm);
    if (lane == 0) {
      s_pf[i - T.node_begin] = make_double2(Fx, Fy);
      s_pz[i - T.node_begin] = zq;
    }
  }
  __syncthreads();
  // phase B: the shares earlier tile nodes left for this node
  for (int64_t i = T.node_begin + threadIdx.x / LPN; i < T.node_end; i += kT / LPN) {
    const int k0 = (int)(s_row[i - p.row0] - kb), k1 = (int)(s_row[i + 1 - p.row0] - kb);
    const int n_uo = (int)(s_meta[i - q.meta0].y >> 16);
    float fx = 0.f, fy = 0.f, zmax = 0.f;
#pragma unroll 4
    for (int k = k0 + n_uo + lane; k < k1; k += LPN) {
      const int slot = (int)s_col[k + col_off];
      const float2 f = s_fj[slot];
      fx += f.x;
      fy += f.y;
      zmax = fmaxf(zmax, s_zq[slot]);
    }
    const double Bx = gsum<LPN>((double)fx, gm);
    const double By = gsum<LPN>((double)fy, gm);
    const float zb = gmax<LPN>(zmax, gm);
    if (lane == 0) {
      const double2 a = s_pf[i - T.node_begin];
      d.f[2 * i] = a.x + Bx;
      d.f[2 * i + 1] = a.y + By;
      const float zq = fmaxf(s_pz[i - T.node_begin], zb);
      d.Z[i] = LAW == LAW_RNP ? sqrtf(zq) * M.inv_rbar : zq * M.inv_s0;
    }
  }
}

// Persistent: a fixed grid (below full occupancy, so that the contact and
// damping passes running beside it find room) claims tiles from a counter in
// the step-control state; the claim for the next tile is made while the
// current one is staged.  The last CTA out resets the counter.
template <int DIM, int LPN, int LAW, typename CT, bool PRE = false, bool SYM = false>
__global__ void __launch_bounds__(kThreadsFor<DIM, LPN>) k_bonds_mixed(DevData d, const BondTile *tiles, int n_tiles,
                                                         const CT *col) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_tile[2];
  if (d.ctrl->error) return;
  constexpr bool state = LAW == LAW_STATE && !PRE;  // the pre-pass needs no m, theta stage
  // learned surrogate: off check steps, its particles' tiles are left out —
  // by claiming from the list of the other tiles the contact rebuild wrote
  // this step where there is one, else by a test of each claimed tile
  const bool sur_step = d.sur_on != nullptr && !d.ctrl->sur_check;
  const bool listed = !PRE && sur_step && d.tile_live != nullptr;
  auto claim = [&]() -> int {
    const int c = (int)atomicAdd(&d.ctrl->tile_next, 1u);
    if (!listed) return c;
    return c < min((int)*d.tile_live_n, d.n_tile_live_src) ? d.tile_live[c] : n_tiles;
  };
  if (threadIdx.x == 0) {
    bar_init(&bar);
    s_tile[0] = claim();
  }
  __syncthreads();
  uint32_t parity = 0;
  int k = 0;
  int t = s_tile[0];
  while (t < n_tiles) {
    const BondTile T = tiles[t];
    if (sur_step && d.sur_on[T.particle] && !d.sur_near[T.particle]) {
      if (threadIdx.x == 0) s_tile[(k + 1) & 1] = claim();
      __syncthreads();
      t = s_tile[(k + 1) & 1];
      k++;
      continue;
    }
    const int w = (int)(T.win_end - T.win_begin);
    const Plan p = plan(DIM, state, (int)sizeof(CT), T.bond_begin, T.bond_end, T.node_begin, T.node_end, w);
    SymPlan q{};
    if constexpr (SYM) q = sym_plan(p, T.node_begin, T.node_end, T.slots);
    CT *s_col = reinterpret_cast<CT *>(smem);
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(smem + p.col_bytes);
    int64_t *s_row = reinterpret_cast<int64_t *>(smem + p.off_row);
    float4 *s_xv = reinterpret_cast<float4 *>(smem + p.off_xv);
    float2 *s_u2 = reinterpret_cast<float2 *>(smem + p.off_u);
    float4 *s_u4 = reinterpret_cast<float4 *>(smem + p.off_u);
    float2 *s_m = reinterpret_cast<float2 *>(smem + p.off_m);

    // columns, bitmap words, row offsets and constant node records of the
    // tile: bulk copies; then the claim of the next tile
    if (threadIdx.x == 0) {
      fence_async_smem();
      bar_arrive_tx(&bar, p.col_bytes + p.bit_bytes + p.row_bytes + 16u * (uint32_t)w + (SYM ? q.meta_bytes : 0u));
      if constexpr (SYM) bulk_load(smem + q.off_meta, d.sym_meta + q.meta0, q.meta_bytes, &bar);
      if (p.col_bytes) bulk_load(s_col, col + p.col0, p.col_bytes, &bar);
      if (p.bit_bytes) bulk_load(s_bits, d.bond_bits + p.word0, p.bit_bytes, &bar);
      bulk_load(s_row, d.pd_row + p.row0, p.row_bytes, &bar);
      bulk_load(s_xv, d.xv_mixed + T.win_begin, 16u * (uint32_t)w, &bar);
      s_tile[(k + 1) & 1] = claim();
    }
    const MixParticle M = d.mixp[T.particle];

    // displacements of the window relative to the particle centre's
    {
      const int st = DIM == 2 ? 2 : 4;
      double uc[DIM];
#pragma unroll
      for (int q = 0; q < DIM; q++) uc[q] = d.u[st * T.center + q];
      for (int a = threadIdx.x; a < w; a += kThreadsFor<DIM, LPN>) {
        const int64_t j = T.win_begin + a;
        if constexpr (DIM == 2) {
          const double2 uj = *reinterpret_cast<const double2 *>(d.u + 2 * j);
          s_u2[a] = make_float2((float)(uj.x - uc[0]), (float)(uj.y - uc[1]));
        } else {
          const double2 u01 = *reinterpret_cast<const double2 *>(d.u + 4 * j);
          const double u2 = d.u[4 * j + 2];
          s_u4[a] = make_float4((float)(u01.x - uc[0]), (float)(u01.y - uc[1]), (float)(u2 - uc[2]), 0.f);
        }
        if (state) {
          const double inv_m = 1.0 / d.mx[j];
          s_m[a] = make_float2((float)(d.theta[j] * M.tf_coef * inv_m), (float)(M.am_coef * inv_m));
        }
      }
    }
    __syncthreads();
    const bool landed = bar_wait(&bar, parity);
    parity ^= 1u;
    if (__syncthreads_or(!landed)) {
      // the copies did not land: record it, give them one more bounded wait
      // so that none is left writing into this CTA's shared memory, and stop
      if (threadIdx.x == 0 && atomicCAS(&d.ctrl->error, 0, DEV_ERR_STAGE_TIMEOUT) == 0)
        d.ctrl->error_info = t;
      if (!landed) bar_wait(&bar, parity ^ 1u);
      return;
    }

    View<DIM> V{s_xv, s_u2, s_u4, s_m};
    if constexpr (PRE) tile_theta<DIM, LPN, CT>(d, T, M, V, s_col, s_bits, s_row, p);
    else if constexpr (SYM && DIM == 2) tile_sym<LPN, LAW, CT>(d, T, M, V, s_col, s_bits, s_row, p, q, smem);
    else tile_nodes<DIM, LPN, LAW, CT>(d, T, M, V, s_col, s_bits, s_row, p);
    const int t_next = s_tile[(k + 1) & 1];
    __syncthreads();  // the stage is free for the next tile's copies
    t = t_next;
    k++;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&d.ctrl->tile_done, 1u) == gridDim.x - 1) {
      atomicExch(&d.ctrl->tile_next, 0u);
      atomicExch(&d.ctrl->tile_done, 0u);
      // the surrogate's tile list is rebuilt by the next step's rebuild kernel
      if (!PRE && d.tile_live) atomicExch(d.tile_live_n, 0u);
    }
  }
}

// CTAs per SM for the persistent bond loop: one below the occupancy limit
// (the occupancy limit itself when it is two or less)
template <class K>
int bond_grid(K kernel, int threads, size_t smem, int n_tiles) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
  // one slot per SM stays free for the contact and damping passes when at
  // least three fit; with two, both go to the bond loop
  const int g = sms * (per > 2 ? per - 1 : (per > 0 ? per : 1));
  return g < n_tiles ? g : n_tiles;
}

template <int DIM, int LPN, int LAW, typename CT, bool PRE = false, bool SYM = false>
void launch_one(const DevData &d, const CT *col, const BondTile *t, int n, size_t smem, cudaStream_t s) {
  auto *k = k_bonds_mixed<DIM, LPN, LAW, CT, PRE, SYM>;
  constexpr int kT = kThreadsFor<DIM, LPN>;
  k<<<bond_grid(k, kT, smem, n), kT, smem, s>>>(d, t, n, col);
}

template <int DIM, int LAW, typename CT, bool PRE = false, bool SYM = false>
void launch_law(const DevData &d, const CT *col, const BondTile *t, int n, int lanes, size_t smem,
                cudaStream_t s) {
  switch (lanes) {
    case 1: launch_one<DIM, 1, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
    case 2: launch_one<DIM, 2, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
    case 4: launch_one<DIM, 4, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
    case 8: launch_one<DIM, 8, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
    case 16: launch_one<DIM, 16, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
    default: launch_one<DIM, 32, LAW, CT, PRE, SYM>(d, col, t, n, smem, s); break;
  }
}

// the symmetric form: 2-D, 16-bit columns
void launch_sym(const DevData &d, const BondTile *t, const int *law_begin, int lanes, size_t smem,
                cudaStream_t s) {
  for (int law = 0; law < 4; law++) {
    const int b = law_begin[law], n = law_begin[law + 1] - b;
    if (n <= 0) continue;
    switch (law) {
      case PDGPU_MAT_RNP: launch_law<2, LAW_RNP, uint16_t, false, true>(d, d.sym_col, t + b, n, lanes, smem, s); break;
      case PDGPU_MAT_PMB: launch_law<2, LAW_PMB, uint16_t, false, true>(d, d.sym_col, t + b, n, lanes, smem, s); break;
      case PDGPU_MAT_PDELASTIC:
        launch_law<2, LAW_ELASTIC, uint16_t, false, true>(d, d.sym_col, t + b, n, lanes, smem, s);
        break;
      default: launch_law<2, LAW_STATE, uint16_t, false, true>(d, d.sym_col, t + b, n, lanes, smem, s); break;
    }
  }
}

// one launch per material law present, each over its run of the tile list
// (the tiles are ordered by law)
template <int DIM, typename CT>
void launch_dim(const DevData &d, const CT *col, const BondTile *t, const int *law_begin, int lanes,
                size_t smem, cudaStream_t s) {
  for (int law = 0; law < 4; law++) {
    const int b = law_begin[law], n = law_begin[law + 1] - b;
    if (n <= 0) continue;
    switch (law) {
      case PDGPU_MAT_RNP: launch_law<DIM, LAW_RNP>(d, col, t + b, n, lanes, smem, s); break;
      case PDGPU_MAT_PMB: launch_law<DIM, LAW_PMB>(d, col, t + b, n, lanes, smem, s); break;
      case PDGPU_MAT_PDELASTIC: launch_law<DIM, LAW_ELASTIC>(d, col, t + b, n, lanes, smem, s); break;
      default: launch_law<DIM, LAW_STATE>(d, col, t + b, n, lanes, smem, s); break;
    }
  }
}

template <int DIM>
void launch_pre(const DevData &d, const BondTile *t, int n, int lanes, size_t smem, cudaStream_t s) {
  using namespace bonds_mixed;
  switch (lanes) {
    case 1: k_prepass_tiled<DIM, 1><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 2: k_prepass_tiled<DIM, 2><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 4: k_prepass_tiled<DIM, 4><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 8: k_prepass_tiled<DIM, 8><<<n, kTileThreads, smem, s>>>(d, t); break;
    case 16: k_prepass_tiled<DIM, 16><<<n, kTileThreads, smem, s>>>(d, t); break;
    default: k_prepass_tiled<DIM, 32><<<n, kTileThreads, smem, s>>>(d, t); break;
  }
}

template <int DIM, int LAW, typename CT, bool PRE = false, bool SYM = false>
bool set_law_limit(size_t bytes) {
  const void *fs[] = {(const void *)k_bonds_mixed<DIM, 1, LAW, CT, PRE, SYM>,
                      (const void *)k_bonds_mixed<DIM, 2, LAW, CT, PRE, SYM>,
                      (const void *)k_bonds_mixed<DIM, 4, LAW, CT, PRE, SYM>,
                      (const void *)k_bonds_mixed<DIM, 8, LAW, CT, PRE, SYM>,
                      (const void *)k_bonds_mixed<DIM, 16, LAW, CT, PRE, SYM>,
                      (const void *)k_bonds_mixed<DIM, 32, LAW, CT, PRE, SYM>};
  for (auto f : fs)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
      return false;
  return true;
}

template <int DIM>
int set_limit(size_t bytes) {
  using bonds_mixed::k_prepass_tiled;
  const void *fs[] = {(const void *)k_prepass_tiled<DIM, 1>, (const void *)k_prepass_tiled<DIM, 2>,
                      (const void *)k_prepass_tiled<DIM, 4>, (const void *)k_prepass_tiled<DIM, 8>,
                      (const void *)k_prepass_tiled<DIM, 16>, (const void *)k_prepass_tiled<DIM, 32>};
  for (auto f : fs)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
      return -1;
  const bool ok = set_law_limit<DIM, LAW_RNP, uint16_t>(bytes) && set_law_limit<DIM, LAW_PMB, uint16_t>(bytes) &&
                  set_law_limit<DIM, LAW_ELASTIC, uint16_t>(bytes) && set_law_limit<DIM, LAW_STATE, uint16_t>(bytes) &&
                  set_law_limit<DIM, LAW_RNP, int32_t>(bytes) && set_law_limit<DIM, LAW_PMB, int32_t>(bytes) &&
                  set_law_limit<DIM, LAW_ELASTIC, int32_t>(bytes) && set_law_limit<DIM, LAW_STATE, int32_t>(bytes) &&
                  set_law_limit<DIM, LAW_STATE, uint16_t, true>(bytes) &&
                  set_law_limit<DIM, LAW_STATE, int32_t, true>(bytes);
  if (!ok) return -1;
  if constexpr (DIM == 2) {
    const bool sym = set_law_limit<2, LAW_RNP, uint16_t, false, true>(bytes) &&
                     set_law_limit<2, LAW_PMB, uint16_t, false, true>(bytes) &&
                     set_law_limit<2, LAW_ELASTIC, uint16_t, false, true>(bytes) &&
                     set_law_limit<2, LAW_STATE, uint16_t, false, true>(bytes);
    if (!sym) return -1;
  }
  return 0;
}

}  // namespace mixed_loop

void launch_pd_tiled_mixed(const DevData &d, const BondTile *t, const int *law_begin, int lanes,
                           size_t smem, cudaStream_t s) {
  using namespace mixed_loop;
  if (d.use_sym && d.dim == 2 && d.use16) {
    launch_sym(d, t, law_begin, lanes, smem, s);
    return;
  }
  if (d.use16) {
    if (d.dim == 2) launch_dim<2>(d, d.pd_col16, t, law_begin, lanes, smem, s);
    else launch_dim<3>(d, d.pd_col16, t, law_begin, lanes, smem, s);
  } else {
    if (d.dim == 2) launch_dim<2>(d, (const int32_t *)d.pd_col, t, law_begin, lanes, smem, s);
    else launch_dim<3>(d, (const int32_t *)d.pd_col, t, law_begin, lanes, smem, s);
  }
}

// PD state pre-pass over the tiles of state-based particles, persistent like
// the bond loop
void launch_prepass_mixed(const DevData &d, const BondTile *t, const int *law_begin, int lanes, size_t smem,
                          cudaStream_t s) {
  using namespace mixed_loop;
  const int b = law_begin[PDGPU_MAT_PDSTATE], n = law_begin[PDGPU_MAT_PDSTATE + 1] - b;
  if (n <= 0) return;
  if (d.use16) {
    if (d.dim == 2) launch_law<2, LAW_STATE, uint16_t, true>(d, d.pd_col16, t + b, n, lanes, smem, s);
    else launch_law<3, LAW_STATE, uint16_t, true>(d, d.pd_col16, t + b, n, lanes, smem, s);
  } else {
    const int32_t *col = (const int32_t *)d.pd_col;
    if (d.dim == 2) launch_law<2, LAW_STATE, int32_t, true>(d, col, t + b, n, lanes, smem, s);
    else launch_law<3, LAW_STATE, int32_t, true>(d, col, t + b, n, lanes, smem, s);
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

size_t tile_smem_mixed_main(int dim, bool state, bool col16, const BondTile &t, bool sym) {
  const mixed_loop::Plan p = mixed_loop::plan(dim, state, col16 ? 2 : 4, t.bond_begin, t.bond_end, t.node_begin,
                                              t.node_end, t.win_end - t.win_begin);
  return sym ? mixed_loop::sym_plan(p, t.node_begin, t.node_end, t.slots).total : p.total;
}

int set_tile_smem_limit_mixed(int dim, size_t bytes) {
  return dim == 2 ? mixed_loop::set_limit<2>(bytes) : mixed_loop::set_limit<3>(bytes);
}

}  // namespace pdgpu
