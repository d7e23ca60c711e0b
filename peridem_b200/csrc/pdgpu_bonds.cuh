// Tiled bond loop of DEMModel::computePeridynamicForces
// (demModel.cpp:602-789): one CTA per tile of one particle's nodes; the
// window of node indices the tile's bonds reach is staged in shared memory
// (reference coordinates, displacements, volumes; m_x and dilatation for the
// state-based law), so every neighbour gather is a shared-memory read.
//
// Included twice: by pdgpu_bonds_fp64.cu (PDGPU_BONDS_FP64 defined, compiled
// with --fmad=false; exactly the arithmetic of the reference) and by
// pdgpu_bonds_mixed.cu (FP32 bond arithmetic on particle-local coordinates,
// cancellation-free stretch, fast intrinsics; FP64 reductions).
#pragma once

#include <cfloat>
#include <cstdint>

#include "pdgpu_internal.h"

// Each inclusion gets its own namespace: the two forms share names but not
// arithmetic, so nothing here may have external linkage in common.
#ifdef PDGPU_BONDS_FP64
#define PDGPU_BONDS_NS bonds_fp64
#else
#define PDGPU_BONDS_NS bonds_mixed
#endif

namespace pdgpu {
namespace PDGPU_BONDS_NS {

constexpr int kTileThreads = 256;

#ifdef PDGPU_BONDS_FP64
typedef double real;
#else
typedef float real;
#endif

__device__ __forceinline__ bool gt(real a, real b) {
  const real fa = fabs(a), fb = fabs(b);
  return (a - b) > ((fa < fb ? fb : fa) * (real)1.0e-5);
}

template <int LPN>
__device__ __forceinline__ unsigned gmask() {
  if constexpr (LPN == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << LPN) - 1u) << (lane / LPN * LPN);
  }
}

template <int LPN>
__device__ __forceinline__ double gsum(double v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}
template <int LPN>
__device__ __forceinline__ float gmax(float v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(m, v, o));
  return v;
}

// shared-memory layout of the staged window (structure of arrays)
template <int DIM>
struct Stage {
  real *x[DIM];  // reference coordinates (particle-local in the mixed form)
  real *u[DIM];  // displacements (minus the particle centre's in the mixed form)
  real *vol;
  real *mx, *th;  // state-based law only
  __device__ Stage(void *base, int w, bool state) {
    real *p = reinterpret_cast<real *>(base);
    for (int q = 0; q < DIM; q++) {
      x[q] = p;
      p += w;
    }
    for (int q = 0; q < DIM; q++) {
      u[q] = p;
      p += w;
    }
    vol = p;
    p += w;
    mx = p;
    th = state ? p + w : p;
  }
};

template <int DIM>
__host__ __device__ constexpr int stage_words(bool state) {
  return 2 * DIM + 1 + (state ? 2 : 0);
}

__device__ __forceinline__ real infl(const DevData &d, real r, real horizon, real inv_horizon) {
#ifdef PDGPU_BONDS_FP64
  (void)inv_horizon;
  const double q = r / horizon;
  if (d.inf.type == PDGPU_INF_LINEAR) return d.inf.p0 + d.inf.p1 * q;
  if (d.inf.type == PDGPU_INF_CONST) return d.inf.p0;
  return d.inf.p0 * exp(-q * q / d.inf.p1);
#else
  (void)horizon;
  const float q = r * inv_horizon;
  if (d.inf.type == PDGPU_INF_LINEAR) return d.inf_p0 + d.inf_p1 * q;
  if (d.inf.type == PDGPU_INF_CONST) return d.inf_p0;
  return d.inf_p0 * __expf(-q * q / d.inf_p1);
#endif
}

// Stage the window [w0, w1) of particle p.  Mixed form: coordinates relative
// to the particle centre (reference and displacement), in FP32.
template <int DIM>
__device__ __forceinline__ void stage_window(const DevData &d, const Stage<DIM> &S, int64_t w0,
                                             int w, int64_t center, bool state) {
  const int st = DIM == 2 ? 2 : 4;
#ifndef PDGPU_BONDS_FP64
  double xc[DIM], uc[DIM];
  for (int q = 0; q < DIM; q++) {
    xc[q] = d.xref[st * center + q];
    uc[q] = d.u[st * center + q];
  }
#endif
  for (int a = threadIdx.x; a < w; a += blockDim.x) {
    const int64_t j = w0 + a;
#pragma unroll
    for (int q = 0; q < DIM; q++) {
#ifdef PDGPU_BONDS_FP64
      S.x[q][a] = __ldg(d.xref + st * j + q);
      S.u[q][a] = d.u[st * j + q];
#else
      S.x[q][a] = (float)(__ldg(d.xref + st * j + q) - xc[q]);
      S.u[q][a] = (float)(d.u[st * j + q] - uc[q]);
#endif
    }
    S.vol[a] = (real)__ldg(d.vol + j);
    if (state) {
      S.mx[a] = (real)d.mx[j];
      S.th[a] = (real)d.theta[j];
    }
  }
}

template <int DIM>
__device__ __forceinline__ real dotr(const real (&a)[3], const real (&b)[3]) {
  real s = a[0] * b[0] + a[1] * b[1];
  if constexpr (DIM == 3) s = s + a[2] * b[2];
  return s;
}

// ---------------------------------------------------------------------------
// state-based pre-pass (demModel.cpp:610-679)
// ---------------------------------------------------------------------------
template <int DIM, int LPN>
__global__ void __launch_bounds__(kTileThreads) k_prepass_tiled(DevData d, const BondTile *tiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (d.ctrl->error) return;
  const BondTile T = tiles[blockIdx.x];
  const DevParticle &P = d.particles[T.particle];
  if (P.material != PDGPU_MAT_PDSTATE) return;
  const int w = T.win_end - T.win_begin;
  Stage<DIM> S(smem, w, false);
  stage_window<DIM>(d, S, T.win_begin, w, P.center, false);
  __syncthreads();
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const real horizon = (real)P.horizon, h = (real)P.h;
  const real inv_h = (real)(1.0 / P.h), inv_hor = (real)(1.0 / P.horizon);
  const real up = (real)P.check_up, low = (real)P.check_low;
  const real sc = (real)P.mat[2];
  const int64_t off = P.start - T.win_begin;
  for (int64_t i = T.node_begin + threadIdx.x / LPN; i < T.node_end; i += kTileThreads / LPN) {
    if (!(d.flags[i] & NODE_ACTIVE)) continue;
    const int li = (int)(i - T.win_begin);
    real xi[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
    for (int q = 0; q < DIM; q++) {
      xi[q] = S.x[q][li];
      ui[q] = S.u[q][li];
    }
    double theta = 0.0;
    real th_lane = 0;
    const int64_t k0 = d.pd_row[i], k1 = d.pd_row[i + 1];
    for (int64_t k = k0 + lane; k < k1; k += LPN) {
      const int lj = d.use16 ? (int)(d.pd_col16[k] + off) : (int)(d.pd_col[k] - T.win_begin);
      real dx[3] = {0, 0, 0}, y[3] = {0, 0, 0};
#ifdef PDGPU_BONDS_FP64
      for (int q = 0; q < DIM; q++) {
        dx[q] = S.x[q][lj] - xi[q];
        y[q] = dx[q] + S.u[q][lj] - ui[q];
      }
      const double rji = sqrt(dotr<DIM>(dx, dx));
      const double cl = sqrt(dotr<DIM>(y, y)) - rji;
      const double s = cl / rji;
#else
      real eta[3] = {0, 0, 0};
      for (int q = 0; q < DIM; q++) {
        dx[q] = S.x[q][lj] - xi[q];
        eta[q] = S.u[q][lj] - ui[q];
        y[q] = dx[q] + eta[q];
      }
      const float r2 = dotr<DIM>(dx, dx);
      const float inv_r = rsqrtf(r2);
      const float rji = r2 * inv_r;
      const float l = sqrtf(dotr<DIM>(y, y));
      const float cl = __fdividef(2.f * dotr<DIM>(dx, eta) + dotr<DIM>(eta, eta), l + rji);
      const float s = cl * inv_r;
#endif
      const uint32_t bit = 1u << (k & 31);
      bool fs = (d.bond_bits[k >> 5] & bit) != 0;
      if (!fs && gt(fabs(s), sc + (real)1.0e-10)) {
        fs = true;
        atomicOr(d.bond_bits + (k >> 5), bit);
      }
      if (!fs) {
        real volj = S.vol[lj];
#ifdef PDGPU_BONDS_FP64
        if (gt(rji, low)) volj *= (up - rji) / h;
        theta += rji * cl * infl(d, rji, horizon, inv_hor) * volj;
#else
        if (gt(rji, low)) volj *= (up - rji) * inv_h;
        th_lane += rji * cl * infl(d, rji, horizon, inv_hor) * volj;
#endif
      }
    }
#ifndef PDGPU_BONDS_FP64
    theta = (double)th_lane;
#endif
    theta = gsum<LPN>(theta, gm);
    if (lane == 0) d.theta[i] = 3.0 * theta / d.mx[i];
  }
}

// ---------------------------------------------------------------------------
// main bond loop (demModel.cpp:685-788)
// ---------------------------------------------------------------------------
template <int DIM, int LPN>
__global__ void __launch_bounds__(kTileThreads) k_pd_tiled(DevData d, const BondTile *tiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (d.ctrl->error) return;
  const BondTile T = tiles[blockIdx.x];
  const DevParticle &P = d.particles[T.particle];
  const int mat = P.material;
  const bool state = mat == PDGPU_MAT_PDSTATE;
  const int w = T.win_end - T.win_begin;
  Stage<DIM> S(smem, w, state);
  stage_window<DIM>(d, S, T.win_begin, w, P.center, state);
  __syncthreads();
  const int st = DIM == 2 ? 2 : 4;
  const int lane = threadIdx.x % LPN;
  const unsigned gm = gmask<LPN>();
  const real horizon = (real)P.horizon, h = (real)P.h;
  const real inv_h = (real)(1.0 / P.h), inv_hor = (real)(1.0 / P.horizon);
  const real up = (real)P.check_up, low = (real)P.check_low;
  const real kn = (real)P.kn, rc = (real)P.rc;
  const int64_t off = P.start - T.win_begin;
#ifdef PDGPU_BONDS_FP64
  const double C = P.mat[0], beta = P.mat[1], rbar = P.mat[2], invf = P.mat[3], fsc = P.mat[4];
  const bool irrev = P.mat[5] != 0.0;
  const double c_pmb = P.mat[0], s0 = mat == PDGPU_MAT_PMB ? P.mat[1] : P.mat[2];
  const double K = P.mat[0], G = P.mat[1];
#else
  const MixParticle M = d.mixp[T.particle];
#endif
  for (int64_t i = T.node_begin + threadIdx.x / LPN; i < T.node_end; i += kTileThreads / LPN) {
    if (!(d.flags[i] & NODE_ACTIVE)) {
      if (lane == 0)
        for (int q = 0; q < DIM; q++) d.f[st * i + q] = 0.0;
      continue;
    }
    const int li = (int)(i - T.win_begin);
    real xi[3] = {0, 0, 0}, ui[3] = {0, 0, 0};
    for (int q = 0; q < DIM; q++) {
      xi[q] = S.x[q][li];
      ui[q] = S.u[q][li];
    }
    const real mi = state ? S.mx[li] : (real)1, thi = state ? S.th[li] : (real)0;
    real fx = 0, fy = 0, fz = 0;
    real zmax = 0;
    const int64_t k0 = d.pd_row[i], k1 = d.pd_row[i + 1];
    for (int64_t k = k0 + lane; k < k1; k += LPN) {
      const int lj = d.use16 ? (int)(d.pd_col16[k] + off) : (int)(d.pd_col[k] - T.win_begin);
      const uint32_t bit = 1u << (k & 31);
      bool fs = (d.bond_bits[k >> 5] & bit) != 0;
      real dx[3] = {0, 0, 0}, du[3] = {0, 0, 0}, y[3] = {0, 0, 0};
      for (int q = 0; q < DIM; q++) {
        dx[q] = S.x[q][lj] - xi[q];
        du[q] = S.u[q][lj] - ui[q];
        y[q] = dx[q] + du[q];
      }
      real volj = S.vol[lj];
#ifdef PDGPU_BONDS_FP64
      // exactly the reference's operation order (material.h, demModel.cpp)
      const double rji = sqrt(dotr<DIM>(dx, dx));
      double S_, sc, ly = 0.0;
      if (mat == PDGPU_MAT_RNP) {
        S_ = dotr<DIM>(dx, du) / dotr<DIM>(dx, dx);
        sc = rbar / sqrt(rji);
      } else {
        ly = sqrt(dotr<DIM>(y, y));
        S_ = (ly - rji) / rji;
        sc = mat == PDGPU_MAT_PDELASTIC ? DBL_MAX : s0;
      }
      if (!fs) {
        if (gt(rji, low)) volj *= (up - rji) / h;
        const double J = infl(d, rji, horizon, inv_hor);
        if (state) {
          const double mj = S.mx[lj], thj = S.th[lj];
          const double cl = S_ * rji;
          const double ai = 15. * G / mi, aj = 15. * G / mj;
          const double fi = (3. * K / mi) - ai / 3., fj = (3. * K / mj) - aj / 3.;
          const double efi = J * (rji * thi * fi + cl * ai);
          const double efj = J * (rji * thj * fj + cl * aj);
          const double sf = (efi + efj) * volj;
          fx += sf * (y[0] / ly);
          fy += sf * (y[1] / ly);
          if constexpr (DIM == 3) fz += sf * (y[2] / ly);
        } else if (mat == PDGPU_MAT_RNP) {
          double ef = 0.0;
          if (irrev && !fs && gt(fabs(S_), fsc * sc)) {
            fs = true;
            atomicOr(d.bond_bits + (k >> 5), bit);
          }
          if (!fs) ef = J * 4. * S_ * C * beta * exp(-beta * rji * S_ * S_) / invf;
          const double sf = ef * volj;
          fx += sf * (dx[0] / rji);
          fy += sf * (dx[1] / rji);
          if constexpr (DIM == 3) fz += sf * (dx[2] / rji);
        } else {
          double ef = 0.0;
          if (mat == PDGPU_MAT_PMB && !fs && gt(fabs(S_), s0 + 1.0e-10)) {
            fs = true;
            atomicOr(d.bond_bits + (k >> 5), bit);
          }
          if (!fs) ef = J * c_pmb * S_;
          const double sf = ef * volj;
          fx += sf * (y[0] / ly);
          fy += sf * (y[1] / ly);
          if constexpr (DIM == 3) fz += sf * (y[2] / ly);
        }
      } else {
        // broken bond: y = (xj + uj) - (xi + ui) (demModel.cpp:762)
        double yb[3] = {0, 0, 0};
        for (int q = 0; q < DIM; q++) yb[q] = (S.x[q][lj] + S.u[q][lj]) - (xi[q] + ui[q]);
        const double R = sqrt(dotr<DIM>(yb, yb));
        double sf = kn * volj * (R - rc) / R;
        if (sf > 0.) sf = 0.;
        fx += sf * yb[0];
        fy += sf * yb[1];
        if constexpr (DIM == 3) fz += sf * yb[2];
      }
      zmax = fmax(zmax, fabs(S_ / sc));
#else
      // FP32: rsqrt-based lengths, cancellation-free stretch
      const float r2 = dotr<DIM>(dx, dx);
      const float inv_r = rsqrtf(r2);
      const float rji = r2 * inv_r;
      float S_, inv_sc, ly = 0.f, inv_ly = 0.f;
      if (mat == PDGPU_MAT_RNP) {
        S_ = dotr<DIM>(dx, du) * inv_r * inv_r;
        inv_sc = sqrtf(rji) * (1.f / M.rbar);
      } else {
        const float y2 = dotr<DIM>(y, y);
        inv_ly = rsqrtf(y2);
        ly = y2 * inv_ly;
        S_ = __fdividef(2.f * dotr<DIM>(dx, du) + dotr<DIM>(du, du), rji * (ly + rji));
        inv_sc = mat == PDGPU_MAT_PDELASTIC ? 0.f : 1.f / M.s0;
      }
      if (!fs) {
        if (gt(rji, low)) volj *= (up - rji) * inv_h;
        const float J = infl(d, rji, horizon, inv_hor);
        if (state) {
          const float mj = S.mx[lj], thj = S.th[lj];
          const float ai = __fdividef(15.f * M.G, mi), aj = __fdividef(15.f * M.G, mj);
          const float fi = __fdividef(3.f * M.K, mi) - ai * (1.f / 3.f);
          const float fj = __fdividef(3.f * M.K, mj) - aj * (1.f / 3.f);
          const float sf = J * (rji * (thi * fi + thj * fj) + S_ * rji * (ai + aj)) * volj * inv_ly;
          fx += sf * y[0];
          fy += sf * y[1];
          if constexpr (DIM == 3) fz += sf * y[2];
        } else if (mat == PDGPU_MAT_RNP) {
          if (M.irreversible && gt(fabsf(S_) * inv_sc, M.factor_sc)) {
            fs = true;
            atomicOr(d.bond_bits + (k >> 5), bit);
          }
          if (!fs) {
            const float sf = J * M.k_force * S_ * __expf(-M.beta * rji * S_ * S_) * volj * inv_r;
            fx += sf * dx[0];
            fy += sf * dx[1];
            if constexpr (DIM == 3) fz += sf * dx[2];
          }
        } else {
          if (mat == PDGPU_MAT_PMB && gt(fabsf(S_), M.s0 + 1.0e-10f)) {
            fs = true;
            atomicOr(d.bond_bits + (k >> 5), bit);
          }
          if (!fs) {
            const float sf = J * M.k_force * S_ * volj * inv_ly;
            fx += sf * y[0];
            fy += sf * y[1];
            if constexpr (DIM == 3) fz += sf * y[2];
          }
        }
      } else {
        const float yy = dotr<DIM>(y, y);
        const float inv_R = rsqrtf(yy);
        float sf = kn * volj * (1.f - rc * inv_R);
        if (sf > 0.f) sf = 0.f;
        fx += sf * y[0];
        fy += sf * y[1];
        if constexpr (DIM == 3) fz += sf * y[2];
      }
      zmax = fmaxf(zmax, fabsf(S_) * inv_sc);
#endif
    }
    const double Fx = gsum<LPN>((double)fx, gm);
    const double Fy = gsum<LPN>((double)fy, gm);
    const double Fz = DIM == 3 ? gsum<LPN>((double)fz, gm) : 0.0;
    const float Z = gmax<LPN>((float)zmax, gm);
    if (lane == 0) {
      d.f[st * i] = Fx;
      d.f[st * i + 1] = Fy;
      if constexpr (DIM == 3) d.f[st * i + 2] = Fz;
      d.Z[i] = Z;
    }
  }
}

inline size_t tile_smem_bytes(int dim, bool state, int window) {
  const int words = dim == 2 ? stage_words<2>(state) : stage_words<3>(state);
  return (size_t)words * (size_t)window * sizeof(real);
}

}  // namespace PDGPU_BONDS_NS
}  // namespace pdgpu
