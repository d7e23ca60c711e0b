// Mixed-precision bond loop: the same bond laws as the FP64 kernels of
// DEMModel::computePeridynamicForces (demModel.cpp:602-789), evaluated in
// FP32 on particle-local reference coordinates.  The relative displacement
// u_j - u_i is formed in FP64 and rounded once, the stretch uses the
// cancellation-free form
//     s = (2 xi.eta + eta.eta) / (|xi| (|xi + eta| + |xi|)),
// and lane partial forces are reduced in FP64.  Integration, boundary
// conditions, contact and all reductions stay in FP64.
#include <cstdint>

#include "pdgpu_internal.h"

namespace pdgpu {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ bool is_greater_f(float a, float b) {
  const float fa = fabsf(a), fb = fabsf(b);
  return (a - b) > ((fa < fb ? fb : fa) * 1.0e-5f);
}

template <int LPN>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (LPN == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << LPN) - 1u) << (lane / LPN * LPN);
  }
}

template <int LPN>
__device__ __forceinline__ double group_sum(double v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
  return v;
}
template <int LPN>
__device__ __forceinline__ float group_max(float v, unsigned m) {
#pragma unroll
  for (int o = LPN / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(m, v, o));
  return v;
}

template <int DIM>
__device__ __forceinline__ void ldxl(const float *__restrict__ a, int64_t i, float (&o)[3]) {
  if constexpr (DIM == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(a) + i);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = 0.f;
  } else {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(a) + i);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
  }
}

template <int DIM>
__device__ __forceinline__ void ldu(const double *__restrict__ a, int64_t i, double (&o)[3]) {
  if constexpr (DIM == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(a) + i);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = 0.0;
  } else {
    const double2 *p = reinterpret_cast<const double2 *>(a) + 2 * i;
    const double2 t0 = __ldg(p), t1 = __ldg(p + 1);
    o[0] = t0.x;
    o[1] = t0.y;
    o[2] = t1.x;
  }
}

template <int DIM>
__device__ __forceinline__ float dotf(const float (&a)[3], const float (&b)[3]) {
  float s = a[0] * b[0] + a[1] * b[1];
  if constexpr (DIM == 3) s += a[2] * b[2];
  return s;
}

__device__ __forceinline__ float influence_f(const DevData &d, float q) {
  if (d.inf.type == PDGPU_INF_LINEAR) return d.inf_p0 + d.inf_p1 * q;
  if (d.inf.type == PDGPU_INF_CONST) return d.inf_p0;
  return d.inf_p0 * __expf(-q * q / d.inf_p1);
}

template <bool USE16>
__device__ __forceinline__ int64_t neighbor(const DevData &d, int64_t k, int64_t start) {
  if constexpr (USE16) return start + (int64_t)__ldg(d.pd_col16 + k);
  else return (int64_t)__ldg(d.pd_col + k);
}

// state-based pre-pass (demModel.cpp:610-679) in FP32
template <int DIM, int LPN, bool USE16>
__global__ void __launch_bounds__(kBlock) k_prepass_mixed(DevData d) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / LPN;
  const int lane = threadIdx.x % LPN;
  if (i >= d.n_nodes) return;
  if (!(d.flags[i] & NODE_ACTIVE) || d.ctrl->error) return;
  const MixParticle P = d.mixp[d.ptid[i]];
  if (P.material != PDGPU_MAT_PDSTATE) return;
  const unsigned gm = group_mask<LPN>();
  float xi[3];
  double ui[3];
  ldxl<DIM>(d.xl, i, xi);
  ldu<DIM>(d.u, i, ui);
  float theta = 0.f;
  const int64_t k0 = d.pd_row[i], k1 = d.pd_row[i + 1];
  for (int64_t k = k0 + lane; k < k1; k += LPN) {
    const int64_t j = neighbor<USE16>(d, k, P.start);
    float xj[3], xi_[3], eta[3];
    double uj[3];
    ldxl<DIM>(d.xl, j, xj);
    ldu<DIM>(d.u, j, uj);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      xi_[q] = xj[q] - xi[q];
      eta[q] = (float)(uj[q] - ui[q]);
    }
    const float r = sqrtf(dotf<DIM>(xi_, xi_));
    float y[3];
#pragma unroll
    for (int q = 0; q < 3; q++) y[q] = xi_[q] + eta[q];
    const float l = sqrtf(dotf<DIM>(y, y));
    const float cl = (2.f * dotf<DIM>(xi_, eta) + dotf<DIM>(eta, eta)) / (l + r);
    const float s = cl / r;
    const uint32_t bit = 1u << (k & 31);
    bool fs = (d.bond_bits[k >> 5] & bit) != 0;
    if (!fs && is_greater_f(fabsf(s), P.s0 + 1.0e-10f)) {
      fs = true;
      atomicOr(d.bond_bits + (k >> 5), bit);
    }
    if (!fs) {
      float volj = __ldg(d.volf + j);
      if (is_greater_f(r, P.check_low)) volj *= (P.check_up - r) * P.inv_h;
      theta += r * cl * influence_f(d, r * P.inv_horizon) * volj;
    }
  }
  const double th = group_sum<LPN>((double)theta, gm);
  if (lane == 0) d.theta[i] = 3.0 * th / d.mx[i];
}

template <int DIM, int LPN, bool USE16>
__global__ void __launch_bounds__(kBlock) k_pd_force_mixed(DevData d) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / LPN;
  const int lane = threadIdx.x % LPN;
  if (i >= d.n_nodes) return;
  if (d.ctrl->error) return;
  const int st = DIM == 2 ? 2 : 4;
  if (!(d.flags[i] & NODE_ACTIVE)) {
    if (lane == 0)
      for (int q = 0; q < DIM; q++) d.f[st * i + q] = 0.0;
    return;
  }
  const unsigned gm = group_mask<LPN>();
  const MixParticle P = d.mixp[d.ptid[i]];
  const int mat = P.material;
  float xi[3];
  double ui[3];
  ldxl<DIM>(d.xl, i, xi);
  ldu<DIM>(d.u, i, ui);
  const float mi = (float)d.mx[i];
  const float thi = (float)d.theta[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, zmax = 0.f;
  const int64_t k0 = d.pd_row[i], k1 = d.pd_row[i + 1];
  for (int64_t k = k0 + lane; k < k1; k += LPN) {
    const int64_t j = neighbor<USE16>(d, k, P.start);
    const uint32_t bit = 1u << (k & 31);
    bool fs = (d.bond_bits[k >> 5] & bit) != 0;
    float xj[3], xi_[3], eta[3];
    double uj[3];
    ldxl<DIM>(d.xl, j, xj);
    ldu<DIM>(d.u, j, uj);
    float volj = __ldg(d.volf + j);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      xi_[q] = xj[q] - xi[q];
      eta[q] = (float)(uj[q] - ui[q]);
    }
    const float r2 = dotf<DIM>(xi_, xi_);
    const float r = sqrtf(r2);
    float y[3];
#pragma unroll
    for (int q = 0; q < 3; q++) y[q] = xi_[q] + eta[q];
    float S, sc, l = 0.f;
    if (mat == PDGPU_MAT_RNP) {
      S = dotf<DIM>(xi_, eta) / r2;
      sc = P.rbar * rsqrtf(r);
    } else {
      l = sqrtf(dotf<DIM>(y, y));
      S = (2.f * dotf<DIM>(xi_, eta) + dotf<DIM>(eta, eta)) / (r * (l + r));
      sc = mat == PDGPU_MAT_PDELASTIC ? 3.4e38f : P.s0;
    }
    if (!fs) {
      if (is_greater_f(r, P.check_low)) volj *= (P.check_up - r) * P.inv_h;
      const float J = influence_f(d, r * P.inv_horizon);
      if (mat == PDGPU_MAT_PDSTATE) {
        const float mj = (float)__ldg(d.mx + j), thj = (float)__ldg(d.theta + j);
        const float cl = S * r;
        const float ai = 15.f * P.G / mi, aj = 15.f * P.G / mj;
        const float fi = 3.f * P.K / mi - ai * (1.f / 3.f), fj = 3.f * P.K / mj - aj * (1.f / 3.f);
        const float sf = J * (r * (thi * fi + thj * fj) + cl * (ai + aj)) * volj / l;
        fx += sf * y[0];
        fy += sf * y[1];
        if constexpr (DIM == 3) fz += sf * y[2];
      } else if (mat == PDGPU_MAT_RNP) {
        if (P.irreversible && is_greater_f(fabsf(S), P.factor_sc * sc)) {
          fs = true;
          atomicOr(d.bond_bits + (k >> 5), bit);
        }
        if (!fs) {
          const float sf = J * P.k_force * S * __expf(-P.beta * r * S * S) * volj / r;
          fx += sf * xi_[0];
          fy += sf * xi_[1];
          if constexpr (DIM == 3) fz += sf * xi_[2];
        }
      } else {
        if (mat == PDGPU_MAT_PMB && is_greater_f(fabsf(S), P.s0 + 1.0e-10f)) {
          fs = true;
          atomicOr(d.bond_bits + (k >> 5), bit);
        }
        if (!fs) {
          const float sf = J * P.k_force * S * volj / l;
          fx += sf * y[0];
          fy += sf * y[1];
          if constexpr (DIM == 3) fz += sf * y[2];
        }
      }
    } else {
      const float R = sqrtf(dotf<DIM>(y, y));
      float sf = P.kn * volj * (R - P.rc) / R;
      if (sf > 0.f) sf = 0.f;
      fx += sf * y[0];
      fy += sf * y[1];
      if constexpr (DIM == 3) fz += sf * y[2];
    }
    zmax = fmaxf(zmax, fabsf(S / sc));
  }
  const double Fx = group_sum<LPN>((double)fx, gm);
  const double Fy = group_sum<LPN>((double)fy, gm);
  const double Fz = DIM == 3 ? group_sum<LPN>((double)fz, gm) : 0.0;
  zmax = group_max<LPN>(zmax, gm);
  if (lane == 0) {
    d.f[st * i] = Fx;
    d.f[st * i + 1] = Fy;
    if constexpr (DIM == 3) d.f[st * i + 2] = Fz;
    d.Z[i] = zmax;
  }
}

// particle-local FP32 reference coordinates and volumes, 16-bit offsets
template <int DIM>
__global__ void k_mixed_setup(DevData d) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n_nodes) return;
  const int st = DIM == 2 ? 2 : 4;
  const int32_t p = d.ptid[i];
  const DevParticle &P = d.particles[p];
  float o[4] = {0.f, 0.f, 0.f, 0.f};
  for (int q = 0; q < DIM; q++) o[q] = (float)(d.xref[st * i + q] - d.xref[st * P.center + q]);
  if (DIM == 2) reinterpret_cast<float2 *>(d.xl)[i] = make_float2(o[0], o[1]);
  else reinterpret_cast<float4 *>(d.xl)[i] = make_float4(o[0], o[1], o[2], 0.f);
  d.volf[i] = (float)d.vol[i];
  if (d.use16)
    for (int64_t k = d.pd_row[i]; k < d.pd_row[i + 1]; k++)
      d.pd_col16[k] = (uint16_t)(d.pd_col[k] - P.start);
}

inline unsigned blocks_for(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

template <int DIM, bool U16>
void force_mixed(const DevData &d, int lanes, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes * lanes, kBlock);
  switch (lanes) {
    case 4: k_pd_force_mixed<DIM, 4, U16><<<g, kBlock, 0, s>>>(d); break;
    case 8: k_pd_force_mixed<DIM, 8, U16><<<g, kBlock, 0, s>>>(d); break;
    case 16: k_pd_force_mixed<DIM, 16, U16><<<g, kBlock, 0, s>>>(d); break;
    default: k_pd_force_mixed<DIM, 32, U16><<<g, kBlock, 0, s>>>(d); break;
  }
}

template <int DIM, bool U16>
void prepass_mixed(const DevData &d, int lanes, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes * lanes, kBlock);
  switch (lanes) {
    case 4: k_prepass_mixed<DIM, 4, U16><<<g, kBlock, 0, s>>>(d); break;
    case 8: k_prepass_mixed<DIM, 8, U16><<<g, kBlock, 0, s>>>(d); break;
    case 16: k_prepass_mixed<DIM, 16, U16><<<g, kBlock, 0, s>>>(d); break;
    default: k_prepass_mixed<DIM, 32, U16><<<g, kBlock, 0, s>>>(d); break;
  }
}

}  // namespace

void launch_pd_force_mixed(const DevData &d, int lanes, cudaStream_t s) {
  if (d.dim == 2) {
    if (d.use16) force_mixed<2, true>(d, lanes, s);
    else force_mixed<2, false>(d, lanes, s);
  } else {
    if (d.use16) force_mixed<3, true>(d, lanes, s);
    else force_mixed<3, false>(d, lanes, s);
  }
}

void launch_pd_prepass_mixed(const DevData &d, int lanes, cudaStream_t s) {
  if (d.dim == 2) {
    if (d.use16) prepass_mixed<2, true>(d, lanes, s);
    else prepass_mixed<2, false>(d, lanes, s);
  } else {
    if (d.use16) prepass_mixed<3, true>(d, lanes, s);
    else prepass_mixed<3, false>(d, lanes, s);
  }
}

void launch_mixed_setup(const DevData &d, cudaStream_t s) {
  const unsigned g = blocks_for(d.n_nodes, 256);
  if (d.dim == 2) k_mixed_setup<2><<<g, 256, 0, s>>>(d);
  else k_mixed_setup<3><<<g, 256, 0, s>>>(d);
}

}  // namespace pdgpu
