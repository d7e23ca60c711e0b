// Learned surrogate of the bond loop (2-D): per reference shape, a particle's
// displacement in its body frame, u_b = R(-theta) (u_i - u_centre) / scale,
// is projected on 32 displacement modes, mapped by an MLP 32-256-256-32
// (tanh) to residual force coefficients, and [network output, projected
// input] is lifted by [residual force modes, tangent force of each mode] to
// the body-frame force density; f_i = fscale R(theta) f_b.  The GEMMs run on
// the tensor cores (pdgpu_tc.cu); this file holds the element-wise and
// data-movement kernels around them, for inference in the step and for
// training:
//   gather   u -> BF16 rows (and FP32 rows for snapshots)
//   scatter  FP32 rows -> f (surrogate particles only) and, on check steps,
//            per-particle error of the surrogate against the bond loop
//   gate     per-particle verdict on check steps
//   training: MSE gradient, tanh backward, column sums (bias gradients),
//            BF16 transpose, Adam
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "pdgpu_internal.h"

namespace pdgpu {
namespace sur {

// one CTA per particle of the list; row k of A holds particle parts[k]
__global__ void k_gather(const double *__restrict__ u, const SurPart *__restrict__ parts, int P, int n_nodes,
                         __nv_bfloat16 *__restrict__ A, int lda, float *__restrict__ Af) {
  const int k = blockIdx.x;
  if (k >= P) return;
  const SurPart sp = parts[k];
  const double uc0 = u[2 * sp.center], uc1 = u[2 * sp.center + 1];
  for (int a = threadIdx.x; a < lda / 2; a += blockDim.x) {
    float b0 = 0.f, b1 = 0.f;
    if (a < n_nodes) {
      const int64_t i = sp.start + a;
      const double d0 = u[2 * i] - uc0, d1 = u[2 * i + 1] - uc1;
      // R(-theta) d / scale
      b0 = (float)((sp.c * d0 + sp.s * d1) * sp.inv_scale);
      b1 = (float)((-sp.s * d0 + sp.c * d1) * sp.inv_scale);
    }
    A[(size_t)k * lda + 2 * a] = __float2bfloat16(b0);
    A[(size_t)k * lda + 2 * a + 1] = __float2bfloat16(b1);
    if (Af) {
      Af[(size_t)k * lda + 2 * a] = b0;
      Af[(size_t)k * lda + 2 * a + 1] = b1;
    }
  }
}

// Body-frame FP32 force rows -> f (k_scatter_all below): row P of F is the
// chain's output for a zero input (row P of the gathered input is never
// written): it is subtracted, so zero deformation gives exactly zero force
// whatever the roundings of the chain.  count[0] counts particle-steps on
// the surrogate, count[1] particle-steps covered.

// Check steps: a particle keeps (or gets) the surrogate when none of its
// bonds is broken, its damage Z = max |S| / s_c stays below z_gate and the
// surrogate's force error against the bond loop, |f_s - f|, is below
// err_gate max(|f|, floor); one CTA per surrogate particle.
__device__ void gate_one(const DevData &d, const SurPart &sp, const double *__restrict__ err2, float z_gate,
                         double err_gate2) {
  __shared__ int broken_s;
  __shared__ float zmax_s;
  if (d.ctrl->error || !d.ctrl->sur_check) return;
  const DevParticle &Pp = d.particles[sp.particle];
  if (threadIdx.x == 0) {
    broken_s = 0;
    zmax_s = 0.f;
  }
  __syncthreads();
  float z = 0.f;
  for (int64_t i = Pp.start + threadIdx.x; i < Pp.end; i += blockDim.x) z = fmaxf(z, d.Z[i]);
  const int64_t b0 = d.pd_row[Pp.start], b1 = d.pd_row[Pp.end];
  int broken = 0;
  if (b1 > b0)
    for (int64_t w = (b0 >> 5) + threadIdx.x; w <= ((b1 - 1) >> 5); w += blockDim.x) {
      uint32_t m = d.bond_bits[w];
      if (w == (b0 >> 5)) m &= ~0u << (b0 & 31);
      if (w == ((b1 - 1) >> 5)) m &= ~0u >> (31 - ((b1 - 1) & 31));
      broken |= m != 0u;
    }
  for (int o = 16; o > 0; o >>= 1) {
    z = fmaxf(z, __shfl_xor_sync(0xffffffffu, z, o));
    broken |= __shfl_xor_sync(0xffffffffu, broken, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(reinterpret_cast<int *>(&zmax_s), __float_as_int(z));  // z >= 0
    if (broken) broken_s = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double e = err2[2 * sp.particle], n = err2[2 * sp.particle + 1];
    const bool ok = !broken_s && zmax_s < z_gate && e <= err_gate2 * fmax(n, sp.floor2);
    d.sur_on[sp.particle] = ok ? 1 : 0;
  }
}

// ---- training ----
// dY = scale (Y - T) (FP32 and BF16); *loss += sum (Y - T)^2
__global__ void k_mse_grad(const float *Y, const float *T, int64_t n, float scale, float *dY,
                           __nv_bfloat16 *dYb, double *loss) {
  __shared__ double red[32];
  double l = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float r = Y[i] - T[i];
    dY[i] = scale * r;
    dYb[i] = __float2bfloat16(scale * r);
    l += (double)r * r;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    atomicAdd(loss, s);
  }
}

// dZ = dH (1 - H^2) for H = tanh(Z) (FP32 and BF16)
__global__ void k_tanh_back(const float *dH, const float *H, int64_t n, float *dZ, __nv_bfloat16 *dZb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float h = H[i];
    const float g = dH[i] * (1.f - h * h);
    dZ[i] = g;
    dZb[i] = __float2bfloat16(g);
  }
}

// out[c] = sum over rows of X[r][c] (a bias gradient), one thread per column
__global__ void k_colsum(const float *X, int rows, int cols, float *out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; r++) s += X[(size_t)r * cols + c];
  out[c] = s;
}

// out (cols x rows) = in (rows x cols)^T, BF16, through a 32 x 32 shared tile
__global__ void k_transpose(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by + j, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[j][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = bx + j, r = by + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][j];
  }
}

// Adam with bias correction on FP32 master weights; wb (if set) receives the
// BF16 copy the GEMMs read
__global__ void k_adam(float *p, float *m, float *v, const float *g, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2, __nv_bfloat16 *wb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (wb) wb[i] = __float2bfloat16(pi);
  }
}

// Gather and projection in one pass.  The projection x = A phi^T has one
// row per particle, 32 columns and K = 2 n_nodes: a long reduction with
// little work per row, which the tensor-core tiles walk serially on a few
// CTAs.  Here a CTA takes kProjRows rows (particles; row P is the zero
// input): their body-frame displacements, rounded to BF16 (the GEMM's A
// operand), go to shared memory, and each warp forms four of the 32 columns
// for all of them with FP32 accumulation, so that every element of phi^T it
// reads (through the read-only cache) serves kProjRows rows.  Written as
// BF16 into xy[:, 32:64].
constexpr int kProjRows = 8;

__global__ void __launch_bounds__(256) k_gather_project(const double *__restrict__ u,
                                                        const SurShapeDev *__restrict__ shapes) {
  extern __shared__ __align__(16) float s_rows[];  // kProjRows x kpad
  const SurShapeDev S = shapes[blockIdx.y];
  const int k0 = blockIdx.x * kProjRows, kpad = S.kpad;
  if (k0 > S.P) return;
  for (int r = 0; r < kProjRows; r++) {
    const int k = k0 + r;
    float *row = s_rows + (size_t)r * kpad;
    if (k < S.P) {
      const SurPart sp = S.parts[k];
      const double uc0 = u[2 * sp.center], uc1 = u[2 * sp.center + 1];
      for (int a = threadIdx.x; a < kpad / 2; a += blockDim.x) {
        float b0 = 0.f, b1 = 0.f;
        if (a < S.n_nodes) {
          const int64_t i = sp.start + a;
          const double d0 = u[2 * i] - uc0, d1 = u[2 * i + 1] - uc1;
          b0 = (float)((sp.c * d0 + sp.s * d1) * sp.inv_scale);
          b1 = (float)((-sp.s * d0 + sp.c * d1) * sp.inv_scale);
        }
        row[2 * a] = __bfloat162float(__float2bfloat16(b0));
        row[2 * a + 1] = __bfloat162float(__float2bfloat16(b1));
      }
    } else {  // the zero input (k == P) and rows past it
      for (int a = threadIdx.x; a < kpad; a += blockDim.x) row[a] = 0.f;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const __nv_bfloat16 *phiT = (const __nv_bfloat16 *)S.phiT;
  __nv_bfloat16 *xy = (__nv_bfloat16 *)S.xy;
  for (int j = warp; j < 32; j += (int)(blockDim.x >> 5)) {
    const __nv_bfloat162 *ph = reinterpret_cast<const __nv_bfloat162 *>(phiT + (size_t)j * kpad);
    float acc[kProjRows];
#pragma unroll
    for (int r = 0; r < kProjRows; r++) acc[r] = 0.f;
    for (int a = lane; a < kpad / 2; a += 32) {
      const float2 w = __bfloat1622float2(__ldg(ph + a));
#pragma unroll
      for (int r = 0; r < kProjRows; r++) {
        const float2 v = reinterpret_cast<const float2 *>(s_rows + (size_t)r * kpad)[a];
        acc[r] += v.x * w.x;
        acc[r] += v.y * w.y;
      }
    }
#pragma unroll
    for (int r = 0; r < kProjRows; r++) {
      float v = acc[r];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      const int k = k0 + r;
      if (lane == 0 && k <= S.P) xy[(size_t)k * 64 + 32 + j] = __float2bfloat16(v);
    }
  }
}

// k_scatter for every shape in one launch, the step's kind read on the
// device: the forces into f on ordinary steps, the comparison on check steps
__global__ void k_scatter_all(double *__restrict__ f, const SurShapeDev *__restrict__ shapes,
                              const uint8_t *__restrict__ on, const uint8_t *__restrict__ near,
                              const CtrlState *ctrl, double *__restrict__ err2,
                              unsigned long long *__restrict__ count) {
  __shared__ double red[2][32];
  const SurShapeDev S = shapes[blockIdx.y];
  const int k = blockIdx.x;
  if (k >= S.P || ctrl->error) return;
  const SurPart sp = S.parts[k];
  const bool check = ctrl->sur_check != 0;
  const bool use = !check && on[sp.particle] && !near[sp.particle];
  if (threadIdx.x == 0) {
    if (use) atomicAdd(&count[0], 1ull);
    atomicAdd(&count[1], 1ull);
  }
  if (!check && !use) return;
  const int ldf = S.kpad;
  const float *F = S.F, *F0 = S.F + (size_t)S.P * ldf;
  double e = 0.0, nrm = 0.0;
  for (int a = threadIdx.x; a < S.n_nodes; a += blockDim.x) {
    const float g0 = F[(size_t)k * ldf + 2 * a] - F0[2 * a];
    const float g1 = F[(size_t)k * ldf + 2 * a + 1] - F0[2 * a + 1];
    const double f0 = sp.fscale * (sp.c * (double)g0 - sp.s * (double)g1);
    const double f1 = sp.fscale * (sp.s * (double)g0 + sp.c * (double)g1);
    const int64_t i = sp.start + a;
    if (check) {
      const double r0 = f[2 * i], r1 = f[2 * i + 1];
      e += (f0 - r0) * (f0 - r0) + (f1 - r1) * (f1 - r1);
      nrm += r0 * r0 + r1 * r1;
    } else {
      f[2 * i] = f0;
      f[2 * i + 1] = f1;
    }
  }
  if (!check) return;
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = e;
    red[1][threadIdx.x >> 5] = nrm;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double se = 0.0, sn = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      se += red[0][w];
      sn += red[1][w];
    }
    err2[2 * sp.particle] = se;
    err2[2 * sp.particle + 1] = sn;
  }
}

// k_gate for every shape in one launch
__global__ void k_gate_all(const DevData d, const SurShapeDev *__restrict__ shapes, const double *__restrict__ err2,
                           float z_gate, double err_gate2) {
  const SurShapeDev S = shapes[blockIdx.y];
  if ((int)blockIdx.x >= S.P) return;
  gate_one(d, S.parts[blockIdx.x], err2, z_gate, err_gate2);
}

unsigned blocks(int64_t n, int t) {
  const int64_t b = (n + t - 1) / t;
  return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace sur

void launch_sur_gather(const double *u, const SurPart *parts, int P, int n_nodes, void *A, int lda, float *Af,
                       cudaStream_t s) {
  if (P > 0) sur::k_gather<<<P, 256, 0, s>>>(u, parts, P, n_nodes, (__nv_bfloat16 *)A, lda, Af);
}

size_t sur_project_smem(int kpad) { return (size_t)4 * sur::kProjRows * kpad; }

void launch_sur_gather_project(const double *u, const SurShapeDev *shapes, int n_shapes, int max_p, int max_kpad,
                               cudaStream_t s) {
  const dim3 g((unsigned)((max_p + 1 + sur::kProjRows - 1) / sur::kProjRows), (unsigned)n_shapes);
  sur::k_gather_project<<<g, 256, sur_project_smem(max_kpad), s>>>(u, shapes);
}

void launch_sur_scatter_all(double *f, const SurShapeDev *shapes, int n_shapes, int max_p, const uint8_t *on,
                            const uint8_t *near, const CtrlState *ctrl, double *err2, unsigned long long *count,
                            cudaStream_t s) {
  if (max_p > 0) sur::k_scatter_all<<<dim3((unsigned)max_p, (unsigned)n_shapes), 256, 0, s>>>(f, shapes, on, near,
                                                                                             ctrl, err2, count);
}

void launch_sur_gate_all(const DevData &d, const SurShapeDev *shapes, int n_shapes, int max_p, const double *err2,
                         float z_gate, double err_gate, cudaStream_t s) {
  if (max_p > 0)
    sur::k_gate_all<<<dim3((unsigned)max_p, (unsigned)n_shapes), 256, 0, s>>>(d, shapes, err2, z_gate,
                                                                             err_gate * err_gate);
}

int sur_fused_setup(int kpad) {
  // the fused kernel keeps kProjRows rows (kpad floats each) in shared memory
  if (sur_project_smem(kpad) > 227 * 1024 - 1024) return 0;
  return cudaFuncSetAttribute(sur::k_gather_project, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sur_project_smem(kpad)) == cudaSuccess;
}

}  // namespace pdgpu

using namespace pdgpu;

// ---- C ABI: training building blocks on caller-owned device arrays ----
extern "C" {

PDGPU_API int pdgpu_sur_mse_grad(const float *Y, const float *T, int64_t n, float scale, float *dY, void *dYb,
                                 double *loss, void *stream) {
  if (!Y || !T || !dY || !dYb || !loss || n <= 0) return PDGPU_ERR_ARG;
  sur::k_mse_grad<<<sur::blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(Y, T, n, scale, dY,
                                                                          (__nv_bfloat16 *)dYb, loss);
  return cudaGetLastError() == cudaSuccess ? PDGPU_OK : PDGPU_ERR_CUDA;
}

PDGPU_API int pdgpu_sur_tanh_back(const float *dH, const float *H, int64_t n, float *dZ, void *dZb, void *stream) {
  if (!dH || !H || !dZ || !dZb || n <= 0) return PDGPU_ERR_ARG;
  sur::k_tanh_back<<<sur::blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(dH, H, n, dZ, (__nv_bfloat16 *)dZb);
  return cudaGetLastError() == cudaSuccess ? PDGPU_OK : PDGPU_ERR_CUDA;
}

PDGPU_API int pdgpu_sur_colsum(const float *X, int32_t rows, int32_t cols, float *out, void *stream) {
  if (!X || !out || rows <= 0 || cols <= 0) return PDGPU_ERR_ARG;
  sur::k_colsum<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(X, rows, cols, out);
  return cudaGetLastError() == cudaSuccess ? PDGPU_OK : PDGPU_ERR_CUDA;
}

PDGPU_API int pdgpu_sur_transpose(const void *in, int32_t rows, int32_t cols, void *out, void *stream) {
  if (!in || !out || rows <= 0 || cols <= 0) return PDGPU_ERR_ARG;
  const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  sur::k_transpose<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)in, rows, cols,
                                                                    (__nv_bfloat16 *)out);
  return cudaGetLastError() == cudaSuccess ? PDGPU_OK : PDGPU_ERR_CUDA;
}

PDGPU_API int pdgpu_sur_adam(float *p, float *m, float *v, const float *g, int64_t n, float lr, float beta1,
                             float beta2, float eps, int32_t step, void *wb, void *stream) {
  if (!p || !m || !v || !g || n <= 0 || step <= 0) return PDGPU_ERR_ARG;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  sur::k_adam<<<sur::blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(p, m, v, g, n, lr, beta1, beta2, eps, c1, c2,
                                                                      (__nv_bfloat16 *)wb);
  return cudaGetLastError() == cudaSuccess ? PDGPU_OK : PDGPU_ERR_CUDA;
}

}  // extern "C"
