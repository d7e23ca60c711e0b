// Learned surrogate of the bond loop (2-D): per reference shape, a particle's
// displacement in its body frame, u_b = R(-theta) (u_i - u_centre) / scale,
// is projected on 32 displacement modes, mapped by an MLP 32-256-256-32
// (tanh) to residual force coefficients, and [network output, projected
// input] is lifted by [residual force modes, tangent force of each mode] to
// the body-frame force density; f_i = fscale R(theta) f_b.  This file holds
//   the step's chain, by warp-level BF16 MMA beside the bond loop:
//            gather + projection (partial sums per node chunk), the three
//            layers, the lift with the scatter into f; after the bond
//            loop, the check-step comparison and the gate
//   the kernels around the tcgen05 GEMMs (pdgpu_tc.cu) of the other chain
//   and of training:
//            gather u -> BF16 rows (and FP32 rows for snapshots), scatter of
//            FP32 rows -> f, gate; MSE gradient, tanh backward, column sums
//            (bias gradients), BF16 transpose, Adam
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

// ---- the CUDA-core chain of the step; the shapes travel by value in the
// kernel parameters, so that no CTA waits on a load of them ----

// ---- warp-level MMA (m16n8k16, BF16 operands, FP32 accumulation) ----
__device__ __forceinline__ void mma_bf16_16816(float *d, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// physical column of logical column c (0..63) of a K-permuted 64-column row
__device__ __forceinline__ int perm_col64(int c) { return 2 * sur_kperm(c >> 1, 4) + (c & 1); }

// A fragments of k-step ks from a row-major BF16 tile in shared memory (ld
// elements per row, logical column order): rows g and g + 8
__device__ __forceinline__ void frag_a(const __nv_bfloat16 *A, int ld, int ks, int g, int tig, uint32_t *a) {
  const uint32_t *r0 = reinterpret_cast<const uint32_t *>(A + g * ld) + 8 * ks + tig;
  const uint32_t *r1 = reinterpret_cast<const uint32_t *>(A + (g + 8) * ld) + 8 * ks + tig;
  a[0] = r0[0];
  a[1] = r1[0];
  a[2] = r0[4];
  a[3] = r1[4];
}

// B fragments of the four k-steps of a 64-input K-permuted chunk (row_chunk:
// the chunk's first 32-bit pair): lane t's eight pairs are adjacent
__device__ __forceinline__ void frag_b_load(const uint32_t *row_chunk, int tig, uint4 *q) {
  const uint4 *src = reinterpret_cast<const uint4 *>(row_chunk + 8 * tig);
  q[0] = __ldg(src);
  q[1] = __ldg(src + 1);
}
__device__ __forceinline__ void frag_b_of(const uint4 *q, int kl, uint32_t *b) {
  const uint4 v = q[kl >> 1];
  b[0] = (kl & 1) ? v.z : v.x;
  b[1] = (kl & 1) ? v.w : v.y;
}

// Gather and projection in one pass, by warp MMA.  The projection
// x = A phi^T has one row per particle, 32 columns and K = 2 n_nodes: a long
// reduction with little work per row.  It is split over CTAs: a CTA takes
// kProjRows rows (particles; row P is the zero input) and kProjNodes nodes
// (256 of K).  Its phi^T fragments (K-permuted rows, 32 bytes per lane and
// 64-input chunk) are requested first; the body-frame displacements,
// rounded to BF16, go to shared memory; warp w forms column tile w % 4 over
// half of the CTA's K, and the two halves are added in a fixed order.  The
// CTA's partial sums go to xpart[row][chunk][32]; the layers' kernel adds
// the chunks in a fixed order, so the result does not depend on scheduling.
constexpr int kProjRows = 16;
constexpr int kProjNodes = 128;
constexpr int kProjThreads = 256;
constexpr int kProjLd = 2 * kProjNodes + 8;  // BF16 per row of the displacement tile

__global__ void __launch_bounds__(kProjThreads) k_gather_project(const double *__restrict__ u,
                                                                 const __grid_constant__ SurShapes shapes) {
  __shared__ __align__(16) __nv_bfloat16 s_a[kProjRows * kProjLd];
  __shared__ __align__(16) float s_red[kProjRows][32];
  __shared__ int64_t s_node[kProjRows][2];  // first node, centre node
  __shared__ double s_rot[kProjRows][3];    // c, s, 1 / scale
  const SurShapeDev &S = shapes.s[blockIdx.z];
  const int k0 = blockIdx.x * kProjRows, a0 = blockIdx.y * kProjNodes;
  if (k0 > S.P || a0 >= S.n_nodes) return;
  const int nrow = min(kProjRows, S.P - k0);  // rows with a particle; the rest are zero
  const int na = min(kProjNodes, S.n_nodes - a0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const int nt = warp & 3, half = warp >> 2;  // column tile, half of the CTA's K
  // phi^T: row 8 nt + g, the two 64-input chunks of this half
  const uint32_t *ph = (const uint32_t *)S.phiT + (size_t)(8 * nt + g) * (S.n_chunks * 128) + blockIdx.y * 128;
  uint4 bq[2][2];
#pragma unroll
  for (int c = 0; c < 2; c++) frag_b_load(ph + 32 * (2 * half + c), tig, bq[c]);
  if ((int)threadIdx.x < nrow) {
    const SurPart sp = S.parts[k0 + threadIdx.x];
    s_node[threadIdx.x][0] = sp.start;
    s_node[threadIdx.x][1] = sp.center;
    s_rot[threadIdx.x][0] = sp.c;
    s_rot[threadIdx.x][1] = sp.s;
    s_rot[threadIdx.x][2] = sp.inv_scale;
  }
  __syncthreads();
  constexpr int kItems = kProjRows * kProjNodes / kProjThreads;  // (row, node) pairs per thread
  constexpr int kBatch = 4;
#pragma unroll
  for (int q0 = 0; q0 < kItems; q0 += kBatch) {
    double2 v[kBatch], c[kBatch];
#pragma unroll
    for (int q = 0; q < kBatch; q++) {
      const int e = threadIdx.x + (q0 + q) * kProjThreads, r = e / kProjNodes, a = e % kProjNodes;
      v[q] = c[q] = make_double2(0.0, 0.0);
      if (r < nrow && a < na) {
        v[q] = *reinterpret_cast<const double2 *>(u + 2 * (s_node[r][0] + a0 + a));
        c[q] = *reinterpret_cast<const double2 *>(u + 2 * s_node[r][1]);
      }
    }
#pragma unroll
    for (int q = 0; q < kBatch; q++) {
      const int e = threadIdx.x + (q0 + q) * kProjThreads, r = e / kProjNodes, a = e % kProjNodes;
      float b0 = 0.f, b1 = 0.f;
      if (r < nrow && a < na) {
        const double *R = s_rot[r];
        const double d0 = v[q].x - c[q].x, d1 = v[q].y - c[q].y;
        // R(-theta) d / scale
        b0 = (float)((R[0] * d0 + R[1] * d1) * R[2]);
        b1 = (float)((-R[1] * d0 + R[0] * d1) * R[2]);
      }
      *reinterpret_cast<__nv_bfloat162 *>(s_a + r * kProjLd + 2 * a) = __floats2bfloat162_rn(b0, b1);
    }
  }
  __syncthreads();
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int kl = 0; kl < 4; kl++) {
      uint32_t a[4], b[2];
      frag_a(s_a, kProjLd, 4 * (2 * half + c) + kl, g, tig, a);
      frag_b_of(bq[c], kl, b);
      mma_bf16_16816(acc, a, b);
    }
  // rows g and g + 8, columns 8 nt + 2 tig (+1): the second half adds its
  // partial sums to the first half's
  const int col = 8 * nt + 2 * tig;
  if (half == 1) {
    s_red[g][col] = acc[0];
    s_red[g][col + 1] = acc[1];
    s_red[g + 8][col] = acc[2];
    s_red[g + 8][col + 1] = acc[3];
  }
  __syncthreads();
  if (half == 1) return;
  float *xp = S.xpart + blockIdx.y * 32 + col;
  const size_t ld = (size_t)S.n_chunks * 32;
  if (k0 + g <= S.P) {
    xp[(k0 + g) * ld] = acc[0] + s_red[g][col];
    xp[(k0 + g) * ld + 1] = acc[1] + s_red[g][col + 1];
  }
  if (k0 + g + 8 <= S.P) {
    xp[(k0 + g + 8) * ld] = acc[2] + s_red[g + 8][col];
    xp[(k0 + g + 8) * ld + 1] = acc[3] + s_red[g + 8][col + 1];
  }
}

// The three layers of the network for 16 rows (rows 0..P, P the zero input)
// per CTA by warp MMA, 16 warps.  The projected input x is the sum of the
// projection's chunks in chunk order, rounded to BF16 (and stored in xy for
// the lift); activations stay in shared memory as BF16 rows (padded so that
// fragment loads do not conflict), with the bias and tanh applied to the
// FP32 accumulators as the tensor-core chain does.  Every weight fragment a
// warp needs (K-permuted rows, 32 bytes per lane and 64-input chunk) is
// requested at the start, so that the layers wait for one round of loads.
//   h1 = tanh(x W1^T + b1), h2 = tanh(h1 W2^T + b2): warp w, columns 16w..16w+15
//   y  = h2 W3^T + b3 -> xy (columns 0..31): warp w, columns 8 (w % 4).., inputs
//        64 (w / 4)..; the four input quarters added in a fixed order
constexpr int kMlpRows = 16;
constexpr int kMlpThreads = 512;
constexpr int kMlpLdX = 32 + 8, kMlpLdH = 256 + 8;

__global__ void __launch_bounds__(kMlpThreads) k_mlp(const __grid_constant__ SurShapes shapes) {
  __shared__ __align__(16) __nv_bfloat16 s_x[kMlpRows * kMlpLdX];
  __shared__ __align__(16) __nv_bfloat16 s_h1[kMlpRows * kMlpLdH];
  __shared__ __align__(16) __nv_bfloat16 s_h2[kMlpRows * kMlpLdH];
  __shared__ float s_y[4][kMlpRows][32];  // layer 3's partial sums per input quarter
  const SurShapeDev &S = shapes.s[blockIdx.y];
  const int k0 = blockIdx.x * kMlpRows;
  if (k0 > S.P) return;
  const int nrow = min(kMlpRows, S.P + 1 - k0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const uint32_t *W1 = (const uint32_t *)S.w1m, *W2 = (const uint32_t *)S.w2m, *W3 = (const uint32_t *)S.w3m;
  // every weight fragment of this warp: layer 1 (32 inputs: one chunk of two
  // k-steps, 16 bytes per lane), layer 2 (four chunks), layer 3 (one chunk)
  uint4 w1q[2], w2q[4][2][2], w3q[2];
#pragma unroll
  for (int t = 0; t < 2; t++)
    w1q[t] = __ldg(reinterpret_cast<const uint4 *>(W1 + (16 * warp + 8 * t + g) * 16) + tig);
#pragma unroll
  for (int ch = 0; ch < 4; ch++)
#pragma unroll
    for (int t = 0; t < 2; t++) frag_b_load(W2 + (16 * warp + 8 * t + g) * 128 + 32 * ch, tig, w2q[ch][t]);
  const int nt3 = warp & 3, q3 = warp >> 2;  // layer 3: column tile, input quarter
  frag_b_load(W3 + (8 * nt3 + g) * 128 + 32 * q3, tig, w3q);
  __nv_bfloat16 *xy = (__nv_bfloat16 *)S.xy;
  {
    const int r = threadIdx.x >> 5, c = threadIdx.x & 31;  // kMlpThreads = kMlpRows x 32
    float x = 0.f;
    if (r < nrow) {
      const float *xp = S.xpart + (size_t)(k0 + r) * S.n_chunks * 32 + c;
      for (int ch = 0; ch < S.n_chunks; ch++) x += xp[32 * ch];
    }
    const __nv_bfloat16 xb = __float2bfloat16(x);
    if (r < nrow) xy[(size_t)(k0 + r) * 64 + perm_col64(32 + c)] = xb;
    s_x[r * kMlpLdX + c] = xb;
  }
  __syncthreads();
  float acc[2][4];
  // layer 1
#pragma unroll
  for (int t = 0; t < 2; t++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[t][q] = 0.f;
#pragma unroll
  for (int kl = 0; kl < 2; kl++) {
    uint32_t a[4];
    frag_a(s_x, kMlpLdX, kl, g, tig, a);
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const uint32_t b[2] = {kl ? w1q[t].z : w1q[t].x, kl ? w1q[t].w : w1q[t].y};
      mma_bf16_16816(acc[t], a, b);
    }
  }
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int col = 16 * warp + 8 * t + 2 * tig;
    const float b0 = S.b1[col], b1 = S.b1[col + 1];
    *reinterpret_cast<__nv_bfloat162 *>(s_h1 + g * kMlpLdH + col) =
        __floats2bfloat162_rn(tanhf(acc[t][0] + b0), tanhf(acc[t][1] + b1));
    *reinterpret_cast<__nv_bfloat162 *>(s_h1 + (g + 8) * kMlpLdH + col) =
        __floats2bfloat162_rn(tanhf(acc[t][2] + b0), tanhf(acc[t][3] + b1));
  }
  __syncthreads();
  // layer 2: four 64-input chunks
#pragma unroll
  for (int t = 0; t < 2; t++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[t][q] = 0.f;
#pragma unroll
  for (int ch = 0; ch < 4; ch++)
#pragma unroll
    for (int kl = 0; kl < 4; kl++) {
      uint32_t a[4];
      frag_a(s_h1, kMlpLdH, 4 * ch + kl, g, tig, a);
#pragma unroll
      for (int t = 0; t < 2; t++) {
        uint32_t b[2];
        frag_b_of(w2q[ch][t], kl, b);
        mma_bf16_16816(acc[t], a, b);
      }
    }
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int col = 16 * warp + 8 * t + 2 * tig;
    const float b0 = S.b2[col], b1 = S.b2[col + 1];
    *reinterpret_cast<__nv_bfloat162 *>(s_h2 + g * kMlpLdH + col) =
        __floats2bfloat162_rn(tanhf(acc[t][0] + b0), tanhf(acc[t][1] + b1));
    *reinterpret_cast<__nv_bfloat162 *>(s_h2 + (g + 8) * kMlpLdH + col) =
        __floats2bfloat162_rn(tanhf(acc[t][2] + b0), tanhf(acc[t][3] + b1));
  }
  __syncthreads();
  // layer 3: this warp's column tile over its quarter of the inputs
  float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int kl = 0; kl < 4; kl++) {
    uint32_t a[4], b[2];
    frag_a(s_h2, kMlpLdH, 4 * q3 + kl, g, tig, a);
    frag_b_of(w3q, kl, b);
    mma_bf16_16816(y, a, b);
  }
  {
    const int col = 8 * nt3 + 2 * tig;
    s_y[q3][g][col] = y[0];
    s_y[q3][g][col + 1] = y[1];
    s_y[q3][g + 8][col] = y[2];
    s_y[q3][g + 8][col + 1] = y[3];
  }
  __syncthreads();
  {
    const int r = threadIdx.x >> 5, c = threadIdx.x & 31;
    if (r < nrow) {
      const float v = ((s_y[0][r][c] + s_y[1][r][c]) + s_y[2][r][c]) + s_y[3][r][c];
      xy[(size_t)(k0 + r) * 64 + perm_col64(c)] = __float2bfloat16(v + S.b3[c]);
    }
  }
}

// The lift fused with the scatter, by warp MMA: a CTA takes kLiftRows - 1
// particles plus the zero input (row P) as the 16 rows of one tile, and
// kLiftNodes nodes (2 kLiftNodes dofs, four 8-dof column tiles per warp);
// K = 64 (the coefficients [y | x], stored K-permuted like the lift's rows,
// so that each lane's fragments of a row are 32 contiguous bytes).  A lane's
// accumulators hold, per column tile, one node's two components for two
// rows, so g = F_k - F_P (the zero input's row of the same tile, fetched
// from the lane that holds it: zero deformation gives exactly zero force) is
// rotated and stored as it stands.  Ordinary steps: f_i = fscale R(theta) g
// for the particles on the surrogate, whose tiles the bond loop skips, so
// that this runs beside it; check steps: g into F for the comparison after
// the bond loop.  count[0] counts particle-steps on the surrogate, count[1]
// particle-steps covered.
constexpr int kLiftRows = 16;           // 15 particles + the zero input
constexpr int kLiftNodes = 128;
constexpr int kLiftThreads = 256;       // 8 warps x 4 column tiles x 4 nodes
constexpr int kLiftTiles = 2 * kLiftNodes / 8 / (kLiftThreads / 32);

__global__ void __launch_bounds__(kLiftThreads) k_lift_scatter(double *__restrict__ f,
                                                               const __grid_constant__ SurShapes shapes,
                                                               const uint8_t *__restrict__ on,
                                                               const uint8_t *__restrict__ near,
                                                               const CtrlState *ctrl,
                                                               unsigned long long *__restrict__ count) {
  __shared__ SurPart s_part[kLiftRows - 1];
  __shared__ int s_use[kLiftRows - 1];
  const SurShapeDev &S = shapes.s[blockIdx.z];
  const int k0 = blockIdx.x * (kLiftRows - 1), a0 = blockIdx.y * kLiftNodes;
  if (k0 >= S.P || a0 >= S.n_nodes) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const int nrow = min(kLiftRows - 1, S.P - k0);
  // B fragments: the lift's K-permuted rows [kpad][64]; the warp's column
  // tiles cover dofs d0 + 8 t .. d0 + 8 t + 7 (rows past 2 n_nodes are zero)
  const uint32_t *L = (const uint32_t *)S.liftm;
  const int d0 = 2 * a0 + warp * 8 * kLiftTiles;
  uint4 bq[kLiftTiles][2];
#pragma unroll
  for (int t = 0; t < kLiftTiles; t++) {
    const int dof = d0 + 8 * t + g;
    if (dof < S.kpad) frag_b_load(L + (size_t)dof * 32, tig, bq[t]);
    else bq[t][0] = bq[t][1] = make_uint4(0, 0, 0, 0);
  }
  // A fragments: rows g and g + 8 of the tile; tile row 15 (and rows past
  // the shape's particles) read the zero input's row P
  const uint32_t *X = (const uint32_t *)S.xy;
  const int ra = (g < nrow) ? k0 + g : S.P;
  const int rb = (g + 8 < nrow) ? k0 + g + 8 : S.P;
  uint4 aq[2][2];
  frag_b_load(X + (size_t)ra * 32, tig, aq[0]);
  frag_b_load(X + (size_t)rb * 32, tig, aq[1]);
  const bool check = ctrl->sur_check != 0;
  const bool error = ctrl->error != 0;
  if (threadIdx.x < kLiftRows - 1) {
    int use = 0;
    if ((int)threadIdx.x < nrow) {
      const SurPart sp = S.parts[k0 + threadIdx.x];
      s_part[threadIdx.x] = sp;
      use = check || (on[sp.particle] && !near[sp.particle]);
    }
    s_use[threadIdx.x] = use;
  }
  __syncthreads();
  if (error) return;
  int n_use = 0;
#pragma unroll
  for (int r = 0; r < kLiftRows - 1; r++) n_use += s_use[r];
  if (threadIdx.x == 0 && blockIdx.y == 0) {
    if (!check && n_use) atomicAdd(&count[0], (unsigned long long)n_use);
    atomicAdd(&count[1], (unsigned long long)nrow);
  }
  if (n_use == 0) return;  // uniform over the CTA
  float acc[kLiftTiles][4];
#pragma unroll
  for (int t = 0; t < kLiftTiles; t++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[t][q] = 0.f;
#pragma unroll
  for (int kl = 0; kl < 4; kl++) {
    uint32_t ar[2], br[2], a[4];
    frag_b_of(aq[0], kl, ar);  // row g: pairs (h = 0, h = 1)
    frag_b_of(aq[1], kl, br);  // row g + 8
    a[0] = ar[0];
    a[1] = br[0];
    a[2] = ar[1];
    a[3] = br[1];
#pragma unroll
    for (int t = 0; t < kLiftTiles; t++) {
      uint32_t b[2];
      frag_b_of(bq[t], kl, b);
      mma_bf16_16816(acc[t], a, b);
    }
  }
  // lanes 28..31 hold tile row 15 (g = 7, second half): the zero input
  const int ua = g < nrow && s_use[g], ub = g + 8 < nrow && s_use[g + 8];
#pragma unroll
  for (int t = 0; t < kLiftTiles; t++) {
    const float p0 = __shfl_sync(0xffffffffu, acc[t][2], 28 + tig);
    const float p1 = __shfl_sync(0xffffffffu, acc[t][3], 28 + tig);
    const int a = (d0 + 8 * t) / 2 + tig;  // node of this lane's dofs 2a, 2a + 1
    if (a >= S.n_nodes) continue;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = g + 8 * h;
      if (!(h ? ub : ua)) continue;
      const float g0 = acc[t][2 * h] - p0, g1 = acc[t][2 * h + 1] - p1;
      if (check) {
        *reinterpret_cast<float2 *>(S.F + (size_t)(k0 + r) * S.kpad + 2 * a) = make_float2(g0, g1);
      } else {
        const SurPart &sp = s_part[r];
        const double f0 = sp.fscale * (sp.c * (double)g0 - sp.s * (double)g1);
        const double f1 = sp.fscale * (sp.s * (double)g0 + sp.c * (double)g1);
        *reinterpret_cast<double2 *>(f + 2 * (sp.start + a)) = make_double2(f0, f1);
      }
    }
  }
}

// Check steps, after the bond loop: per particle |f_s - f|^2 and |f|^2 from
// the body-frame rows F, then the gate; a grid of one CTA per SM that leaves
// at once on other steps.
__global__ void __launch_bounds__(256) k_check_all(const DevData d, const __grid_constant__ SurShapes shapes,
                                                   double *__restrict__ err2, float z_gate, double err_gate2) {
  __shared__ double red[2][8];
  if (d.ctrl->error || !d.ctrl->sur_check) return;
  for (int sh = 0; sh < shapes.n; sh++) {
    const SurShapeDev &S = shapes.s[sh];
    for (int k = blockIdx.x; k < S.P; k += gridDim.x) {
      const SurPart sp = S.parts[k];
      const float *F = S.F + (size_t)k * S.kpad;
      double e = 0.0, nrm = 0.0;
      for (int a = threadIdx.x; a < S.n_nodes; a += blockDim.x) {
        const double g0 = F[2 * a], g1 = F[2 * a + 1];
        const double f0 = sp.fscale * (sp.c * g0 - sp.s * g1);
        const double f1 = sp.fscale * (sp.s * g0 + sp.c * g1);
        const int64_t i = sp.start + a;
        const double r0 = d.f[2 * i], r1 = d.f[2 * i + 1];
        e += (f0 - r0) * (f0 - r0) + (f1 - r1) * (f1 - r1);
        nrm += r0 * r0 + r1 * r1;
      }
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
      gate_one(d, sp, err2, z_gate, err_gate2);
      __syncthreads();  // before red and the gate's shared words are reused
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

void launch_sur_gather_project(const double *u, const SurShapes &shapes, int max_p, int max_nodes, cudaStream_t s) {
  const dim3 g((unsigned)((max_p + 1 + sur::kProjRows - 1) / sur::kProjRows),
               (unsigned)((max_nodes + sur::kProjNodes - 1) / sur::kProjNodes), (unsigned)shapes.n);
  sur::k_gather_project<<<g, sur::kProjThreads, 0, s>>>(u, shapes);
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

void launch_sur_mlp(const SurShapes &shapes, int max_p, cudaStream_t s) {
  const dim3 g((unsigned)((max_p + 1 + sur::kMlpRows - 1) / sur::kMlpRows), (unsigned)shapes.n);
  sur::k_mlp<<<g, sur::kMlpThreads, 0, s>>>(shapes);
}

void launch_sur_lift_scatter(double *f, const SurShapes &shapes, int max_p, int max_nodes, const uint8_t *on,
                             const uint8_t *near, const CtrlState *ctrl, unsigned long long *count, cudaStream_t s) {
  if (max_p <= 0) return;
  const dim3 g((unsigned)((max_p + sur::kLiftRows - 2) / (sur::kLiftRows - 1)),
               (unsigned)((max_nodes + sur::kLiftNodes - 1) / sur::kLiftNodes), (unsigned)shapes.n);
  sur::k_lift_scatter<<<g, sur::kLiftThreads, 0, s>>>(f, shapes, on, near, ctrl, count);
}

void launch_sur_check_all(const DevData &d, const SurShapes &shapes, double *err2, float z_gate, double err_gate,
                          cudaStream_t s) {
  sur::k_check_all<<<(unsigned)sm_count(), 256, 0, s>>>(d, shapes, err2, z_gate, err_gate * err_gate);
}

int sur_n_chunks(int n_nodes) { return (n_nodes + sur::kProjNodes - 1) / sur::kProjNodes; }

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
