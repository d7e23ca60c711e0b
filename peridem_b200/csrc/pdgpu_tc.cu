// Tensor-core GEMM of the learned surrogate: C = act(A B^T + bias), BF16
// operands, FP32 accumulation in tensor memory (tcgen05.mma, kind::f16,
// cta_group::1), one 128-row tile of C per CTA and up to 256 columns per
// tile (blockIdx.y walks wider outputs).
//
//   A: M x K, row-major (K contiguous), BF16
//   B: N x K, row-major (K contiguous), BF16   (a weight matrix W[out][in])
//   C: M x N, row-major, FP32 and/or BF16; act: 0 none, 1 tanh
//
// Operand tiles are written by the CTA's threads into shared memory in the
// canonical no-swizzle K-major layout of the tensor core (8-row x 16-byte
// core matrices; the next core along K is LBO bytes on, the next along M/N
// SBO bytes on); one elected thread issues the MMAs and commits them to an
// mbarrier; the accumulator is read back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = rows 32w..32w+31 of the tile).
//
// Limits: K a multiple of 16, N a multiple of 16, lda/ldb/ldc multiples of 8
// elements, A, B, bias and C 16-byte aligned.  Waits are bounded: on timeout the kernel sets
// *err and returns after a further bounded wait for its own MMAs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "pdgpu_internal.h"

namespace pdgpu {
namespace tc {

constexpr int kRows = 128;     // tile rows (MMA M)
// K per shared-memory stage: 64, or 32 for 256-column tiles (48 KB static limit)
constexpr int kThreads = 128;  // 4 warps: one per 32 TMEM lanes
constexpr unsigned kTries = 1u << 24;

__device__ __forceinline__ uint32_t sa(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm100)
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4)                    // D format F32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((uint32_t)(n >> 3) << 17)  // N / 8
         | ((uint32_t)(kRows >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   sa(bar))
               : "memory");
}

// non-blocking test of the phase (test_wait, not try_wait: no suspension
// window between polls)
__device__ __forceinline__ bool bar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  for (unsigned t = 0; t < kTries; t++)
    if (bar_try(bar, parity)) return true;
  return false;
}

// 8 columns of this warp's 32 TMEM lanes into registers; the caller waits
// (tcgen05.wait::ld) before reading them
__device__ __forceinline__ void ld8_nowait(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int q = 0; q < 8; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 8; q++) v[q] = __uint_as_float(r[q]);
}

// byte offset of element (r, k) of an R-row tile in the canonical layout:
// core (r / 8, k / 8) at ((k / 8) * (R / 8) + r / 8) * 128, row r % 8 at 16 B
__device__ __forceinline__ uint32_t tile_off(int r, int k8, int R) {
  return (uint32_t)((k8 * (R / 8) + (r >> 3)) * 128 + (r & 7) * 16);
}

// one 128 x N tile of C at (row0, col0); called by every thread of the CTA
template <int N>
__device__ __forceinline__ void gemm_tile(const __nv_bfloat16 *__restrict__ A, int lda,
                                          const __nv_bfloat16 *__restrict__ B, int ldb, int M, int Ntot, int K,
                                          const float *__restrict__ bias, int act, float *__restrict__ Cf,
                                          __nv_bfloat16 *__restrict__ Cb, int ldc, int *err, int row0, int col0) {
  constexpr uint32_t kCols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  constexpr int kKc = N >= 256 ? 32 : 64;
  __shared__ __align__(128) unsigned char sA[kRows * kKc * 2];
  __shared__ __align__(128) unsigned char sB[N * kKc * 2];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(&tmem_base)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t id = idesc(N);
  bool ok = true;
  uint32_t parity = 0;
  // stage tiles: every thread issues all its global loads first (fixed trip
  // counts, so they are in flight together), then writes shared memory; rows
  // past M / Ntot and columns past K are zero.  The loads of stage s + 1 are
  // issued right after the MMAs of stage s, so they overlap them.
  constexpr int k8f = kKc / 8;                // 16-byte vectors per row in a full stage
  constexpr int kA = kRows * k8f / kThreads;  // per thread
  constexpr int kB = (N * k8f + kThreads - 1) / kThreads;
  uint4 ra[kA], rb[kB];
  auto load_stage = [&](int k0) {
    const int kc = min(kKc, K - k0);
#pragma unroll
    for (int t = 0; t < kA; t++) {
      const int v = threadIdx.x + t * kThreads;
      const int r = v / k8f, k8 = v % k8f;
      ra[t] = make_uint4(0, 0, 0, 0);
      if (row0 + r < M && 8 * k8 < kc)
        ra[t] = *reinterpret_cast<const uint4 *>(A + (size_t)(row0 + r) * lda + k0 + 8 * k8);
    }
#pragma unroll
    for (int t = 0; t < kB; t++) {
      const int v = threadIdx.x + t * kThreads;
      const int r = v / k8f, k8 = v % k8f;
      rb[t] = make_uint4(0, 0, 0, 0);
      if (v < N * k8f && col0 + r < Ntot && 8 * k8 < kc)
        rb[t] = *reinterpret_cast<const uint4 *>(B + (size_t)(col0 + r) * ldb + k0 + 8 * k8);
    }
  };
  load_stage(0);
  for (int k0 = 0; k0 < K; k0 += kKc) {
    const int kc = min(kKc, K - k0);  // a multiple of 16
#pragma unroll
    for (int t = 0; t < kA; t++) {
      const int v = threadIdx.x + t * kThreads;
      *reinterpret_cast<uint4 *>(sA + tile_off(v / k8f, v % k8f, kRows)) = ra[t];
    }
#pragma unroll
    for (int t = 0; t < kB; t++) {
      const int v = threadIdx.x + t * kThreads;
      if (v < N * k8f) *reinterpret_cast<uint4 *>(sB + tile_off(v / k8f, v % k8f, N)) = rb[t];
    }
    // generic-proxy writes become visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t lboA = (kRows / 8) * 128, lboB = (N / 8) * 128;
      for (int s = 0; s < kc / 16; s++) {
        const uint64_t da = sdesc(sa(sA) + 2 * s * lboA, lboA, 128);
        const uint64_t db = sdesc(sa(sB) + 2 * s * lboB, lboB, 128);
        mma(tmem, da, db, id, (k0 > 0 || s > 0) ? 1u : 0u);
      }
      commit(&bar);
    }
    if (k0 + kKc < K) load_stage(k0 + kKc);  // in flight during the MMAs
    // the stage is reused only after the MMAs that read it completed
    const bool landed = bar_wait(&bar, parity);
    parity ^= 1u;
    if (__syncthreads_or(!landed)) {
      ok = false;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (ok) {
    // epilogue: warp w owns rows 32w + lane; 32 columns per TMEM wait; each
    // thread writes its 8 consecutive columns as one 32-byte sector (FP32)
    // or 16 bytes (BF16)
    const int r = row0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < N; c += 32) {
      float v[32];
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (c + 8 * j < N) ld8_nowait(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c + 8 * j), v + 8 * j);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int col = col0 + c + 8 * j;
        if (c + 8 * j >= N || col >= Ntot || r >= M) continue;
        float x[8];
        if (bias) {
          const float4 b0 = *reinterpret_cast<const float4 *>(bias + col);
          const float4 b1 = *reinterpret_cast<const float4 *>(bias + col + 4);
          const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
          for (int q = 0; q < 8; q++) x[q] = v[8 * j + q] + bb[q];
        } else {
#pragma unroll
          for (int q = 0; q < 8; q++) x[q] = v[8 * j + q];
        }
        if (act == 1) {
#pragma unroll
          for (int q = 0; q < 8; q++) x[q] = tanhf(x[q]);
        }
        if (Cf) {
          float4 *o = reinterpret_cast<float4 *>(Cf + (size_t)r * ldc + col);
          o[0] = make_float4(x[0], x[1], x[2], x[3]);
          o[1] = make_float4(x[4], x[5], x[6], x[7]);
        }
        if (Cb) {
          __nv_bfloat162 h[4];
#pragma unroll
          for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
          *reinterpret_cast<uint4 *>(Cb + (size_t)r * ldc + col) = *reinterpret_cast<const uint4 *>(h);
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
    bar_wait(&bar, parity ^ 1u);  // let the committed MMAs finish before TMEM is freed
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
  }
}

template <int N>
__global__ void __launch_bounds__(kThreads) k_gemm(const __nv_bfloat16 *__restrict__ A, int lda,
                                                   const __nv_bfloat16 *__restrict__ B, int ldb, int M,
                                                   int Ntot, int K, const float *__restrict__ bias, int act,
                                                   float *__restrict__ Cf, __nv_bfloat16 *__restrict__ Cb,
                                                   int ldc, int *err) {
  gemm_tile<N>(A, lda, B, ldb, M, Ntot, K, bias, act, Cf, Cb, ldc, err, blockIdx.x * kRows, blockIdx.y * N);
}

// several independent problems in one launch: blockIdx.z picks the problem,
// CTAs outside its M x N extent return before touching tensor memory
template <int N>
__global__ void __launch_bounds__(kThreads) k_gemm_grouped(const GemmProblem *__restrict__ probs, int *err) {
  const GemmProblem p = probs[blockIdx.z];
  const int row0 = blockIdx.x * kRows, col0 = blockIdx.y * N;
  if (row0 >= p.M || col0 >= p.N) return;  // uniform over the CTA
  gemm_tile<N>(static_cast<const __nv_bfloat16 *>(p.A), p.lda, static_cast<const __nv_bfloat16 *>(p.B), p.ldb,
               p.M, p.N, p.K, p.bias, p.act, p.Cf, static_cast<__nv_bfloat16 *>(p.Cb), p.ldc, err, row0, col0);
}

}  // namespace tc

// C = act(A B^T + bias) on `stream`; returns a CUDA error code of the launch
int launch_tc_gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K, const float *bias,
                   int act, float *Cf, void *Cb, int ldc, int *err, cudaStream_t s) {
  using namespace tc;
  if (M <= 0 || N <= 0 || K <= 0 || K % 16 || N % 16 || lda % 8 || ldb % 8 || ldc % 8) return (int)cudaErrorInvalidValue;
  auto a16 = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  if (!a16(A) || !a16(B) || !a16(bias) || !a16(Cf) || !a16(Cb)) return (int)cudaErrorInvalidValue;
  const auto *a = static_cast<const __nv_bfloat16 *>(A);
  const auto *b = static_cast<const __nv_bfloat16 *>(B);
  auto *cb = static_cast<__nv_bfloat16 *>(Cb);
  const unsigned gx = (unsigned)((M + kRows - 1) / kRows);
  if (N <= 32) k_gemm<32><<<dim3(gx, 1), kThreads, 0, s>>>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, ldc, err);
  else if (N <= 64) k_gemm<64><<<dim3(gx, 1), kThreads, 0, s>>>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, ldc, err);
  else if (N <= 128) k_gemm<128><<<dim3(gx, 1), kThreads, 0, s>>>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, ldc, err);
  else k_gemm<256><<<dim3(gx, (unsigned)((N + 255) / 256)), kThreads, 0, s>>>(a, lda, b, ldb, M, N, K, bias, act, Cf, cb, ldc, err);
  return (int)cudaGetLastError();
}

// n_probs problems (device array) in one launch with tiles of ncol (32,
// 64, 128 or 256) columns; max_m / max_n bound every problem's M / N.  The
// problems' K, N, lda, ldb obey the limits above (checked by the caller).
int launch_tc_gemm_grouped(const GemmProblem *probs, int n_probs, int max_m, int max_n, int ncol, int *err,
                           cudaStream_t s) {
  using namespace tc;
  if (n_probs <= 0 || max_m <= 0 || max_n <= 0) return (int)cudaErrorInvalidValue;
  const dim3 grid((unsigned)((max_m + kRows - 1) / kRows), (unsigned)((max_n + ncol - 1) / ncol), (unsigned)n_probs);
  switch (ncol) {
    case 32: k_gemm_grouped<32><<<grid, kThreads, 0, s>>>(probs, err); break;
    case 64: k_gemm_grouped<64><<<grid, kThreads, 0, s>>>(probs, err); break;
    case 128: k_gemm_grouped<128><<<grid, kThreads, 0, s>>>(probs, err); break;
    case 256: k_gemm_grouped<256><<<grid, kThreads, 0, s>>>(probs, err); break;
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

}  // namespace pdgpu

extern "C" PDGPU_API int pdgpu_tc_gemm(const void *A, int32_t lda, const void *B, int32_t ldb, int32_t M,
                                      int32_t N, int32_t K, const float *bias, int32_t act, float *Cf,
                                      void *Cb, int32_t ldc, int32_t *err, void *stream) {
  if (!A || !B || !err || (!Cf && !Cb)) return PDGPU_ERR_ARG;
  const int rc = pdgpu::launch_tc_gemm(A, lda, B, ldb, M, N, K, bias, act, Cf, Cb, ldc, err,
                                       (cudaStream_t)stream);
  return rc == 0 ? PDGPU_OK : (rc == (int)cudaErrorInvalidValue ? PDGPU_ERR_ARG : PDGPU_ERR_CUDA);
}
