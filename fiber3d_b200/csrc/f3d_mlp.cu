// Tensor-core (tcgen05, sm_100a) BF16 GEMM with FP32 accumulation in tensor
// memory, and the small kernels around it that train and run the per-fiber
// warm-start network (input 192 -> 3 x 256 hidden (ReLU) -> 128 output).
//
// GEMM: C[M x N] (fp32) = op(A[M x K] B[N x K]^T) with A, B given as fp32 with
// arbitrary (row, column) strides — so X W^T, dY W and dY^T X all use the same
// kernel without transposed copies.  Operands are rounded to BF16 while a
// CTA stages them into shared memory in the canonical K-major, no-swizzle
// UMMA layout (8x8 core matrices of 128 bytes; adjacent rows-of-8 are SBO =
// 128 B apart, adjacent K-groups-of-8 are LBO = (rows/8)*128 B apart).  One
// elected thread issues tcgen05.mma.cta_group::1.kind::f16 (M = 128, N <= 256,
// K = 16 per instruction) into a 128 x 256 fp32 accumulator in TMEM, and
// tcgen05.commit signals an mbarrier that the CTA waits on (bounded by
// %globaltimer).  The epilogue reads TMEM with tcgen05.ld.32x32b (warp w owns
// lanes 32w..32w+31 = rows) and fuses bias, ReLU and the ReLU mask of the
// backward pass.  One CTA (128 threads) computes a 128-row x ntile tile
// (grid.y splits N into ntile-column tiles when there are too few row tiles to
// fill the GPU); no TMA multicast, no clusters.
#include <cuda_bf16.h>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kGemmThreads = 128;
constexpr int kKChunk = 64;      // K elements staged per round
constexpr int kTmemCols = 256;   // fp32 accumulator columns (N <= 256)

struct GemmArgs {
  const float *A;  // element (m, k) at A[m * a_rs + k * a_cs]
  const float *B;  // element (n, k) at B[n * b_rs + k * b_cs]
  float *C;        // element (m, n) at C[m * ldc + n]
  const float *bias;      // [N] or null
  const float *mask_src;  // [M x ldm]: epilogue multiplies by (mask_src > 0) when non-null
  float *pre;             // [M x ldc]: pre-activation copy when non-null
  int64_t a_rs, a_cs, b_rs, b_cs, ldc, ldm;
  int M, N, K;
  int ntile;       // columns per CTA (multiple of 16, <= 256)
  int relu;        // apply max(0, .) in the epilogue
  int accumulate;  // C += result
  float alpha;
  int *err;
  uint64_t wait_ns;  // limit of each bounded mbarrier wait
};

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32;
  d |= static_cast<uint64_t>(1) << 46;  // descriptor version (sm_100)
  // base offset 0, legacy LBO mode, layout type 0 = no swizzle
  return d;
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4)                                  // C format F32
         | (1u << 7)                                // A format BF16
         | (1u << 10)                               // B format BF16
         | (static_cast<uint32_t>(N >> 3) << 17)    // N / 8
         | (static_cast<uint32_t>(M >> 4) << 24);   // M / 16
}

// Byte offset of element (r, k) in a K-major no-swizzle tile of `rows` rows.
__device__ __forceinline__ uint32_t core_offset(int r, int k, int rows) {
  return static_cast<uint32_t>(((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Stage a rows x kKChunk operand tile (rows = 128 or ntile) to shared memory.
__device__ __forceinline__ void stage_operand(unsigned char *dst, const float *src, int64_t rs,
                                              int64_t cs, int nrows_valid, int rows, int k0,
                                              int K) {
  // one thread per (row, 8-wide K group): 16-byte shared store
  const int groups = rows * (kKChunk / 8);
  for (int gi = threadIdx.x; gi < groups; gi += kGemmThreads) {
    const int r = gi / (kKChunk / 8);
    const int kg = gi - r * (kKChunk / 8);
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + kg * 8 + j;
      float x = 0.f;
      if (r < nrows_valid && k < K) x = src[static_cast<int64_t>(r) * rs + static_cast<int64_t>(k) * cs];
      v[j] = __float2bfloat16_rn(x);
    }
    *reinterpret_cast<uint4 *>(dst + core_offset(r, kg * 8, rows)) = *reinterpret_cast<const uint4 *>(v);
  }
}

__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_tcgen05_kernel(const GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char gsm[];
  // layout: [A tile 128 x 64 bf16 = 16 KB][B tile 256 x 64 bf16 = 32 KB]
  unsigned char *sA = gsm;
  unsigned char *sB = gsm + 128 * kKChunk * 2;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128;
  const int mvalid = min(128, g.M - m0);
  const int n0 = blockIdx.y * g.ntile;
  const int N = min(g.ntile, g.N - n0);  // multiple of 16, <= 256

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    fence_mbar_init();
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  const uint32_t idesc = umma_idesc_bf16(128, N);
  const uint32_t a_lbo = (128 / 8) * 128, b_lbo = (N / 8) * 128, sbo = 128;
  const int nchunks = (g.K + kKChunk - 1) / kKChunk;
  uint32_t phase = 0;
  bool ok = true;
  for (int c = 0; c < nchunks; ++c) {
    const int k0 = c * kKChunk;
    stage_operand(sA, g.A + static_cast<int64_t>(m0) * g.a_rs, g.a_rs, g.a_cs, mvalid, 128, k0, g.K);
    stage_operand(sB, g.B + static_cast<int64_t>(n0) * g.b_rs, g.b_rs, g.b_cs, N, N, k0, g.K);
    fence_proxy_async_smem();  // generic-proxy stores -> async-proxy (MMA) reads
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int ksteps = min(kKChunk, g.K - k0 + 15) / 16;
      for (int s = 0; s < ksteps && s < kKChunk / 16; ++s) {
        const uint64_t da = umma_smem_desc(smem_addr(sA) + s * 2 * a_lbo, a_lbo, sbo);
        const uint64_t db = umma_smem_desc(smem_addr(sB) + s * 2 * b_lbo, b_lbo, sbo);
        const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&mbar))
                   : "memory");
    }
    // all threads wait for the MMAs of this chunk (shared memory is reused next round)
    const bool done = mbar_wait_bounded(&mbar, phase, g.wait_ns);
    phase ^= 1u;
    if (!done) s_fail = 1;
    __syncthreads();
    if (s_fail) { ok = false; break; }
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 (rows), 16 columns per load
    const int row = warp * 32 + lane;
    const int m = m0 + row;
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t r[16];
      const uint32_t addr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
            "=r"(r[14]), "=r"(r[15])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c0 + j;
          float v = g.alpha * __uint_as_float(r[j]);
          if (g.bias) v += g.bias[n];
          if (g.pre) g.pre[static_cast<int64_t>(m) * g.ldc + n] = v;
          if (g.relu) v = fmaxf(v, 0.f);
          if (g.mask_src && !(g.mask_src[static_cast<int64_t>(m) * g.ldm + n] > 0.f)) v = 0.f;
          float *dst = g.C + static_cast<int64_t>(m) * g.ldc + n;
          *dst = g.accumulate ? *dst + v : v;
        }
      }
    }
  } else if (threadIdx.x == 0) {
    record_error(g.err, F3D_ERR_TIMEOUT);
    (void)mbar_wait_bounded(&mbar, phase ^ 1u, g.wait_ns);  // MMAs still in flight, bounded
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// out[n] (+)= sum_m G[m * ld + n]  (bias gradient), fixed order.
__global__ void colsum_kernel(const float *G, int64_t ld, int M, int N, float *out, int accumulate) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += G[static_cast<int64_t>(m) * ld + n];
  out[n] = accumulate ? out[n] + s : s;
}

// Adam step on fp32 parameters (bias-corrected), gradient already averaged.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int64_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// D = 2 (Y - T) / (M * N) (mean-squared-error gradient); loss partials per row.
__global__ void mse_grad_kernel(const float *Y, const float *T, float *D, float *row_loss, int M,
                                int N) {
  const int m = blockIdx.x;
  if (m >= M) return;
  float s = 0.f;
  const float sc = 2.f / (static_cast<float>(M) * N);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const float d = Y[static_cast<int64_t>(m) * N + n] - T[static_cast<int64_t>(m) * N + n];
    D[static_cast<int64_t>(m) * N + n] = sc * d;
    s += d * d;
  }
  __shared__ float red[32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    row_loss[m] = t;
  }
}

}  // namespace f3d

extern "C" {

int f3d_gemm_bf16(const float *A, int64_t a_rs, int64_t a_cs, const float *B, int64_t b_rs,
                  int64_t b_cs, float *C, int64_t ldc, int32_t M, int32_t N, int32_t K,
                  const float *bias, int relu, const float *mask_src, int64_t ldm, float *pre,
                  float alpha, int accumulate, void *stream) {
  if (!A || !B || !C) return F3D_ERR_NULL;
  if (M < 0 || K < 0 || N < 16 || N > 256 || (N % 16) != 0 || ldc < N) return F3D_ERR_SHAPE;
  if (M == 0) return F3D_OK;
  if (K == 0) return F3D_ERR_SHAPE;
  if (mask_src && ldm < N) return F3D_ERR_SHAPE;
  // Few row tiles (small batches, e.g. one time step's fibers): split N so
  // that more CTAs run; each re-stages its A tile (an L2 hit).
  const int mtiles = (M + 127) / 128;
  int ntile = N;
  while (ntile > 32 && ntile % 32 == 0 && mtiles * (N / ntile) < f3d::sm_count()) ntile /= 2;
  f3d::GemmArgs g{A, B, C, bias, mask_src, pre, a_rs, a_cs, b_rs, b_cs, ldc, ldm,
                  M, N, K, ntile, relu, accumulate, alpha, f3d::device_error_word(),
                  f3d::wait_limit_ns()};
  // 48 KB of operand tiles; ~100 KB is requested so that at most two CTAs
  // share an SM and their two 256-column TMEM allocations always fit.
  const size_t smem = 100 * 1024;
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    if (cudaFuncSetAttribute(f3d::gemm_bf16_tcgen05_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
      return F3D_ERR_CUDA;
    attr[dev] = true;
  }
  const dim3 grid(static_cast<unsigned>(mtiles), static_cast<unsigned>((N + ntile - 1) / ntile));
  f3d::gemm_bf16_tcgen05_kernel<<<grid, f3d::kGemmThreads, smem, static_cast<cudaStream_t>(stream)>>>(g);
  return f3d::launch_status();
}

int f3d_colsum(const float *G, int64_t ld, int32_t M, int32_t N, float *out, int accumulate,
               void *stream) {
  if (!G || !out) return F3D_ERR_NULL;
  if (M < 0 || N < 0 || ld < N) return F3D_ERR_SHAPE;
  if (N == 0) return F3D_OK;
  f3d::colsum_kernel<<<(N + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(G, ld, M, N, out,
                                                                                      accumulate);
  return f3d::launch_status();
}

int f3d_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr, float beta1,
             float beta2, float eps, int32_t step, void *stream) {
  if (!p || !g || !m || !v) return F3D_ERR_NULL;
  if (n < 0 || step < 1) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  const float c1 = 1.f - powf(beta1, static_cast<float>(step));
  const float c2 = 1.f - powf(beta2, static_cast<float>(step));
  f3d::adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return f3d::launch_status();
}

int f3d_mse_grad(const float *Y, const float *T, float *D, float *row_loss, int32_t M, int32_t N,
                 void *stream) {
  if (!Y || !T || !D || !row_loss) return F3D_ERR_NULL;
  if (M < 0 || N < 0) return F3D_ERR_SHAPE;
  if (M == 0) return F3D_OK;
  f3d::mse_grad_kernel<<<M, 128, 0, static_cast<cudaStream_t>(stream)>>>(Y, T, D, row_loss, M, N);
  return f3d::launch_status();
}

}  // extern "C"
