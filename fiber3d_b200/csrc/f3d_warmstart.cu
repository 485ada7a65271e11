// Input features and guess assembly of the learned GMRES warm start (no
// counterpart in fiber3d, whose GMRES starts from zero, tstep/tstep.py:1209).
//
// Solutions are fiber3d's unknown vectors (tstep_utils.py:906-931); fiber f's
// block of 4N entries starts at o_fib + 4N f and holds X_x, X_y, X_z, T (N
// each).  From the last four solutions h0 (oldest) .. h3 (newest):
//   D1 = h3 - h2,  D2 = D1 - (h2 - h1),  D3 = h3 - 3 h2 + 3 h1 - h0,
//   sK_X = rms over the 3N position entries of DK, sK_T over the N tensions,
//   features (4N + 4N + 4): D2_X / s2_X, D3_X / s2_X, D2_T / s2_T,
//   D3_T / s2_T, log10(s3_X / s2_X), log10(s3_T / s2_T), log10(s2_X / s1_X),
//   log10(s2_T / s1_T), each optionally standardised as (v - mean) / std
//   with the network's input statistics.
// Guess: x0 = 3 h3 - 3 h2 + h1 (quadratic extrapolation) everywhere, plus on
// fiber block f the network's normalised correction times s2_X (positions)
// or s2_T (tensions).  One warp per fiber for the features (N = 32: lane j
// owns positions j, j+32, j+64 and tension j); one thread per entry for the
// guess.
#include <math.h>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kWsPts = 32;  // points per fiber the network is built for

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__global__ void warmstart_features_kernel(const double *__restrict__ h0, const double *__restrict__ h1,
                                          const double *__restrict__ h2, const double *__restrict__ h3,
                                          int64_t o_fib, int nfib, const float *__restrict__ mean,
                                          const float *__restrict__ stdev, float *__restrict__ feats,
                                          double *__restrict__ sx, double *__restrict__ st) {
  const int lane = threadIdx.x & 31;
  const int f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (f >= nfib) return;
  const int64_t base = o_fib + static_cast<int64_t>(4 * kWsPts) * f;
  double d1[4], d2[4], d3[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int64_t i = base + lane + 32 * q;
    const double a = h0[i], b = h1[i], c = h2[i], d = h3[i];
    // explicit rounding steps (no contraction): the same arithmetic as the
    // host restatement of the features
    d1[q] = __dsub_rn(d, c);
    d2[q] = __dsub_rn(d1[q], __dsub_rn(c, b));
    d3[q] = __dsub_rn(__dadd_rn(__dsub_rn(d, __dmul_rn(3.0, c)), __dmul_rn(3.0, b)), a);
  }
  const double n3 = 3.0 * kWsPts, n1 = kWsPts;
  const double s1x = sqrt(warp_sum(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]) / n3) + 1e-300;
  const double s2x = sqrt(warp_sum(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]) / n3) + 1e-300;
  const double s3x = sqrt(warp_sum(d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2]) / n3) + 1e-300;
  const double s1t = sqrt(warp_sum(d1[3] * d1[3]) / n1) + 1e-300;
  const double s2t = sqrt(warp_sum(d2[3] * d2[3]) / n1) + 1e-300;
  const double s3t = sqrt(warp_sum(d3[3] * d3[3]) / n1) + 1e-300;
  float *o = feats + static_cast<int64_t>(8 * kWsPts + 4) * f;
  auto put = [&](int j, double v) {
    float x = static_cast<float>(v);
    if (mean) x = (x - mean[j]) / stdev[j];
    o[j] = x;
  };
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    put(lane + 32 * q, d2[q] / s2x);
    put(3 * kWsPts + lane + 32 * q, d3[q] / s2x);
  }
  put(6 * kWsPts + lane, d2[3] / s2t);
  put(7 * kWsPts + lane, d3[3] / s2t);
  if (lane == 0) {
    put(8 * kWsPts + 0, log10(s3x / s2x));
    put(8 * kWsPts + 1, log10(s3t / s2t));
    put(8 * kWsPts + 2, log10(s2x / s1x));
    put(8 * kWsPts + 3, log10(s2t / s1t));
    sx[f] = s2x;
    st[f] = s2t;
  }
}

__global__ void warmstart_guess_kernel(const double *__restrict__ h1, const double *__restrict__ h2,
                                       const double *__restrict__ h3, int64_t n, int64_t o_fib,
                                       int nfib, const float *__restrict__ corr,
                                       const double *__restrict__ sx, const double *__restrict__ st,
                                       double *__restrict__ x0) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    // rounded step by step, as 3 h3 - 3 h2 + h1 evaluates elementwise
    double v = __dadd_rn(__dsub_rn(__dmul_rn(3.0, h3[i]), __dmul_rn(3.0, h2[i])), h1[i]);
    if (corr && i >= o_fib) {
      const int64_t j = i - o_fib;
      const int64_t f = j / (4 * kWsPts);
      const int k = static_cast<int>(j - f * 4 * kWsPts);
      if (f < nfib)
        v = __dadd_rn(v, __dmul_rn(static_cast<double>(corr[f * 4 * kWsPts + k]), k < 3 * kWsPts ? sx[f] : st[f]));
    }
    x0[i] = v;
  }
}

}  // namespace f3d

extern "C" {

int f3d_warmstart_features(const double *h0, const double *h1, const double *h2, const double *h3,
                           int64_t n, int64_t o_fib, int32_t nfib, int32_t npts, const float *mean,
                           const float *stdev, float *feats, double *scale_x, double *scale_t,
                           void *stream) {
  if (!h0 || !h1 || !h2 || !h3 || !feats || !scale_x || !scale_t) return F3D_ERR_NULL;
  if ((mean == nullptr) != (stdev == nullptr)) return F3D_ERR_NULL;
  if (npts != f3d::kWsPts) return F3D_ERR_ARG;
  if (nfib < 0 || o_fib < 0 || o_fib + static_cast<int64_t>(4 * npts) * nfib > n) return F3D_ERR_SHAPE;
  if (nfib == 0) return F3D_OK;
  const int threads = 256;
  const unsigned grid = static_cast<unsigned>((static_cast<int64_t>(nfib) * 32 + threads - 1) / threads);
  f3d::warmstart_features_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      h0, h1, h2, h3, o_fib, nfib, mean, stdev, feats, scale_x, scale_t);
  return f3d::launch_status();
}

int f3d_warmstart_guess(const double *h1, const double *h2, const double *h3, int64_t n,
                        int64_t o_fib, int32_t nfib, int32_t npts, const float *corr,
                        const double *scale_x, const double *scale_t, double *x0, void *stream) {
  if (!h1 || !h2 || !h3 || !x0) return F3D_ERR_NULL;
  if (corr && (!scale_x || !scale_t)) return F3D_ERR_NULL;
  if (npts != f3d::kWsPts) return F3D_ERR_ARG;
  if (n < 0 || nfib < 0 || o_fib < 0 || o_fib + static_cast<int64_t>(4 * npts) * nfib > n)
    return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  const int threads = 256;
  const int64_t want = (n + threads - 1) / threads;
  const unsigned grid = static_cast<unsigned>(want < 8 * 148 ? want : 8 * 148);
  f3d::warmstart_guess_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      h1, h2, h3, n, o_fib, nfib, corr, scale_x, scale_t, x0);
  return f3d::launch_status();
}

}  // extern "C"
