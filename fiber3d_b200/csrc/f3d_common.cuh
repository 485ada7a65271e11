// Shared device helpers of the fiber3d_b200 kernels (sm_100a).
//
// PTX wrappers for mbarriers and the bulk (TMA, non-tensor) global->shared
// copy, a bounded mbarrier wait, and the host-side plumbing every entry point
// uses (status mapping, the per-device error word).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fiber3d_b200.h"

namespace f3d {

// A bounded wait gives up after this many nanoseconds of %globaltimer by
// default; f3d_set_wait_limit_ns changes the limit the entry points pass to
// their kernels.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// Split-reduction counters of the pair sums: one word per target block, in
// a fixed region at the start of the pair workspace.
constexpr int64_t kMaxCounters = 65536;
constexpr size_t kCounterBytes = kMaxCounters * sizeof(unsigned);

// ---------------------------------------------------------------- device --
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes the initialised barriers visible to the async proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders earlier generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes into the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One arrival on `bar` (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// 1-D bulk copy global -> shared, completion signalled on `bar` as tx bytes.
// dst, src 16-byte aligned; bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of `bar` to complete, for at most limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
}

// D += A B on the FP64 tensor cores for one 16 x 8 x 16 step
// (mma.sync.m16n8k16.f64): a[i] holds A(g + 8 (i & 1), t + 4 (i >> 1)),
// b[j] holds B(t + 4 j, g), d[i] holds D(g + 8 (i >> 1), 2 t + (i & 1)), with
// g = lane / 4, t = lane % 4.
__device__ __forceinline__ void mma_f64_16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void record_error(int *err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// ------------------------------------------------------------------ host --
// Device address of this device's error word (set up on first use per device).
int *device_error_word();

// The limit (ns) that entry points hand to their kernels' bounded waits.
uint64_t wait_limit_ns();

inline bool aligned(const void *p, uintptr_t a) {
  return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

inline int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? F3D_OK : F3D_ERR_CUDA;
}

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

constexpr double kPi = 3.14159265358979323846;

}  // namespace f3d
