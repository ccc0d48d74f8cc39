// Shared device helpers for the sm_100a beamforming kernels: the packed
// max/argmax key, mbarrier and bulk-copy (TMA engine) wrappers, bounded waits.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "beampower_b200.h"

namespace bp {

constexpr int kWarp = 32;

// ---------------------------------------------------------------------------
// Packed (beam value, source index) key.
//
// The reference keeps, per sample, the first source (ascending index) whose
// beam is strictly larger than the running max seeded with -FLT_MAX
// (beampower/src/beamform.c:269-334).  One unsigned 64-bit key per candidate
// reproduces that under an unordered max-reduction:
//   high 32 bits: the float mapped to an order-preserving unsigned integer,
//   low 32 bits : 0xFFFFFFFF - source index (smaller index => larger key).
// A beam that is NaN or <= -FLT_MAX can never beat the seed, so it gets key 0
// ("no candidate").  Beams are never -0.0 (the accumulator starts at +0.0 and
// round-to-nearest addition cannot reach -0.0 from there), but -0.0 is folded
// onto +0.0 anyway so that the key order equals the float order.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t ordered_bits(float v) {
  uint32_t b;
#ifdef __CUDA_ARCH__
  b = __float_as_uint(v);
#else
  __builtin_memcpy(&b, &v, 4);
#endif
  if (b == 0x80000000u) b = 0u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ __forceinline__ float float_from_ordered(uint32_t o) {
  uint32_t b = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
  float v;
#ifdef __CUDA_ARCH__
  v = __uint_as_float(b);
#else
  __builtin_memcpy(&v, &b, 4);
#endif
  return v;
}

__host__ __device__ __forceinline__ unsigned long long make_key(float beam, int source) {
  // `beam > -FLT_MAX` is false for NaN, -inf and -FLT_MAX itself.
  if (!(beam > -FLT_MAX)) return 0ull;
  return ((unsigned long long)ordered_bits(beam) << 32) |
         (unsigned long long)(0xFFFFFFFFu - (uint32_t)source);
}

__host__ __device__ __forceinline__ int key_source(unsigned long long key) {
  return (int)(0xFFFFFFFFu - (uint32_t)(key & 0xFFFFFFFFull));
}

__host__ __device__ __forceinline__ float key_value(unsigned long long key) {
  return float_from_ordered((uint32_t)(key >> 32));
}

// ---------------------------------------------------------------------------
// Status word written by kernels (bit flags, OR-ed).
// ---------------------------------------------------------------------------
enum : int {
  kStatusWaitTimeout = 1,   // an mbarrier wait gave up after its time limit
  kStatusBadWindow = 2,     // a trace window did not fit the shared-memory row
  kStatusBadIndex = 4,      // checked build: an index check failed, the access was skipped
};

// Wall-clock limit of one mbarrier wait.  A stage normally lands within
// microseconds; the limit only bounds a wait that can no longer complete.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on one phase of an mbarrier.  Returns false (and raises the
// block's abort flag and the global status) if the phase did not complete
// within kWaitLimitNs, or if another thread of the block already aborted.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  volatile int* abort_flag, int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long start = globaltimer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer_ns() - start > kWaitLimitNs) {
      *abort_flag = 1;
      if (status) atomicOr(status, kStatusWaitTimeout);
      return false;
    }
  }
}

// Same with a caller-given limit (diagnostics).
__device__ __forceinline__ bool mbar_wait_limit(uint64_t* bar, uint32_t parity,
                                                unsigned long long limit_ns, int* status) {
  const unsigned long long start = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - start > limit_ns) {
      if (status) atomicOr(status, kStatusWaitTimeout);
      return false;
    }
  }
  return true;
}

// 1-D bulk copy global -> shared through the TMA engine, completing on an
// mbarrier.  Both addresses 16-byte aligned, size a multiple of 16 bytes.
// No multicast: every copy reads this GPU's own memory into this CTA.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Packed FP32 pair add (sm_100 .f32x2); each lane equals __fadd_rn.  Only
// used where no multiply precedes it, so there is nothing to fuse.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\t"
      "mov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}

__device__ __forceinline__ void named_barrier_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void red_max_u64(unsigned long long* addr, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(addr), "l"(v) : "memory");
}

}  // namespace bp
