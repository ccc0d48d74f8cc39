// Source-sharded max/argmax across GPUs: the reduction step between ranks.
//
// The reference splits sources over the visible GPUs and merges the partial
// maxima on the host (beampower/src/beamform.cu:227-276, 430-445).  Here each
// rank beamforms a contiguous block of sources into the packed keys
// ordered(beam) << 32 | (0xFFFFFFFF - source); the keys are rebased to global
// source indexes and mapped from unsigned to signed order, one elementwise
// max all-reduce over ranks merges them (NCCL's int64 max), and the merged
// keys are decoded.  The lowest global source index keeps winning ties, as in
// the single-GPU path.
#define BP_TEMPLATE_KERNELS_ONLY
#include <cstdint>

#include <cuda_runtime.h>

#include "beampower_b200.h"
#include "bp_host.h"

using namespace bp_host;

namespace {

constexpr unsigned long long kSignBit = 1ull << 63;

// Local source index -> global (low 32 bits hold 0xFFFFFFFF - index), then
// the sign bit flipped so that signed int64 order is the keys' unsigned
// order (0, "no candidate", becomes the smallest int64).
__global__ void keys_to_shared_kernel(unsigned long long* __restrict__ keys, long long n,
                                      uint32_t offset) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long k = keys[i];
  if (k != 0ull) k -= (unsigned long long)offset;
  keys[i] = k ^ kSignBit;
}

// Merged keys back to unsigned order, then decoded: beam_max keeps its
// content and argmax gets 0 where no rank had a candidate.
__global__ void keys_from_shared_kernel(const unsigned long long* __restrict__ keys, long long n,
                                        float* __restrict__ beam_max,
                                        int32_t* __restrict__ argmax) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = keys[i] ^ kSignBit;
  if (k != 0ull) {
    beam_max[i] = bp::key_value(k);
    argmax[i] = bp::key_source(k);
  } else {
    argmax[i] = 0;
  }
}

}  // namespace

extern "C" {

int bp_keys_to_shared_dev(unsigned long long* d_keys, size_t n, size_t source_offset,
                          void* stream) {
  BP_NVTX("bp_keys_to_shared_dev");
  if (n == 0) return BP_OK;
  if (!d_keys) return fail(BP_ERR_INVALID_ARGUMENT, "NULL keys");
  if (source_offset > 0x7FFFFFFFull)
    return fail(BP_ERR_INVALID_ARGUMENT, "source offset beyond 2^31 - 1");
  keys_to_shared_kernel<<<(unsigned)((n + 255) / 256), 256, 0,
                          reinterpret_cast<cudaStream_t>(stream)>>>(d_keys, (long long)n,
                                                                    (uint32_t)source_offset);
  BP_LAUNCHED("keys_to_shared_kernel");
  return BP_OK;
}

int bp_keys_from_shared_dev(const unsigned long long* d_keys, size_t n, float* d_beam_max,
                            int32_t* d_argmax, void* stream) {
  BP_NVTX("bp_keys_from_shared_dev");
  if (n == 0) return BP_OK;
  if (!d_keys || !d_beam_max || !d_argmax) return fail(BP_ERR_INVALID_ARGUMENT, "NULL pointer");
  keys_from_shared_kernel<<<(unsigned)((n + 255) / 256), 256, 0,
                            reinterpret_cast<cudaStream_t>(stream)>>>(d_keys, (long long)n,
                                                                      d_beam_max, d_argmax);
  BP_LAUNCHED("keys_from_shared_kernel");
  return BP_OK;
}

}  // extern "C"
