// synth.cu -- seeded synthetic inputs generated on the device.
//
// The counter-based generator of lzx_b200/synth.py, bit for bit:
//   H(seed, stream, i) = mix64(mix64(seed*G + stream*C2 + C3) + i*G)
// with the SplitMix64 finaliser mix64; uniform residues by rejection on a
// retry lane (stream + r<<40): u32 candidates below 2^32 - 2^32 mod q (the
// rule of lattice-ring/src/ring.rs:123), Goldilocks candidates below p; int8
// digits are the low byte of H.  Lets benchmarks and large tests fill
// gigabytes in milliseconds instead of uploading them.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/lattice_cuda.h"
#include "arith.cuh"
#include "common.cuh"
#include "internal.h"

namespace lc {

constexpr uint64_t kG = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kC2 = 0xC2B2AE3D27D4EB4Full;
constexpr uint64_t kC3 = 0x165667B19E3779F9ull;
constexpr int kMaxRetries = 64;  // rejection never needs more than a few

LC_HD uint64_t mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xBF58476D1CE4E5B9ull;
  z ^= z >> 27;
  z *= 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

LC_HD uint64_t synth_base(uint64_t seed, uint64_t stream) { return mix64(seed * kG + stream * kC2 + kC3); }

// kind: 0 = u64 raw, 1 = u32 residues mod q, 2 = Goldilocks residues, 3 = int8 digits
__global__ void synth_kernel(int kind, uint64_t seed, uint64_t stream, uint32_t q, void* out,
                             size_t count, size_t offset, uint32_t* err) {
  const uint64_t base0 = synth_base(seed, stream);
  const uint64_t limit32 = (1ull << 32) - ((1ull << 32) % (q ? q : 1));
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint64_t idx = offset + i;
    uint64_t v = mix64(base0 + idx * kG);
    if (kind == 0) {
      static_cast<uint64_t*>(out)[i] = v;
    } else if (kind == 3) {
      static_cast<int8_t*>(out)[i] = (int8_t)(uint8_t)v;
    } else {
      bool ok = kind == 1 ? (v & 0xFFFFFFFFull) < limit32 : v < kGlP;
      for (int r = 1; !ok && r <= kMaxRetries; ++r) {
        v = mix64(synth_base(seed, stream + ((uint64_t)r << 40)) + idx * kG);
        ok = kind == 1 ? (v & 0xFFFFFFFFull) < limit32 : v < kGlP;
      }
      if (!ok) record_error(err, 2);
      if (kind == 1)
        static_cast<uint32_t*>(out)[i] = (uint32_t)((v & 0xFFFFFFFFull) % q);
      else
        static_cast<uint64_t*>(out)[i] = v;
    }
  }
}

}  // namespace lc

extern "C" LC_API int lc_synth_fill(int kind, uint64_t seed, uint64_t stream, uint32_t q, void* out,
                                    size_t count, size_t offset, lc_stream stream_handle) {
  using namespace lc;
  if (kind < 0 || kind > 3 || (!out && count) || (kind == 1 && (q < 2))) return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  const int sms = device_sm_count();
  if (sms <= 0) return LC_ERR_NO_DEVICE;
  const size_t blocks = std::min<size_t>((count + 255) / 256, (size_t)sms * 32);
  synth_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream_handle>>>(kind, seed, stream, q, out,
                                                                          count, offset, nullptr);
  return map_cuda(cudaGetLastError());
}
