// decompose.cu -- digit decompositions of Goldilocks vectors on the device.
//
// decomp_b (lattice-folding/src/neo.rs:253-266): unsigned base-2^b digits of
// the canonical residue, ceil(64/b) rows, row r = the r-th digits of every
// element ([rows][count] bytes, b <= 8) -- the digit vectors a folding step
// commits to.
// GadgetDecomposition::decompose (lattice-core/src/decomposition.rs:48-70):
// balanced digits of a u64 in base 2^log_b: the low digit t in [0, 2^log_b)
// becomes t - 2^log_b when t > 2^(log_b - 1), the remainder moves on with the
// borrow; values not exhausted after num_digits digits are counted as
// ValueTooLarge.  ([num_digits][count] int16.)
// Both are one pass over HBM: 8 bytes in, rows x (1 or 2) bytes out per element.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/lattice_cuda.h"
#include "arith.cuh"
#include "common.cuh"
#include "internal.h"

namespace lc {

// 8 consecutive elements per thread: one 8-byte store per row when the rows
// are 8-byte aligned (count % 8 == 0), else byte stores.
__global__ void decomp_b_kernel(const uint64_t* __restrict__ z, size_t count, uint32_t b_bits, uint32_t rows,
                                uint8_t* __restrict__ out) {
  const uint64_t mask = (1ull << b_bits) - 1;
  const bool vec = (count & 7) == 0 && (reinterpret_cast<uintptr_t>(out) & 7) == 0;
  const size_t groups = (count + 7) / 8;
  for (size_t gi = blockIdx.x * (size_t)blockDim.x + threadIdx.x; gi < groups;
       gi += (size_t)gridDim.x * blockDim.x) {
    const size_t e0 = gi * 8;
    uint64_t x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = e0 + u < count ? gl_canon(__ldg(z + e0 + u)) : 0;
    for (uint32_t r = 0; r < rows; ++r) {
      const uint32_t sh = r * b_bits;
      if (vec) {
        uint64_t packed = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) packed |= ((x[u] >> sh) & mask) << (8 * u);
        *reinterpret_cast<uint64_t*>(out + (size_t)r * count + e0) = packed;
      } else {
        for (int u = 0; u < 8 && e0 + u < count; ++u)
          out[(size_t)r * count + e0 + u] = (uint8_t)((x[u] >> sh) & mask);
      }
    }
  }
}

__global__ void gadget_kernel(const uint64_t* __restrict__ z, size_t count, uint32_t log_b, uint32_t nd,
                              int16_t* __restrict__ out, uint32_t* __restrict__ too_large) {
  const uint64_t base = 1ull << log_b, mask = base - 1, half = base >> 1;
  uint32_t fails = 0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x) {
    uint64_t rem = __ldg(z + e);
    for (uint32_t i = 0; i < nd; ++i) {
      const uint64_t t = rem & mask;
      const bool borrow = t > half;
      // (rem - d) / base with d = t - base*borrow: the quotient plus the borrow
      rem = (rem >> log_b) + (borrow ? 1 : 0);
      out[(size_t)i * count + e] = (int16_t)(borrow ? (int64_t)t - (int64_t)base : (int64_t)t);
    }
    fails += rem != 0;
  }
  if (too_large && fails) atomicAdd(too_large, fails);
}

// pack_field_elements (lattice-ring/src/packing.rs:30-52): value e -> limbs
// raw & (2^22-1), (raw >> 22) & (2^22-1), raw >> 44 at coefficients 3e..3e+2
// of the flattened [elems][n] output; the rest zero.
__global__ void pack_kernel(const uint64_t* __restrict__ v, size_t count, uint32_t* __restrict__ out,
                            size_t total) {
  constexpr uint64_t mask = (1ull << 22) - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t e = i / 3;
    uint32_t c = 0;
    if (e < count) {
      const uint64_t raw = gl_canon(__ldg(v + e));
      const uint32_t part = (uint32_t)(i - 3 * e);
      c = (uint32_t)(part == 0 ? raw & mask : part == 1 ? (raw >> 22) & mask : raw >> 44);
    }
    out[i] = c;
  }
}

static unsigned grid_for(size_t items) {
  const int sms = std::max(device_sm_count(), 1);
  return (unsigned)std::max<size_t>(1, std::min<size_t>((items + 255) / 256, (size_t)sms * 16));
}

}  // namespace lc

extern "C" {

LC_API int lc_decomp_b(const uint64_t* z, size_t count, uint32_t b_bits, uint8_t* out, lc_stream stream) {
  using namespace lc;
  if (b_bits < 1 || b_bits > 8 || (count && (!z || !out))) return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  const uint32_t rows = (64 + b_bits - 1) / b_bits;
  decomp_b_kernel<<<grid_for((count + 7) / 8), 256, 0, (cudaStream_t)stream>>>(z, count, b_bits, rows, out);
  return map_cuda(cudaGetLastError());
}

LC_API int lc_gadget_decompose(const uint64_t* z, size_t count, uint32_t log_base, uint32_t num_digits,
                               int16_t* out, uint32_t* too_large, lc_stream stream) {
  using namespace lc;
  if (log_base < 1 || log_base > 15 || num_digits < 1 || (count && (!z || !out)))
    return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  gadget_kernel<<<grid_for(count), 256, 0, (cudaStream_t)stream>>>(z, count, log_base, num_digits, out,
                                                                    too_large);
  return map_cuda(cudaGetLastError());
}

LC_API int lc_pack_field_elements(const uint64_t* values, size_t count, uint32_t log_n, size_t out_elems,
                                  uint32_t* out, lc_stream stream) {
  using namespace lc;
  if (log_n < 1 || log_n > 11 || !out || (count && !values)) return LC_ERR_INVALID_ARGUMENT;
  const size_t n = (size_t)1 << log_n;
  const size_t need = std::max<size_t>(1, (3 * count + n - 1) / n);
  if (out_elems < need) return LC_ERR_DIMENSION_MISMATCH;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  const size_t total = out_elems * n;
  pack_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(values, count, out, total);
  return map_cuda(cudaGetLastError());
}

}  // extern "C"
