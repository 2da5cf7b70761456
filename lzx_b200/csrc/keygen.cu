// keygen.cu -- seeded ring elements and Ajtai keys derived on the device.
//
// RingConfig::uniform_from_seed (lattice-ring/src/ring.rs:102-180): for index
// i the coefficients are the accepted 4-byte little-endian windows, from byte
// 8 on, of  SHAKE256("LZXX" || le32(7) || "uniform" || le32(|salt|) || salt)
// (Transcript::xof, lattice-core/src/transcript.rs:229-237) with
// salt = domain || seed || le64(i); a window c is accepted when
// c < 2^32 - (2^32 mod q) and gives c mod q.  The reference squeezes
// 8 + 4(n + slack) bytes and continues window by window past them if needed
// -- the same stream, since SHAKE output is prefix-consistent -- so the
// coefficients are exactly the first n accepted windows.  One thread per ring
// element: the state stays in registers, 136-byte output blocks hold 34 whole
// windows, and AjtaiPublicKey::from_seed (lattice-commitment/src/ajtai.rs:
// 87-103) becomes one launch over the k*m indices plus the cached NTT.
//
// Keccak-f[1600] follows FIPS 202 (keccak.rs:52 in the reference): theta,
// rho, pi, chi, iota over 24 rounds; the round constants come from the
// rc(t) LFSR and the rotation offsets from the (x, y) -> (y, 2x + 3y) walk,
// both evaluated at compile time from those definitions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace lc {

struct KeccakTables {
  uint64_t rc[24];
  unsigned rho[25];
};

// rc(t): the output bit of the LFSR x^8 + x^6 + x^5 + x^4 + 1 after t steps
__host__ __device__ constexpr int keccak_rc_bit(unsigned t) {
  unsigned r = 1;  // R[0] = 1, bit i of r holds R[i]
  for (unsigned i = 0; i < t % 255; ++i) {
    const unsigned r8 = (r >> 7) & 1;  // the bit shifted out
    r = (r << 1) & 0xFF;
    if (r8) r ^= 0x71;  // R[0], R[4], R[5], R[6] ^= R[8]
  }
  return r & 1;
}

__host__ __device__ constexpr KeccakTables keccak_tables() {
  KeccakTables t{};
  for (unsigned ir = 0; ir < 24; ++ir) {
    uint64_t rc = 0;
    for (unsigned j = 0; j <= 6; ++j)
      if (keccak_rc_bit(j + 7 * ir)) rc |= (uint64_t)1 << ((1u << j) - 1);
    t.rc[ir] = rc;
  }
  t.rho[0] = 0;
  unsigned x = 1, y = 0;
  for (unsigned s = 0; s < 24; ++s) {
    t.rho[x + 5 * y] = ((s + 1) * (s + 2) / 2) % 64;
    const unsigned nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  return t;
}

__constant__ KeccakTables c_keccak = keccak_tables();

template <unsigned R>
LC_D uint64_t rotl64(uint64_t v) {
  if constexpr (R == 0)
    return v;
  else
    return (v << R) | (v >> (64 - R));
}

// rotation of lane x + 5y, known at compile time after unrolling
template <int L>
LC_D uint64_t rho_rot(uint64_t v) {
  constexpr KeccakTables t = keccak_tables();
  return rotl64<t.rho[L]>(v);
}

template <int X, int Y>
LC_D void rho_pi_one(const uint64_t (&a)[25], uint64_t (&b)[25]) {
  b[Y + 5 * ((2 * X + 3 * Y) % 5)] = rho_rot<X + 5 * Y>(a[X + 5 * Y]);
}

template <int I>
LC_D void rho_pi_all(const uint64_t (&a)[25], uint64_t (&b)[25]) {
  if constexpr (I < 25) {
    rho_pi_one<I % 5, I / 5>(a, b);
    rho_pi_all<I + 1>(a, b);
  }
}

LC_D void keccak_f1600(uint64_t (&a)[25]) {
#pragma unroll 1
  for (int round = 0; round < 24; ++round) {
    uint64_t c[5], b[25];
#pragma unroll
    for (int x = 0; x < 5; ++x) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
    for (int x = 0; x < 5; ++x) {
      const uint64_t d = c[(x + 4) % 5] ^ rotl64<1>(c[(x + 1) % 5]);
#pragma unroll
      for (int y = 0; y < 5; ++y) a[x + 5 * y] ^= d;
    }
    rho_pi_all<0>(a, b);
#pragma unroll
    for (int y = 0; y < 5; ++y)
#pragma unroll
      for (int x = 0; x < 5; ++x)
        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
    a[0] ^= c_keccak.rc[round];
  }
}

constexpr int kRateLanes = 17;  // SHAKE256: 136-byte rate
constexpr int kMaxAbsorbBlocks = 4;

struct UniformParams {
  uint64_t tmpl[kMaxAbsorbBlocks * kRateLanes];  // padded message, index bytes zero
  uint32_t blocks;      // absorb blocks
  uint32_t ioff;        // byte offset of le64(index) in the message
  uint64_t index0;
  uint64_t count;
  uint32_t q, log_n;
  uint64_t limit;       // 2^32 - (2^32 mod q)
  uint32_t* out;        // [count][n]
};

__global__ void __launch_bounds__(128) uniform_from_seed_kernel(const __grid_constant__ UniformParams p) {
  const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e >= p.count) return;
  const uint64_t index = p.index0 + e;
  const uint32_t gl = p.ioff / 8, sh = (p.ioff % 8) * 8;
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) a[i] = 0;
  for (uint32_t blk = 0; blk < p.blocks; ++blk) {
#pragma unroll
    for (int l = 0; l < kRateLanes; ++l) {
      const uint32_t g = blk * kRateLanes + l;
      uint64_t v = p.tmpl[g];
      if (g == gl) v ^= index << sh;
      if (sh && g == gl + 1) v ^= index >> (64 - sh);
      a[l] ^= v;
    }
    keccak_f1600(a);
  }
  const uint32_t n = 1u << p.log_n;
  uint32_t* out = p.out + e * n;
  uint32_t got = 0;
  bool first = true;  // the stream's windows start at byte 8 (word 2)
  while (true) {
#pragma unroll
    for (int w = 0; w < 2 * kRateLanes; ++w) {
      const uint32_t cand = (uint32_t)(a[w / 2] >> (32 * (w & 1)));
      if ((w >= 2 || !first) && got < n && cand < p.limit) out[got++] = cand % p.q;
    }
    if (got >= n) break;
    first = false;
    keccak_f1600(a);
  }
}

// The padded message "LZXX" || le32(7) || "uniform" || le32(|salt|) || domain
// || seed || le64(0) as rate-sized 64-bit lanes, plus where the index goes.
static int uniform_params(const lc_ntt_plan* plan, const uint8_t* domain, size_t dlen, const uint8_t* seed,
                          size_t slen, UniformParams& p) {
  std::vector<uint8_t> msg;
  auto put32 = [&](uint32_t v) {
    for (int i = 0; i < 4; ++i) msg.push_back((uint8_t)(v >> (8 * i)));
  };
  const char* tag = "LZXX";
  msg.insert(msg.end(), tag, tag + 4);
  put32(7);
  const char* lbl = "uniform";
  msg.insert(msg.end(), lbl, lbl + 7);
  put32((uint32_t)(dlen + slen + 8));
  msg.insert(msg.end(), domain, domain + dlen);
  msg.insert(msg.end(), seed, seed + slen);
  p.ioff = (uint32_t)msg.size();
  for (int i = 0; i < 8; ++i) msg.push_back(0);
  const size_t rate = kRateLanes * 8;
  const size_t blocks = msg.size() / rate + 1;  // room for at least the padding byte
  if (blocks > (size_t)kMaxAbsorbBlocks) return LC_ERR_INVALID_ARGUMENT;
  std::vector<uint8_t> padded(blocks * rate, 0);
  std::memcpy(padded.data(), msg.data(), msg.size());
  padded[msg.size()] ^= 0x1F;   // SHAKE domain bits + first pad bit
  padded[blocks * rate - 1] ^= 0x80;  // last pad bit
  std::memset(p.tmpl, 0, sizeof(p.tmpl));
  for (size_t g = 0; g < blocks * kRateLanes; ++g) {
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v |= (uint64_t)padded[g * 8 + b] << (8 * b);
    p.tmpl[g] = v;
  }
  p.blocks = (uint32_t)blocks;
  p.q = plan->q[0];
  p.log_n = plan->log_n;
  p.limit = ((uint64_t)1 << 32) - (((uint64_t)1 << 32) % p.q);
  return LC_OK;
}

int uniform_from_seed(const lc_ntt_plan* plan, const uint8_t* domain, size_t dlen, const uint8_t* seed,
                      size_t slen, uint64_t index0, size_t count, uint32_t* out, cudaStream_t st) {
  UniformParams p{};
  const int rc = uniform_params(plan, domain, dlen, seed, slen, p);
  if (rc) return rc;
  p.index0 = index0;
  p.count = count;
  p.out = out;
  if (count == 0) return LC_OK;
  uniform_from_seed_kernel<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(p);
  return map_cuda(cudaGetLastError());
}

}  // namespace lc

extern "C" {

LC_API int lc_uniform_from_seed(const lc_ntt_plan* plan, const uint8_t* domain, size_t domain_len,
                                const uint8_t* seed, size_t seed_len, uint64_t index0, size_t count,
                                uint32_t* out, lc_stream stream) {
  using namespace lc;
  if (!plan || (domain_len && !domain) || (seed_len && !seed) || (count && !out)) return LC_ERR_INVALID_ARGUMENT;
  if (plan->kind == PlanKind::Goldilocks || plan->num_moduli != 1) return LC_ERR_UNSUPPORTED;
  if (count > ((size_t)1 << 32)) return LC_ERR_INVALID_ARGUMENT;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  return uniform_from_seed(plan, domain, domain_len, seed, seed_len, index0, count, out, (cudaStream_t)stream);
}

LC_API int lc_ajtai_key_from_seed(const lc_ntt_plan* plan, uint32_t k, uint32_t m, const uint8_t seed[32],
                                  lc_ajtai_key** out) {
  using namespace lc;
  if (!plan || !seed || !out || k == 0 || m == 0) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (plan->kind == PlanKind::Goldilocks || plan->num_moduli != 1) return LC_ERR_UNSUPPORTED;
  int rc = key_create_check(plan, k, m, 0);
  if (rc) return rc;
  const size_t count = (size_t)k * m, n = (size_t)1 << plan->log_n;
  uint32_t* mat = nullptr;
  if (cudaMalloc(&mat, count * n * 4) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  // the expansion is written straight into the buffer the key is built from
  static const uint8_t dom[7] = {'a', 'j', 't', 'a', 'i', '-', 'A'};
  rc = uniform_from_seed(plan, dom, 7, seed, 32, 0, count, mat, nullptr);
  if (rc) {
    cudaFree(mat);
    return rc;
  }
  return key_create_from(plan, k, m, mat, 0, out);  // takes over mat
}

}  // extern "C"
