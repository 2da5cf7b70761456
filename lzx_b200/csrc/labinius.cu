// labinius.cu -- the labinius Ajtai commitment over R_648 = Z_q[X]/Phi_1944(X).
//
// CommitmentKey::commit (lattice-labinius/src/key.rs:223-474, scalar path
// :382-474 as the specification): the witness is a stream of F162 elements;
// ring element i of chunk c lifts elements 4i..4i+3 of the chunk into the
// binary coefficients c[4m + k] = bit m of element 4i + k (binfield.rs:
// 128-143).  Per limb prime q (seven primes below 2^15, params.rs:20-30,
// :306-308) each lifted element is transformed on the limb's tree
// (scalar.rs:37-86 for q = 1 mod 1944: Phi_6 split, radix 2, 2, 3, 3, 3, 3,
// slot j = a(psi^SLOT_EXP[j]); scalar.rs:165-213 for the quadratic primes:
// Phi_6 split, radix 2, 3, 3, 3, 3 down to 324 leaves X^2 - psi'^u), then
// y += A_i (.) t (pointwise, or the per-leaf product of mul_quad_slots,
// scalar.rs:229-243).  The raw commitment yc = y mod q is decomposed into four
// R_162 slot elements (ring.rs:193-319).
//
// GPU mapping: one warp per lifted ring element (648 residues in shared
// memory, __syncwarp between tree levels), grid (chunk split, chunk, limb);
// each lane accumulates its 21 slots (11 leaf pairs) over the warp's ring
// elements in u64 registers, the CTA sums its warps, and a finish kernel adds
// the splits, reduces mod q and decomposes.  Every transform value is
// canonical in [0, q) and every product is exact, so the results equal the
// scalar reference bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace lc {

constexpr int kLbN = 648, kLbN162 = 162, kLbQSlots = 324;
constexpr int kLbCond = 1944, kLbCondQ = 972;
constexpr int kLbTw = 326;  // twiddles of levels 1..6 of the split tree (2+4+8+24+72+216)
constexpr int kLbWarps = 8;
constexpr int kLbSlotsPerLane = (kLbN + 31) / 32;       // 21
constexpr int kLbPairsPerLane = (kLbQSlots + 31) / 32;  // 11
static_assert(2 * kLbPairsPerLane >= kLbSlotsPerLane, "accumulators");

// Per-limb constants: Shoup pairs (w, floor(w 2^32 / q)) for every twiddle.
struct LbLimb {
  uint32_t q, quad;
  uint32_t z6, z6s, om, oms;
  uint32_t tw[kLbTw], tws[kLbTw], tw2[kLbTw], tw2s[kLbTw];  // zeta, zeta^2 per (level, subring)
  uint32_t leaf[kLbQSlots];                                // quadratic leaves: psi'^QUAD_SLOT_EXP[j]
  uint32_t dtw[4][kLbN162];                                // decomposition factors
  uint32_t i_root, inv2;
};

// Index maps shared by every prime (params.rs:88-97, ring.rs:68-99, params.rs:318-355).
struct LbMaps {
  uint16_t slot_648[4][kLbN162];
  uint16_t quad_class_slot[2][kLbN162];
};

__constant__ LbMaps c_lb_maps;

}  // namespace lc

struct lc_lb_key {
  size_t len_f162 = 0, nr = 0;
  uint32_t limbs = 0;
  std::vector<uint16_t> primes;
  std::vector<int16_t> a_host;  // centered rows [limbs][nr][648]
  uint16_t* d_a = nullptr;      // canonical rows [limbs][nr][648]
  lc::LbLimb* d_limb = nullptr;
  uint32_t* d_partial = nullptr;
  size_t partial_bytes = 0;
  uint64_t* d_in = nullptr;  // host-API staging
  size_t in_bytes = 0;
  void* d_out = nullptr;
  size_t out_bytes = 0;
};

namespace lc {

// ------------------------------------------------------------------ host tables

static uint64_t lb_pow(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t r = 1;
  b %= q;
  while (e) {
    if (e & 1) r = r * b % q;
    b = b * b % q;
    e >>= 1;
  }
  return r;
}

static const int kRadix[7] = {2, 2, 2, 3, 3, 3, 3};
static const int kSub[8] = {1, 2, 4, 8, 24, 72, 216, 648};
static const int kRadixQ[6] = {2, 2, 3, 3, 3, 3};
static const int kSubQ[7] = {1, 2, 4, 12, 36, 108, 324};

// exponent of sub-ring k at a level (params.rs:73-85, :273-285)
static uint32_t sub_exp(bool quad, int level, int k) {
  if (level == 1) return quad ? (k == 0 ? 162 : 810) : (k == 0 ? 324 : 1620);
  const uint32_t p = (uint32_t)(quad ? kRadixQ[level - 1] : kRadix[level - 1]);
  const uint32_t cond = quad ? kLbCondQ : kLbCond;
  return (sub_exp(quad, level - 1, k / (int)p) + cond * ((uint32_t)k % p)) / p;
}

static bool lb_is_quad(uint32_t q) { return (q - 1) % kLbCondQ == 0 && (q - 1) % kLbCond != 0; }

static bool lb_prime_ok(uint32_t q) {
  switch (q) {
    case 2917: case 3889: case 4861: case 9721: case 12637: case 17497: case 19441: return true;
    default: return false;
  }
}

static uint32_t find_root(uint32_t q, bool quad) {  // params.rs:61-70, :262-270
  const uint64_t ord = quad ? 972 : 1944;
  for (uint64_t x = 2;; ++x)
    if (lb_pow(x, ord, q) == 1 && lb_pow(x, ord / 2, q) != 1 && lb_pow(x, ord / 3, q) != 1) return (uint32_t)x;
}

static uint32_t shoup32(uint32_t w, uint32_t q) { return (uint32_t)(((uint64_t)w << 32) / q); }

static void build_maps(LbMaps& m) {
  uint16_t slot_exp[kLbN], quad_exp[kLbQSlots], pow3[kLbN162];
  for (int j = 0; j < kLbN; ++j) slot_exp[j] = (uint16_t)sub_exp(false, 7, j);
  for (int j = 0; j < kLbQSlots; ++j) quad_exp[j] = (uint16_t)sub_exp(true, 6, j);
  int pos[486];
  std::fill(pos, pos + 486, -1);
  int n = 0;
  for (int j = 0; j < kLbN; ++j) {
    const int u = slot_exp[j], v = u % 486, t = (u - v) / 486;
    if (pos[v] < 0) {
      pos[v] = n;
      pow3[n++] = (uint16_t)v;
    }
    m.slot_648[t][pos[v]] = (uint16_t)j;
  }
  for (int s = 0; s < kLbN162; ++s)
    for (int j = 0; j < kLbQSlots; ++j) {
      if (quad_exp[j] == pow3[s]) m.quad_class_slot[0][s] = (uint16_t)j;
      if (quad_exp[j] == pow3[s] + 486) m.quad_class_slot[1][s] = (uint16_t)j;
    }
}

static void build_limb(uint32_t q, LbLimb& L) {
  const bool quad = lb_is_quad(q);
  std::memset(&L, 0, sizeof(L));
  L.q = q;
  L.quad = quad;
  const uint32_t psi = find_root(q, quad);
  L.z6 = (uint32_t)lb_pow(psi, quad ? 162 : 324, q);
  L.om = (uint32_t)lb_pow(psi, quad ? 324 : 648, q);
  L.z6s = shoup32(L.z6, q);
  L.oms = shoup32(L.om, q);
  const int levels = quad ? 5 : 6;
  int off = 0;
  for (int level = 1; level <= levels; ++level) {
    const int subs = quad ? kSubQ[level] : kSub[level];
    const int p = quad ? kRadixQ[level] : kRadix[level];
    for (int k = 0; k < subs; ++k) {
      const uint32_t z = (uint32_t)lb_pow(psi, sub_exp(quad, level, k) / (uint32_t)p, q);
      const uint32_t z2 = (uint32_t)((uint64_t)z * z % q);
      L.tw[off + k] = z;
      L.tws[off + k] = shoup32(z, q);
      L.tw2[off + k] = z2;
      L.tw2s[off + k] = shoup32(z2, q);
    }
    off += subs;
  }
  uint16_t pow3[kLbN162];
  {
    uint16_t slot_exp[kLbN];
    for (int j = 0; j < kLbN; ++j) slot_exp[j] = (uint16_t)sub_exp(false, 7, j);
    bool seen[486] = {};
    int n = 0;
    for (int j = 0; j < kLbN; ++j) {
      const int v = slot_exp[j] % 486;
      if (!seen[v]) {
        seen[v] = true;
        pow3[n++] = (uint16_t)v;
      }
    }
  }
  L.inv2 = (uint32_t)lb_pow(2, q - 2, q);
  if (quad) {
    for (int j = 0; j < kLbQSlots; ++j) L.leaf[j] = (uint32_t)lb_pow(psi, sub_exp(true, 6, j), q);
    for (int s = 0; s < kLbN162; ++s)  // inv2 * psi'^{-v}, ring.rs:248-262
      L.dtw[0][s] = (uint32_t)((uint64_t)L.inv2 * lb_pow(psi, (kLbCondQ - pow3[s]) % kLbCondQ, q) % q);
  } else {
    const uint64_t inv4 = lb_pow(4, q - 2, q);
    L.i_root = (uint32_t)lb_pow(psi, 486, q);
    for (int s = 0; s < kLbN162; ++s)  // inv4 * psi^{-v k}, ring.rs:167-187
      for (int k = 0; k < 4; ++k)
        L.dtw[k][s] = (uint32_t)(inv4 * lb_pow(psi, (kLbCond - (uint32_t)pow3[s] * k % kLbCond) % kLbCond, q) % q);
  }
}

// c_lb_maps is constant memory of each device: uploaded once per device (one
// bit per device; devices past 63 upload on every call).
static std::mutex g_maps_mu;
static uint64_t g_maps_done = 0;

static int ensure_maps() {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return map_cuda(e);
  const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t)1 << dev : 0;
  std::lock_guard<std::mutex> lk(g_maps_mu);
  if (bit && (g_maps_done & bit)) return LC_OK;
  LbMaps m;
  build_maps(m);
  const int rc = map_cuda(cudaMemcpyToSymbol(c_lb_maps, &m, sizeof(m)));
  if (rc == LC_OK) g_maps_done |= bit;
  return rc;
}

// ------------------------------------------------------------------ device arithmetic

// x * w mod q, x < 2^32, w < q with ws = floor(w 2^32 / q): a representative in [0, 2q)
LC_D uint32_t lb_mulc(uint32_t x, uint32_t w, uint32_t ws, uint32_t q) { return x * w - __umulhi(x, ws) * q; }

struct LbTw {  // shared-memory copy of the limb's twiddles
  uint32_t tw[kLbTw], tws[kLbTw], tw2[kLbTw], tw2s[kLbTw];
};

// One radix-P level: NSUB sub-rings of degree DEG, twiddles at offset OFF.
// Lazy: products are representatives in [0, 2q) and differences add 2q or 4q,
// so a radix-2 level raises the bound on every value by 2q and a radix-3 level
// by 4q; the transform's values stay below 24q < 2^20.
template <int NSUB, int DEG, int P, int OFF>
LC_D void lb_level(uint32_t* v, const LbTw& T, uint32_t q, uint32_t om, uint32_t oms, uint32_t lane) {
  constexpr int M = DEG / P, BF = NSUB * M;
  const uint32_t q2 = 2 * q;
  for (int b = lane; b < BF; b += 32) {
    const int k = b / M, i = b - k * M, base = k * DEG;
    if (P == 2) {
      const uint32_t a0 = v[base + i];
      const uint32_t t = lb_mulc(v[base + M + i], T.tw[OFF + k], T.tws[OFF + k], q);
      v[base + i] = a0 + t;
      v[base + M + i] = a0 + q2 - t;
    } else {
      // a0 + w t1 + w^2 t2 = a0 - t2 + w (t1 - t2) and a0 + w^2 t1 + w t2 = a0 - t1 - w (t1 - t2)
      const uint32_t a0 = v[base + i];
      const uint32_t t1 = lb_mulc(v[base + M + i], T.tw[OFF + k], T.tws[OFF + k], q);
      const uint32_t t2 = lb_mulc(v[base + 2 * M + i], T.tw2[OFF + k], T.tw2s[OFF + k], q);
      const uint32_t u = lb_mulc(t1 + q2 - t2, om, oms, q);
      v[base + i] = a0 + t1 + t2;
      v[base + M + i] = a0 + q2 - t2 + u;
      v[base + 2 * M + i] = a0 + 2 * q2 - t1 - u;
    }
  }
  __syncwarp();
}

// The whole forward transform of one ring element in warp-private shared
// memory, canonical residues out.  Inputs are canonical; BINARY inputs
// (0/1 coefficients) take the Phi_6 split's product a1 * zeta6 as a select.
template <bool BINARY>
LC_D void lb_transform(uint32_t* v, const LbTw& T, const LbLimb& L, uint32_t lane) {
  const uint32_t q = L.q;
  for (int i = lane; i < 324; i += 32) {  // Phi_6 split: (a0 + t, a0 + a1 - t), t = zeta6 a1
    const uint32_t a0 = v[i], a1 = v[i + 324];
    const uint32_t t = BINARY ? (a1 ? L.z6 : 0u) : lb_mulc(a1, L.z6, L.z6s, q);
    v[i] = a0 + t;
    v[i + 324] = a0 + a1 + 2 * q - t;
  }
  __syncwarp();
  if (L.quad) {
    lb_level<2, 324, 2, 0>(v, T, q, L.om, L.oms, lane);
    lb_level<4, 162, 3, 2>(v, T, q, L.om, L.oms, lane);
    lb_level<12, 54, 3, 6>(v, T, q, L.om, L.oms, lane);
    lb_level<36, 18, 3, 18>(v, T, q, L.om, L.oms, lane);
    lb_level<108, 6, 3, 54>(v, T, q, L.om, L.oms, lane);
  } else {
    lb_level<2, 324, 2, 0>(v, T, q, L.om, L.oms, lane);
    lb_level<4, 162, 2, 2>(v, T, q, L.om, L.oms, lane);
    lb_level<8, 81, 3, 6>(v, T, q, L.om, L.oms, lane);
    lb_level<24, 27, 3, 14>(v, T, q, L.om, L.oms, lane);
    lb_level<72, 9, 3, 38>(v, T, q, L.om, L.oms, lane);
    lb_level<216, 3, 3, 110>(v, T, q, L.om, L.oms, lane);
  }
  // canonical: Barrett with floor(2^32 / q) leaves [0, 2q) for values < 2^20
  const uint32_t bm = 0xFFFFFFFFu / q;
  for (int x = lane; x < kLbN; x += 32) {
    uint32_t r = v[x] - __umulhi(v[x], bm) * q;
    v[x] = r >= q ? r - q : r;
  }
  __syncwarp();
}

struct LbCommitParams {
  const uint64_t* witness;  // [r * len_f162][3]
  const uint16_t* a;        // [limbs][nr][648] canonical
  const LbLimb* limbs;
  uint32_t* partial;        // [limbs][r][S][648]
  uint32_t* batches;        // [r * nr][648] (limb 0) or null
  uint32_t nr, splits, per_split, r;
  size_t len_f162;
};

__global__ void __launch_bounds__(kLbWarps * 32) lb_commit_kernel(const __grid_constant__ LbCommitParams p) {
  __shared__ LbTw s_tw;
  __shared__ uint32_t s_leaf[kLbQSlots];
  __shared__ uint32_t s_v[kLbWarps][kLbN];
  __shared__ uint64_t s_w[kLbWarps][12];
  const uint32_t split = blockIdx.x, c = blockIdx.y, k = blockIdx.z;
  const LbLimb& L = p.limbs[k];
  const uint32_t q = L.q;
  const bool quad = L.quad != 0;
  for (int e = threadIdx.x; e < kLbTw; e += blockDim.x) {
    s_tw.tw[e] = L.tw[e];
    s_tw.tws[e] = L.tws[e];
    s_tw.tw2[e] = L.tw2[e];
    s_tw.tw2s[e] = L.tw2s[e];
  }
  if (quad)
    for (int e = threadIdx.x; e < kLbQSlots; e += blockDim.x) s_leaf[e] = L.leaf[e];
  __syncthreads();
  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  uint32_t* v = s_v[warp];
  uint64_t* w = s_w[warp];
  // 21 slots per lane (split limbs) or 11 leaf pairs = 22 sums (quadratic limbs)
  uint64_t acc[2 * kLbPairsPerLane];
#pragma unroll
  for (int j = 0; j < 2 * kLbPairsPerLane; ++j) acc[j] = 0;
  const uint32_t i0 = split * p.per_split, i1 = min(p.nr, i0 + p.per_split);
  const uint64_t* wc = p.witness + (size_t)c * p.len_f162 * 3;
  const uint16_t* ak = p.a + (size_t)k * p.nr * kLbN;
  for (uint32_t i = i0 + warp; i < i1; i += kLbWarps) {
    if (lane < 12) w[lane] = wc[(size_t)12 * i + lane];  // elements 4i..4i+3, 3 words each
    __syncwarp();
    for (int x = lane; x < kLbN; x += 32) {  // coefficient 4m + kk = bit m of element 4i + kk
      const int m = x >> 2, kk = x & 3;
      v[x] = (uint32_t)(w[3 * kk + (m >> 6)] >> (m & 63)) & 1u;
    }
    __syncwarp();
    lb_transform<true>(v, s_tw, L, lane);
    if (k == 0 && p.batches) {
      uint32_t* dst = p.batches + ((size_t)c * p.nr + i) * kLbN;
      for (int x = lane; x < kLbN; x += 32) dst[x] = v[x];
    }
    const uint16_t* arow = ak + (size_t)i * kLbN;
    if (!quad) {
#pragma unroll
      for (int j = 0; j < kLbSlotsPerLane; ++j) {
        const int u = lane + 32 * j;
        if (u < kLbN) acc[j] += (uint64_t)__ldg(arow + u) * v[u];
      }
    } else {
      // leaf j: (a0 + a1 X)(b0 + b1 X) mod (X^2 - c_j), accumulated without reduction
#pragma unroll
      for (int j = 0; j < kLbPairsPerLane; ++j) {
        const int s = lane + 32 * j;
        if (s < kLbQSlots) {
          const uint32_t a0 = __ldg(arow + 2 * s), a1 = __ldg(arow + 2 * s + 1);
          const uint32_t b0 = v[2 * s], b1 = v[2 * s + 1];
          acc[2 * j] += (uint64_t)a0 * b0 + (uint64_t)s_leaf[s] * (a1 * b1);
          acc[2 * j + 1] += (uint64_t)a0 * b1 + (uint64_t)a1 * b0;
        }
      }
    }
    __syncwarp();
  }
  // CTA sum of the warps' accumulators, reduced mod q
  __syncthreads();
  if (!quad) {
#pragma unroll
    for (int j = 0; j < kLbSlotsPerLane; ++j) {
      const int u = lane + 32 * j;
      if (u < kLbN) s_v[warp][u] = (uint32_t)(acc[j] % q);
    }
  } else {
#pragma unroll
    for (int j = 0; j < kLbPairsPerLane; ++j) {
      const int s = lane + 32 * j;
      if (s < kLbQSlots) {
        s_v[warp][2 * s] = (uint32_t)(acc[2 * j] % q);
        s_v[warp][2 * s + 1] = (uint32_t)(acc[2 * j + 1] % q);
      }
    }
  }
  __syncthreads();
  uint32_t* out = p.partial + (((size_t)k * p.r + c) * p.splits + split) * kLbN;
  for (int u = threadIdx.x; u < kLbN; u += blockDim.x) {
    uint32_t sum = 0;
#pragma unroll
    for (int ww = 0; ww < kLbWarps; ++ww) sum += s_v[ww][u];
    out[u] = sum % q;
  }
}

LC_D int16_t lb_center(uint32_t r, uint32_t q) { return r > (q - 1) / 2 ? (int16_t)((int32_t)r - (int32_t)q) : (int16_t)r; }

struct LbFinishParams {
  const uint32_t* partial;
  const LbLimb* limbs;
  uint32_t* raw;      // [limbs][r][648]
  int16_t* matrix;    // [4][r][limbs][162]
  uint32_t splits, r, nlimbs;
};

__global__ void __launch_bounds__(256) lb_finish_kernel(const __grid_constant__ LbFinishParams p) {
  __shared__ uint32_t y[kLbN];
  const uint32_t c = blockIdx.x, k = blockIdx.y;
  const LbLimb& L = p.limbs[k];
  const uint32_t q = L.q;
  const uint32_t* part = p.partial + ((size_t)k * p.r + c) * p.splits * kLbN;
  for (int u = threadIdx.x; u < kLbN; u += blockDim.x) {
    uint64_t s = 0;
    for (uint32_t sp = 0; sp < p.splits; ++sp) s += part[(size_t)sp * kLbN + u];
    y[u] = (uint32_t)(s % q);
    p.raw[((size_t)k * p.r + c) * kLbN + u] = y[u];
  }
  __syncthreads();
  for (int s = threadIdx.x; s < kLbN162; s += blockDim.x) {
    int16_t o[4];
    if (!L.quad) {  // length-4 inverse DFT over the class, ring.rs:193-245
      uint32_t e[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) e[t] = y[c_lb_maps.slot_648[t][s]];
      const uint64_t a = e[0] + e[2], d0 = e[0] + q - e[2], cc = e[1] + e[3], d1 = e[1] + q - e[3];
      const uint64_t id = (d1 % q) * L.i_root % q;
      const uint64_t m[4] = {a + cc, d0 + q - id, a + 2ull * q - cc, d0 + id};
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) o[kk] = lb_center((uint32_t)((m[kk] % q) * L.dtw[kk][s] % q), q);
    } else {  // 2-point butterfly over the class's two leaves, ring.rs:264-306
      const int jp = c_lb_maps.quad_class_slot[0][s], jm = c_lb_maps.quad_class_slot[1][s];
#pragma unroll
      for (int kk = 0; kk < 2; ++kk) {
        const uint64_t ep = y[2 * jp + kk], em = y[2 * jm + kk];
        o[kk] = lb_center((uint32_t)((ep + em) % q * L.inv2 % q), q);
        o[kk + 2] = lb_center((uint32_t)((ep + q - em) % q * L.dtw[0][s] % q), q);
      }
    }
#pragma unroll
    for (int row = 0; row < 4; ++row) p.matrix[(((size_t)row * p.r + c) * p.nlimbs + k) * kLbN162 + s] = o[row];
  }
}

// general-input transform of `count` ring elements (key derivation, lc_lb_ntt)
__global__ void __launch_bounds__(kLbWarps * 32)
    lb_ntt_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t count, const LbLimb* limb) {
  __shared__ LbTw s_tw;
  __shared__ uint32_t s_v[kLbWarps][kLbN];
  const LbLimb& L = *limb;
  for (int e = threadIdx.x; e < kLbTw; e += blockDim.x) {
    s_tw.tw[e] = L.tw[e];
    s_tw.tws[e] = L.tws[e];
    s_tw.tw2[e] = L.tw2[e];
    s_tw.tw2s[e] = L.tw2s[e];
  }
  __syncthreads();
  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  uint32_t* v = s_v[warp];
  for (size_t i = (size_t)blockIdx.x * kLbWarps + warp; i < count; i += (size_t)gridDim.x * kLbWarps) {
    for (int x = lane; x < kLbN; x += 32) v[x] = in[i * kLbN + x] % L.q;
    __syncwarp();
    lb_transform<false>(v, s_tw, L, lane);
    for (int x = lane; x < kLbN; x += 32) out[i * kLbN + x] = v[x];
    __syncwarp();
  }
}

static int lb_ntt_run(const LbLimb* d_limb, const uint32_t* in, uint32_t* out, size_t count, cudaStream_t st) {
  if (count == 0) return LC_OK;
  const size_t blocks = std::min<size_t>((count + kLbWarps - 1) / kLbWarps, (size_t)std::max(1, device_sm_count()) * 8);
  lb_ntt_kernel<<<(unsigned)blocks, kLbWarps * 32, 0, st>>>(in, out, count, d_limb);
  return map_cuda(cudaGetLastError());
}

// xorshift64* of the reference (binfield.rs:158-175)
struct LbRng {
  uint64_t s;
  explicit LbRng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull | 1) {}
  uint64_t next() {
    uint64_t x = s;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    s = x;
    return x * 0x2545F4914F6CDD1Dull;
  }
  uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * n) >> 32); }
};

static int lb_key_finish(lc_lb_key* key) {
  // canonical rows on the device
  std::vector<uint16_t> canon(key->a_host.size());
  for (uint32_t k = 0; k < key->limbs; ++k) {
    const int32_t q = key->primes[k];
    for (size_t e = 0; e < key->nr * kLbN; ++e) {
      const size_t idx = (size_t)k * key->nr * kLbN + e;
      int32_t x = key->a_host[idx] % q;
      canon[idx] = (uint16_t)(x < 0 ? x + q : x);
    }
  }
  if (cudaMalloc(&key->d_a, canon.size() * 2) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  return map_cuda(cudaMemcpy(key->d_a, canon.data(), canon.size() * 2, cudaMemcpyHostToDevice));
}

static int lb_key_alloc(size_t len_f162, const uint16_t* primes, uint32_t limbs, lc_lb_key** out) {
  if (!out || !primes || limbs == 0 || limbs > 7) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  // key.rs:96-100: len_f162 > 0 and a multiple of 4; no limb listed twice (:102-106)
  if (len_f162 == 0 || len_f162 % 4 || len_f162 / 4 > (1u << 16)) return LC_ERR_INVALID_ARGUMENT;  // nr <= 2^16 keeps the u64 sums exact
  for (uint32_t k = 0; k < limbs; ++k) {
    if (!lb_prime_ok(primes[k])) return LC_ERR_INVALID_ARGUMENT;
    for (uint32_t j = 0; j < k; ++j)
      if (primes[j] == primes[k]) return LC_ERR_INVALID_ARGUMENT;
  }
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  int rc = ensure_maps();
  if (rc) return rc;
  lc_lb_key* key = new (std::nothrow) lc_lb_key();
  if (!key) return LC_ERR_OUT_OF_MEMORY;
  key->len_f162 = len_f162;
  key->nr = len_f162 / 4;
  key->limbs = limbs;
  key->primes.assign(primes, primes + limbs);
  std::vector<LbLimb> tabs(limbs);
  for (uint32_t k = 0; k < limbs; ++k) build_limb(primes[k], tabs[k]);
  if (cudaMalloc(&key->d_limb, sizeof(LbLimb) * limbs) != cudaSuccess) {
    cudaGetLastError();
    delete key;
    return LC_ERR_OUT_OF_MEMORY;
  }
  rc = map_cuda(cudaMemcpy(key->d_limb, tabs.data(), sizeof(LbLimb) * limbs, cudaMemcpyHostToDevice));
  if (rc) {
    lc_lb_key_destroy(key);
    return rc;
  }
  *out = key;
  return LC_OK;
}

static int grow(void** p, size_t* have, size_t need) {
  if (need <= *have) return LC_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(p, need) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  *have = need;
  return LC_OK;
}

}  // namespace lc

extern "C" {

LC_API int lc_lb_key_create(size_t len_f162, const uint16_t* primes, uint32_t limbs, const int16_t* a,
                            lc_lb_key** out) {
  using namespace lc;
  if (!a) return LC_ERR_INVALID_ARGUMENT;
  lc_lb_key* key = nullptr;
  int rc = lb_key_alloc(len_f162, primes, limbs, &key);
  if (rc) return rc;
  key->a_host.assign(a, a + (size_t)limbs * key->nr * kLbN);
  rc = lb_key_finish(key);
  if (rc) {
    lc_lb_key_destroy(key);
    return rc;
  }
  *out = key;
  return LC_OK;
}

// CommitmentKey::random (key.rs:94-137): per limb k an xorshift64* stream
// seeded with seed ^ 0x9E3779B9 (k + 1) draws nr x 648 uniform coefficients
// below q; the rows are their transforms, centered.
LC_API int lc_lb_key_random(size_t len_f162, uint64_t seed, const uint16_t* primes, uint32_t limbs,
                            lc_lb_key** out) {
  using namespace lc;
  lc_lb_key* key = nullptr;
  int rc = lb_key_alloc(len_f162, primes, limbs, &key);
  if (rc) return rc;
  const size_t per = key->nr * kLbN;
  std::vector<uint32_t> coeffs(per), t(per);
  uint32_t* d_buf = nullptr;
  if (cudaMalloc(&d_buf, per * 4 * 2) != cudaSuccess) {
    cudaGetLastError();
    lc_lb_key_destroy(key);
    return LC_ERR_OUT_OF_MEMORY;
  }
  key->a_host.resize((size_t)limbs * per);
  for (uint32_t k = 0; k < limbs && !rc; ++k) {
    const uint32_t q = primes[k];
    LbRng rng(seed ^ (0x9E3779B9ull * (uint64_t)(k + 1)));
    for (size_t e = 0; e < per; ++e) coeffs[e] = rng.below(q);
    rc = map_cuda(cudaMemcpy(d_buf, coeffs.data(), per * 4, cudaMemcpyHostToDevice));
    if (!rc) rc = lb_ntt_run(key->d_limb + k, d_buf, d_buf + per, key->nr, nullptr);
    if (!rc) rc = map_cuda(cudaMemcpy(t.data(), d_buf + per, per * 4, cudaMemcpyDeviceToHost));
    const int32_t half = (int32_t)((q - 1) / 2);
    for (size_t e = 0; e < per && !rc; ++e)
      key->a_host[(size_t)k * per + e] = (int16_t)((int32_t)t[e] > half ? (int32_t)t[e] - (int32_t)q : (int32_t)t[e]);
  }
  cudaFree(d_buf);
  if (!rc) rc = lb_key_finish(key);
  if (rc) {
    lc_lb_key_destroy(key);
    return rc;
  }
  *out = key;
  return LC_OK;
}

LC_API void lc_lb_key_destroy(lc_lb_key* key) {
  if (!key) return;
  cudaFree(key->d_a);
  cudaFree(key->d_limb);
  cudaFree(key->d_partial);
  cudaFree(key->d_in);
  cudaFree(key->d_out);
  delete key;
}

LC_API int lc_lb_key_info(const lc_lb_key* key, size_t* len_f162, uint32_t* limbs, uint16_t* primes, int16_t* a) {
  if (!key) return LC_ERR_INVALID_ARGUMENT;
  if (len_f162) *len_f162 = key->len_f162;
  if (limbs) *limbs = key->limbs;
  if (primes) std::copy(key->primes.begin(), key->primes.end(), primes);
  if (a) std::copy(key->a_host.begin(), key->a_host.end(), a);
  return LC_OK;
}

LC_API int lc_lb_ntt(const lc_lb_key* key, uint32_t limb, const uint32_t* in, uint32_t* out, size_t count,
                     lc_stream stream) {
  using namespace lc;
  if (!key || limb >= key->limbs || ((!in || !out) && count)) return LC_ERR_INVALID_ARGUMENT;
  return lb_ntt_run(key->d_limb + limb, in, out, count, (cudaStream_t)stream);
}

LC_API int lc_lb_commit(lc_lb_key* key, const uint64_t* witness, uint32_t r, uint32_t* raw, int16_t* matrix,
                        uint32_t* batches, lc_stream stream) {
  using namespace lc;
  if (!key || !witness || !raw || !matrix) return LC_ERR_INVALID_ARGUMENT;
  if (r < 2 || (r & (r - 1)) || r > (1u << 15)) return LC_ERR_INVALID_ARGUMENT;  // key.rs:388-391
  const uint32_t nr = (uint32_t)key->nr;
  const int sms = std::max(1, device_sm_count());
  // at least 16 CTAs per SM when the problem allows, about 8 ring elements per
  // warp (64 per CTA), so the last wave is a small fraction of the launch
  uint32_t splits = (uint32_t)std::max<size_t>(1, (size_t)16 * sms / ((size_t)r * key->limbs));
  splits = std::max<uint32_t>(splits, nr / (8 * kLbWarps));
  splits = std::min<uint32_t>(splits, std::max<uint32_t>(1, nr / kLbWarps));
  // at most about 64 CTAs per SM in all: bounds the partial sums [limb][column][split][648]
  splits = std::min<uint32_t>(splits, (uint32_t)std::max<size_t>(1, (size_t)64 * sms / ((size_t)r * key->limbs)));
  const uint32_t per = (nr + splits - 1) / splits;
  splits = (nr + per - 1) / per;
  int rc = grow((void**)&key->d_partial, &key->partial_bytes, (size_t)key->limbs * r * splits * kLbN * 4);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  LbCommitParams p{witness, key->d_a, key->d_limb, key->d_partial, batches, nr, splits, per, r, key->len_f162};
  lb_commit_kernel<<<dim3(splits, r, key->limbs), kLbWarps * 32, 0, st>>>(p);
  rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  LbFinishParams f{key->d_partial, key->d_limb, raw, matrix, splits, r, key->limbs};
  lb_finish_kernel<<<dim3(r, key->limbs), 256, 0, st>>>(f);
  return map_cuda(cudaGetLastError());
}

// Host buffers: witness [r * len_f162][3] u64 in, raw / matrix / batches out
// (batches may be null); synchronous.
LC_API int lc_lb_commit_host(lc_lb_key* key, const uint64_t* witness, uint32_t r, uint32_t* raw, int16_t* matrix,
                             uint32_t* batches) {
  using namespace lc;
  if (!key || !witness || !raw || !matrix) return LC_ERR_INVALID_ARGUMENT;
  if (r < 2 || (r & (r - 1)) || r > (1u << 15)) return LC_ERR_INVALID_ARGUMENT;
  const size_t wbytes = (size_t)r * key->len_f162 * 24;
  const size_t raw_b = (size_t)key->limbs * r * kLbN * 4, mat_b = (size_t)4 * r * key->limbs * kLbN162 * 2;
  const size_t bat_b = batches ? (size_t)r * key->nr * kLbN * 4 : 0;
  int rc = grow((void**)&key->d_in, &key->in_bytes, wbytes);
  if (!rc) rc = grow(&key->d_out, &key->out_bytes, raw_b + mat_b + bat_b);
  if (rc) return rc;
  char* o = static_cast<char*>(key->d_out);
  rc = map_cuda(cudaMemcpy(key->d_in, witness, wbytes, cudaMemcpyHostToDevice));
  if (!rc)
    rc = lc_lb_commit(key, key->d_in, r, (uint32_t*)o, (int16_t*)(o + raw_b),
                      batches ? (uint32_t*)(o + raw_b + mat_b) : nullptr, nullptr);
  if (!rc) rc = map_cuda(cudaMemcpy(raw, o, raw_b, cudaMemcpyDeviceToHost));
  if (!rc) rc = map_cuda(cudaMemcpy(matrix, o + raw_b, mat_b, cudaMemcpyDeviceToHost));
  if (!rc && batches) rc = map_cuda(cudaMemcpy(batches, o + raw_b + mat_b, bat_b, cudaMemcpyDeviceToHost));
  return rc;
}

// random_elems (binfield.rs:186-189): n uniform F162 elements as [n][3] u64 (host)
LC_API int lc_lb_random_elems(size_t n, uint64_t seed, uint64_t* out) {
  if (n && !out) return LC_ERR_INVALID_ARGUMENT;
  lc::LbRng rng(seed);
  for (size_t i = 0; i < n; ++i) {
    out[3 * i] = rng.next();
    out[3 * i + 1] = rng.next();
    out[3 * i + 2] = rng.next() & ((1ull << 34) - 1);
  }
  return LC_OK;
}

}  // extern "C"
