// commit.cu -- Ajtai commitment c = A.w, cached-NTT form (sm_100a).
//
// Restates AjtaiPublicKey::commit (lattice-commitment/src/ajtai.rs:118-153):
//   t_i = INTT( sum_j NTT(A_ij) (.) NTT(s_j) ),  i < k, j < m,
// for a batch of B witnesses at once, over a u32 modulus (Modulus32, e.g.
// Q_32) or over Goldilocks.  Zero witness elements contribute nothing, which
// is exactly the reference's skip (ajtai.rs:128-137); every output is a
// canonical residue, bit-identical to the reference.
//
// Device layouts (t = NTT slot, j = witness element, i = row, b = witness):
//   key   Ahat_T[t][j][i_pad]      cached NTT(A), i padded to 16 with zeros
//   Ŵ     What_T[t][j][b_pad]      witness NTT, written frequency-major
//   parts partial[split][t][i][b] K-split partial sums, canonical residues
//   Ĉ     Chat[b][i][t]            summed evaluations -> inverse NTT -> out
// so that the per-frequency products C_t = A_t^T . W_t read contiguous rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "internal.h"
#include "mac.cuh"
#include "ntt_kernels.cuh"

namespace lc {

constexpr int kBTile = 128;  // witnesses per MAC tile


// ------------------------------------------------------------------ kernels

// Cached-key layout: Ahat[i][j][t] (k x m ring elements, natural NTT output)
// -> Ahat_T[t][j][i_pad], rows i >= k zero.  One CTA per witness slot j.
template <class E>
__global__ void key_transpose_kernel(const E* __restrict__ ahat, E* __restrict__ out, uint32_t k,
                                     uint32_t m, uint32_t n) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  E* tile = reinterpret_cast<E*>(smem_raw);  // [kIPad][n]
  const uint32_t j = blockIdx.x;
  for (uint32_t e = threadIdx.x; e < (uint32_t)kIPad * n; e += blockDim.x) {
    const uint32_t i = e / n, t = e % n;
    tile[e] = i < k ? ahat[((size_t)i * m + j) * n + t] : E(0);
  }
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < (uint32_t)kIPad * n; e += blockDim.x) {
    const uint32_t t = e / kIPad, i = e % kIPad;
    out[((size_t)t * m + j) * kIPad + i] = tile[i * n + t];
  }
}

// Input element conversion for the witness: residues pass through, int8
// digits map to their residue (NeoRing::small, lattice-folding/src/neo.rs:98-109).
template <class E, class S>
LC_D E to_residue(S x, uint32_t q);
template <>
LC_D uint64_t to_residue<uint64_t, uint64_t>(uint64_t x, uint32_t) {
  return x;
}
template <>
LC_D uint32_t to_residue<uint32_t, uint32_t>(uint32_t x, uint32_t) {
  return x;
}
template <>
LC_D uint64_t to_residue<uint64_t, int8_t>(int8_t x, uint32_t) {
  return x >= 0 ? (uint64_t)x : kGlP - (uint64_t)(-(int)x);
}
template <>
LC_D uint32_t to_residue<uint32_t, int8_t>(int8_t x, uint32_t q) {
  return x >= 0 ? (uint32_t)x : q - (uint32_t)(-(int)x);
}
// unsigned digits (decomp_b rows, lattice-folding/src/neo.rs:253-266); every
// supported modulus exceeds 255
template <>
LC_D uint64_t to_residue<uint64_t, uint8_t>(uint8_t x, uint32_t) {
  return x;
}
template <>
LC_D uint32_t to_residue<uint32_t, uint8_t>(uint8_t x, uint32_t) {
  return x;
}

// Witness NTT, frequency-major output.  CTA (j, b-block of BB witnesses):
// loads the BB polynomials w[b][j][*] (16-byte vector loads when aligned),
// transforms them in shared memory and writes What_T[t][j][b0 + b] -- for
// each NTT slot t one contiguous run of BB values -- with zeros for
// b >= batch so the padded columns of the product tiles are exact zeros.
// Slots are SS elements apart: odd strides keep the transposed store
// bank-conflict free.
template <class A, int LOG_N>
struct WitnessSlotStride;
template <class A>
struct WitnessSlotStride<A, 6> {
  static constexpr int value = sizeof(typename A::T) == 8 ? 73 : 75;
};
template <class A>
struct WitnessSlotStride<A, 7> {
  static constexpr int value = 137;
};
template <class A>
struct WitnessSlotStride<A, 8> {
  static constexpr int value = 273;
};

// A CTA takes JB consecutive ring elements j of BB witnesses (JB = 1 for the
// tiled batches; small batches take several j so that a CTA still holds about
// a hundred polynomials).  Polynomial p = jj*BB + b of the tile sits in slot p.
template <class A, class S, int LOG_N, int LOG_V, int NT, int BB, int JB = 1>
__global__ void __launch_bounds__(NT)
    witness_ntt_kernel(const S* __restrict__ w, typename A::T* __restrict__ what_t, uint32_t m,
                       uint32_t batch, uint32_t b_pad, const typename A::Tw* __restrict__ twg,
                       uint32_t q, uint32_t qinv) {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int PP = BB * JB;  // polynomials per CTA
  constexpr int N = G::N, GROUPS = NT / G::T, IT = PP / GROUPS;
  constexpr int SS = WitnessSlotStride<A, LOG_N>::value;
  static_assert(PP % GROUPS == 0, "tile");
  static_assert(SS >= Slots<A, LOG_N, LOG_V>::S, "slot stride");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Tw* tw = reinterpret_cast<Tw*>(smem_raw);
  T* slots = reinterpret_cast<T*>(smem_raw + ((G::fwd_entries() * sizeof(Tw) + 15) / 16 * 16));
  const uint32_t j0 = blockIdx.x * JB;
  const uint32_t b0 = blockIdx.y * BB;
  for (int i = threadIdx.x; i < G::fwd_entries(); i += NT) tw[i] = twg[i];
  constexpr int EPC = 16 / sizeof(S);  // elements per 16-byte chunk
  constexpr int CH = N / EPC;          // chunks per polynomial
  const bool vec = (N * sizeof(S)) % 16 == 0 && (reinterpret_cast<uintptr_t>(w) & 15) == 0;
  if (vec) {
    for (int e = threadIdx.x; e < PP * CH; e += NT) {
      const int pp = e / CH, k = e % CH;
      const int jj = pp / BB, b = pp % BB;
      T* dst = slots + pp * SS + k * EPC;
      if (b0 + b < batch && j0 + jj < m) {
        const uint4 v =
            *reinterpret_cast<const uint4*>(w + ((size_t)(b0 + b) * m + j0 + jj) * N + (size_t)k * EPC);
        const S* x = reinterpret_cast<const S*>(&v);
#pragma unroll
        for (int u = 0; u < EPC; ++u) dst[u] = to_residue<T, S>(x[u], q);
      } else {
#pragma unroll
        for (int u = 0; u < EPC; ++u) dst[u] = 0;
      }
    }
  } else {
    for (int e = threadIdx.x; e < PP * N; e += NT) {
      const int pp = e / N, c = e % N;
      const int jj = pp / BB, b = pp % BB;
      T v = 0;
      if (b0 + b < batch && j0 + jj < m) v = to_residue<T, S>(w[((size_t)(b0 + b) * m + j0 + jj) * N + c], q);
      slots[pp * SS + c] = v;
    }
  }
  __syncthreads();
  const A ar = make_arith_q<A>(q, qinv);
  const int grp = threadIdx.x / G::T;
  const uint32_t t = threadIdx.x % G::T;
#pragma unroll 1
  for (int it = 0; it < IT; ++it)
    transform_slot<A, LOG_N, LOG_V, false>(slots + (it * GROUPS + grp) * SS, tw, ar, t);
  __syncthreads();
  // for each slot tt the tile's (jj, b) values are one contiguous run when BB == b_pad
  for (int e = threadIdx.x; e < PP * N; e += NT) {
    const int tt = e / PP, pp = e % PP;
    const int jj = pp / BB, b = pp % BB;
    if (b0 + b < b_pad && j0 + jj < m)
      what_t[((size_t)tt * m + j0 + jj) * b_pad + b0 + b] = slots[pp * SS + tt];
  }
}

// Generic witness path (ring degrees without a fused kernel): element
// conversion into [b][j][t] residues, then the batched NTT, then this
// transpose into What_T[t][j][b_pad] (zero columns b >= batch).
template <class E, class S>
__global__ void witness_convert_kernel(const S* __restrict__ w, E* __restrict__ out, size_t count,
                                       uint32_t q) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = to_residue<E, S>(w[i], q);
}

template <class E>
__global__ void witness_transpose_kernel(const E* __restrict__ in, E* __restrict__ what_t, uint32_t m,
                                         uint32_t n, uint32_t batch, uint32_t b_pad) {
  __shared__ E tile[32][33];
  const uint32_t j = blockIdx.z;
  const uint32_t t0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
  for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t b = b0 + k, t = t0 + threadIdx.x;
    tile[k][threadIdx.x] = (b < batch && t < n) ? in[((size_t)b * m + j) * n + t] : E(0);
  }
  __syncthreads();
  for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t t = t0 + k, b = b0 + threadIdx.x;
    if (t < n && b < b_pad) what_t[((size_t)t * m + j) * b_pad + b] = tile[threadIdx.x][k];
  }
}

// Per-frequency product, tiled: CTA (t, b-tile, split) accumulates
// C_t[i][b] = sum_j Ahat_T[t][j][i] What_T[t][j][b] over its j-range for all
// 16 (padded) rows and 128 witnesses; 256 threads, each 2 rows x 4 witnesses
// (witnesses tb, tb+32, tb+64, tb+96).  Shared-memory rows are double-buffered
// with TMA bulk copies.
template <class E, int JB>
struct MacCfg {
  static constexpr int NT = 256;
  static constexpr size_t A_BYTES = (size_t)JB * kIPad * sizeof(E);
  static constexpr size_t W_BYTES = (size_t)JB * kBTile * sizeof(E);
  static constexpr size_t STAGE = A_BYTES + W_BYTES;
  static constexpr size_t SMEM = 2 * STAGE + 16;
};

// One product work item (slot t, b-tile bt, K split) of the tiled form.  The
// caller initialises the two stage barriers once; `parity` carries their
// phases across the items a CTA runs.  Returns false after a timed-out wait
// (the error word is set and the CTA's copies have been waited for).
template <class E, int JB>
LC_D bool mac_tile(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t, E* __restrict__ partial,
                   uint32_t m, uint32_t b_pad, uint32_t n, uint32_t splits, uint32_t q, uint32_t* err, uint32_t t,
                   uint32_t bt, uint32_t split, unsigned char* smem_raw, uint64_t* bar, uint32_t& parity) {
  using C = MacCfg<E, JB>;
  const uint32_t per = (m + splits - 1) / splits;
  const uint32_t j0 = split * per, j1 = min(m, j0 + per);
  const int tid = threadIdx.x;
  const int ti = tid >> 5, tb = tid & 31;
  auto stage_a = [&](int s) { return reinterpret_cast<E*>(smem_raw + s * C::STAGE); };
  auto stage_w = [&](int s) { return reinterpret_cast<E*>(smem_raw + s * C::STAGE + C::A_BYTES); };
  auto issue = [&](uint32_t jb, int s) {
    const uint32_t rows = min((uint32_t)JB, j1 - jb);
    const uint32_t a_bytes = rows * kIPad * sizeof(E);
    mbar_arrive_expect_tx(&bar[s], a_bytes + rows * kBTile * (uint32_t)sizeof(E));
    bulk_g2s(stage_a(s), ahat_t + ((size_t)t * am + jb) * kIPad, a_bytes, &bar[s]);
    if (b_pad == kBTile) {
      bulk_g2s(stage_w(s), what_t + ((size_t)t * m + jb) * b_pad, rows * kBTile * sizeof(E), &bar[s]);
    } else {
      for (uint32_t r = 0; r < rows; ++r)
        bulk_g2s(stage_w(s) + r * kBTile, what_t + ((size_t)t * m + jb + r) * b_pad + bt * kBTile,
                 kBTile * sizeof(E), &bar[s]);
    }
  };
  Acc160 acc[2][4];
  const uint32_t nblk = (j1 > j0) ? (j1 - j0 + JB - 1) / JB : 0;
  if (tid == 0 && nblk > 0) issue(j0, 0);
  bool failed = false;
  uint32_t failed_blk = 0;
  for (uint32_t k = 0; k < nblk; ++k) {
    const int s = k & 1;
    if (tid == 0 && k + 1 < nblk) issue(j0 + (k + 1) * JB, s ^ 1);
    const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
    parity ^= 1u << s;
    if (__syncthreads_or(!ok)) {
      failed = true;
      failed_blk = k;
      break;
    }
    const E* As = stage_a(s);
    const E* Ws = stage_w(s);
    const uint32_t rows = min((uint32_t)JB, j1 - (j0 + k * JB));
#pragma unroll 2
    for (uint32_t r = 0; r < rows; ++r) {
      const E a0 = As[r * kIPad + 2 * ti], a1 = As[r * kIPad + 2 * ti + 1];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const E wv = Ws[r * kBTile + tb + 32 * u];
        mac<E>(acc[0][u], a0, wv);
        mac<E>(acc[1][u], a1, wv);
      }
    }
    __syncthreads();  // stage s is refilled by the next iteration's issue
  }
  if (failed) {
    if (tid == 0) {
      record_error(err, LC_DEVERR_TIMEOUT);
      // Copies that may still be landing must finish before the CTA moves on:
      // the block whose wait expired (its phase is the one before the
      // toggle) and the prefetch of the following block.  Bounded waits; if
      // either expires again, the error word is marked poisoned.
      const int f = failed_blk & 1;
      bool landed = mbar_wait(&bar[f], ((parity >> f) & 1u) ^ 1u);
      if (failed_blk + 1 < nblk) {
        const int o = f ^ 1;
        landed = mbar_wait(&bar[o], (parity >> o) & 1u) && landed;
      }
      if (!landed) record_poisoned(err);
    }
    return false;
  }
  // partial[split][t][i][b]
  for (int ii = 0; ii < 2; ++ii)
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = 2 * ti + ii, b = bt * kBTile + tb + 32 * u;
      partial[(((size_t)split * n + t) * kIPad + i) * b_pad + b] = acc_reduce<E>(acc[ii][u], q);
    }
  return true;
}

template <class E, int JB>
__global__ void __launch_bounds__(256)
    mac_tiled_kernel(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t, E* __restrict__ partial,
                     uint32_t m, uint32_t b_pad, uint32_t n, uint32_t splits, uint32_t q,
                     uint32_t* err) {
  using C = MacCfg<E, JB>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * C::STAGE);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t parity = 0;
  mac_tile<E, JB>(ahat_t, am, what_t, partial, m, b_pad, n, splits, q, err, blockIdx.x, blockIdx.y, blockIdx.z,
                  smem_raw, bar, parity);
}

// Small-batch product for b_pad a multiple of 4: one thread per (split, t,
// row pair, 4 witnesses), 8 accumulators, so each A pair and each witness
// quad is loaded once per 8 multiply-adds.  Lanes run along the row pairs
// (one 128-byte A row per slot), then the witness quads (broadcast loads);
// both streams are prefetched into L2 16 ring elements ahead (the loop is
// otherwise bound by DRAM latency).
template <class E>
LC_D void mac_quad_items(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t,
                         E* __restrict__ partial, uint32_t m, uint32_t b_pad, uint32_t n, uint32_t splits,
                         uint32_t kappa, uint32_t q, size_t first, size_t stride) {
  const uint32_t npair = (kappa + 1) / 2, nquad = b_pad / 4;
  const size_t total = (size_t)splits * n * nquad * npair;
  for (size_t idx = first; idx < total; idx += stride) {
    const uint32_t ip = idx % npair;
    const uint32_t bq = (idx / npair) % nquad;
    const uint32_t t = (idx / ((size_t)npair * nquad)) % n;
    const uint32_t split = (uint32_t)(idx / ((size_t)npair * nquad * n));
    const uint32_t per = (m + splits - 1) / splits;
    const uint32_t j0 = split * per, j1 = min(m, j0 + per);
    Acc160 acc[2][4];
    const E* ap = ahat_t + ((size_t)t * am + j0) * kIPad + 2 * ip;
    const E* wp = what_t + ((size_t)t * m + j0) * b_pad + 4 * bq;
#pragma unroll 2
    for (uint32_t j = j0; j < j1; ++j) {
      // both streams run along j: bring the rows 16 ring elements ahead into L2
      if (j + 16 < j1) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(ap + 16 * kIPad));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(wp + (size_t)16 * b_pad));
      }
      const E a0 = ap[0], a1 = ap[1];
      E wv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) wv[u] = wp[u];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        mac<E>(acc[0][u], a0, wv[u]);
        mac<E>(acc[1][u], a1, wv[u]);
      }
      ap += kIPad;
      wp += b_pad;
    }
    for (int ii = 0; ii < 2; ++ii)
      for (int u = 0; u < 4; ++u)
        partial[(((size_t)split * n + t) * kIPad + 2 * ip + ii) * b_pad + 4 * bq + u] =
            acc_reduce<E>(acc[ii][u], q);
  }
}

template <class E>
__global__ void __launch_bounds__(256)
    mac_quad_kernel(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t, E* __restrict__ partial,
                    uint32_t m, uint32_t b_pad, uint32_t n, uint32_t splits, uint32_t kappa, uint32_t q) {
  mac_quad_items<E>(ahat_t, am, what_t, partial, m, b_pad, n, splits, kappa, q,
                    blockIdx.x * (size_t)blockDim.x + threadIdx.x, (size_t)gridDim.x * blockDim.x);
}

// Small-batch product: one thread per (split, t, i, b).
template <class E>
LC_D void mac_small_items(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t,
                          E* __restrict__ partial, uint32_t m, uint32_t b_pad, uint32_t n, uint32_t splits,
                          uint32_t kappa, uint32_t batch, uint32_t q, size_t first, size_t stride) {
  const size_t total = (size_t)splits * n * kappa * batch;
  for (size_t idx = first; idx < total; idx += stride) {
    const uint32_t b = idx % batch;
    const uint32_t i = (idx / batch) % kappa;
    const uint32_t t = (idx / ((size_t)batch * kappa)) % n;
    const uint32_t split = idx / ((size_t)batch * kappa * n);
    const uint32_t per = (m + splits - 1) / splits;
    const uint32_t j0 = split * per, j1 = min(m, j0 + per);
    Acc160 acc;
    for (uint32_t j = j0; j < j1; ++j)
      mac<E>(acc, ahat_t[((size_t)t * am + j) * kIPad + i], what_t[((size_t)t * m + j) * b_pad + b]);
    partial[(((size_t)split * n + t) * kIPad + i) * b_pad + b] = acc_reduce<E>(acc, q);
  }
}

template <class E>
__global__ void mac_small_kernel(const E* __restrict__ ahat_t, uint32_t am, const E* __restrict__ what_t,
                                 E* __restrict__ partial, uint32_t m, uint32_t b_pad, uint32_t n,
                                 uint32_t splits, uint32_t kappa, uint32_t batch, uint32_t q) {
  mac_small_items<E>(ahat_t, am, what_t, partial, m, b_pad, n, splits, kappa, batch, q,
                     blockIdx.x * (size_t)blockDim.x + threadIdx.x, (size_t)gridDim.x * blockDim.x);
}

// ------------------------------------------------------------------ single-launch commit
//
// A small commitment (at most 4 witnesses, a few thousand ring elements) in
// one kernel: CTA c takes ring elements [c*jc, c*jc + jc) of every witness,
// runs their forward transforms in shared memory, multiplies them against
// the cached NTT(A) slots of every row and adds each canonical partial sum v
// into two 64-bit accumulators in global memory, one for the low and one for
// the high 32 bits of v (atomic adds whose result is not read back; neither
// sum can wrap for fewer than 2^32 CTAs).  The CTA that takes the last
// ticket forms low + high * 2^32 as a 128-bit value, reduces it mod q, zeroes
// the accumulators and the ticket for the next call, runs the batch x kappa
// inverse transforms in shared memory and writes the rows.  No CTA ever
// waits for another; the accumulators and the ticket are zero between calls.
struct FusedCommitParams {
  const void* w;      // [batch][m][n] witness (residues or byte digits)
  const void* ahat_t; // Ahat_T[t][j][i_pad]
  unsigned long long* acc;  // [batch][kappa][n] x {sum of low halves, sum of high halves}
  uint32_t* ticket;
  void* out;          // [batch][kappa][n]
  const void* twf;    // forward / inverse twiddle tables of the plan
  const void* twi;
  uint32_t batch, m, am, kappa, jc, nc, q, qinv;
};

template <class A, int LOG_N, int LOG_V>
struct FusedCommitCfg {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  static constexpr int NT = 256;
  static constexpr int GROUPS = NT / G::T;  // polynomials per transform pass
  static constexpr int SS = WitnessSlotStride<A, LOG_N>::value;
  static constexpr int MAX_ROWS = 4 * kIPad;  // batch x kappa rows of the last CTA
  static constexpr int SLOTS = GROUPS > MAX_ROWS ? GROUPS : MAX_ROWS;
  static constexpr size_t TWF = ((size_t)G::fwd_entries() * sizeof(Tw) + 15) / 16 * 16;
  static constexpr size_t TWI = ((size_t)G::inv_entries() * sizeof(Tw) + 15) / 16 * 16;
  static constexpr size_t SMEM = TWF + TWI + (size_t)SLOTS * SS * sizeof(T);
  static_assert(MAX_ROWS % GROUPS == 0, "inverse passes stay inside the slots");
};

template <class A, class S, int LOG_N, int LOG_V>
__global__ void __launch_bounds__(256) commit_fused_kernel(const __grid_constant__ FusedCommitParams p) {
  using C = FusedCommitCfg<A, LOG_N, LOG_V>;
  using G = typename C::G;
  using E = typename A::T;
  using Tw = typename A::Tw;
  constexpr int N = G::N, SS = C::SS, NT = C::NT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint32_t is_last;
  Tw* twf = reinterpret_cast<Tw*>(smem_raw);
  Tw* twi = reinterpret_cast<Tw*>(smem_raw + C::TWF);
  E* slots = reinterpret_cast<E*>(smem_raw + C::TWF + C::TWI);
  const int tid = threadIdx.x;
  const uint32_t j0 = blockIdx.x * p.jc;
  const uint32_t jn = min(p.jc, p.m - j0);
  const E* ahat = reinterpret_cast<const E*>(p.ahat_t);
  // this CTA's rows of Ahat_T (one run of jn * 16 entries per slot) into L2
  // while the witness is loaded and transformed
  {
    constexpr uint32_t kLine = 128 / sizeof(E);
    const uint32_t run = jn * kIPad, lines = (run + kLine - 1) / kLine;
    for (uint32_t e = tid; e < N * lines; e += NT) {
      const E* a = ahat + ((size_t)(e / lines) * p.am + j0) * kIPad + (e % lines) * kLine;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
    }
  }
  for (int i = tid; i < G::fwd_entries(); i += NT) twf[i] = reinterpret_cast<const Tw*>(p.twf)[i];
  for (int i = tid; i < G::inv_entries(); i += NT) twi[i] = reinterpret_cast<const Tw*>(p.twi)[i];

  // ---- witness ring elements of this CTA: polynomial jj*batch + b in slot jj*batch + b
  const uint32_t pp = jn * p.batch;
  const S* w = reinterpret_cast<const S*>(p.w);
  for (int e = tid; e < C::GROUPS * N; e += NT) {
    const uint32_t pi = e / N, c = e % N;
    E v = 0;
    if (pi < pp) {
      const uint32_t jj = pi / p.batch, b = pi % p.batch;
      v = to_residue<E, S>(w[((size_t)b * p.m + j0 + jj) * N + c], p.q);
    }
    slots[pi * SS + c] = v;
  }
  __syncthreads();
  const A ar = make_arith_q<A>(p.q, p.qinv);
  const int grp = tid / G::T;
  const uint32_t t = (uint32_t)(tid % G::T);
  transform_slot<A, LOG_N, LOG_V, false>(slots + grp * SS, twf, ar, t);
  __syncthreads();

  // ---- products of this CTA's ring elements; output (b, slot tt, row i), i fastest
  const uint32_t outs = p.batch * N * p.kappa;
  for (uint32_t o = tid; o < outs; o += NT) {
    const uint32_t i = o % p.kappa, tt = (o / p.kappa) % N, b = o / (p.kappa * N);
    const E* ap = ahat + ((size_t)tt * p.am + j0) * kIPad + i;
    Acc160 acc;
#pragma unroll 4
    for (uint32_t jj = 0; jj < jn; ++jj) mac<E>(acc, ap[(size_t)jj * kIPad], slots[(jj * p.batch + b) * SS + tt]);
    const uint64_t v = (uint64_t)acc_reduce<E>(acc, p.q);
    unsigned long long* a2 = p.acc + 2 * (((size_t)b * p.kappa + i) * N + tt);
    atomicAdd(a2, (unsigned long long)(v & 0xffffffffu));
    if (v >> 32) atomicAdd(a2 + 1, (unsigned long long)(v >> 32));
  }
  __threadfence();  // this thread's additions are visible before the ticket
  __syncthreads();
  if (tid == 0) is_last = atomicAdd(p.ticket, 1u) == p.nc - 1 ? 1u : 0u;
  __syncthreads();
  if (!is_last) return;
  __threadfence();

  // ---- last CTA: accumulators -> canonical evaluations -> inverse transforms
  const uint32_t rows = p.batch * p.kappa;
  for (uint32_t e = tid; e < rows * N; e += NT) {
    const uint32_t r = e / N, tt = e % N;
    unsigned long long* a2 = p.acc + 2 * ((size_t)r * N + tt);
    const uint64_t sl = __ldcg(a2), sh = __ldcg(a2 + 1);
    // x = sl + sh * 2^32 < 2^96
    const uint64_t lo = sl + (sh << 32);
    const uint64_t hi = (sh >> 32) + (lo < sl ? 1u : 0u);
    slots[r * SS + tt] = Field<E>::reduce160((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi,
                                             (uint32_t)(hi >> 32), 0, p.q);
    __stcg(a2, 0ull);
    __stcg(a2 + 1, 0ull);
  }
  if (tid == 0) *p.ticket = 0;
  __syncthreads();
  // whole passes of GROUPS slots: groups past `rows` transform unused slots
  for (uint32_t base = 0; base < rows; base += C::GROUPS)
    transform_slot<A, LOG_N, LOG_V, true>(slots + (base + grp) * SS, twi, ar, t);
  __syncthreads();
  E* out = reinterpret_cast<E*>(p.out);
  for (uint32_t e = tid; e < rows * N; e += NT) out[e] = slots[(e / N) * SS + e % N];
}

// Chat[b][i][t] = sum_split partial[split][t][i][b]  (mod q)
template <class E>
__global__ void reduce_partials_kernel(const E* __restrict__ partial, E* __restrict__ chat,
                                       uint32_t splits, uint32_t n, uint32_t kappa, uint32_t batch,
                                       uint32_t b_pad, uint32_t q) {
  const size_t total = (size_t)batch * kappa * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const uint32_t t = idx % n;
    const uint32_t i = (idx / n) % kappa;
    const uint32_t b = idx / ((size_t)n * kappa);
    E s = 0;
    for (uint32_t sp = 0; sp < splits; ++sp)
      s = Field<E>::add(s, partial[(((size_t)sp * n + t) * kIPad + i) * b_pad + b], q);
    chat[idx] = s;
  }
}

// ------------------------------------------------------------------ products, split sum and inverse NTT in one launch
//
// The staged form's last three launches -- the products with K split across
// CTAs, the modular sum of the splits, the batched inverse NTT -- as one
// cooperative kernel, i.e. the whole of ajtai.rs:139-150 after the witness
// transforms, in three phases separated by grid barriers (bounded spins on a
// counter zeroed in the stream before the launch; the cooperative launch
// makes every CTA resident): (1) the product items of the shape's form
// (tiled, quad or small) over the persistent grid, partial[split][t][i][b];
// (2) every thread of the grid sums the splits of some outputs into
// Chat[b][i][t]; (3) groups of 32 rows (b, i) are loaded into shared memory,
// inverse-transformed there and written straight to out[b][i][..].
enum : int { kFormTiled = 0, kFormQuad = 1, kFormSmall = 2 };
constexpr uint32_t kInttRows = 32;  // rows (b, i) per phase-3 item

struct MacInttParams {
  const void* ahat_t;
  const void* what_t;
  void* partial;
  void* chat;
  void* out;
  const void* twi;
  uint32_t am, m, b_pad, n, splits, kappa, batch, q, qinv, btiles;
  uint32_t* err;
  unsigned int* barrier;
};

template <class A, int LOG_N, int LOG_V, int JB, int FORM>
struct MacInttCfg {
  using E = typename A::T;
  using Tw = typename A::Tw;
  using G = Geo<LOG_N, LOG_V>;
  static constexpr int NT = 256;
  static constexpr size_t PH1 = FORM == kFormTiled ? MacCfg<E, JB>::SMEM : 0;  // stages + barriers
  static constexpr size_t OFF2 = (PH1 + 127) / 128 * 128;
  static constexpr size_t TWI = ((size_t)G::inv_entries() * sizeof(Tw) + 15) / 16 * 16;
  static constexpr int SS = WitnessSlotStride<A, LOG_N>::value;
  static constexpr size_t SMEM = OFF2 + TWI + (size_t)kInttRows * SS * sizeof(E);
  static constexpr int GROUPS = NT / G::T;
  static_assert(kInttRows % GROUPS == 0, "whole transform passes");
};

// Every CTA arrives once per barrier (the `round`-th barrier of the launch
// waits for round * gridDim arrivals); false if the others did not all arrive
// within the spin bound (the error word is set).
LC_D bool grid_barrier(unsigned int* ctr, uint32_t round, uint32_t* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this CTA's writes are visible before it arrives
    atomicAdd(ctr, 1u);
    const unsigned int target = round * gridDim.x;
    // polls back off from 64 ns to 2 us, so that CTAs which finished early do
    // not flood the counter's L2 line while the others still load; at most
    // 2^20 polls (about two seconds)
    bool ok = false;
    uint32_t ns = 64;
    for (uint32_t i = 0; i < (1u << 20); ++i) {
      if (*reinterpret_cast<volatile unsigned int*>(ctr) >= target) {
        ok = true;
        break;
      }
      __nanosleep(ns);
      ns = ns < 2048 ? 2 * ns : ns;
    }
    __threadfence();
    if (!ok) record_error(err, LC_DEVERR_TIMEOUT);
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <class A, int LOG_N, int LOG_V, int JB, int FORM>
__global__ void __launch_bounds__(256, 2) commit_mac_intt_kernel(const __grid_constant__ MacInttParams p) {
  using C = MacInttCfg<A, LOG_N, LOG_V, JB, FORM>;
  using E = typename A::T;
  using Tw = typename A::Tw;
  using G = typename C::G;
  constexpr int N = G::N, SS = C::SS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const E* ahat = static_cast<const E*>(p.ahat_t);
  const E* what = static_cast<const E*>(p.what_t);
  E* part = static_cast<E*>(p.partial);
  E* chat = static_cast<E*>(p.chat);
  const int tid = threadIdx.x;
  const size_t gtid = blockIdx.x * (size_t)blockDim.x + tid, gthreads = (size_t)gridDim.x * blockDim.x;

  // ---- phase 1: the product items
  bool ok = true;
  if constexpr (FORM == kFormTiled) {
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * MacCfg<E, JB>::STAGE);
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    uint32_t parity = 0;
    const uint32_t items = p.n * p.btiles * p.splits;
    for (uint32_t it = blockIdx.x; it < items && ok; it += gridDim.x) {
      const uint32_t t = it % p.n, rest = it / p.n;
      ok = mac_tile<E, JB>(ahat, p.am, what, part, p.m, p.b_pad, p.n, p.splits, p.q, p.err, t, rest % p.btiles,
                           rest / p.btiles, smem_raw, bar, parity);
    }
  } else if constexpr (FORM == kFormQuad) {
    mac_quad_items<E>(ahat, p.am, what, part, p.m, p.b_pad, p.n, p.splits, p.kappa, p.q, gtid, gthreads);
  } else {
    mac_small_items<E>(ahat, p.am, what, part, p.m, p.b_pad, p.n, p.splits, p.kappa, p.batch, p.q, gtid,
                       gthreads);
  }
  // a CTA whose products timed out still arrives, so no other CTA waits on it
  if (!grid_barrier(p.barrier, 1, p.err)) return;

  // ---- phase 2: Chat[b][i][t] = sum over the splits, every thread of the grid
  const size_t outs = (size_t)p.batch * p.kappa * N;
  for (size_t idx = gtid; idx < outs; idx += gthreads) {
    const uint32_t t = idx % N, i = (idx / N) % p.kappa;
    const uint32_t b = (uint32_t)(idx / ((size_t)N * p.kappa));
    const E* src = part + ((size_t)t * kIPad + i) * p.b_pad + b;
    const size_t sstride = (size_t)N * kIPad * p.b_pad;
    E s0 = 0, s1 = 0, s2 = 0, s3 = 0;  // four loads in flight
    uint32_t sp = 0;
    for (; sp + 4 <= p.splits; sp += 4) {
      const E v0 = __ldcg(src + sp * sstride), v1 = __ldcg(src + (sp + 1) * sstride);
      const E v2 = __ldcg(src + (sp + 2) * sstride), v3 = __ldcg(src + (sp + 3) * sstride);
      s0 = Field<E>::add(s0, v0, p.q);
      s1 = Field<E>::add(s1, v1, p.q);
      s2 = Field<E>::add(s2, v2, p.q);
      s3 = Field<E>::add(s3, v3, p.q);
    }
    for (; sp < p.splits; ++sp) s0 = Field<E>::add(s0, __ldcg(src + sp * sstride), p.q);
    chat[idx] = Field<E>::add(Field<E>::add(s0, s1, p.q), Field<E>::add(s2, s3, p.q), p.q);
  }
  if (!grid_barrier(p.barrier, 2, p.err)) return;
  if (*reinterpret_cast<volatile uint32_t*>(p.err) != 0) return;  // some CTA failed: outputs are not formed

  // ---- phase 3: inverse transforms of 32 rows (b, i) per item, into the output
  Tw* twi = reinterpret_cast<Tw*>(smem_raw + C::OFF2);
  E* slots = reinterpret_cast<E*>(smem_raw + C::OFF2 + C::TWI);
  for (int i = tid; i < G::inv_entries(); i += C::NT) twi[i] = static_cast<const Tw*>(p.twi)[i];
  const A ar = make_arith_q<A>(p.q, p.qinv);
  const int grp = tid / G::T;
  const uint32_t lt = (uint32_t)(tid % G::T);
  const uint32_t rows = p.batch * p.kappa;
  E* out = static_cast<E*>(p.out);
  for (uint32_t r0 = blockIdx.x * kInttRows; r0 < rows; r0 += gridDim.x * kInttRows) {
    const uint32_t nr = min(kInttRows, rows - r0);
    __syncthreads();  // twiddles written; the previous item's slots are read out
    for (uint32_t e = tid; e < kInttRows * N; e += C::NT) {
      const uint32_t rr = e / N, c = e % N;
      slots[rr * SS + c] = rr < nr ? __ldcg(chat + (size_t)(r0 + rr) * N + c) : E(0);
    }
    __syncthreads();
#pragma unroll 1
    for (uint32_t base = 0; base < kInttRows; base += C::GROUPS)
      transform_slot<A, LOG_N, LOG_V, true>(slots + (base + grp) * SS, twi, ar, lt);
    __syncthreads();
    for (uint32_t e = tid; e < nr * N; e += C::NT) out[(size_t)r0 * N + e] = slots[(e / N) * SS + e % N];
  }
}

// ------------------------------------------------------------------ split sums and inverse NTT in one launch
//
// After the tiled products (a handful of K splits), the rest of ajtai.rs:
// 139-150 for ROWS output rows per CTA: rows (b0 .. b0 + ROWS - 1, i),
// summed over the splits straight into shared-memory slots (consecutive
// threads take consecutive witnesses b, so every read of
// partial[split][t][i][b] is one contiguous run), inverse-transformed there
// and written to out[b][i][..] -- no Chat round trip and no second launch.
struct SumInttParams {
  const void* partial;  // [splits][n][kIPad][b_pad]
  void* out;            // [batch][kappa][n]
  const void* twi;      // inverse twiddle table of the plan
  uint32_t splits, kappa, batch, b_pad, q, qinv;
};

template <class A, int LOG_N, int LOG_V>
struct SumInttCfg {
  using E = typename A::T;
  using G = Geo<LOG_N, LOG_V>;
  static constexpr int NT = 256;          // the split sums: all threads
  static constexpr int XT = 128;          // the transform: the first four warps
  static constexpr int ROWS = XT / G::T;  // one transform pass
  static constexpr int SS = WitnessSlotStride<A, LOG_N>::value;
  static constexpr size_t TWI = ((size_t)G::inv_entries() * sizeof(typename A::Tw) + 15) / 16 * 16;
  static constexpr size_t SMEM = TWI + (size_t)ROWS * SS * sizeof(E);
};

template <class A, int LOG_N, int LOG_V>
__global__ void __launch_bounds__(256) sum_intt_kernel(const __grid_constant__ SumInttParams p) {
  using C = SumInttCfg<A, LOG_N, LOG_V>;
  using E = typename A::T;
  using Tw = typename A::Tw;
  using G = typename C::G;
  constexpr int N = G::N, SS = C::SS, ROWS = C::ROWS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Tw* twi = reinterpret_cast<Tw*>(smem_raw);
  E* slots = reinterpret_cast<E*>(smem_raw + C::TWI);
  const int tid = threadIdx.x;
  for (int e = tid; e < G::inv_entries(); e += C::NT) twi[e] = static_cast<const Tw*>(p.twi)[e];
  const uint32_t i = blockIdx.x % p.kappa, b0 = (blockIdx.x / p.kappa) * ROWS;
  const E* part = static_cast<const E*>(p.partial);
  const size_t sstride = (size_t)N * kIPad * p.b_pad;  // one K split
  for (int e = tid; e < ROWS * N; e += C::NT) {
    const uint32_t rr = e % ROWS, t = e / ROWS, b = b0 + rr;
    E s = 0;
    if (b < p.batch) {
      const E* src = part + ((size_t)t * kIPad + i) * p.b_pad + b;
      for (uint32_t sp = 0; sp < p.splits; sp += 8) {  // up to eight loads in flight, then their sum
        E v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = sp + k < p.splits ? __ldg(src + (sp + k) * sstride) : E(0);
#pragma unroll
        for (int k = 0; k < 8; ++k) s = Field<E>::add(s, v[k], p.q);
      }
    }
    slots[rr * SS + t] = s;
  }
  __syncthreads();
  if (tid < C::XT) {  // whole warps: the transform's __syncwarp sees all its lanes
    const A ar = make_arith_q<A>(p.q, p.qinv);
    transform_slot<A, LOG_N, LOG_V, true>(slots + (tid / G::T) * SS, twi, ar, (uint32_t)(tid % G::T));
  }
  __syncthreads();
  E* out = static_cast<E*>(p.out);
  for (int e = tid; e < ROWS * N; e += C::NT) {
    const uint32_t rr = e / N, c = e % N, b = b0 + rr;
    if (b < p.batch) out[((size_t)b * p.kappa + i) * N + c] = slots[rr * SS + c];
  }
}

}  // namespace lc

using namespace lc;

// ------------------------------------------------------------------ key object

// struct lc_ajtai_key is defined in internal.h


namespace lc {

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

static uint32_t choose_splits(uint32_t n, uint32_t btiles, uint32_t m) {
  const int sms = device_sm_count();
  const uint32_t target = (uint32_t)std::max(1, sms * 3);  // about three CTAs per SM
  uint32_t s = std::max<uint32_t>(1, target / std::max<uint32_t>(1, n * btiles));
  s = std::min<uint32_t>(s, std::max<uint32_t>(1, m / 64));
  return std::max<uint32_t>(s, 1);
}

template <class A, int LOG_N, int LOG_V, class S, int NT, int BB, int JB = 1>
static int launch_witness_cfg(const lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                              typename A::T* dst, cudaStream_t st) {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  constexpr int SS = WitnessSlotStride<A, LOG_N>::value;
  const size_t smem = ((G::fwd_entries() * sizeof(typename A::Tw) + 15) / 16 * 16) +
                      (size_t)BB * JB * SS * sizeof(T);
  auto kern = witness_ntt_kernel<A, S, LOG_N, LOG_V, NT, BB, JB>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return map_cuda(e);
  dim3 grid((key->m + JB - 1) / JB, (unsigned)((b_pad + BB - 1) / BB));
  const lc_ntt_plan* plan = key->plan;
  kern<<<grid, NT, smem, st>>>(w, dst, key->m, (uint32_t)batch, b_pad,
                               reinterpret_cast<const typename A::Tw*>(plan->d_tw_fwd), plan->q[0],
                               plan->qinv[0]);
  return map_cuda(cudaGetLastError());
}

// Polynomials per CTA of the small-batch tiles: as many slots as fit in
// 96 KB, a multiple of the 128-thread CTA's polynomial groups, at most 128.
template <class A, int LOG_N, int LOG_V>
struct SmallWitnessTile {
  static constexpr int groups = 128 / Geo<LOG_N, LOG_V>::T;
  static constexpr int fit = (96 * 1024) / (WitnessSlotStride<A, LOG_N>::value * (int)sizeof(typename A::T));
  static constexpr int polys = (fit > 128 ? 128 : fit) / groups * groups;
};

// 128 witnesses per CTA when the batch is tiled and 128 slots fit in 160 KB of
// shared memory (64 otherwise); small batches: 8, 4 or 1 witnesses by as many
// ring elements as fill SmallWitnessTile, 32 witnesses when b_pad is neither.
template <class A, int LOG_N, int LOG_V, class S>
static int launch_witness_to(const lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                             typename A::T* dst, cudaStream_t st) {
  constexpr bool fits128 =
      (size_t)128 * WitnessSlotStride<A, LOG_N>::value * sizeof(typename A::T) <= 160 * 1024;
  if (b_pad % 128 == 0) {
    if constexpr (fits128)
      return launch_witness_cfg<A, LOG_N, LOG_V, S, 256, 128>(key, w, batch, b_pad, dst, st);
    else
      return launch_witness_cfg<A, LOG_N, LOG_V, S, 256, 64>(key, w, batch, b_pad, dst, st);
  }
  constexpr int PP = SmallWitnessTile<A, LOG_N, LOG_V>::polys;
  constexpr int G = SmallWitnessTile<A, LOG_N, LOG_V>::groups;
  static_assert(PP >= 8 && PP % 8 == 0 && G % 8 == 0, "small tile");
  // tiny problems (fewer polynomials than full tiles for every SM): one
  // polynomial per thread group, so the grid still spreads over the SMs
  const bool tiny = (size_t)key->m * b_pad < (size_t)std::max(1, device_sm_count()) * PP;
  if (b_pad % 8 == 0)
    return tiny ? launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 8, G / 8>(key, w, batch, b_pad, dst, st)
                : launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 8, PP / 8>(key, w, batch, b_pad, dst, st);
  if (b_pad % 4 == 0)
    return tiny ? launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 4, G / 4>(key, w, batch, b_pad, dst, st)
                : launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 4, PP / 4>(key, w, batch, b_pad, dst, st);
  if (b_pad < 4)
    return tiny ? launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 1, G>(key, w, batch, b_pad, dst, st)
                : launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 1, PP>(key, w, batch, b_pad, dst, st);
  return launch_witness_cfg<A, LOG_N, LOG_V, S, 128, 32>(key, w, batch, b_pad, dst, st);
}

template <class A, int LOG_N, int LOG_V, class S>
static int launch_witness_ntt(lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                              cudaStream_t st) {
  return launch_witness_to<A, LOG_N, LOG_V, S>(key, w, batch, b_pad,
                                               reinterpret_cast<typename A::T*>(key->d_what_t), st);
}

template <class E, class S>
static int witness_ntt_generic(lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                               cudaStream_t st) {
  const size_t count = batch * key->m * key->n;
  int rc = grow(&key->d_wtmp, &key->wtmp_bytes, count * sizeof(E));
  if (rc) return rc;
  E* tmp = reinterpret_cast<E*>(key->d_wtmp);
  const unsigned blocks = (unsigned)std::min<size_t>((count + 255) / 256, 65535);
  witness_convert_kernel<E, S><<<blocks, 256, 0, st>>>(w, tmp, count, key->plan->q[0]);
  rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  rc = run_ntt(key->plan, tmp, tmp, batch * key->m, false, st);
  if (rc) return rc;
  dim3 grid((key->n + 31) / 32, (b_pad + 31) / 32, key->m);
  witness_transpose_kernel<E><<<grid, dim3(32, 8), 0, st>>>(tmp, reinterpret_cast<E*>(key->d_what_t),
                                                             key->m, key->n, (uint32_t)batch, b_pad);
  return map_cuda(cudaGetLastError());
}

template <class A, class S>
static int witness_ntt_as(lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad, cudaStream_t st) {
  switch (key->log_n) {
    case 6: return launch_witness_ntt<A, 6, 3, S>(key, w, batch, b_pad, st);
    case 7: return launch_witness_ntt<A, 7, 4, S>(key, w, batch, b_pad, st);
    case 8: return launch_witness_ntt<A, 8, 4, S>(key, w, batch, b_pad, st);
    default: return witness_ntt_generic<typename A::T, S>(key, w, batch, b_pad, st);
  }
}

template <class S>
static int witness_ntt(lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad, cudaStream_t st) {
  const PlanKind kind = key->plan->kind;
  if constexpr (std::is_same<S, int8_t>::value || std::is_same<S, uint8_t>::value) {
    // d = 64 Goldilocks byte digits: the transform as exact INT8 tensor-core
    // products when the shape allows (large problems), identical residues
    if (kind == PlanKind::Goldilocks && key->log_n == 6) {
      const int rc = tc_witness_ntt(w, std::is_same<S, int8_t>::value, batch, key->m, b_pad,
                                    reinterpret_cast<uint64_t*>(key->d_what_t), key->d_err, st);
      if (rc != LC_ERR_UNSUPPORTED) return rc;
    }
  }
  if constexpr (!std::is_same<S, uint32_t>::value) {
    if (kind == PlanKind::Goldilocks) return witness_ntt_as<Goldilocks, S>(key, w, batch, b_pad, st);
  }
  if constexpr (!std::is_same<S, uint64_t>::value) {
    if (kind == PlanKind::U32Lazy) return witness_ntt_as<ShoupLazy, S>(key, w, batch, b_pad, st);
    if (kind == PlanKind::U32Mont) return witness_ntt_as<MontCanon, S>(key, w, batch, b_pad, st);
  }
  return LC_ERR_INVALID_ARGUMENT;
}

// One cooperative launch: products of `form`, split sums, inverse transforms.
template <class A, int LOG_N, int LOG_V, int FORM>
static int launch_mac_intt(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, uint32_t btiles,
                           void* out, cudaStream_t st) {
  using E = typename A::T;
  constexpr int JB = sizeof(E) == 8 ? 16 : 32;
  using C = MacInttCfg<A, LOG_N, LOG_V, JB, FORM>;
  auto kern = commit_mac_intt_kernel<A, LOG_N, LOG_V, JB, FORM>;
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = smem_attr_once(attr_done, kern, C::SMEM);
  if (e != cudaSuccess) return map_cuda(e);
  if (!key->d_grid) {
    if (cudaMalloc(&key->d_grid, 256) != cudaSuccess) {
      cudaGetLastError();
      return LC_ERR_OUT_OF_MEMORY;
    }
  }
  e = cudaMemsetAsync(key->d_grid, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return map_cuda(e);
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, C::SMEM);
  if (e != cudaSuccess) return map_cuda(e);
  if (per_sm < 1) return LC_ERR_UNSUPPORTED;
  const uint32_t n = key->n, kappa = key->k;
  const size_t resident = (size_t)per_sm * device_sm_count();
  if (FORM == kFormTiled) {
    // enough K splits for at least four waves of the resident grid, so the
    // last, partly filled wave is short (at least 64 ring elements per item)
    const size_t per_split = (size_t)n * btiles;
    const size_t want = (4 * resident + per_split - 1) / per_split;
    splits = (uint32_t)std::max<size_t>(
        splits, std::min<size_t>(want, std::max<uint32_t>(1, key->m / 64)));
    const int rc = grow(&key->d_partial, &key->partial_bytes, (size_t)splits * n * kIPad * b_pad * sizeof(E));
    if (rc) return rc;
  }
  size_t work1;
  if (FORM == kFormTiled)
    work1 = (size_t)n * btiles * splits;
  else if (FORM == kFormQuad)
    work1 = ((size_t)splits * n * (b_pad / 4) * ((kappa + 1) / 2) + C::NT - 1) / C::NT;
  else
    work1 = ((size_t)splits * n * kappa * batch + C::NT - 1) / C::NT;
  const size_t work2 = ((size_t)batch * kappa + kInttRows - 1) / kInttRows;
  const size_t grid = std::max<size_t>(1, std::min<size_t>(resident, std::max(work1, work2)));
  MacInttParams prm{};
  prm.ahat_t = key->d_ahat_t;
  prm.what_t = key->d_what_t;
  prm.partial = key->d_partial;
  prm.chat = key->d_chat;
  prm.out = out;
  prm.twi = key->plan->d_tw_inv;
  prm.am = key->a_m;
  prm.m = key->m;
  prm.b_pad = b_pad;
  prm.n = n;
  prm.splits = splits;
  prm.kappa = kappa;
  prm.batch = (uint32_t)batch;
  prm.q = key->plan->q[0];
  prm.qinv = key->plan->qinv[0];
  prm.btiles = btiles;
  prm.err = key->d_err;
  prm.barrier = key->d_grid;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(C::NT);
  cfg.dynamicSmemBytes = C::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return map_cuda(cudaLaunchKernelEx(&cfg, kern, prm));
}

template <class A, int FORM>
static int mac_intt_as(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, uint32_t btiles, void* out,
                       cudaStream_t st) {
  switch (key->log_n) {
    case 6: return launch_mac_intt<A, 6, 3, FORM>(key, batch, b_pad, splits, btiles, out, st);
    case 7: return launch_mac_intt<A, 7, 4, FORM>(key, batch, b_pad, splits, btiles, out, st);
    case 8: return launch_mac_intt<A, 8, 4, FORM>(key, batch, b_pad, splits, btiles, out, st);
    default: return LC_ERR_UNSUPPORTED;
  }
}

template <class E, int FORM>
static int mac_intt(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, uint32_t btiles, void* out,
                    cudaStream_t st) {
  const PlanKind kind = key->plan->kind;
  if constexpr (std::is_same<E, uint64_t>::value) {
    if (kind == PlanKind::Goldilocks) return mac_intt_as<Goldilocks, FORM>(key, batch, b_pad, splits, btiles, out, st);
  } else {
    if (kind == PlanKind::U32Lazy) return mac_intt_as<ShoupLazy, FORM>(key, batch, b_pad, splits, btiles, out, st);
    if (kind == PlanKind::U32Mont) return mac_intt_as<MontCanon, FORM>(key, batch, b_pad, splits, btiles, out, st);
  }
  return LC_ERR_UNSUPPORTED;
}

template <class A, int LOG_N, int LOG_V>
static int launch_sum_intt(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, void* out,
                           cudaStream_t st) {
  using C = SumInttCfg<A, LOG_N, LOG_V>;
  auto kern = sum_intt_kernel<A, LOG_N, LOG_V>;
  static std::atomic<uint64_t> attr_done{0};
  const cudaError_t e = smem_attr_once(attr_done, kern, C::SMEM);
  if (e != cudaSuccess) return map_cuda(e);
  SumInttParams prm{};
  prm.partial = key->d_partial;
  prm.out = out;
  prm.twi = key->plan->d_tw_inv;
  prm.splits = splits;
  prm.kappa = key->k;
  prm.batch = (uint32_t)batch;
  prm.b_pad = b_pad;
  prm.q = key->plan->q[0];
  prm.qinv = key->plan->qinv[0];
  const size_t grid = (size_t)key->k * ((batch + C::ROWS - 1) / C::ROWS);
  kern<<<(unsigned)grid, C::NT, C::SMEM, st>>>(prm);
  return map_cuda(cudaGetLastError());
}

template <class A>
static int sum_intt_as(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, void* out,
                       cudaStream_t st) {
  switch (key->log_n) {
    case 6: return launch_sum_intt<A, 6, 3>(key, batch, b_pad, splits, out, st);
    case 7: return launch_sum_intt<A, 7, 4>(key, batch, b_pad, splits, out, st);
    case 8: return launch_sum_intt<A, 8, 4>(key, batch, b_pad, splits, out, st);
    default: return LC_ERR_UNSUPPORTED;
  }
}

// The tiled form's split sums and inverse transforms as one launch
// (sum_intt_kernel); LC_ERR_UNSUPPORTED outside d = 64 .. 256.
template <class E>
static int sum_intt(lc_ajtai_key* key, size_t batch, uint32_t b_pad, uint32_t splits, void* out, cudaStream_t st) {
  const PlanKind kind = key->plan->kind;
  if constexpr (std::is_same<E, uint64_t>::value) {
    if (kind == PlanKind::Goldilocks) return sum_intt_as<Goldilocks>(key, batch, b_pad, splits, out, st);
  } else {
    if (kind == PlanKind::U32Lazy) return sum_intt_as<ShoupLazy>(key, batch, b_pad, splits, out, st);
    if (kind == PlanKind::U32Mont) return sum_intt_as<MontCanon>(key, batch, b_pad, splits, out, st);
  }
  return LC_ERR_UNSUPPORTED;
}

template <class E>
static int commit_core(lc_ajtai_key* key, size_t batch, uint32_t b_pad, void* out, cudaStream_t st) {
  const uint32_t n = key->n, m = key->m, kappa = key->k;
  const uint32_t q = key->plan->q[0];
  // the per-slot products as byte-limb GEMMs on the tensor cores
  if (key->slot_products == LC_PRODUCTS_TENSOR) {
    int rc = grow(&key->d_chat, &key->chat_bytes, (size_t)batch * kappa * n * sizeof(E));
    if (rc) return rc;
    rc = tc_slot_products(key->d_ahat_t, key->a_m, key->d_what_t, (uint32_t)sizeof(E), q, m, n, kappa, batch,
                          b_pad, &key->d_partial, &key->partial_bytes, key->d_chat, key->d_err, st);
    if (rc == LC_OK) return run_ntt(key->plan, key->d_chat, out, (size_t)batch * kappa, true, st);
    if (rc != LC_ERR_UNSUPPORTED) return rc;
  }
  const bool tiled = b_pad % kBTile == 0;
  const bool quad = !tiled && b_pad % 4 == 0;
  const uint32_t btiles = tiled ? b_pad / kBTile : 1;
  // small batches: about 2^18 threads (2^19 quad threads), each summing a
  // contiguous j-range
  const size_t outs = quad ? (size_t)n * ((kappa + 1) / 2) * (b_pad / 4) : (size_t)n * kappa * batch;
  const size_t want = quad ? ((size_t)1 << 19) : ((size_t)1 << 18);
  // (each product thread sums at least 32 ring elements, so small commits keep
  // few partial sums to add up afterwards)
  const uint32_t splits =
      tiled ? choose_splits(n, btiles, m)
            : (uint32_t)std::max<size_t>(
                  1, std::min<size_t>(std::max<size_t>(1, m / 32), want / std::max<size_t>(1, outs)));
  int rc = grow(&key->d_partial, &key->partial_bytes, (size_t)splits * n * kIPad * b_pad * sizeof(E));
  if (rc) return rc;
  rc = grow(&key->d_chat, &key->chat_bytes, (size_t)batch * kappa * n * sizeof(E));
  if (rc) return rc;
  // the products, their split sums and the inverse transforms in one launch:
  // by default for the smallest batches (at most 3 witnesses), where it
  // measured faster than the three launches below; for every form when the
  // key asks for it (lc_ajtai_key_set_fused(key, 2)); never with 0
  const int form = tiled ? kFormTiled : quad ? kFormQuad : kFormSmall;
  if (key->fused && key->log_n >= 6 && key->log_n <= 8 && (key->fused == 2 || form == kFormSmall)) {
    rc = form == kFormTiled ? mac_intt<E, kFormTiled>(key, batch, b_pad, splits, btiles, out, st)
         : form == kFormQuad ? mac_intt<E, kFormQuad>(key, batch, b_pad, splits, btiles, out, st)
                             : mac_intt<E, kFormSmall>(key, batch, b_pad, splits, btiles, out, st);
    if (rc != LC_ERR_UNSUPPORTED) return rc;
  }
  const E* ahat = reinterpret_cast<const E*>(key->d_ahat_t);
  const E* what = reinterpret_cast<const E*>(key->d_what_t);
  E* part = reinterpret_cast<E*>(key->d_partial);
  if (tiled) {
    constexpr int JB = sizeof(E) == 8 ? 16 : 32;
    using MC = MacCfg<E, JB>;
    auto kern = mac_tiled_kernel<E, JB>;
    static std::atomic<uint64_t> attr_done{0};
    {
      const cudaError_t e = smem_attr_once(attr_done, kern, MC::SMEM);
      if (e != cudaSuccess) return map_cuda(e);
    }
    kern<<<dim3(n, btiles, splits), MC::NT, MC::SMEM, st>>>(ahat, key->a_m, what, part, m, b_pad, n, splits, q,
                                                           key->d_err);
  } else if (quad) {
    const size_t total = (size_t)splits * n * ((kappa + 1) / 2) * (b_pad / 4);
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 65535);
    mac_quad_kernel<E><<<blocks, 256, 0, st>>>(ahat, key->a_m, what, part, m, b_pad, n, splits, kappa, q);
  } else {
    const size_t total = (size_t)splits * n * kappa * batch;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 65535);
    mac_small_kernel<E><<<blocks, 256, 0, st>>>(ahat, key->a_m, what, part, m, b_pad, n, splits, kappa,
                                                (uint32_t)batch, q);
  }
  rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  if (tiled) {
    // few K splits: their sums and the inverse transforms in one launch
    rc = sum_intt<E>(key, batch, b_pad, splits, out, st);
    if (rc != LC_ERR_UNSUPPORTED) return rc;
  }
  {
    const size_t total = (size_t)batch * kappa * n;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 65535);
    reduce_partials_kernel<E><<<blocks, 256, 0, st>>>(part, reinterpret_cast<E*>(key->d_chat), splits,
                                                      n, kappa, (uint32_t)batch, b_pad, q);
    rc = map_cuda(cudaGetLastError());
    if (rc) return rc;
  }
  // inverse NTT of the batch*kappa summed rows, straight into the output
  return run_ntt(key->plan, key->d_chat, out, (size_t)batch * kappa, true, st);
}

// Single-launch commit (commit_fused_kernel) for small problems: at most
// kFusedMaxBatch witnesses, kFusedMaxM ring elements and kFusedMaxMacs
// multiply-adds, where the staged launches cost more than their work.
constexpr size_t kFusedMaxBatch = 4;
constexpr uint32_t kFusedMaxM = 2048;
constexpr size_t kFusedMaxMacs = (size_t)1 << 20;

template <class A, class S, int LOG_N, int LOG_V>
static int launch_commit_fused(lc_ajtai_key* key, const S* w, size_t batch, void* out, cudaStream_t st) {
  using C = FusedCommitCfg<A, LOG_N, LOG_V>;
  constexpr uint32_t N = 1u << LOG_N;
  // accumulators for the largest batch of this key, zeroed once; every call
  // leaves them zero again
  if (!key->d_fused) {
    const size_t bytes = 16 + kFusedMaxBatch * key->k * N * 16;
    int rc = grow(&key->d_fused, &key->fused_bytes, bytes);
    if (rc) return rc;
    rc = map_cuda(cudaMemsetAsync(key->d_fused, 0, bytes, st));
    if (rc) return rc;
  }
  auto kern = commit_fused_kernel<A, S, LOG_N, LOG_V>;
  static std::atomic<uint64_t> attr_done{0};
  {
    const cudaError_t e = smem_attr_once(attr_done, kern, C::SMEM);
    if (e != cudaSuccess) return map_cuda(e);
  }
  // ring elements per CTA: about 16 multiply-adds per thread and at least 8
  // (few atomic additions per product), within one transform pass
  const uint32_t per_thread = (uint32_t)((batch * N * key->k + C::NT - 1) / C::NT);
  uint32_t jc = std::max<uint32_t>(8, 16 / std::max<uint32_t>(1, per_thread));
  jc = std::max<uint32_t>(1, std::min<uint32_t>(jc, (uint32_t)(C::GROUPS / batch)));
  FusedCommitParams p{};
  p.w = w;
  p.ahat_t = key->d_ahat_t;
  p.ticket = static_cast<uint32_t*>(key->d_fused);
  p.acc = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(key->d_fused) + 16);
  p.out = out;
  p.twf = key->plan->d_tw_fwd;
  p.twi = key->plan->d_tw_inv;
  p.batch = (uint32_t)batch;
  p.m = key->m;
  p.am = key->a_m;
  p.kappa = key->k;
  p.jc = jc;
  p.nc = (key->m + jc - 1) / jc;
  p.q = key->plan->q[0];
  p.qinv = key->plan->qinv[0];
  kern<<<p.nc, C::NT, C::SMEM, st>>>(p);
  return map_cuda(cudaGetLastError());
}

template <class A, class S>
static int commit_fused_as(lc_ajtai_key* key, const S* w, size_t batch, void* out, cudaStream_t st) {
  switch (key->log_n) {
    case 6: return launch_commit_fused<A, S, 6, 3>(key, w, batch, out, st);
    case 7: return launch_commit_fused<A, S, 7, 4>(key, w, batch, out, st);
    case 8: return launch_commit_fused<A, S, 8, 4>(key, w, batch, out, st);
    default: return LC_ERR_UNSUPPORTED;
  }
}

// LC_ERR_UNSUPPORTED when the problem is not small enough for one launch.
template <class S>
static int commit_fused(lc_ajtai_key* key, const S* w, size_t batch, void* out, cudaStream_t st) {
  if (!key->fused || batch > kFusedMaxBatch || key->m > kFusedMaxM || key->log_n < 6 || key->log_n > 8)
    return LC_ERR_UNSUPPORTED;
  if ((size_t)key->m * batch * key->n * key->k > kFusedMaxMacs) return LC_ERR_UNSUPPORTED;
  const PlanKind kind = key->plan->kind;
  if constexpr (!std::is_same<S, uint32_t>::value) {
    if (kind == PlanKind::Goldilocks) return commit_fused_as<Goldilocks, S>(key, w, batch, out, st);
  }
  if constexpr (!std::is_same<S, uint64_t>::value) {
    if (kind == PlanKind::U32Lazy) return commit_fused_as<ShoupLazy, S>(key, w, batch, out, st);
    if (kind == PlanKind::U32Mont) return commit_fused_as<MontCanon, S>(key, w, batch, out, st);
  }
  return LC_ERR_UNSUPPORTED;
}

template <class S>
static int commit_any(lc_ajtai_key* key, const S* w, size_t batch, void* out, cudaStream_t st) {
  if (batch == 0) return LC_OK;
  if (batch > (1u << 24)) return LC_ERR_INVALID_ARGUMENT;
  {
    const int rc = commit_fused<S>(key, w, batch, out, st);
    key->last_fused = rc == LC_OK;
    if (rc != LC_ERR_UNSUPPORTED) return rc;
  }
  // tiles of 128 witnesses from 64 on; from 4 on a multiple of 4 (zero
  // columns) for the quad product
  const uint32_t b_pad = batch >= 64 ? (uint32_t)((batch + kBTile - 1) / kBTile * kBTile)
                                     : batch >= 4 ? (uint32_t)((batch + 3) / 4 * 4) : (uint32_t)batch;
  const size_t eb = key->wide ? 8 : 4;
  int rc = grow(&key->d_what_t, &key->what_bytes, (size_t)key->n * key->m * b_pad * eb);
  if (rc) return rc;
  rc = witness_ntt<S>(key, w, batch, b_pad, st);
  if (rc) return rc;
  return key->wide ? commit_core<uint64_t>(key, batch, b_pad, out, st)
                   : commit_core<uint32_t>(key, batch, b_pad, out, st);
}

// ------------------------------------------------------------------ no-allocation commit
//
// Scratch of lc_ajtai_commit_noalloc: one fixed array in device memory, part
// of this library's module, so a commit through that entry point never calls
// cudaMalloc/cudaFree.  Every GPU that loads the library holds these bytes
// until the process exits.  In host code the symbol is only a stand-in; its
// device address comes from cudaGetSymbolAddress, once per device.
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static void* g_noalloc_addr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device (set up on the
// first call per device).
static int noalloc_scratch_addr(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return map_cuda(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return LC_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return map_cuda(e);
    g_noalloc_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  return LC_OK;
}

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Witness NTT of the fused path into an explicit destination.
template <class A, int LOG_N, int LOG_V, class S>
static int noalloc_witness_ntt(const lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                               typename A::T* dst, cudaStream_t st) {
  return launch_witness_to<A, LOG_N, LOG_V, S>(key, w, batch, b_pad, dst, st);
}

template <class A, class S>
static int noalloc_witness_as(const lc_ajtai_key* key, const S* w, size_t batch, uint32_t b_pad,
                              typename A::T* dst, cudaStream_t st) {
  switch (key->log_n) {
    case 6: return noalloc_witness_ntt<A, 6, 3, S>(key, w, batch, b_pad, dst, st);
    case 7: return noalloc_witness_ntt<A, 7, 4, S>(key, w, batch, b_pad, dst, st);
    case 8: return noalloc_witness_ntt<A, 8, 4, S>(key, w, batch, b_pad, dst, st);
    default: return LC_ERR_UNSUPPORTED;
  }
}

// The commit of commit_any/commit_core with every scratch buffer carved out
// of the fixed array; rejects requests that do not fit.
template <class E>
static int noalloc_commit(const lc_ajtai_key* key, const E* s, size_t batch, void* out, cudaStream_t st) {
  if (batch == 0) return LC_OK;
  if (key->log_n < 6 || key->log_n > 8) return LC_ERR_UNSUPPORTED;
  const uint32_t n = key->n, m = key->m, kappa = key->k;
  const uint32_t b_pad = batch >= 64 ? (uint32_t)((batch + kBTile - 1) / kBTile * kBTile) : (uint32_t)batch;
  const bool tiled = b_pad % kBTile == 0;
  const uint32_t btiles = tiled ? b_pad / kBTile : 1;
  const size_t what_bytes = align256((size_t)n * m * b_pad * sizeof(E));
  const size_t chat_bytes = align256((size_t)batch * kappa * n * sizeof(E));
  const size_t part_unit = (size_t)n * kIPad * b_pad * sizeof(E);  // one K-split
  if (what_bytes + chat_bytes + part_unit > kNoAllocScratchBytes) return LC_ERR_INVALID_ARGUMENT;
  const size_t outs = (size_t)n * kappa * batch;
  uint32_t splits =
      tiled ? choose_splits(n, btiles, m)
            : (uint32_t)std::max<size_t>(1, std::min<size_t>(m, ((size_t)1 << 18) / std::max<size_t>(1, outs)));
  const size_t fit = (kNoAllocScratchBytes - what_bytes - chat_bytes) / part_unit;
  splits = (uint32_t)std::max<size_t>(1, std::min<size_t>(splits, fit));

  unsigned char* base = nullptr;
  int rc = noalloc_scratch_addr(&base);
  if (rc) return rc;
  E* what = reinterpret_cast<E*>(base);
  E* chat = reinterpret_cast<E*>(base + what_bytes);
  E* part = reinterpret_cast<E*>(base + what_bytes + chat_bytes);

  const PlanKind kind = key->plan->kind;
  if constexpr (std::is_same<E, uint64_t>::value) {
    rc = noalloc_witness_as<Goldilocks, E>(key, s, batch, b_pad, what, st);
  } else {
    rc = kind == PlanKind::U32Lazy ? noalloc_witness_as<ShoupLazy, E>(key, s, batch, b_pad, what, st)
                                   : noalloc_witness_as<MontCanon, E>(key, s, batch, b_pad, what, st);
  }
  if (rc) return rc;
  const uint32_t q = key->plan->q[0];
  if (tiled) {
    constexpr int JB = sizeof(E) == 8 ? 16 : 32;
    using MC = MacCfg<E, JB>;
    auto kern = mac_tiled_kernel<E, JB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MC::SMEM);
    if (e != cudaSuccess) return map_cuda(e);
    kern<<<dim3(n, btiles, splits), MC::NT, MC::SMEM, st>>>(
        reinterpret_cast<const E*>(key->d_ahat_t), key->a_m, what, part, m, b_pad, n, splits, q, key->d_err);
  } else {
    const size_t total = (size_t)splits * n * kappa * batch;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 65535);
    mac_small_kernel<E><<<blocks, 256, 0, st>>>(reinterpret_cast<const E*>(key->d_ahat_t), key->a_m, what, part,
                                                m, b_pad, n, splits, kappa, (uint32_t)batch, q);
  }
  rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  const size_t total = (size_t)batch * kappa * n;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 65535);
  reduce_partials_kernel<E><<<blocks, 256, 0, st>>>(part, chat, splits, n, kappa, (uint32_t)batch,
                                                    b_pad, q);
  rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  return run_ntt(key->plan, chat, out, (size_t)batch * kappa, true, st);
}

}  // namespace lc

namespace lc {

// Arguments a key can be created with (LC_OK) or the status that refuses them.
int key_create_check(const lc_ntt_plan* plan, uint32_t k, uint32_t m, uint32_t flags) {
  if (flags & ~LC_KEY_TENSOR_I8) return LC_ERR_INVALID_ARGUMENT;
  if (plan->num_moduli != 1) return LC_ERR_UNSUPPORTED;
  if ((flags & LC_KEY_TENSOR_I8) && (plan->kind != PlanKind::Goldilocks || plan->log_n != 6))
    return LC_ERR_UNSUPPORTED;
  if (k > (uint32_t)kIPad) return LC_ERR_UNSUPPORTED;
  if (plan->log_n > (plan->kind == PlanKind::Goldilocks ? 9u : 10u)) return LC_ERR_UNSUPPORTED;
  (void)m;
  return LC_OK;
}

// A key from the coefficient-form matrix in `tmp` (device memory holding
// k*m*n residues, row-major (i, j)), which the call takes over: it is
// transformed in place, transposed into the key's Ahat_T and freed, on every
// return path.  One device synchronisation reports the kernels' errors.
int key_create_from(const lc_ntt_plan* plan, uint32_t k, uint32_t m, void* tmp, uint32_t flags,
                    lc_ajtai_key** out) {
  lc_ajtai_key* key = new (std::nothrow) lc_ajtai_key();
  if (!key) {
    cudaFree(tmp);
    return LC_ERR_OUT_OF_MEMORY;
  }
  key->k = k;
  key->m = m;
  key->a_m = m;
  key->log_n = plan->log_n;
  key->n = 1u << plan->log_n;
  key->wide = plan->kind == PlanKind::Goldilocks;
  int rc;
  if (key->wide)
    rc = lc_ntt_plan_create_goldilocks(plan->log_n, &key->plan);
  else
    rc = lc_ntt_plan_create_u32(plan->log_n, plan->q, plan->two_adicity, plan->generator, 1, &key->plan);
  if (rc) {
    cudaFree(tmp);
    delete key;
    return rc;
  }
  const size_t eb = key->wide ? 8 : 4;
  if (cudaMalloc(&key->d_ahat_t, (size_t)key->n * m * kIPad * eb) != cudaSuccess ||
      cudaMalloc(&key->d_err, 4) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(tmp);
    lc_ajtai_key_destroy(key);
    return LC_ERR_OUT_OF_MEMORY;
  }
  cudaMemsetAsync(key->d_err, 0, 4, nullptr);
  // the tensor-core witness transform's matrix image (once per device; a
  // failure only leaves the CUDA-core transform in use)
  if (plan->kind == PlanKind::Goldilocks && plan->log_n == 6) tc_ntt_prepare();
  // rotation-limb tables from the coefficient form (before it is transformed in place)
  if (flags & LC_KEY_TENSOR_I8) {
    rc = tc_tables_create(static_cast<const uint64_t*>(tmp), k, m, &key->tc);
    if (rc) {
      cudaFree(tmp);
      lc_ajtai_key_destroy(key);
      return rc;
    }
    key->engine = LC_ENGINE_TENSOR_I8;
  }
  // cached NTT of every entry (AjtaiPublicKey::from_seed, ajtai.rs:91-96)
  rc = run_ntt(key->plan, tmp, tmp, (size_t)k * m, false, nullptr);
  if (!rc) {
    const size_t smem = (size_t)kIPad * key->n * eb;
    if (smem > 48 * 1024) {
      cudaFuncSetAttribute(key_transpose_kernel<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      cudaFuncSetAttribute(key_transpose_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
    }
    if (key->wide)
      key_transpose_kernel<uint64_t><<<m, 256, smem>>>((const uint64_t*)tmp, (uint64_t*)key->d_ahat_t,
                                                        k, m, key->n);
    else
      key_transpose_kernel<uint32_t><<<m, 256, smem>>>((const uint32_t*)tmp, (uint32_t*)key->d_ahat_t,
                                                        k, m, key->n);
    rc = map_cuda(cudaGetLastError());
  }
  // one synchronisation: the kernels' errors, and nothing reads tmp any more
  const cudaError_t e = cudaDeviceSynchronize();
  if (!rc) rc = map_cuda(e);
  cudaFree(tmp);
  if (rc) {
    lc_ajtai_key_destroy(key);
    return rc;
  }
  *out = key;
  return LC_OK;
}

}  // namespace lc

extern "C" {

LC_API int lc_ajtai_key_create(const lc_ntt_plan* plan, uint32_t k, uint32_t m, const void* matrix,
                               int matrix_on_device, lc_ajtai_key** out) {
  return lc_ajtai_key_create_ex(plan, k, m, matrix, matrix_on_device, 0, out);
}

LC_API int lc_ajtai_key_create_ex(const lc_ntt_plan* plan, uint32_t k, uint32_t m, const void* matrix,
                                  int matrix_on_device, uint32_t flags, lc_ajtai_key** out) {
  if (!plan || !matrix || !out || k == 0 || m == 0) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int rc = lc::key_create_check(plan, k, m, flags);
  if (rc) return rc;
  const size_t eb = plan->kind == PlanKind::Goldilocks ? 8 : 4;
  const size_t bytes = (size_t)k * m * ((size_t)1 << plan->log_n) * eb;
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, bytes) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  const cudaError_t e =
      cudaMemcpy(tmp, matrix, bytes, matrix_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(tmp);
    return map_cuda(e);
  }
  return lc::key_create_from(plan, k, m, tmp, flags, out);
}

LC_API void lc_ajtai_key_destroy(lc_ajtai_key* key) {
  if (!key) return;
  if (key->owns_ahat && key->d_ahat_t) cudaFree(key->d_ahat_t);
  for (void* p : {key->d_what_t, key->d_partial, key->d_chat, key->d_wtmp, key->d_fused, (void*)key->d_grid, key->d_in,
                  key->d_out, (void*)key->d_err})
    if (p) cudaFree(p);
  if (key->host_stream) cudaStreamDestroy(key->host_stream);
  if (key->h_flags) cudaFreeHost(key->h_flags);
  if (key->h_stage_in) cudaFreeHost(key->h_stage_in);
  if (key->h_stage_out) cudaFreeHost(key->h_stage_out);
  if (key->plan) lc_ntt_plan_destroy(key->plan);
  tc_tables_destroy(key->tc);
  delete key;
}

LC_API int lc_ajtai_key_view(const lc_ajtai_key* parent, uint32_t k, uint32_t m, lc_ajtai_key** out) {
  if (!parent || !out || k == 0 || m == 0 || k > parent->k || m > parent->m) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  lc_ajtai_key* key = new (std::nothrow) lc_ajtai_key();
  if (!key) return LC_ERR_OUT_OF_MEMORY;
  key->k = k;
  key->m = m;
  key->a_m = parent->a_m;
  key->log_n = parent->log_n;
  key->n = parent->n;
  key->wide = parent->wide;
  key->d_ahat_t = parent->d_ahat_t;
  key->owns_ahat = false;
  const lc_ntt_plan* pp = parent->plan;
  int rc = key->wide ? lc_ntt_plan_create_goldilocks(pp->log_n, &key->plan)
                     : lc_ntt_plan_create_u32(pp->log_n, pp->q, pp->two_adicity, pp->generator, 1, &key->plan);
  if (!rc && cudaMalloc(&key->d_err, 4) != cudaSuccess) {
    cudaGetLastError();
    rc = LC_ERR_OUT_OF_MEMORY;
  }
  if (!rc) rc = map_cuda(cudaMemset(key->d_err, 0, 4));
  if (rc) {
    lc_ajtai_key_destroy(key);
    return rc;
  }
  *out = key;
  return LC_OK;
}

LC_API int lc_ajtai_key_set_engine(lc_ajtai_key* key, int engine) {
  if (!key || (engine != LC_ENGINE_NTT && engine != LC_ENGINE_TENSOR_I8)) return LC_ERR_INVALID_ARGUMENT;
  if (engine == LC_ENGINE_TENSOR_I8 && !key->tc) return LC_ERR_UNSUPPORTED;
  key->engine = engine;
  return LC_OK;
}

LC_API int lc_ajtai_key_get_engine(const lc_ajtai_key* key) { return key ? key->engine : -1; }

LC_API int lc_ajtai_key_set_fused(lc_ajtai_key* key, int enable) {
  if (!key || enable < 0 || enable > 2) return LC_ERR_INVALID_ARGUMENT;
  key->fused = enable;
  return LC_OK;
}

LC_API int lc_ajtai_key_get_fused(const lc_ajtai_key* key) { return key ? key->fused : -1; }

LC_API int lc_ajtai_key_set_slot_products(lc_ajtai_key* key, int mode) {
  if (!key || (mode != LC_PRODUCTS_INT64 && mode != LC_PRODUCTS_TENSOR)) return LC_ERR_INVALID_ARGUMENT;
  key->slot_products = mode;
  return LC_OK;
}

LC_API int lc_ajtai_key_get_slot_products(const lc_ajtai_key* key) { return key ? key->slot_products : -1; }

}  // extern "C"

namespace lc {
// Identity of the scratch buffers a commit on this key writes; changes when
// any of them is reallocated (a captured graph of a commit is only valid
// while it stays the same).
uint64_t commit_scratch_signature(const lc_ajtai_key* key) {
  uint64_t h = 1469598103934665603ull;
  for (uintptr_t v : {(uintptr_t)key->d_what_t, (uintptr_t)key->d_partial, (uintptr_t)key->d_chat,
                      (uintptr_t)key->d_wtmp, (uintptr_t)key->what_bytes, (uintptr_t)key->partial_bytes,
                      (uintptr_t)key->chat_bytes, (uintptr_t)key->wtmp_bytes, (uintptr_t)key->d_fused,
                      (uintptr_t)key->d_grid})
    h = (h ^ (uint64_t)v) * 1099511628211ull;
  return h;
}
}  // namespace lc

extern "C" {

LC_API int lc_ajtai_commit(lc_ajtai_key* key, const void* s, size_t batch, void* out, lc_stream stream) {
  if (!key || (!s && batch) || (!out && batch)) return LC_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)out) & 15) return LC_ERR_INVALID_ARGUMENT;
  if (key->wide) return commit_any<uint64_t>(key, (const uint64_t*)s, batch, out, (cudaStream_t)stream);
  return commit_any<uint32_t>(key, (const uint32_t*)s, batch, out, (cudaStream_t)stream);
}

LC_API int lc_ajtai_commit_i8(lc_ajtai_key* key, const int8_t* s, size_t batch, void* out,
                              lc_stream stream) {
  if (!key || (!s && batch) || (!out && batch)) return LC_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)out) & 15) return LC_ERR_INVALID_ARGUMENT;
  if (key->engine == LC_ENGINE_TENSOR_I8)
    return tc_commit(key->tc, s, true, batch, static_cast<uint64_t*>(out), key->d_err, (cudaStream_t)stream);
  return commit_any<int8_t>(key, s, batch, out, (cudaStream_t)stream);
}

LC_API int lc_ajtai_commit_u8(lc_ajtai_key* key, const uint8_t* s, size_t batch, void* out,
                              lc_stream stream) {
  if (!key || (!s && batch) || (!out && batch)) return LC_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)out) & 15) return LC_ERR_INVALID_ARGUMENT;
  if (key->engine == LC_ENGINE_TENSOR_I8)
    return tc_commit(key->tc, s, false, batch, static_cast<uint64_t*>(out), key->d_err, (cudaStream_t)stream);
  return commit_any<uint8_t>(key, s, batch, out, (cudaStream_t)stream);
}

// Host buffers of at most kHostStageMax bytes that are not page-locked go
// through pinned staging buffers of the key: a CPU copy of a few KB costs far
// less than the driver's synchronous path for pageable memory.  Page-locked
// (or larger) buffers are copied directly.
constexpr size_t kHostStageMax = (size_t)1 << 20;

static bool host_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Device address of page-locked host memory (mapped into the device address
// space under unified addressing); false for pageable and device memory.
static bool mapped_host(const void* p, void** dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeHost || a.devicePointer == nullptr) return false;
  *dev = a.devicePointer;
  return true;
}

static int grow_pinned(void** p, size_t* have, size_t need) {
  if (need <= *have) return LC_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMallocHost(p, need) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return LC_ERR_OUT_OF_MEMORY;
  }
  *have = need;
  return LC_OK;
}

static int commit_host(lc_ajtai_key* key, const void* s, size_t in_elem, size_t batch, void* out,
                       bool i8) {
  if (!key || (!s && batch) || (!out && batch)) return LC_ERR_INVALID_ARGUMENT;
  if (batch == 0) return LC_OK;
  const size_t eb = key->wide ? 8 : 4;
  const size_t in_bytes = batch * key->m * key->n * in_elem;
  const size_t out_bytes = batch * key->k * key->n * eb;
  int rc = grow(&key->d_in, &key->in_bytes, in_bytes);
  if (!rc) rc = grow(&key->d_out, &key->out_bytes, out_bytes);
  if (rc) return rc;
  if (!key->host_stream && cudaStreamCreateWithFlags(&key->host_stream, cudaStreamNonBlocking) != cudaSuccess)
    return map_cuda(cudaGetLastError());
  if (!key->h_flags && cudaMallocHost(&key->h_flags, 2 * sizeof(uint32_t)) != cudaSuccess) {
    key->h_flags = nullptr;
    return map_cuda(cudaGetLastError());
  }
  const bool stage_in = in_bytes <= kHostStageMax && !host_pinned(s);
  const bool stage_out = out_bytes <= kHostStageMax && !host_pinned(out);
  if (stage_in) {
    rc = grow_pinned(&key->h_stage_in, &key->h_stage_in_bytes, in_bytes);
    if (rc) return rc;
    std::memcpy(key->h_stage_in, s, in_bytes);
  }
  if (stage_out) {
    rc = grow_pinned(&key->h_stage_out, &key->h_stage_out_bytes, out_bytes);
    if (rc) return rc;
  }
  cudaStream_t st = key->host_stream;
  {
    // a commitment small enough for the single-launch kernel, with input and
    // output in page-locked host memory (the staging buffers or the caller's):
    // the kernel reads the witness and writes the rows over the host link
    // itself, so neither copy is queued.  Only for witnesses of up to 256 KiB,
    // where the copies' fixed cost outweighs the kernel's slower loads over
    // the link; larger ones are copied at the copy engine's rate
    const void* hin = stage_in ? key->h_stage_in : s;
    void* hout = stage_out ? key->h_stage_out : out;
    void* din = nullptr;
    void* dout = nullptr;
    if (key->engine == LC_ENGINE_NTT && in_bytes <= ((size_t)256 << 10) && mapped_host(hin, &din) &&
        mapped_host(hout, &dout) &&
        reinterpret_cast<uintptr_t>(din) % in_elem == 0 && (reinterpret_cast<uintptr_t>(dout) & 15) == 0) {
      int frc = LC_ERR_UNSUPPORTED;
      if (in_elem == 1)
        frc = i8 ? commit_fused<int8_t>(key, static_cast<const int8_t*>(din), batch, dout, st)
                 : commit_fused<uint8_t>(key, static_cast<const uint8_t*>(din), batch, dout, st);
      else if (key->wide)
        frc = commit_fused<uint64_t>(key, static_cast<const uint64_t*>(din), batch, dout, st);
      else
        frc = commit_fused<uint32_t>(key, static_cast<const uint32_t*>(din), batch, dout, st);
      if (frc != LC_ERR_UNSUPPORTED) {
        // the single-launch kernel has no bounded waits and sets no error word
        const cudaError_t e = cudaStreamSynchronize(st);
        if (frc) return frc;
        if (e != cudaSuccess) return map_cuda(e);
        if (stage_out) std::memcpy(out, key->h_stage_out, out_bytes);
        return LC_OK;
      }
    }
  }
  if (cudaMemcpyAsync(key->d_in, stage_in ? key->h_stage_in : s, in_bytes, cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return map_cuda(cudaGetLastError());
  key->last_fused = false;
  rc = in_elem == 1 ? (i8 ? lc_ajtai_commit_i8(key, (const int8_t*)key->d_in, batch, key->d_out, st)
                          : lc_ajtai_commit_u8(key, (const uint8_t*)key->d_in, batch, key->d_out, st))
                    : lc_ajtai_commit(key, key->d_in, batch, key->d_out, st);
  if (rc) {
    // the input copy may still be reading the caller's (pinned) buffer
    cudaStreamSynchronize(st);
    cudaGetLastError();
    return rc;
  }
  // the single-launch kernel has no bounded waits and never sets an error word
  const bool flags = !key->last_fused;
  if (cudaMemcpyAsync(stage_out ? key->h_stage_out : out, key->d_out, out_bytes, cudaMemcpyDeviceToHost, st) !=
      cudaSuccess) {
    const int err = map_cuda(cudaGetLastError());
    cudaStreamSynchronize(st);  // nothing queued may still read the caller's input
    cudaGetLastError();
    return err;
  }
  // both error words come back with the result: one synchronisation per call
  if (flags) {
    cudaMemcpyAsync(key->h_flags, key->d_err, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(key->h_flags + 1, key->plan->d_err, 4, cudaMemcpyDeviceToHost, st);
  }
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return map_cuda(e);
  if (stage_out) std::memcpy(out, key->h_stage_out, out_bytes);
  if (flags && (key->h_flags[0] | key->h_flags[1])) {
    if (key->h_flags[0] != LC_DEVERR_POISONED) cudaMemsetAsync(key->d_err, 0, 4, st);
    cudaMemsetAsync(key->plan->d_err, 0, 4, st);
    cudaStreamSynchronize(st);
    return LC_ERR_TIMEOUT;
  }
  return LC_OK;
}

LC_API int lc_ajtai_commit_host(lc_ajtai_key* key, const void* s, size_t batch, void* out) {
  return commit_host(key, s, key ? (key->wide ? 8 : 4) : 0, batch, out, false);
}

LC_API int lc_ajtai_commit_i8_host(lc_ajtai_key* key, const int8_t* s, size_t batch, void* out) {
  return commit_host(key, s, 1, batch, out, true);
}

LC_API int lc_ajtai_commit_u8_host(lc_ajtai_key* key, const uint8_t* s, size_t batch, void* out) {
  return commit_host(key, s, 1, batch, out, false);
}

LC_API int lc_ajtai_key_check(lc_ajtai_key* key, lc_stream stream) {
  if (!key) return LC_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return map_cuda(e);
  uint32_t flag = 0;
  if (cudaMemcpy(&flag, key->d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return map_cuda(cudaGetLastError());
  if (flag) {
    if (flag != LC_DEVERR_POISONED) cudaMemset(key->d_err, 0, 4);  // a poisoned word stays set
    return LC_ERR_TIMEOUT;
  }
  return lc_ntt_plan_check(key->plan, stream);
}

LC_API int lc_ajtai_key_info(const lc_ajtai_key* key, uint32_t* k, uint32_t* m, uint32_t* log_n) {
  if (!key) return LC_ERR_INVALID_ARGUMENT;
  if (k) *k = key->k;
  if (m) *m = key->m;
  if (log_n) *log_n = key->log_n;
  return LC_OK;
}

LC_API int lc_ajtai_commit_noalloc(const lc_ajtai_key* key, const void* s, size_t batch, void* out,
                                   lc_stream stream) {
  if (!key || (!s && batch) || (!out && batch)) return LC_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)out) & 15) return LC_ERR_INVALID_ARGUMENT;
  if (batch > (1u << 24)) return LC_ERR_INVALID_ARGUMENT;
  if (key->wide)
    return noalloc_commit<uint64_t>(key, (const uint64_t*)s, batch, out, (cudaStream_t)stream);
  return noalloc_commit<uint32_t>(key, (const uint32_t*)s, batch, out, (cudaStream_t)stream);
}

}  // extern "C"
