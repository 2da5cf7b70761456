// batch.cu -- many Ajtai commitments of uneven ring degree, length, row count
// and modulus in three persistent launches fed by device work counters.
//
// Every job is AjtaiPublicKey::commit (lattice-commitment/src/ajtai.rs:
// 118-153) of one int8-digit witness with the first kappa rows and n columns
// of its class's key(s).  Jobs that share a key form lanes of at most 128
// jobs, sorted by n (longest first).  At ring element j only the jobs with
// n_b > j take part, so a lane's transformed witnesses are stored as a
// staircase: slot t, ring element j, job b at  what[t*Sp + Rp[j] + b],  where
// R[j] = sum over j' < j of the number of jobs longer than j' (S = sum n_b),
// Rp[j] the same with every row of active jobs padded to 16 bytes (so each
// row starts 16-byte aligned) and Sp = Rp[n_max] the entries per slot.
//   1. witness NTT: an item is PB consecutive staircase polynomials; their
//      (j, b) come from a per-item start table and a short walk over R;
//   2. product: a warp's item is (chunk of ring elements, slot t, block of 16
//      jobs active at the chunk's start); each thread holds 2 rows x 4 jobs
//      (160-bit accumulators) and streams the key's rows Ahat[t][j][..] --
//      read once per lane of jobs, not once per job -- and the staircase,
//      with the next 32 ring elements' rows prefetched into L2;
//   3. finish: an item is one job: the sum over its chunks (mod q), then the
//      inverse NTT of its kappa rows straight into the job's output.
// A CTA claims `claim` items at a time from the phase's counter
// (atomicAdd), so uneven items balance across the SMs.  The three launches
// and the counter reset are captured into a CUDA graph when asked.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "arith.cuh"
#include "common.cuh"
#include "internal.h"
#include "mac.cuh"
#include "ntt_kernels.cuh"
#include "tcgen05.cuh"

namespace lc {

constexpr int kBatchThreads = 256;
constexpr uint32_t kLaneJobs = 128;
// tensor-core products: jobs per block (MMA N = 32 limbs-bytes per job) and
// ring elements per exact int32 sum (32768 * 255^2 < 2^31)
constexpr int kTpJobs = 32;
constexpr uint32_t kTpChunk = 32768;
constexpr uint32_t kMinChunk = 1024;

// Slot strides (odd, >= N + T) that keep the transposed reads of the
// staircase store free of bank conflicts: the commit witness tiles' values.
template <class A, int LOG_N>
struct BatchSlotStride;
template <class A>
struct BatchSlotStride<A, 6> {
  static constexpr int value = sizeof(typename A::T) == 8 ? 73 : 75;
};
template <class A>
struct BatchSlotStride<A, 7> {
  static constexpr int value = 137;
};
template <class A>
struct BatchSlotStride<A, 8> {
  static constexpr int value = 273;
};

struct LaneDesc {
  uint32_t kind;   // PlanKind
  uint32_t log_n;
  uint32_t q, qinv;
  const void* tw_fwd;
  const void* tw_inv;
  const void* ahat;  // [d][a_m][16]
  uint32_t a_m;
  uint32_t nb;      // jobs in the lane
  uint32_t n_max;   // longest job
  uint32_t nchunks;
  uint64_t S;       // staircase polynomials
  const uint64_t* R;       // [n_max + 1]: jobs longer than j' summed over j' < j
  const uint64_t* Rp;      // [n_max + 1]: the same with every row padded to 16 bytes (where row j starts)
  uint64_t Sp;             // entries per slot of `what` (16-byte rows, 16-byte slots)
  const uint32_t* item_j;  // witness items: ring element of the first polynomial
  uint32_t sub0;           // first job of the lane in the sub-job table
  uint32_t pb;             // polynomials per witness item
  void* what;              // [d][S]
  void* partial;           // [nchunks][d][16][nb]
  const uint64_t* citem;   // [nchunks + 1]: first product item of each chunk (lane-relative)
  const uint8_t* cblk;     // [nchunks]: 16-job blocks with jobs active at the chunk's start
  uint64_t item0[3];       // first item of the lane in each launch
  int32_t* tpart;          // tensor-core products: limb-pair sums of the lane (null: CUDA-core partials)
  const uint32_t* tchunk0; // [blocks + 1]: first K chunk of each 32-job block in tpart
};

struct SubJob {
  const int8_t* w;  // [n][d]
  void* out;        // [kappa][d] of this lane's modulus
  uint32_t n, kappa;
};

struct BatchParams {
  const LaneDesc* lanes;
  const SubJob* subs;
  unsigned long long* counters;  // [4]: witness, Goldilocks products, finish, u32 products
  uint32_t* err;
  uint64_t total[3];
  uint64_t prod_split;  // product items of the Goldilocks lanes (they come first)
  uint32_t nlanes, chunk, claim;
  uint32_t lane_split;  // first lane of a u32 modulus
};

template <class A, int LOG_N, int LOG_V>
struct BCfg {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  static constexpr int N = G::N;
  static constexpr int GROUPS = kBatchThreads / G::T;
  static constexpr int SS = BatchSlotStride<A, LOG_N>::value;
  // polynomials per thread group in a witness item: as many as keep the
  // item's slots within 72 KB (a few per group amortise the item's fixed
  // costs: counter claim, twiddles, four barriers), so three witness CTAs
  // fit in an SM's shared memory
  static constexpr size_t POLY_BYTES = (size_t)SS * sizeof(T);
  static constexpr int IT = (size_t)GROUPS * 4 * POLY_BYTES <= 72 * 1024   ? 4
                            : (size_t)GROUPS * 2 * POLY_BYTES <= 72 * 1024 ? 2
                                                                           : 1;
  static constexpr int PB = GROUPS * IT;  // polynomials per witness item
  static constexpr int TWE = G::fwd_entries() > G::inv_entries() ? G::fwd_entries() : G::inv_entries();
  static constexpr size_t TWB = ((size_t)TWE * sizeof(Tw) + 15) / 16 * 16;
  static constexpr size_t SMEM1 = TWB + (size_t)PB * SS * sizeof(T) + (size_t)PB * 16 + (size_t)(PB + 2) * 16;
  static constexpr size_t SMEM3 = TWB + (size_t)16 * SS * sizeof(T);
  static_assert(SS >= Slots<A, LOG_N, LOG_V>::S, "slot stride");
};

template <class T>
LC_D T digit_residue(int8_t x, uint32_t q);
template <>
LC_D uint64_t digit_residue<uint64_t>(int8_t x, uint32_t) {
  return x >= 0 ? (uint64_t)x : kGlP - (uint64_t)(-(int)x);
}
template <>
LC_D uint32_t digit_residue<uint32_t>(int8_t x, uint32_t q) {
  return x >= 0 ? (uint32_t)x : q - (uint32_t)(-(int)x);
}

LC_D uint64_t add_mod(uint64_t a, uint64_t b, uint32_t) { return gl_add(a, b); }
LC_D uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) {
  const uint64_t s = (uint64_t)a + b;  // canonical inputs; q may exceed 2^31
  return (uint32_t)(s >= q ? s - q : s);
}

// ---- launch 1: witness NTT of PB staircase polynomials
template <class A, int LOG_N, int LOG_V>
LC_D void witness_item(const LaneDesc& L, const SubJob* __restrict__ subs, uint64_t k, unsigned char* smem) {
  using C = BCfg<A, LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int N = C::N, PB = C::PB, SS = C::SS;
  Tw* tw = reinterpret_cast<Tw*>(smem);
  T* slots = reinterpret_cast<T*>(smem + C::TWB);
  const int8_t** ssrc = reinterpret_cast<const int8_t**>(slots + PB * SS);  // digits of each polynomial (or null)
  uint64_t* sdst = reinterpret_cast<uint64_t*>(ssrc + PB);                 // its row offset Rp[j] + b in a slot
  uint64_t* sR = sdst + PB;                                                // R[j_lo .. j_lo + PB + 1]
  uint64_t* sRp = sR + PB + 2;                                             // Rp[j_lo .. j_lo + PB + 1]
  __shared__ uint32_t s_jlo;
  const int tid = threadIdx.x;
  const uint64_t p0 = k * PB;
  for (int i = tid; i < Geo<LOG_N, LOG_V>::fwd_entries(); i += kBatchThreads)
    tw[i] = reinterpret_cast<const Tw*>(L.tw_fwd)[i];
  if (tid == 0) s_jlo = L.item_j[k];
  __syncthreads();
  // consecutive staircase polynomials advance the ring element by at most one,
  // so the item's PB polynomials lie in ring elements j_lo .. j_lo + PB - 1
  const uint32_t jlo = s_jlo;
  if (tid < PB + 2) {
    sR[tid] = jlo + tid <= L.n_max ? L.R[jlo + tid] : L.S;
    sRp[tid] = jlo + tid <= L.n_max ? L.Rp[jlo + tid] : L.Sp;
  }
  __syncthreads();
  // polynomial p of the staircase: ring element j, job b; its digits and its
  // place in every slot of `what`, looked up once here
  if (tid < PB) {
    const uint64_t p = p0 + tid;
    const int8_t* src = nullptr;
    uint64_t dst = 0;
    if (p < L.S) {
      uint32_t x = 0;
      while (sR[x + 1] <= p) ++x;
      const uint32_t br = (uint32_t)(p - sR[x]);
      src = subs[L.sub0 + br].w + (size_t)(jlo + x) * N;
      dst = sRp[x] + br;
    }
    ssrc[tid] = src;
    sdst[tid] = dst;
  }
  __syncthreads();
  // the item's 16-digit chunks: every load of a thread issued before its
  // conversions, so several loads are in flight
  constexpr int CH = N / 16;  // 16-digit chunks per polynomial
  constexpr int PER = (PB * CH + kBatchThreads - 1) / kBatchThreads;
  uint4 v[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * kBatchThreads;
    v[u] = make_uint4(0, 0, 0, 0);
    if (e < PB * CH) {
      const int8_t* src = ssrc[e / CH];
      if (src) v[u] = __ldg(reinterpret_cast<const uint4*>(src + (e % CH) * 16));
    }
  }
  // Lanes of a warp hold neighbouring 16-digit chunks 16 words apart; lane l
  // stores its chunk starting at digit (l % 16), so that one store
  // instruction of the warp touches 16 distinct banks per polynomial instead
  // of 2.  The 16 bytes are rotated once (word selects, then byte funnel
  // shifts), so every digit is then taken from a fixed register position.
  const uint32_t rot = (uint32_t)tid & 15u;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * kBatchThreads;
    if (e < PB * CH) {
      T* dst = slots + (e / CH) * SS + (e % CH) * 16;
      // byte i of (r0 r1 r2 r3) = byte (i + rot) mod 16 of the chunk
      const bool w1 = rot & 4u, w2 = rot & 8u;
      const uint32_t t0 = w1 ? v[u].y : v[u].x, t1 = w1 ? v[u].z : v[u].y;
      const uint32_t t2 = w1 ? v[u].w : v[u].z, t3 = w1 ? v[u].x : v[u].w;
      const uint32_t q0 = w2 ? t2 : t0, q1 = w2 ? t3 : t1, q2 = w2 ? t0 : t2, q3 = w2 ? t1 : t3;
      const uint32_t sh = 8u * (rot & 3u);
      const uint32_t r[4] = {__funnelshift_r(q0, q1, sh), __funnelshift_r(q1, q2, sh), __funnelshift_r(q2, q3, sh),
                             __funnelshift_r(q3, q0, sh)};
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int8_t x = (int8_t)(uint8_t)(r[i >> 2] >> (8 * (i & 3)));
        dst[(i + rot) & 15u] = digit_residue<T>(x, L.q);
      }
    }
  }
  __syncthreads();
  const A ar = make_arith_q<A>(L.q, L.qinv);
#pragma unroll 1
  for (int it = 0; it < C::IT; ++it)
    transform_slot<A, LOG_N, LOG_V, false>(slots + (it * C::GROUPS + tid / Geo<LOG_N, LOG_V>::T) * SS, tw, ar,
                                           tid % Geo<LOG_N, LOG_V>::T);
  __syncthreads();
  // PB divides the block, so a thread keeps one polynomial s and walks its
  // slots tt = tid / PB, + 256 / PB, ...: one slot-strided store each
  static_assert(kBatchThreads % PB == 0, "a thread keeps its polynomial");
  {
    constexpr int TSTEP = kBatchThreads / PB;
    const int s = tid % PB;
    if (ssrc[s]) {
      T* wp = reinterpret_cast<T*>(L.what) + sdst[s] + (size_t)(tid / PB) * L.Sp;
      const size_t step = (size_t)TSTEP * L.Sp;
      for (int tt = tid / PB; tt < N; tt += TSTEP, wp += step) *wp = slots[s * SS + tt];
    }
  }
  __syncthreads();
}

// ---- launch 2: products, one warp per item = (chunk c, slot t, block of 16 jobs)
//
// The planner lists, for every chunk of ring elements, the 16-job blocks with
// jobs active at the chunk's first element (jobs are sorted longest first, so
// the active jobs are a prefix) and one item per (slot t, block).  A warp
// claims items from the launch's counter on its own -- no CTA-wide barrier,
// so a warp whose jobs end early simply takes the next item.  Lane
// (ip, g) holds rows 2ip, 2ip+1 of jobs 4(4*blk + g) .. +3 in 160-bit
// accumulators and streams, two ring elements at a time (loads before the
// multiply-adds), the key pair Ahat[t][j][2ip..2ip+1] and the witness values
// what[t*Sp + Rp[j] + b] from L2.
template <class E>
LC_D void load_pair(const E* p, E& a0, E& a1);
template <>
LC_D void load_pair<uint64_t>(const uint64_t* p, uint64_t& a0, uint64_t& a1) {
  const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
  a0 = ((uint64_t)v.y << 32) | v.x;
  a1 = ((uint64_t)v.w << 32) | v.z;
}
template <>
LC_D void load_pair<uint32_t>(const uint32_t* p, uint32_t& a0, uint32_t& a1) {
  const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
  a0 = v.x;
  a1 = v.y;
}

template <class E>
LC_D void product_warp_item(const LaneDesc& L, const SubJob* __restrict__ subs, uint32_t chunk, uint64_t k) {
  // chunk of the item: citem[c] <= k < citem[c + 1]
  uint32_t lo = 0, hi = L.nchunks;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (L.citem[mid] <= k)
      lo = mid;
    else
      hi = mid;
  }
  const uint32_t c = lo, nblk = L.cblk[c];
  const uint32_t r = (uint32_t)(k - L.citem[c]);
  const uint32_t t = r / nblk, blk = r % nblk;
  const uint32_t d = 1u << L.log_n;
  const uint32_t j0 = c * chunk, j1 = min(L.n_max, j0 + chunk);
  const int lane = threadIdx.x & 31;
  const uint32_t ip = lane & 7, bq = blk * 4 + (lane >> 3);  // rows 2ip, 2ip+1; jobs 4bq..4bq+3
  uint32_t nq[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const uint32_t b = 4 * bq + u;
    nq[u] = b < L.nb ? subs[L.sub0 + b].n : 0;  // sorted: nq[0] >= nq[1] >= ...
  }
  // warp-uniform end: lanes 0-7 hold the block's first (longest) job, the
  // other quads' shorter jobs are masked by j < nq[u]
  const uint32_t jend = __shfl_sync(0xffffffffu, min(j1, nq[0]), 0);
  const E* A = reinterpret_cast<const E*>(L.ahat) + (size_t)t * L.a_m * kIPad + 2 * ip;
  const E* W = reinterpret_cast<const E*>(L.what) + (size_t)t * L.Sp + 4 * bq;
  const uint64_t* R = L.Rp;  // where each ring element's row of active jobs starts
  // The staircase offsets of 32 ring elements arrive in one coalesced load and
  // are broadcast by shuffles; the key and witness loads of JU ring elements
  // issue together before their multiply-adds, so a warp keeps several
  // independent loads in flight instead of one dependent pair per element.
  constexpr int JU = sizeof(E) == 8 ? 2 : 4;
  Acc160 acc[2][4];
  // Lane l also prefetches into L2 the key row and this block's 16 staircase
  // entries of ring element jb + 32 + l, so the next block's loads hit L2.
  const uint32_t b16 = 16 * blk;
  for (uint32_t jb = j0; jb < jend; jb += 32) {
    const uint32_t nj = min(32u, jend - jb);
    const uint64_t rl = (uint32_t)lane < nj ? __ldg(R + jb + lane) : 0;
    const uint32_t jp = jb + 32 + lane;
    if (jp < jend) {
      asm volatile("prefetch.global.L2 [%0];" ::"l"(A - 2 * ip + (size_t)jp * kIPad));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(W - 4 * bq + __ldg(R + jp) + b16));
    }
    uint32_t s = 0;
    for (; s + JU <= nj; s += JU) {
      E a[JU][2], w[JU][4];
#pragma unroll
      for (int x = 0; x < JU; ++x) {
        const uint32_t j = jb + s + x;
        const uint64_t rj = __shfl_sync(0xffffffffu, rl, s + x);
        load_pair<E>(A + (size_t)j * kIPad, a[x][0], a[x][1]);
#pragma unroll
        for (int u = 0; u < 4; ++u) w[x][u] = j < nq[u] ? __ldg(W + rj + u) : E(0);
      }
#pragma unroll
      for (int x = 0; x < JU; ++x)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          mac<E>(acc[0][u], a[x][0], w[x][u]);
          mac<E>(acc[1][u], a[x][1], w[x][u]);
        }
    }
    for (; s < nj; ++s) {
      const uint32_t j = jb + s;
      const uint64_t rj = __shfl_sync(0xffffffffu, rl, s);
      E a0, a1;
      load_pair<E>(A + (size_t)j * kIPad, a0, a1);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const E wv = j < nq[u] ? __ldg(W + rj + u) : E(0);
        mac<E>(acc[0][u], a0, wv);
        mac<E>(acc[1][u], a1, wv);
      }
    }
  }
  // jobs active at j0 own a partial of this chunk (the finish launch reads
  // chunks c with c*chunk < n_b)
  E* P = reinterpret_cast<E*>(L.partial) + ((size_t)c * d + t) * kIPad * L.nb;
#pragma unroll
  for (int ii = 0; ii < 2; ++ii)
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (j0 < nq[u]) P[(size_t)(2 * ip + ii) * L.nb + 4 * bq + u] = acc_reduce<E>(acc[ii][u], L.q);
}

// ---- launch 3: one job's chunk sums and inverse NTT
template <class A, int LOG_N, int LOG_V>
LC_D void finish_item(const LaneDesc& L, const SubJob* __restrict__ subs, uint32_t chunk, uint64_t b,
                      unsigned char* smem) {
  using C = BCfg<A, LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int N = C::N, SS = C::SS, GROUPS = C::GROUPS;
  Tw* tw = reinterpret_cast<Tw*>(smem);
  T* slots = reinterpret_cast<T*>(smem + C::TWB);
  const int tid = threadIdx.x;
  const SubJob J = subs[L.sub0 + b];
  const uint32_t nch = (J.n + chunk - 1) / chunk;
  for (int i = tid; i < Geo<LOG_N, LOG_V>::inv_entries(); i += kBatchThreads)
    tw[i] = reinterpret_cast<const Tw*>(L.tw_inv)[i];
  if (L.tpart) {
    // tensor-core partials: D[(b, lw)][(i, la)] per (chunk, slot) of the
    // job's 32-job block; the 2L - 1 sums of equal la + lw over the chunks
    // fit 64 bits (< 2^31 * L * chunks) and are folded with 2^(8k) mod q.
    // Consecutive threads take consecutive rows i, i.e. adjacent words.
    constexpr int LL = sizeof(T);
    const uint32_t blk = (uint32_t)b / kTpJobs, bl = (uint32_t)b % kTpJobs;
    const uint32_t c0 = L.tchunk0[blk], nchk = L.tchunk0[blk + 1] - c0;
    const size_t tile = (size_t)kTpJobs * LL * 128;
    for (uint32_t e = tid; e < J.kappa * N; e += kBatchThreads) {
      const uint32_t i = e % J.kappa, tt = e / J.kappa;
      uint64_t tk[2 * LL - 1];
#pragma unroll
      for (int k = 0; k < 2 * LL - 1; ++k) tk[k] = 0;
      for (uint32_t c = 0; c < nchk; ++c) {
        const int32_t* D = L.tpart + ((size_t)(c0 + c) * N + tt) * tile + (size_t)bl * LL * 128 + i * LL;
#pragma unroll
        for (int lw = 0; lw < LL; ++lw)
#pragma unroll
          for (int la = 0; la < LL; ++la) tk[la + lw] += (uint32_t)__ldg(D + (size_t)lw * 128 + la);
      }
      T res;
      if constexpr (LL == 8) {
        unsigned __int128 v = 0;
        uint64_t cw = 1;  // 2^(8k) mod p
#pragma unroll
        for (int k = 0; k < 2 * LL - 1; ++k) {
          v += (unsigned __int128)tk[k] * cw;
          cw = gl_mul(cw, 256);
        }
        res = (T)gl_canon(gl_reduce128_lazy((uint64_t)(v >> 64), (uint64_t)v));
      } else {
        const uint64_t q = L.q;
        uint64_t v = 0, cw = 1 % q;  // 2^(8k) mod q
#pragma unroll
        for (int k = 0; k < 2 * LL - 1; ++k) {
          v = (v + (tk[k] % q) * cw % q) % q;
          cw = (cw << 8) % q;
        }
        res = (T)v;
      }
      slots[i * SS + tt] = res;
    }
  } else {
    const T* P = reinterpret_cast<const T*>(L.partial);
    for (uint32_t e = tid; e < J.kappa * N; e += kBatchThreads) {
      const uint32_t i = e / N, tt = e % N;
      T s = 0;
      for (uint32_t c = 0; c < nch; ++c) s = add_mod(s, P[(((size_t)c * N + tt) * kIPad + i) * L.nb + b], L.q);
      slots[i * SS + tt] = s;
    }
  }
  __syncthreads();
  const A ar = make_arith_q<A>(L.q, L.qinv);
  const int grp = tid / Geo<LOG_N, LOG_V>::T;
  const uint32_t lt = tid % Geo<LOG_N, LOG_V>::T;
  for (uint32_t p0 = 0; p0 < J.kappa; p0 += GROUPS)
    if (p0 + grp < J.kappa) transform_slot<A, LOG_N, LOG_V, true>(slots + (p0 + grp) * SS, tw, ar, lt);
  __syncthreads();
  T* out = reinterpret_cast<T*>(J.out);
  for (uint32_t e = tid; e < J.kappa * N; e += kBatchThreads) out[e] = slots[(e / N) * SS + e % N];
  __syncthreads();
}

template <int PHASE>
LC_D void run_item(const BatchParams& p, const LaneDesc& L, uint64_t k, unsigned char* smem) {
  const int key = (int)L.kind * 16 + (int)L.log_n;
  constexpr int GL = (int)PlanKind::Goldilocks * 16, SL = (int)PlanKind::U32Lazy * 16, MC = (int)PlanKind::U32Mont * 16;
#define LC_BATCH_CASE(K, A, LN, LV)                       \
  case K + LN:                                            \
    if (PHASE == 0)                                       \
      witness_item<A, LN, LV>(L, p.subs, k, smem);        \
    else                                                  \
      finish_item<A, LN, LV>(L, p.subs, p.chunk, k, smem); \
    return;
  switch (key) {
    LC_BATCH_CASE(GL, Goldilocks, 6, 3)
    LC_BATCH_CASE(GL, Goldilocks, 7, 4)
    LC_BATCH_CASE(GL, Goldilocks, 8, 4)
    LC_BATCH_CASE(SL, ShoupLazy, 6, 3)
    LC_BATCH_CASE(SL, ShoupLazy, 7, 4)
    LC_BATCH_CASE(SL, ShoupLazy, 8, 4)
    LC_BATCH_CASE(MC, MontCanon, 6, 3)
    LC_BATCH_CASE(MC, MontCanon, 7, 4)
    LC_BATCH_CASE(MC, MontCanon, 8, 4)
    default:
      if (threadIdx.x == 0) record_error(p.err, 2);
  }
#undef LC_BATCH_CASE
}

// the witness launch at three CTAs per SM (79 registers, no spills)
template <int PHASE>
__global__ void __launch_bounds__(kBatchThreads, PHASE == 0 ? 3 : 2) batch_kernel(const __grid_constant__ BatchParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long s_base;
  const uint64_t total = p.total[PHASE];
  uint32_t lane = 0;
  for (;;) {
    if (threadIdx.x == 0) s_base = atomicAdd(&p.counters[PHASE], (unsigned long long)p.claim);
    __syncthreads();
    const uint64_t base = s_base;
    __syncthreads();
    if (base >= total) break;
    const uint64_t end = min(base + p.claim, total);
    for (uint64_t it = base; it < end; ++it) {
      // claims only grow, so the lane index only moves forward
      while (lane + 1 < p.nlanes && p.lanes[lane + 1].item0[PHASE] <= it) ++lane;
      run_item<PHASE>(p, p.lanes[lane], it - p.lanes[lane].item0[PHASE], smem);
    }
  }
}

// Products of one element type: the Goldilocks lanes' items [0, prod_split)
// or the u32 lanes' items [prod_split, total), each launch with its own
// counter, so neither carries the other's registers.
template <class E>
__global__ void __launch_bounds__(kBatchThreads, sizeof(E) == 8 ? 2 : 3)
    product_kernel(const __grid_constant__ BatchParams p) {
  constexpr bool WIDE = sizeof(E) == 8;
  const int lane = threadIdx.x & 31;
  const uint64_t lo = WIDE ? 0 : p.prod_split, hi = WIDE ? p.prod_split : p.total[1];
  unsigned long long* ctr = &p.counters[WIDE ? 1 : 3];
  uint32_t li = WIDE ? 0 : p.lane_split;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(ctr, (unsigned long long)p.claim);
    base = __shfl_sync(0xffffffffu, base, 0);
    const uint64_t first = lo + base;
    if (first >= hi) return;
    const uint64_t end = min(first + p.claim, hi);
    for (uint64_t it = first; it < end; ++it) {
      // a warp's claims only grow, so its lane index only moves forward
      while (li + 1 < p.nlanes && p.lanes[li + 1].item0[1] <= it) ++li;
      const LaneDesc& L = p.lanes[li];
      product_warp_item<E>(L, p.subs, p.chunk, it - L.item0[1]);
    }
  }
}

// ---- launch 1 on the tensor cores: witness transforms, d = 64 / 128 / 256
//
// For ring degree d the forward transform of a digit row w (natural order,
// out[t] = sum_c w_c psi^((2t+1) c), ntt.rs:118-146) is the fixed product
// What[t] = sum_c V[t][c] w[c] (mod q), V[t][c] = psi^((2t+1) c).  With V's
// residues split into L byte limbs (4 for a 30-bit q, 8 for Goldilocks) it
// is L exact INT8 GEMMs,
//   D[p][(t,l)] = sum_c w_p[c] V_l[t][c]   (s8 x u8 -> s32, |D| <= d 128 255 < 2^23),
// folded per output: for q = 2^30 - c (c <= 2^20) v = sum_l 2^(8l) D
// (|v| < 2^48), u = v + q 2^19 > 0, two folds by 2^30 == c and one
// conditional subtract (tw_fold); for Goldilocks tw_fold_gl.  A tile is 128
// consecutive staircase polynomials of a lane (M = 128), gathered from the
// jobs' digit rows by four warps with cp.async into the K-major
// 128-byte-swizzled layout (K = d bytes in 128-byte atoms; d = 64 fills half
// an atom and runs 2 K-steps); N = the L d columns (t, l) in passes of PN
// (PN / L slots), each pass's V-limb rows loaded by TMA from the lane's
// [L d][max(d, 128)] image in global memory (L2-resident) into one of
// NS = 512 / PN stages; NS TMEM accumulators of PN columns rotate between
// passes, so the epilogue warps fold pass k and store What[t][Rp[j] + b]
// while the next passes load and run.
// EW epilogue warps (8 or 16; warp w reads TMEM lanes 32 (w % 4).. and a
// PN / (EW / 4)-column share of each pass), then 4 gather warps, the TMA
// warp and the MMA warp.
template <int EW, int PN>
struct TwCfg {
  static_assert(EW == 8 || EW == 16, "epilogue warps");
  static_assert(PN == 128 || PN == 256, "pass width");
  static constexpr int THREADS = 32 * (EW + 6);
  static constexpr int GATHER = EW, TMA = EW + 4, MMA = EW + 5;
  static constexpr uint32_t COLS = PN / (EW / 4);  // TMEM columns per epilogue warp and pass
  static constexpr uint32_t NS = 512 / PN;         // B stages = TMEM accumulators
  static constexpr uint32_t BSTAGE = PN * 256;     // bytes of a B stage (PN rows x d <= 256)
  // D = s32, A = s8, B = u8, both K-major, N = PN, M = 128
  static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | ((uint32_t)(PN >> 3) << 17) | ((128u >> 4) << 24);
};
constexpr int kTwEpi = 16;
constexpr int kTwPN = 256;
constexpr int kTwRows = 128;          // polynomials per tile
constexpr int kTwABytes = kTwRows * 256;  // A stage (d <= 256)
constexpr int kTwOffB = 2 * kTwABytes;
constexpr int kTwOffInfo = kTwOffB + 512 * 256;              // per A stage: 128 x u64 destinations
constexpr int kTwOffBar = kTwOffInfo + 2 * kTwRows * 8;
constexpr size_t kTwSmem = 1024 + kTwOffBar + 256;
static_assert(kTwSmem <= 227 * 1024, "shared memory");

struct TwItem {
  uint32_t lane, tile, jlo, pad;
};

// OR of `v` over the `count` threads of named barrier `id` (all of them
// receive it): keeps a warp group's loop decisions uniform.
LC_D bool named_bar_or(bool v, uint32_t id, uint32_t count) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(count)
      : "memory");
  return r != 0;
}

// One output from its four limb sums x[l]: v = sum_l 2^(8l) D_l (|v| < 2^48)
// mod q, canonical, for the q tw_fold_exact accepts (2^30 - c, c <= 2^20):
// u = v + off (off = q 2^19) in (0, 2^50), two folds by 2^30 == c, and
// min(y, y - q) for the final subtract (y < 2q).
LC_D uint32_t tw_fold(const uint32_t* x, uint32_t q, uint32_t c, int64_t off) {
  int64_t v = off + (int32_t)x[0];
  v += (int64_t)(int32_t)x[1] * 256;
  v += (int64_t)(int32_t)x[2] * 65536;
  v += (int64_t)(int32_t)x[3] * 16777216;
  const uint64_t u = (uint64_t)v;
  const uint64_t w = (uint64_t)(uint32_t)(u >> 30) * c + ((uint32_t)u & 0x3FFFFFFFu);  // < 2^40 + 2^30
  const uint32_t y = (uint32_t)(w >> 30) * c + ((uint32_t)w & 0x3FFFFFFFu);            // < 2q
  return min(y, y - q);
}

// Goldilocks: v = A + 2^32 B with A, B the limb sums 0-3 and 4-7 (|A|, |B|
// <= 256 128 255 (1 + 2^8 + 2^16 + 2^24) < 2^47.01), returned as a 64-bit
// value congruent mod p, not necessarily canonical (the products read any
// 64-bit representative): S = A + hi(B) (2^32 - 1), |S| < 2^48.02; U = S +
// 2^32 lo(B) = R + k 2^64 with R = U mod 2^64, k = carry - [S < 0], and the
// value R + k (2^32 - 1) stays inside [0, 2^64) (the reasoning of tn_fold).
LC_D uint64_t tw_fold_gl(const uint32_t* x) {
  int64_t A = (int32_t)x[0], B = (int32_t)x[4];
  A += (int64_t)(int32_t)x[1] * 256;
  B += (int64_t)(int32_t)x[5] * 256;
  A += (int64_t)(int32_t)x[2] * 65536;
  B += (int64_t)(int32_t)x[6] * 65536;
  A += (int64_t)(int32_t)x[3] * 16777216;
  B += (int64_t)(int32_t)x[7] * 16777216;
  const int64_t S = A + (B >> 32) * (int64_t)0xFFFFFFFFll;
  const uint64_t lo = (uint64_t)(uint32_t)B << 32;
  const uint64_t R = (uint64_t)S + lo;
  const int k = (int)(R < lo) - (int)(S < 0);
  return R + (uint64_t)(int64_t)k * 0xFFFFFFFFull;
}

// limbs of a lane's V image (8 Goldilocks, 4 u32) and its passes of PN columns
LC_D uint32_t tw_limbs(const LaneDesc& L) { return L.kind == (uint32_t)PlanKind::Goldilocks ? 8u : 4u; }

template <int EW, int PN>
__global__ void __launch_bounds__(TwCfg<EW, PN>::THREADS, 1)
    lane_witness_tc_kernel(const TwItem* __restrict__ items, uint64_t nitems, const LaneDesc* __restrict__ lanes,
                           const SubJob* __restrict__ subs, const CUtensorMap* __restrict__ vmaps, uint32_t* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* info = reinterpret_cast<uint64_t*>(base + kTwOffInfo);  // [2][128] staircase offset, ~0 = none
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kTwOffBar);
  uint64_t* a_full = bars;        // [2] 128 gather threads
  uint64_t* a_free = bars + 2;    // [2] MMA commit + EW epilogue warps
  uint64_t* b_full = bars + 4;    // [NS] V rows landed (tx)
  uint64_t* b_empty = bars + 8;   // [NS] MMA commit
  uint64_t* acc_full = bars + 12;   // [NS] MMA commit
  uint64_t* acc_empty = bars + 16;  // [NS] EW epilogue warps
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 20);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 21);
  uint64_t* done = bars + 22;     // every MMA issued has finished
  using Cfg = TwCfg<EW, PN>;
  constexpr uint32_t NS = Cfg::NS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    mbar_init(done, 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(&a_full[s], 128);
      mbar_init(&a_free[s], 1 + EW);
    }
    for (uint32_t s = 0; s < NS; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], EW);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == Cfg::MMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint64_t n_my = nitems > blockIdx.x ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto item_at = [&](uint64_t i) { return items[blockIdx.x + i * gridDim.x]; };
  auto fail = [&]() {
    record_error(err, LC_DEVERR_TIMEOUT);
    *abort_flag = 1;
  };
  auto a_stage = [&](uint64_t i) { return base + (i & 1) * kTwABytes; };
  auto b_stage = [&](uint64_t g) { return base + kTwOffB + (g % NS) * Cfg::BSTAGE; };
  int64_t tma_last = -1;    // TMA thread: last pass index loaded

  if (warp == Cfg::TMA) {
    // ---------------- TMA: V-limb rows of each pass
    if (lane == 0) {
      uint64_t g = 0;
      for (uint64_t i = 0; i < n_my && !*abort_flag; ++i) {
        const TwItem it = item_at(i);
        const LaneDesc& L = lanes[it.lane];
        const uint32_t d = 1u << L.log_n, passes = tw_limbs(L) * d / PN, kb = d > 128 ? d / 128 : 1;
        const CUtensorMap* vm = vmaps + it.lane;
        for (uint32_t k = 0; k < passes && !*abort_flag; ++k, ++g) {
          if (g >= NS && !mbar_wait(&b_empty[g % NS], (uint32_t)(((g - NS) / NS) & 1))) {
            fail();
            break;
          }
          mbar_arrive_expect_tx(&b_full[g % NS], PN * 128 * kb);
          for (uint32_t kk = 0; kk < kb; ++kk)
            tma_load_2d(b_stage(g) + kk * (PN * 128), vm, (int)(kk * 128), (int)(k * PN), &b_full[g % NS]);
          tma_last = (int64_t)g;
        }
      }
    }
  } else if (warp == Cfg::MMA) {
    // ---------------- MMA issuer
    if (lane == 0) {
      uint64_t g = 0;
      bool ok = true;
      for (uint64_t i = 0; i < n_my && ok && !*abort_flag; ++i) {
        const TwItem it = item_at(i);
        const LaneDesc& L = lanes[it.lane];
        const uint32_t d = 1u << L.log_n, passes = tw_limbs(L) * d / PN;
        if (!mbar_wait(&a_full[i & 1], (uint32_t)((i >> 1) & 1))) {
          fail();
          break;
        }
        const uint32_t aa = smem_u32(a_stage(i));
        for (uint32_t k = 0; k < passes; ++k, ++g) {
          if (!mbar_wait(&b_full[g % NS], (uint32_t)((g / NS) & 1)) ||
              (g >= NS && !mbar_wait(&acc_empty[g % NS], (uint32_t)(((g - NS) / NS) & 1)))) {
            fail();
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t bb = smem_u32(b_stage(g));
          for (uint32_t ks = 0; ks < d / 32; ++ks) {
            const uint32_t off = (ks >> 2) * 16384u + (ks & 3) * 32u;
            mma_i8(tmem + (uint32_t)(g % NS) * PN, umma_desc_sw128(aa + off),
                   umma_desc_sw128(bb + (ks >> 2) * (PN * 128u) + (ks & 3) * 32u), Cfg::IDESC, ks > 0 ? 1u : 0u);
          }
          mma_commit(&acc_full[g % NS]);
          mma_commit(&b_empty[g % NS]);
        }
        if (ok) mma_commit(&a_free[i & 1]);
      }
      mma_commit(done);
      if (!mbar_wait(done, 0)) fail();
    }
  } else if (warp >= Cfg::GATHER) {
    // ---------------- gather: row info (thread r = row r), then the digit rows.
    // A tile's row table is worked out while the previous tile's copies are
    // in flight: R[jlo .. jlo + 128] staged in shared memory, each row's ring
    // element found there, then its source row and staircase destination.
    const int gt = tid - 32 * Cfg::GATHER;  // 0..127
    __shared__ uint64_t s_R[kTwRows + 1];
    __shared__ const int8_t* s_src[kTwRows];
    auto row_of = [&](uint64_t ii, const int8_t*& src, uint64_t& dst) {
      const TwItem it = item_at(ii);
      const LaneDesc& L = lanes[it.lane];
      const uint32_t hi = min(L.n_max, it.jlo + kTwRows);  // R[jlo] <= the tile's polynomials < R[hi]
      if (it.jlo + gt <= hi) s_R[gt] = __ldg(L.R + it.jlo + gt);
      if (gt == 0 && it.jlo + kTwRows <= hi) s_R[kTwRows] = __ldg(L.R + it.jlo + kTwRows);
      asm volatile("bar.sync 1, 128;" ::: "memory");
      // row r: staircase polynomial p = 128 tile + r -> ring element j (R[j] <= p < R[j + 1]), job b
      const uint64_t p = (uint64_t)it.tile * kTwRows + gt;
      src = nullptr;
      dst = ~0ull;
      if (p < L.S) {
        uint32_t lo = 0, h = hi - it.jlo;
        while (h - lo > 1) {
          const uint32_t mid = (lo + h) >> 1;
          if (s_R[mid] <= p) lo = mid; else h = mid;
        }
        const uint32_t b = (uint32_t)(p - s_R[lo]);
        src = subs[L.sub0 + b].w + (size_t)(it.jlo + lo) * (1u << L.log_n);
        dst = __ldg(L.Rp + it.jlo + lo) + b;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");  // s_R is rewritten by the next call
    };
    const int8_t* src = nullptr;
    uint64_t dst = ~0ull;
    if (n_my) row_of(0, src, dst);
    for (uint64_t i = 0; i < n_my; ++i) {
      // one decision for the four gather warps (they share named barrier 1)
      bool timed_out = false;
      if (!*abort_flag && i >= 2) timed_out = !mbar_wait(&a_free[i & 1], (uint32_t)(((i - 2) >> 1) & 1));
      if (timed_out) fail();
      if (named_bar_or(timed_out || *abort_flag, 1, 128)) break;
      const TwItem it = item_at(i);
      const LaneDesc& L = lanes[it.lane];
      const uint32_t d = 1u << L.log_n;
      info[(i & 1) * kTwRows + gt] = dst;
      s_src[gt] = src;
      asm volatile("bar.sync 1, 128;" ::: "memory");  // the four gather warps
      const uint32_t cpr = d / 16;                 // 16-byte chunks per row
      const uint32_t rpi = 128 / cpr;              // rows per pass of the 128 threads
      const uint32_t c = (uint32_t)gt % cpr;
      const uint32_t a = smem_u32(a_stage(i));
      for (uint32_t r = (uint32_t)gt / cpr; r < kTwRows; r += rpi) {
        const int8_t* sp = s_src[r];
        const uint32_t dsto = a + (c >> 3) * 16384u + (r >> 3) * 1024u + (r & 7) * 128u + (((c & 7) ^ (r & 7)) << 4);
        cp_async16_zfill(dsto, sp ? (const void*)(sp + c * 16) : (const void*)L.what, sp ? 16u : 0u);
      }
      cp_async_commit();
      // the next tile's rows while these copies fly (its first barrier also
      // ends this tile's reads of s_src; the barrier at the top of the next
      // iteration does when there is none)
      if (i + 1 < n_my) row_of(i + 1, src, dst);
      cp_async_wait<0>();
      fence_proxy_async_smem();
      mbar_arrive(&a_full[i & 1]);
    }
    cp_async_wait<0>();
  } else {
    // ---------------- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31
    // (rows = polynomials) and columns COLS (w / 4) .. + COLS - 1 of each pass
    const uint32_t quad = warp & 3, row = 32 * quad + lane, cbeg = (uint32_t)(warp >> 2) * Cfg::COLS;
    uint64_t g = 0;
    for (uint64_t i = 0; i < n_my; ++i) {
      const TwItem it = item_at(i);
      const LaneDesc& L = lanes[it.lane];
      const bool gl = L.kind == (uint32_t)PlanKind::Goldilocks;
      const uint32_t d = 1u << L.log_n, passes = tw_limbs(L) * d / PN, q = L.q, cq = (1u << 30) - q;
      const int64_t off = (int64_t)q << 19;
      const size_t Sp = L.Sp;
      bool stop = false;
      // the gather's row table of this tile (its a_full phase; the stage is
      // not refilled before this warp releases it)
      const bool rows_ok = !*abort_flag && mbar_wait(&a_full[i & 1], (uint32_t)((i >> 1) & 1));
      if (!__all_sync(0xffffffffu, rows_ok)) {
        if (lane == 0) fail();
        break;
      }
      const uint64_t dst = info[(i & 1) * kTwRows + row];
      for (uint32_t k = 0; k < passes; ++k, ++g) {
        const bool ok = !*abort_flag && mbar_wait(&acc_full[g % NS], (uint32_t)((g / NS) & 1));
        if (!__all_sync(0xffffffffu, ok)) {  // warp-uniform: the TMEM loads are .sync.aligned
          if (lane == 0) fail();
          stop = true;
          break;
        }
        tc_fence_after();
        const uint32_t taddr = tmem + ((32 * quad) << 16) + (uint32_t)(g % NS) * PN + cbeg;
        if (gl) {
          // output slot t = (PN / 8) k + (cbeg + c0) / 8 + u, row dst of the staircase
          uint64_t* what = reinterpret_cast<uint64_t*>(L.what) + (dst == ~0ull ? 0 : dst) +
                           (size_t)((PN / 8) * k + cbeg / 8) * Sp;
#pragma unroll 1
          for (uint32_t c0 = 0; c0 < Cfg::COLS; c0 += 32) {
            uint32_t v0[16], v1[16];
            tmem_ld16(taddr + c0, v0);
            tmem_ld16(taddr + c0 + 16, v1);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              if (dst != ~0ull) *what = tw_fold_gl(u < 2 ? v0 + 8 * u : v1 + 8 * (u - 2));
              what += Sp;
            }
          }
        } else {
          // output slot t = (PN / 4) k + (cbeg + c0) / 4 + u, row dst of the staircase
          uint32_t* what = reinterpret_cast<uint32_t*>(L.what) + (dst == ~0ull ? 0 : dst) +
                           (size_t)((PN / 4) * k + cbeg / 4) * Sp;
#pragma unroll 1
          for (uint32_t c0 = 0; c0 < Cfg::COLS; c0 += 32) {
            uint32_t v0[16], v1[16];
            tmem_ld16(taddr + c0, v0);
            tmem_ld16(taddr + c0 + 16, v1);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              if (dst != ~0ull) *what = tw_fold(u < 4 ? v0 + 4 * u : v1 + 4 * (u - 4), q, cq, off);
              what += Sp;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[g % NS]);
      }
      if (stop) break;
      if (lane == 0) mbar_arrive(&a_free[i & 1]);
    }
  }
  // ---------------- nothing in flight when TMEM and shared memory go
  __syncthreads();
  if (warp == Cfg::TMA && lane == 0) {
    for (int64_t g = tma_last >= (int64_t)NS - 1 ? tma_last - (NS - 1) : 0; g <= tma_last; ++g)
      mbar_wait(&b_full[g % NS], (uint32_t)((g / NS) & 1));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == Cfg::MMA) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ---- launch 2 on the tensor cores: lane products as exact byte-limb GEMMs
//
// C_t[i][b] = sum_j Ahat[t][j][i] * What[t][j][b] over j < n_b, with both
// residues split into L byte limbs (L = 8 Goldilocks, 4 for u32 moduli):
// C_t = sum_{la,lw} 2^(8 (la + lw)) D_t and
//   D_t[(i,la)][(b,lw)] = sum_j Ahat_la[t][j][i] * What_lw[t][j][b]   (u8 x u8 -> s32),
// exact for at most 32768 ring elements j per sum (32768 * 255^2 < 2^31).
// An item is (lane, slot t, block of 32 jobs, chunk of 32768 ring elements):
// M = 128 (the key row's 16 x L bytes (i, la); u32 keys fill half and the
// second A atom is a zero tile), N = 32 L bytes (b, lw), K = the chunk.  The
// key rows Ahat[t][j][16] arrive by TMA (a 3-D map per lane: row bytes,
// j < a_m, slot); the witness rows come from the staircase, where row j of
// the block is the 32 L contiguous bytes at what[t Sp + Rp[j] + 32 blk]
// (16-byte aligned) of which only the first cnt(j) - 32 blk jobs are active:
// four gather warps copy them in 16-byte chunks with zero-filling cp.async
// straight into the 128-byte-swizzled MN-major layout the MMA descriptor
// reads (chunk c of row r at c ^ (r & 7)),
// so the shorter jobs of a block contribute zeros and nothing outside the
// staircase is read.  The epilogue (the same four warps) writes D, one
// [32 L columns][128 rows] int32 tile per item; the finish launch folds the
// limb pairs over the block's chunks.
constexpr int kTpRows = 64;            // ring elements per stage
constexpr int kTpStages = 4;
constexpr int kTpLag = 2;              // gather stages in flight before a stage is handed to the MMA
constexpr int kTpAhead = 2;            // stages the staircase offsets are loaded ahead of their copies
constexpr int kTpThreads = 192;        // warp 0 TMA, 1 MMA + TMEM, 2..5 gather + epilogue

struct TpItem {
  uint32_t lane, t, blk, chunk;
};

template <int EB>
struct TpCfg {
  static constexpr int NB = kTpJobs * EB;        // B row bytes = MMA N (256 or 128)
  static constexpr int AW = 16 * EB;             // key row bytes (128 or 64)
  static constexpr int A_LOAD = kTpRows * AW;    // bytes the TMA writes per stage
  static constexpr int A_BYTES = kTpRows * 128;  // A region (for AW = 64 the zero atom follows)
  static constexpr int B_ATOM = kTpRows * 128;   // one 128-byte swizzle atom along N, all K rows
  static constexpr int ATOMS = NB / 128;
  static constexpr int STAGE = A_BYTES + ATOMS * B_ATOM;
  static constexpr size_t SMEM = 1024 + (size_t)kTpStages * STAGE + 128;
  static constexpr uint32_t A_LAYOUT = AW == 128 ? 2u : 4u;  // 128- or 64-byte swizzle
  static_assert(STAGE % 1024 == 0, "swizzle atoms stay aligned");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// D = s32, A = B = u8, both MN-major, N, M = 128
template <int N>
struct TpIdesc {
  static constexpr uint32_t value =
      (2u << 4) | (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
};


template <int EB>
__global__ void __launch_bounds__(kTpThreads, 1)
    lane_products_tc_kernel(const TpItem* __restrict__ items, const LaneDesc* __restrict__ lanes,
                            const SubJob* __restrict__ subs, const CUtensorMap* __restrict__ amaps, uint32_t* err) {
  using C = TpCfg<EB>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kTpStages * C::STAGE);
  uint64_t* full = bars;                  // [4] key rows landed (tx) and 128 gather threads arrived
  uint64_t* empty = bars + kTpStages;     // [4] the stage's MMAs finished
  uint64_t* done = bars + 2 * kTpStages;  // every MMA finished
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kTpStages + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 2 * kTpStages + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const TpItem it = items[blockIdx.x];
  const LaneDesc& L = lanes[it.lane];
  const uint32_t d = 1u << L.log_n;
  const uint32_t nblk = subs[L.sub0 + kTpJobs * it.blk].n;  // the block's longest job
  const uint32_t j0 = it.chunk * kTpChunk;
  const uint32_t j1 = min(nblk, j0 + kTpChunk);
  const int nst = (int)((j1 - j0 + kTpRows - 1) / kTpRows);

  if (tid == 0) {
    for (int s = 0; s < kTpStages; ++s) {
      mbar_init(&full[s], 1 + 128);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if constexpr (C::AW == 64) {
    // the second A atom of every stage: rows (i, la) 64..127 are zero
    for (int s = 0; s < kTpStages; ++s) {
      uint4* z = reinterpret_cast<uint4*>(base + s * C::STAGE + C::A_LOAD);
      for (int e = tid; e < (C::A_BYTES - C::A_LOAD) / 16; e += kTpThreads) z[e] = make_uint4(0, 0, 0, 0);
    }
    fence_proxy_async_smem();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(C::NB));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto stage = [&](int s) { return base + (s % kTpStages) * C::STAGE; };
  auto fail = [&]() {
    record_error(err, LC_DEVERR_TIMEOUT);
    *abort_flag = 1;
  };
  int last_loaded = -1, last_mma = -1;

  if (warp == 0) {
    // ---------------- TMA: key rows (i, la) of slot t
    if (lane == 0) {
      const CUtensorMap* amap = amaps + it.lane;
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (s >= kTpStages && !mbar_wait(&empty[s % kTpStages], (uint32_t)(((s - kTpStages) / kTpStages) & 1))) {
          fail();
          break;
        }
        mbar_arrive_expect_tx(&full[s % kTpStages], (uint32_t)C::A_LOAD);
        tma_load_3d(stage(s), amap, 0, (int)(j0 + kTpRows * s), (int)it.t, &full[s % kTpStages]);
        last_loaded = s;
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (!mbar_wait(&full[s % kTpStages], (uint32_t)((s / kTpStages) & 1))) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(stage(s)), sb = sa + C::A_BYTES;
#pragma unroll
        for (int ks = 0; ks < kTpRows / 32; ++ks) {
          const uint64_t ad = umma_desc_mn(sa + ks * 32 * C::AW, C::A_LOAD, 8 * C::AW, C::A_LAYOUT);
          const uint64_t bd = umma_desc_mn(sb + ks * 32 * 128, C::B_ATOM, 8 * 128, 2);
          mma_i8(tmem, ad, bd, TpIdesc<C::NB>::value, (s > 0 || ks > 0) ? 1u : 0u);
        }
        mma_commit(&empty[s % kTpStages]);
        last_mma = s;
      }
      if (last_mma >= 0) mma_commit(done);
    }
  } else {
    // ---------------- gather: warp g = warp - 2 fills rows 16 g .. 16 g + 15 of
    // every stage in 16-byte chunks.  Row j of the block starts at
    // what[t Sp + Rp[j] + 32 blk], 16-byte aligned; chunk k holds jobs
    // 32 blk + k J .. + J - 1 (J = 16 / EB), of which the first
    // cnt(j) - 32 blk - k J are active and copied, the rest zero-filled.
    constexpr int J = 16 / EB;           // jobs per chunk
    constexpr int CPR = C::NB / 16;      // chunks per row (16 or 8)
    constexpr int RPI = 32 / CPR;        // rows per warp instruction (2 or 4)
    const int g = warp - 2;
    using E = typename std::conditional<EB == 8, uint64_t, uint32_t>::type;
    const E* W = reinterpret_cast<const E*>(L.what) + (size_t)it.t * L.Sp + (size_t)kTpJobs * it.blk;
    const uint32_t k = (uint32_t)lane % CPR, rsub = (uint32_t)lane / CPR;
    const uint32_t boff = (k >> 3) * C::B_ATOM;  // swizzle atom of the chunk
    const uint32_t kc = k & 7;
    const int first_job = kTpJobs * (int)it.blk + (int)(k * J);
    // R[jb .. jb + 16] (job counts) and Rp[jb .. jb + 15] (row starts) of a
    // stage, loaded kTpAhead stages ahead (a register queue) so their
    // latency hides behind the copies and waits of the stages between
    auto offsets = [&](int s, uint64_t& r, uint64_t& rp) {
      const uint32_t jb = j0 + kTpRows * s + 16 * g;
      const bool in_r = s < nst && lane <= 16 && jb + lane <= L.n_max;
      r = in_r ? __ldg(L.R + jb + lane) : 0;
      rp = in_r ? __ldg(L.Rp + jb + lane) : 0;
    };
    uint64_t rq[kTpAhead], rpq[kTpAhead];
#pragma unroll
    for (int a = 0; a < kTpAhead; ++a) offsets(a, rq[a], rpq[a]);
    bool ok = true;
    for (int s = 0; s < nst; ++s) {
      if (*abort_flag) {
        ok = false;
        break;
      }
      if (s >= kTpStages && !mbar_wait(&empty[s % kTpStages], (uint32_t)(((s - kTpStages) / kTpStages) & 1))) {
        fail();
        ok = false;
        break;
      }
      const uint32_t jb = j0 + kTpRows * s + 16 * g;
      const uint64_t rl = rq[0], rpl = rpq[0];
#pragma unroll
      for (int a = 0; a + 1 < kTpAhead; ++a) {
        rq[a] = rq[a + 1];
        rpq[a] = rpq[a + 1];
      }
      offsets(s + kTpAhead, rq[kTpAhead - 1], rpq[kTpAhead - 1]);
      const uint32_t sb = smem_u32(stage(s)) + C::A_BYTES + boff;
#pragma unroll
      for (int rr = 0; rr < 16; rr += RPI) {
        const int r = rr + (int)rsub;
        const uint64_t r0 = __shfl_sync(0xffffffffu, rl, r);
        const uint64_t r1 = __shfl_sync(0xffffffffu, rl, r + 1);
        const uint64_t rp = __shfl_sync(0xffffffffu, rpl, r);
        const uint32_t j = jb + r, row = 16 * g + r;
        const int act = (j < j1) ? (int)(r1 - r0) - first_job : 0;  // active jobs from this chunk's first
        const uint32_t bytes = act <= 0 ? 0u : act >= J ? 16u : (uint32_t)act * EB;
        const uint32_t dst = sb + row * 128 + ((kc ^ (row & 7)) << 4);
        cp_async16_zfill(dst, bytes ? (const void*)(W + rp + k * J) : L.what, bytes);
      }
      cp_async_commit();
      if (s >= kTpLag) {
        cp_async_wait<kTpLag>();
        fence_proxy_async_smem();
        mbar_arrive(&full[(s - kTpLag) % kTpStages]);
      }
    }
    cp_async_wait<0>();
    fence_proxy_async_smem();
    if (ok)
      for (int s = max(0, nst - kTpLag); s < nst; ++s) mbar_arrive(&full[s % kTpStages]);
    // ---------------- epilogue: lane = row (i, la); column = (b, lw)
    const bool fin = ok && nst > 0 && !*abort_flag && mbar_wait(done, 0);
    if (__all_sync(0xffffffffu, fin)) {
      tc_fence_after();
      const uint32_t lq = warp & 3, row = 32 * lq + lane;
      int32_t* out = L.tpart + ((size_t)(L.tchunk0[it.blk] + it.chunk) * d + it.t) * (size_t)C::NB * 128;
#pragma unroll 1
      for (int c0 = 0; c0 < C::NB; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + ((32 * lq) << 16) + c0, v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int u = 0; u < 16; ++u) out[(size_t)(c0 + u) * 128 + row] = (int32_t)v[u];
      }
    } else if (nst > 0 && lane == 0) {
      fail();
    }
  }
  // ---------------- nothing in flight when TMEM and shared memory go
  __syncthreads();
  if (warp == 0 && lane == 0) {
    for (int s = max(0, last_loaded - (kTpStages - 1)); s <= last_loaded; ++s)
      mbar_wait(&full[s % kTpStages], (uint32_t)((s / kTpStages) & 1));
  }
  if (warp == 1 && lane == 0 && last_mma >= 0) mbar_wait(done, 0);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::NB));
  }
}

template <class A, int LOG_N, int LOG_V>
static void smem_need(size_t& s1, size_t& s3, uint32_t& pb) {
  using C = BCfg<A, LOG_N, LOG_V>;
  s1 = C::SMEM1;
  s3 = C::SMEM3;
  pb = C::PB;
}

static bool lane_geometry(PlanKind kind, uint32_t log_n, size_t& s1, size_t& s3, uint32_t& pb) {
  switch ((int)kind * 16 + (int)log_n) {
#define LC_GEO(K, A, LN, LV)            \
  case (int)K * 16 + LN:                \
    smem_need<A, LN, LV>(s1, s3, pb);   \
    return true;
    LC_GEO(PlanKind::Goldilocks, Goldilocks, 6, 3)
    LC_GEO(PlanKind::Goldilocks, Goldilocks, 7, 4)
    LC_GEO(PlanKind::Goldilocks, Goldilocks, 8, 4)
    LC_GEO(PlanKind::U32Lazy, ShoupLazy, 6, 3)
    LC_GEO(PlanKind::U32Lazy, ShoupLazy, 7, 4)
    LC_GEO(PlanKind::U32Lazy, ShoupLazy, 8, 4)
    LC_GEO(PlanKind::U32Mont, MontCanon, 6, 3)
    LC_GEO(PlanKind::U32Mont, MontCanon, 7, 4)
    LC_GEO(PlanKind::U32Mont, MontCanon, 8, 4)
#undef LC_GEO
    default:
      return false;
  }
}

}  // namespace lc

struct lc_batch {
  std::vector<lc::LaneDesc> lanes;     // host copies (device pointers inside)
  std::vector<std::vector<uint64_t>> R;  // staircase offsets per lane (host)
  uint64_t* d_citem = nullptr;
  uint8_t* d_cblk = nullptr;
  std::vector<uint64_t> lane_elem;     // element bytes per lane
  lc::LaneDesc* d_lanes = nullptr;
  lc::SubJob* d_subs = nullptr;
  uint64_t* d_R = nullptr;
  uint32_t* d_itemj = nullptr;
  unsigned char* d_what = nullptr;
  unsigned char* d_partial = nullptr;
  unsigned long long* d_counters = nullptr;
  uint32_t* d_err = nullptr;
  uint64_t total[3] = {0, 0, 0};
  uint64_t prod_split = 0;  // product items of the Goldilocks lanes, which come first
  uint32_t lane_split = 0;
  size_t smem[3] = {0, 0, 0};
  uint32_t chunk = 4096, ctas = 2, claim = 1;
  uint32_t flags = 0;
  // tensor-core products (lane_products_tc_kernel)
  int products = LC_PRODUCTS_INT64;
  bool tensor_ok = false;
  std::vector<uint32_t> h_nfirst;        // per lane: n of each 32-job block's first job, concatenated
  std::vector<size_t> nfirst_off;
  int32_t* d_tpart = nullptr;
  uint32_t* d_tchunk0 = nullptr;
  CUtensorMap* d_amaps = nullptr;
  lc::TpItem* d_titems = nullptr;
  uint64_t titems[2] = {0, 0};           // Goldilocks items, then u32 items
  std::vector<int32_t*> lane_tpart;
  std::vector<const uint32_t*> lane_tchunk0;
  // tensor-core witness transforms (lane_witness_tc_kernel): u32 lanes with q < 2^30, d = 128 / 256
  std::vector<uint8_t> lane_tw;            // per lane: its witness transforms run there
  std::vector<std::pair<uint64_t, void*>> vimgs;  // V-limb images by (q << 16 | d)
  CUtensorMap* d_vmaps = nullptr;
  lc::TwItem* d_twitems = nullptr;
  uint64_t twitems = 0;
  bool warmed = false, dirty = true;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace lc {

static void batch_free(lc_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  for (void* p : {(void*)b->d_lanes, (void*)b->d_subs, (void*)b->d_R, (void*)b->d_itemj, (void*)b->d_what,
                  (void*)b->d_partial, (void*)b->d_counters, (void*)b->d_err, (void*)b->d_citem,
                  (void*)b->d_cblk, (void*)b->d_tpart, (void*)b->d_tchunk0, (void*)b->d_amaps,
                  (void*)b->d_titems, (void*)b->d_vmaps, (void*)b->d_twitems})
    if (p) cudaFree(p);
  for (auto& v : b->vimgs) cudaFree(v.second);
  delete b;
}

// Tensor-core products: per lane a TMA map of its key rows, per 32-job block
// the K chunks, the items (longest first, Goldilocks lanes then u32 lanes)
// and the partial tiles.  Leaves tensor_ok false when a lane cannot run
// there (no tensor-map encoder, or an element width other than 8 / 4 bytes).
static int batch_tensor_setup(lc_batch* b) {
  EncodeTiledFn enc = encode_fn();
  if (!enc || b->lanes.empty()) return LC_OK;
  const size_t nl = b->lanes.size();
  std::vector<CUtensorMap> maps(nl);
  std::vector<uint32_t> tchunk0;
  std::vector<size_t> tc_off(nl), part_off(nl);
  std::vector<std::pair<uint32_t, TpItem>> items[2];  // (rows, item)
  size_t part_elems = 0;
  for (size_t l = 0; l < nl; ++l) {
    const LaneDesc& L = b->lanes[l];
    const uint32_t eb = L.kind == (uint32_t)PlanKind::Goldilocks ? 8 : 4;
    const uint32_t d = 1u << L.log_n, aw = 16 * eb;
    const cuuint64_t dims[3] = {aw, (cuuint64_t)L.a_m, (cuuint64_t)d};
    const cuuint64_t strides[2] = {aw, (cuuint64_t)L.a_m * aw};
    const cuuint32_t box[3] = {aw, (cuuint32_t)kTpRows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&maps[l], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(L.ahat), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, aw == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return LC_OK;
    tc_off[l] = tchunk0.size();
    part_off[l] = part_elems;
    const uint32_t nblk = (L.nb + kTpJobs - 1) / kTpJobs;
    uint32_t acc = 0;
    for (uint32_t blk = 0; blk < nblk; ++blk) {
      const uint32_t nfirst = b->h_nfirst[b->nfirst_off[l] + blk];
      const uint32_t chunks = (nfirst + kTpChunk - 1) / kTpChunk;
      tchunk0.push_back(acc);
      for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t rows = std::min(nfirst, (c + 1) * kTpChunk) - c * kTpChunk;
        for (uint32_t t = 0; t < d; ++t) items[eb == 8 ? 0 : 1].push_back({rows, TpItem{(uint32_t)l, t, blk, c}});
      }
      acc += chunks;
    }
    tchunk0.push_back(acc);
    part_elems += (size_t)acc * d * kTpJobs * eb * 128;
  }
  for (auto& v : items)
    std::stable_sort(v.begin(), v.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  std::vector<TpItem> flat;
  for (auto& v : items)
    for (auto& x : v) flat.push_back(x.second);
  if (cudaMalloc(&b->d_amaps, nl * sizeof(CUtensorMap)) != cudaSuccess ||
      cudaMalloc(&b->d_tchunk0, tchunk0.size() * 4) != cudaSuccess ||
      cudaMalloc(&b->d_titems, std::max<size_t>(1, flat.size()) * sizeof(TpItem)) != cudaSuccess ||
      cudaMalloc(&b->d_tpart, std::max<size_t>(256, part_elems * 4)) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  cudaMemcpy(b->d_amaps, maps.data(), nl * sizeof(CUtensorMap), cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_tchunk0, tchunk0.data(), tchunk0.size() * 4, cudaMemcpyHostToDevice);
  if (!flat.empty()) cudaMemcpy(b->d_titems, flat.data(), flat.size() * sizeof(TpItem), cudaMemcpyHostToDevice);
  b->titems[0] = items[0].size();
  b->titems[1] = items[1].size();
  b->lane_tpart.resize(nl);
  b->lane_tchunk0.resize(nl);
  for (size_t l = 0; l < nl; ++l) {
    b->lane_tpart[l] = b->d_tpart + part_off[l];
    b->lane_tchunk0[l] = b->d_tchunk0 + tc_off[l];
  }
  b->tensor_ok = true;
  return map_cuda(cudaGetLastError());
}

static uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((unsigned __int128)a * b % q); }
static uint64_t powmod64(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  for (a %= q; e; e >>= 1, a = mulmod64(a, a, q))
    if (e & 1) r = mulmod64(r, a, q);
  return r;
}

// The [limbs d rows (t, l)][max(d, 128) bytes c] image of V[t][c] =
// psi^((2t+1) c) mod q split into byte limbs l (zero for c >= d), psi =
// g^((q - 1) >> (log d + 1)) as the plan's forward transform uses (natural
// output order, ntt.rs:118-146; Goldilocks: g = 7, field.rs:195-200).
static void tw_image(uint64_t q, uint64_t g, uint32_t log_d, uint32_t limbs, std::vector<uint8_t>& img) {
  const uint32_t d = 1u << log_d, cols = std::max(d, 128u);
  const uint64_t psi = powmod64(g, (q - 1) >> (log_d + 1), q);
  img.assign((size_t)limbs * d * cols, 0);
  for (uint32_t t = 0; t < d; ++t) {
    const uint64_t step = powmod64(psi, 2 * t + 1, q);
    uint64_t v = 1;
    for (uint32_t c = 0; c < d; ++c, v = mulmod64(v, step, q))
      for (uint32_t l = 0; l < limbs; ++l) img[((size_t)t * limbs + l) * cols + c] = (uint8_t)(v >> (8 * l));
  }
}

// Whether tw_fold is exact for q and ring degree d: the offset q 2^19 must
// exceed the largest |v| = d 128 255 (1 + 2^8 + 2^16 + 2^24), c = 2^30 - q
// at most 2^20, and after two folds by 2^30 == c the value below 2q (so q
// close to 2^30, as the 30-bit CRT primes are; other q keep the CUDA cores).
static bool tw_fold_exact(uint64_t q, uint32_t d) {
  if (q >= (1ull << 30) || q < (1ull << 29)) return false;
  const uint64_t vmax = (uint64_t)d * 128 * 255 * 16843009ull, off = q << 19;
  if (off <= vmax) return false;
  const uint64_t c = (1ull << 30) - q, m = (1ull << 30) - 1;
  if (c > (1ull << 20)) return false;  // the second fold multiplies in 32 bits
  const uint64_t umax = vmax + off;
  const uint64_t xmax = (umax >> 30) * c + m;
  const uint64_t ymax = (xmax >> 30) * c + m;
  return ymax < 2 * q;
}

// Tensor-core witness transforms: per eligible lane a TMA map of its (q, d)
// image and the tiles of 128 staircase polynomials with their first ring
// element.  Lanes that cannot run there keep the CUDA-core transforms.
static int batch_tw_setup(lc_batch* b, const std::vector<uint32_t>& plan_gen) {
  EncodeTiledFn enc = encode_fn();
  const size_t nl = b->lanes.size();
  b->lane_tw.assign(nl, 0);
  if (!enc || !nl) return LC_OK;
  std::vector<CUtensorMap> maps(nl);
  std::vector<TwItem> items;
  for (size_t l = 0; l < nl; ++l) {
    const LaneDesc& L = b->lanes[l];
    const bool gl = L.kind == (uint32_t)PlanKind::Goldilocks;
    if (L.log_n < 6 || L.log_n > 8 || L.S == 0) continue;
    const uint32_t d = 1u << L.log_n, limbs = gl ? 8 : 4, cols = std::max(d, 128u);
    if (!gl && (L.kind != (uint32_t)PlanKind::U32Lazy || !tw_fold_exact(L.q, d))) continue;
    const uint64_t key = gl ? (1ull << 63) | d : ((uint64_t)L.q << 16) | d;
    void* img = nullptr;
    for (auto& v : b->vimgs)
      if (v.first == key) img = v.second;
    if (!img) {
      std::vector<uint8_t> h;
      tw_image(gl ? kGlP : L.q, gl ? 7 : plan_gen[l], L.log_n, limbs, h);
      if (cudaMalloc(&img, h.size()) != cudaSuccess) {
        cudaGetLastError();
        return LC_ERR_OUT_OF_MEMORY;
      }
      cudaMemcpy(img, h.data(), h.size(), cudaMemcpyHostToDevice);
      b->vimgs.push_back({key, img});
    }
    const cuuint64_t dims[2] = {cols, (cuuint64_t)limbs * d};
    const cuuint64_t strides[1] = {cols};
    const cuuint32_t box[2] = {128, kTwPN};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&maps[l], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, img, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      continue;
    const std::vector<uint64_t>& R = b->R[l];
    uint32_t j = 0;
    for (uint64_t tile = 0; tile * kTwRows < L.S; ++tile) {
      while (R[j + 1] <= tile * kTwRows) ++j;
      items.push_back(TwItem{(uint32_t)l, (uint32_t)tile, j, 0});
    }
    b->lane_tw[l] = 1;
  }
  if (items.empty()) return LC_OK;
  if (cudaMalloc(&b->d_vmaps, nl * sizeof(CUtensorMap)) != cudaSuccess ||
      cudaMalloc(&b->d_twitems, items.size() * sizeof(TwItem)) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  cudaMemcpy(b->d_vmaps, maps.data(), nl * sizeof(CUtensorMap), cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_twitems, items.data(), items.size() * sizeof(TwItem), cudaMemcpyHostToDevice);
  b->twitems = items.size();
  return map_cuda(cudaGetLastError());
}

// The lanes' partial pointers for the current product mode.
static void batch_apply_products(lc_batch* b) {
  for (size_t l = 0; l < b->lanes.size(); ++l) {
    const bool tc = b->products == LC_PRODUCTS_TENSOR && b->tensor_ok;
    b->lanes[l].tpart = tc ? b->lane_tpart[l] : nullptr;
    b->lanes[l].tchunk0 = tc ? b->lane_tchunk0[l] : nullptr;
  }
}

// chunk-dependent fields, item bases and the device copy of the lanes
static int batch_layout(lc_batch* b) {
  // product items per chunk: one per slot and 16-job block active at the chunk's start
  std::vector<uint64_t> citem;
  std::vector<uint8_t> cblk;
  std::vector<size_t> coff;
  for (size_t l = 0; l < b->lanes.size(); ++l) {
    LaneDesc& L = b->lanes[l];
    const std::vector<uint64_t>& R = b->R[l];
    L.nchunks = (L.n_max + b->chunk - 1) / b->chunk;
    coff.push_back(citem.size());
    const uint32_t d = 1u << L.log_n;
    uint64_t acc = 0;
    for (uint32_t c = 0; c < L.nchunks; ++c) {
      const uint64_t j0 = (uint64_t)c * b->chunk;
      const uint64_t cnt = R[j0 + 1] - R[j0];
      const uint32_t nblk = (uint32_t)((cnt + 15) / 16);
      citem.push_back(acc);
      cblk.push_back((uint8_t)nblk);
      acc += (uint64_t)d * nblk;
    }
    citem.push_back(acc);
    cblk.push_back(0);
  }
  if (b->d_citem) cudaFree(b->d_citem);
  if (b->d_cblk) cudaFree(b->d_cblk);
  b->d_citem = nullptr;
  b->d_cblk = nullptr;
  if (cudaMalloc(&b->d_citem, std::max<size_t>(1, citem.size()) * 8) != cudaSuccess ||
      cudaMalloc(&b->d_cblk, std::max<size_t>(1, cblk.size())) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  if (!citem.empty()) {
    cudaMemcpy(b->d_citem, citem.data(), citem.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_cblk, cblk.data(), cblk.size(), cudaMemcpyHostToDevice);
  }
  uint64_t base[3] = {0, 0, 0};
  for (size_t l = 0; l < b->lanes.size(); ++l) {
    LaneDesc& L = b->lanes[l];
    L.citem = b->d_citem + coff[l];
    L.cblk = b->d_cblk + coff[l];
    const bool tw = b->products == LC_PRODUCTS_TENSOR && b->tensor_ok && b->twitems && b->lane_tw[l];
    const uint64_t items[3] = {tw ? 0 : (L.S + L.pb - 1) / L.pb, citem[coff[l] + L.nchunks], L.nb};
    for (int ph = 0; ph < 3; ++ph) {
      L.item0[ph] = base[ph];
      base[ph] += items[ph];
    }
  }
  for (int ph = 0; ph < 3; ++ph) b->total[ph] = base[ph];
  b->lane_split = (uint32_t)b->lanes.size();
  b->prod_split = b->total[1];
  for (size_t l = 0; l < b->lanes.size(); ++l)
    if (b->lanes[l].kind != (uint32_t)PlanKind::Goldilocks) {
      b->lane_split = (uint32_t)l;
      b->prod_split = b->lanes[l].item0[1];
      break;
    }
  if (cudaMemcpy(b->d_lanes, b->lanes.data(), b->lanes.size() * sizeof(LaneDesc), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return map_cuda(cudaGetLastError());
  b->dirty = true;
  return LC_OK;
}

static int batch_launch(lc_batch* b, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(b->d_counters, 0, 4 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return map_cuda(e);
  BatchParams p{};
  p.lanes = b->d_lanes;
  p.subs = b->d_subs;
  p.counters = b->d_counters;
  p.err = b->d_err;
  for (int ph = 0; ph < 3; ++ph) p.total[ph] = b->total[ph];
  p.nlanes = (uint32_t)b->lanes.size();
  p.prod_split = b->prod_split;
  p.lane_split = b->lane_split;
  p.chunk = b->chunk;
  p.claim = b->claim;
  const unsigned grid = (unsigned)std::max(1, device_sm_count()) * b->ctas;
  if (b->smem[0] > 48 * 1024) {
    e = cudaFuncSetAttribute(batch_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem[0]);
    if (e != cudaSuccess) return map_cuda(e);
  }
  if (b->total[0]) batch_kernel<0><<<grid, kBatchThreads, b->smem[0], st>>>(p);
  if (b->products == LC_PRODUCTS_TENSOR && b->tensor_ok && b->twitems) {
    static std::atomic<uint64_t> attr_tw{0};
    e = smem_attr_once(attr_tw, lane_witness_tc_kernel<kTwEpi, kTwPN>, kTwSmem);
    if (e != cudaSuccess) return map_cuda(e);
    const unsigned tgrid = (unsigned)std::min<uint64_t>(b->twitems, (uint64_t)std::max(1, device_sm_count()));
    lane_witness_tc_kernel<kTwEpi, kTwPN><<<tgrid, TwCfg<kTwEpi, kTwPN>::THREADS, kTwSmem, st>>>(b->d_twitems, b->twitems, b->d_lanes, b->d_subs,
                                                                b->d_vmaps, b->d_err);
  }
  if (b->products == LC_PRODUCTS_TENSOR && b->tensor_ok) {
    static std::atomic<uint64_t> attr8{0}, attr4{0};
    e = smem_attr_once(attr8, lane_products_tc_kernel<8>, TpCfg<8>::SMEM);
    if (e == cudaSuccess) e = smem_attr_once(attr4, lane_products_tc_kernel<4>, TpCfg<4>::SMEM);
    if (e != cudaSuccess) return map_cuda(e);
    // one CTA per item; grids above 2^31 - 1 items are refused at creation
    if (b->titems[0])
      lane_products_tc_kernel<8><<<(unsigned)b->titems[0], kTpThreads, TpCfg<8>::SMEM, st>>>(
          b->d_titems, b->d_lanes, b->d_subs, b->d_amaps, b->d_err);
    if (b->titems[1])
      lane_products_tc_kernel<4><<<(unsigned)b->titems[1], kTpThreads, TpCfg<4>::SMEM, st>>>(
          b->d_titems + b->titems[0], b->d_lanes, b->d_subs, b->d_amaps, b->d_err);
  } else {
    product_kernel<uint64_t><<<grid, kBatchThreads, 0, st>>>(p);
    product_kernel<uint32_t><<<grid, kBatchThreads, 0, st>>>(p);
  }
  batch_kernel<2><<<grid, kBatchThreads, b->smem[2], st>>>(p);
  return map_cuda(cudaGetLastError());
}

}  // namespace lc

extern "C" {

LC_API int lc_batch_create(const lc_commit_class* classes, uint32_t num_classes, const lc_commit_job* jobs,
                           uint32_t num_jobs, uint32_t flags, lc_batch** out) {
  using namespace lc;
  if (!out || (num_classes && !classes) || (num_jobs && !jobs) || (flags & ~LC_BATCH_GRAPH))
    return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  // ---- validate
  for (uint32_t c = 0; c < num_classes; ++c) {
    const lc_commit_class& C = classes[c];
    if (C.num_keys < 1 || C.num_keys > 4) return LC_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < C.num_keys; ++k) {
      const lc_ajtai_key* K = C.keys[k];
      if (!K || K->log_n != C.keys[0]->log_n || K->wide != C.keys[0]->wide) return LC_ERR_INVALID_ARGUMENT;
      if (K->log_n < 6 || K->log_n > 8) return LC_ERR_UNSUPPORTED;
    }
    if (C.keys[0]->wide && C.num_keys != 1) return LC_ERR_INVALID_ARGUMENT;
  }
  for (uint32_t i = 0; i < num_jobs; ++i) {
    const lc_commit_job& J = jobs[i];
    if (J.cls >= num_classes || !J.w || !J.out || J.n == 0 || J.kappa == 0) return LC_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(J.w) & 15) return LC_ERR_INVALID_ARGUMENT;
    for (uint32_t k = 0; k < classes[J.cls].num_keys; ++k) {
      const lc_ajtai_key* K = classes[J.cls].keys[k];
      if (J.kappa > K->k || J.n > K->m) return LC_ERR_DIMENSION_MISMATCH;
    }
  }
  lc_batch* b = new (std::nothrow) lc_batch();
  if (!b) return LC_ERR_OUT_OF_MEMORY;
  b->flags = flags;
  // ---- lanes: per class and key, jobs sorted by n (longest first), 128 at a time
  std::vector<SubJob> subs;
  std::vector<uint64_t> Rall;
  std::vector<uint32_t> itemj_all;
  std::vector<size_t> r_off, ij_off;
  size_t what_bytes = 0, partial_bytes = 0;
  std::vector<size_t> what_off, part_off;
  std::vector<uint32_t> lane_gen;  // generator of each lane's modulus (for the V-limb images)
  // Goldilocks classes first, so each element type's product items are one range
  std::vector<uint32_t> corder;
  for (int pass = 0; pass < 2; ++pass)
    for (uint32_t c = 0; c < num_classes; ++c)
      if (classes[c].keys[0]->wide == (pass == 0)) corder.push_back(c);
  for (uint32_t c : corder) {
    std::vector<uint32_t> idx;
    for (uint32_t i = 0; i < num_jobs; ++i)
      if (jobs[i].cls == c) idx.push_back(i);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return jobs[x].n > jobs[y].n; });
    for (uint32_t k = 0; k < classes[c].num_keys; ++k) {
      const lc_ajtai_key* K = classes[c].keys[k];
      const size_t eb = K->wide ? 8 : 4;
      const uint32_t d = 1u << K->log_n;
      for (size_t g0 = 0; g0 < idx.size(); g0 += kLaneJobs) {
        const size_t g1 = std::min(idx.size(), g0 + (size_t)kLaneJobs);
        LaneDesc L{};
        lane_gen.push_back(K->plan->generator[0]);
        L.kind = (uint32_t)K->plan->kind;
        L.log_n = K->log_n;
        L.q = K->plan->q[0];
        L.qinv = K->plan->qinv[0];
        L.tw_fwd = K->plan->d_tw_fwd;
        L.tw_inv = K->plan->d_tw_inv;
        L.ahat = K->d_ahat_t;
        L.a_m = K->a_m;
        L.nb = (uint32_t)(g1 - g0);
        L.sub0 = (uint32_t)subs.size();
        size_t s1, s3;
        uint32_t pb;
        if (!lane_geometry(K->plan->kind, K->log_n, s1, s3, pb)) {
          batch_free(b);
          return LC_ERR_UNSUPPORTED;
        }
        b->smem[0] = std::max(b->smem[0], s1);
        b->smem[2] = std::max(b->smem[2], s3);
        L.pb = pb;
        for (size_t g = g0; g < g1; ++g) {
          const lc_commit_job& J = jobs[idx[g]];
          SubJob sj{J.w, static_cast<unsigned char*>(J.out) + (size_t)k * J.kappa * d * eb, J.n, J.kappa};
          subs.push_back(sj);
        }
        L.n_max = jobs[idx[g0]].n;
        b->nfirst_off.push_back(b->h_nfirst.size());
        for (size_t g = g0; g < g1; g += kTpJobs) b->h_nfirst.push_back(jobs[idx[g]].n);
        // staircase offsets R[j] and the witness items' first ring elements
        r_off.push_back(Rall.size());
        std::vector<uint64_t> R(L.n_max + 1);
        uint64_t acc = 0;
        size_t active = g1 - g0;  // jobs longer than j
        for (uint32_t j = 0; j < L.n_max; ++j) {
          while (active > 0 && jobs[idx[g0 + active - 1]].n <= j) --active;
          R[j] = acc;
          acc += active;
        }
        R[L.n_max] = acc;
        L.S = acc;
        // the same offsets with each row of active jobs padded to 16 bytes, so
        // that every row of `what` starts 16-byte aligned
        const uint64_t pad = 16 / eb;
        std::vector<uint64_t> Rp(L.n_max + 1);
        uint64_t accp = 0;
        for (uint32_t j = 0; j < L.n_max; ++j) {
          Rp[j] = accp;
          accp += (R[j + 1] - R[j] + pad - 1) / pad * pad;
        }
        Rp[L.n_max] = accp;
        L.Sp = accp;
        ij_off.push_back(itemj_all.size());
        const uint64_t items = (L.S + pb - 1) / pb;
        uint32_t j = 0;
        for (uint64_t it = 0; it < items; ++it) {
          const uint64_t p = it * pb;
          while (R[j + 1] <= p) ++j;
          itemj_all.push_back(j);
        }
        Rall.insert(Rall.end(), R.begin(), R.end());
        Rall.insert(Rall.end(), Rp.begin(), Rp.end());
        b->R.push_back(std::move(R));
        what_off.push_back(what_bytes);
        what_bytes += ((size_t)d * L.Sp * eb + 255) / 256 * 256;
        part_off.push_back(partial_bytes);
        partial_bytes += (((size_t)(L.n_max + kMinChunk - 1) / kMinChunk) * d * kIPad * L.nb * eb + 255) / 256 * 256;
        b->lanes.push_back(L);
      }
    }
  }
  // ---- device buffers
  const size_t nl = std::max<size_t>(1, b->lanes.size());
  if (cudaMalloc(&b->d_lanes, nl * sizeof(LaneDesc)) != cudaSuccess ||
      cudaMalloc(&b->d_subs, std::max<size_t>(1, subs.size()) * sizeof(SubJob)) != cudaSuccess ||
      cudaMalloc(&b->d_R, (Rall.size() + 2) * 8) != cudaSuccess ||  // + slack for 16-byte copy rounding
      cudaMalloc(&b->d_itemj, std::max<size_t>(1, itemj_all.size()) * 4) != cudaSuccess ||
      cudaMalloc(&b->d_what, what_bytes + 256) != cudaSuccess ||  // + slack for 16-byte copy rounding
      cudaMalloc(&b->d_partial, std::max<size_t>(256, partial_bytes)) != cudaSuccess ||
      cudaMalloc(&b->d_counters, 4 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_err, 4) != cudaSuccess) {
    cudaGetLastError();
    batch_free(b);
    return LC_ERR_OUT_OF_MEMORY;
  }
  cudaMemset(b->d_err, 0, 4);
  if (!subs.empty()) cudaMemcpy(b->d_subs, subs.data(), subs.size() * sizeof(SubJob), cudaMemcpyHostToDevice);
  if (!Rall.empty()) cudaMemcpy(b->d_R, Rall.data(), Rall.size() * 8, cudaMemcpyHostToDevice);
  if (!itemj_all.empty())
    cudaMemcpy(b->d_itemj, itemj_all.data(), itemj_all.size() * 4, cudaMemcpyHostToDevice);
  for (size_t l = 0; l < b->lanes.size(); ++l) {
    LaneDesc& L = b->lanes[l];
    L.R = b->d_R + r_off[l];
    L.Rp = L.R + L.n_max + 1;
    L.item_j = b->d_itemj + ij_off[l];
    L.what = b->d_what + what_off[l];
    L.partial = b->d_partial + part_off[l];
  }
  // products on the tensor cores by default, where every lane can run there
  int rc = batch_tensor_setup(b);
  if (rc) {
    batch_free(b);
    return rc;
  }
  if (b->titems[0] > 0x7FFFFFFFull || b->titems[1] > 0x7FFFFFFFull) b->tensor_ok = false;
  if (b->tensor_ok) {
    rc = batch_tw_setup(b, lane_gen);
    if (rc) {
      batch_free(b);
      return rc;
    }
  }
  b->products = b->tensor_ok ? LC_PRODUCTS_TENSOR : LC_PRODUCTS_INT64;
  batch_apply_products(b);
  rc = batch_layout(b);
  if (rc) {
    batch_free(b);
    return rc;
  }
  *out = b;
  return LC_OK;
}

LC_API int lc_batch_set_config(lc_batch* b, uint32_t chunk, uint32_t ctas_per_sm, uint32_t claim) {
  using namespace lc;
  if (!b || chunk < kMinChunk || chunk > 16384 || (chunk & (chunk - 1)) || ctas_per_sm < 1 || ctas_per_sm > 4 ||
      claim < 1 || claim > 16)
    return LC_ERR_INVALID_ARGUMENT;
  b->chunk = chunk;
  b->ctas = ctas_per_sm;
  b->claim = claim;
  return batch_layout(b);
}

LC_API int lc_batch_set_products(lc_batch* b, int mode) {
  using namespace lc;
  if (!b || (mode != LC_PRODUCTS_TENSOR && mode != LC_PRODUCTS_INT64)) return LC_ERR_INVALID_ARGUMENT;
  if (mode == LC_PRODUCTS_TENSOR && !b->tensor_ok) return LC_ERR_UNSUPPORTED;
  b->products = mode;
  batch_apply_products(b);
  return batch_layout(b);
}

LC_API int lc_batch_get_products(const lc_batch* b) { return b ? b->products : -1; }

LC_API int lc_batch_get_config(const lc_batch* b, uint32_t* chunk, uint32_t* ctas_per_sm, uint32_t* claim) {
  if (!b) return LC_ERR_INVALID_ARGUMENT;
  if (chunk) *chunk = b->chunk;
  if (ctas_per_sm) *ctas_per_sm = b->ctas;
  if (claim) *claim = b->claim;
  return LC_OK;
}

LC_API int lc_batch_info(const lc_batch* b, uint64_t* items_ntt, uint64_t* items_product, uint64_t* items_finish,
                         uint32_t* lanes) {
  if (!b) return LC_ERR_INVALID_ARGUMENT;
  const bool tw = b->products == LC_PRODUCTS_TENSOR && b->tensor_ok;
  if (items_ntt) *items_ntt = b->total[0] + (tw ? b->twitems : 0);
  if (items_product)
    *items_product = b->products == LC_PRODUCTS_TENSOR && b->tensor_ok ? b->titems[0] + b->titems[1] : b->total[1];
  if (items_finish) *items_finish = b->total[2];
  if (lanes) *lanes = (uint32_t)b->lanes.size();
  return LC_OK;
}

LC_API int lc_batch_run(lc_batch* b, lc_stream stream) {
  using namespace lc;
  if (!b) return LC_ERR_INVALID_ARGUMENT;
  if (b->lanes.empty()) return LC_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (!(b->flags & LC_BATCH_GRAPH) || !b->warmed) {
    const int rc = batch_launch(b, st);
    if (!rc) b->warmed = true;
    return rc;
  }
  if (b->dirty && b->exec) {
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  if (!b->exec) {
    if (!b->cap && cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess)
      return map_cuda(cudaGetLastError());
    cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return map_cuda(e);
    const int rc = batch_launch(b, b->cap);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->cap, &g);
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc ? rc : map_cuda(e);
    }
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      b->exec = nullptr;
      return map_cuda(e);
    }
    b->graph = g;
    b->dirty = false;
  }
  return map_cuda(cudaGraphLaunch(b->exec, st));
}

LC_API int lc_batch_check(lc_batch* b, lc_stream stream) {
  using namespace lc;
  if (!b) return LC_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return map_cuda(e);
  uint32_t flag = 0;
  if (cudaMemcpy(&flag, b->d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return map_cuda(cudaGetLastError());
  if (flag) {
    cudaMemset(b->d_err, 0, 4);
    return flag == LC_DEVERR_TIMEOUT ? LC_ERR_TIMEOUT : LC_ERR_UNSUPPORTED;
  }
  return LC_OK;
}

LC_API void lc_batch_destroy(lc_batch* b) {
  if (b) lc::batch_free(b);
}

}  // extern "C"
