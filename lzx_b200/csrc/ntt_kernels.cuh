// ntt_kernels.cuh -- batched negacyclic NTT / INTT kernels (sm_100a).
//
// Computes exactly the reference transforms NttTables::forward_fast and
// NttTables::inverse_fast (lattice-ring/src/ntt.rs:118-146, 187-216):
//   forward:  out[j] = sum_i a_i psi^((2j+1) i)      (natural order, j = 0..n-1)
//   inverse:  the exact inverse of forward.
// The reference pre-scales by psi^i, bit-reverses and runs cyclic CT levels;
// here the psi powers are merged into the butterfly twiddles (negacyclic
// CT/GS "merged psi" form), so no pre/post-scaling pass exists, and the
// bit-reversal permutation is folded into the shared-memory addressing of the
// output store (forward) / input load (inverse).  Results are bit-identical
// residues.
//
// Work decomposition (one CTA iteration = one tile of P polynomials):
//   * TMA: thread 0 issues one 1-D bulk copy per polynomial into a padded
//     shared-memory slot; completion on an mbarrier (bounded wait).
//   * T = 2^(LOG_N-LOG_V) threads own one polynomial, V = 2^LOG_V values
//     each, in registers.  Phase 0 runs the butterfly levels whose bit lies
//     in the thread's register index (no data exchange); the group then
//     transposes through a padded copy of the slot (bank-conflict free) and phase 1 runs the remaining levels.  T <= 32, so a group
//     lives inside one warp and synchronises with __syncwarp.
//   * Results go back to the same slot in output order and thread 0 issues
//     1-D bulk stores.
// Twiddles for levels whose index depends only on the register number are
// read as shared-memory broadcasts; the rest come from a host-transposed
// table so that consecutive lanes read consecutive words.
#pragma once

#include "arith.cuh"
#include "common.cuh"

namespace lc {

constexpr int kMaxModuli = 8;

struct NttParams {
  const void* in;
  void* out;
  unsigned long long count;  // polynomials per modulus
  const void* tw;            // twiddle tables, one per modulus, tw_stride entries apart
  uint32_t tw_stride;
  uint32_t num_moduli;
  uint32_t q[kMaxModuli];
  uint32_t qinv[kMaxModuli];
  uint32_t* err;
};

template <int LOG_N, int LOG_V>
struct Geo {
  static constexpr int N = 1 << LOG_N;
  static constexpr int V = 1 << LOG_V;
  static constexpr int LO0 = LOG_N - LOG_V;  // lane bits per polynomial
  static constexpr int T = 1 << LO0;         // threads per polynomial
  static_assert(LO0 >= 1 && LO0 <= 5 && LOG_N <= 2 * LOG_V, "two-phase geometry");
  // Twiddle table layout (entries), see the host-side generator.
  __host__ __device__ static constexpr int fwd_phase1_off(int b) {
    // blocks for b = LO0-1 .. 0 follow the 2^LOG_V phase-0 entries
    int off = V;
    for (int bb = LO0 - 1; bb > b; --bb) off += 1 << (LOG_N - 1 - bb);
    return off;
  }
  __host__ __device__ static constexpr int fwd_entries() { return fwd_phase1_off(-1); }
  __host__ __device__ static constexpr int inv_phase0_off(int b) {
    int off = 0;
    for (int bb = 0; bb < b; ++bb) off += 1 << (LOG_N - 1 - bb);
    return off;
  }
  __host__ __device__ static constexpr int inv_phase1_off() { return inv_phase0_off(LOG_V); }
  __host__ __device__ static constexpr int inv_entries() { return inv_phase1_off() + T; }
};

LC_HD constexpr uint32_t brv_bits(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

template <class A>
LC_D A make_arith(const NttParams& p, uint32_t mi);

template <>
LC_D ShoupLazy make_arith<ShoupLazy>(const NttParams& p, uint32_t mi) {
  return ShoupLazy(p.q[mi]);
}
template <>
LC_D MontCanon make_arith<MontCanon>(const NttParams& p, uint32_t mi) {
  return MontCanon(p.q[mi], p.qinv[mi]);
}
template <>
LC_D Goldilocks make_arith<Goldilocks>(const NttParams&, uint32_t) {
  return Goldilocks();
}

template <class A>
LC_D A make_arith_q(uint32_t q, uint32_t qinv);
template <>
LC_D ShoupLazy make_arith_q<ShoupLazy>(uint32_t q, uint32_t) {
  return ShoupLazy(q);
}
template <>
LC_D MontCanon make_arith_q<MontCanon>(uint32_t q, uint32_t qinv) {
  return MontCanon(q, qinv);
}
template <>
LC_D Goldilocks make_arith_q<Goldilocks>(uint32_t, uint32_t) {
  return Goldilocks();
}

// Shared-memory slot geometry for a tile.
template <class A, int LOG_N, int LOG_V>
struct Slots {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  // One pad word per 2^LOG_V words: the transposing copy lives at
  // idx + (idx >> LOG_V), which keeps both access patterns bank-conflict free
  // and every address a per-thread base plus a compile-time offset.  N + T
  // words also spread the polynomials that share a warp over disjoint banks.
  static constexpr int S = G::N + G::T;
  LC_HD static constexpr int padded(int idx) { return idx + (idx >> LOG_V); }
};

template <class A, int LOG_N, int LOG_V, int NT, int IT, int STAGES, bool INVERSE>
struct NttKernelCfg {
  using G = Geo<LOG_N, LOG_V>;
  using SL = Slots<A, LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  static constexpr int GROUPS = NT / G::T;
  static constexpr int P = GROUPS * IT;  // polynomials per tile
  static constexpr int TW_ENTRIES = INVERSE ? G::inv_entries() : G::fwd_entries();
  static constexpr size_t TW_BYTES = ((size_t)TW_ENTRIES * sizeof(Tw) + 15) / 16 * 16;
  static constexpr size_t STAGE_BYTES = (size_t)P * SL::S * sizeof(T);
  static constexpr size_t SMEM = TW_BYTES + STAGES * STAGE_BYTES + 8 * STAGES;
  static_assert(NT % G::T == 0, "block size");
  static_assert(STAGES >= 1 && STAGES <= 4, "stages");
  static_assert((SL::S * sizeof(T)) % 16 == 0, "slot alignment for bulk copies");
  static_assert(STAGE_BYTES % 16 == 0, "stage alignment");
};

// Twiddles whose index includes the thread's lane bits (forward phase 1,
// inverse phase 0), one set per thread for the whole kernel.  With
// LOG_V == LOG_N - LOG_V there are V - 1 of them: level b holds
// V >> (b + 1) entries, at register offset (V >> (b + 1)) - 1 (forward,
// levels LO0-1 .. 0) or V - (V >> b) (inverse, levels 0 .. LOG_V-1).
template <class A, int LOG_N, int LOG_V>
struct LaneTw {
  using G = Geo<LOG_N, LOG_V>;
  static constexpr bool kHeld = G::LO0 == LOG_V;
  typename A::Tw w[kHeld ? G::V - 1 : 1];
};

template <class A, int LOG_N, int LOG_V, bool INVERSE>
LC_D void load_lane_tw(LaneTw<A, LOG_N, LOG_V>& lt, const typename A::Tw* tw, uint32_t t) {
  using G = Geo<LOG_N, LOG_V>;
  constexpr int V = G::V, TT = G::T;
  static_assert(LaneTw<A, LOG_N, LOG_V>::kHeld, "register twiddles need LOG_V == LOG_N - LOG_V");
#pragma unroll
  for (int b = 0; b < LOG_V; ++b) {
#pragma unroll
    for (int j = 0; j < (V >> (b + 1)); ++j) {
      if (!INVERSE)
        lt.w[((V >> (b + 1)) - 1) + j] = tw[G::fwd_phase1_off(b) + j * TT + t];
      else
        lt.w[(V - (V >> b)) + j] = tw[G::inv_phase0_off(b) + j * TT + t];
    }
  }
}

// Transposing copy for u32 values, V = T = 16: element e = 16*row + col is
// kept at row*16 + ((col>>2) ^ ((row>>1)&3))*4 + (col&3), an XOR swizzle of
// the 16-byte chunks of each row.  Column accesses (16 lanes, one row) hit
// 16 distinct banks; row accesses go as four 16-byte vector accesses, and
// every quarter-warp of them covers 8 distinct chunk banks.
LC_HD constexpr int swz16(int e) { return (e & ~12) | ((((e >> 2) & 3) ^ ((e >> 5) & 3)) << 2); }

// Options of the transform: kOptRegTw takes the lane twiddles from `lt`
// (registers); kOptSwz, for u32 values with V = T = 16, uses the swizzled
// transposing copy with 16-byte vector accesses on its row side.
enum : int { kOptRegTw = 1, kOptSwz = 2 };

// One polynomial held by a group of T threads: the complete forward
// (natural coefficients -> natural evaluations) or inverse transform of the
// shared-memory slot, in place.
template <class A, int LOG_N, int LOG_V, bool INVERSE, int OPT>
LC_D void transform_slot_x(typename A::T* slot, const typename A::Tw* tw, const A& ar, uint32_t t,
                           const LaneTw<A, LOG_N, LOG_V>& lt) {
  using G = Geo<LOG_N, LOG_V>;
  using SL = Slots<A, LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int V = G::V, LO0 = G::LO0, TT = G::T;
  constexpr bool REGTW = (OPT & kOptRegTw) != 0;
  constexpr bool SWZ = (OPT & kOptSwz) != 0 && sizeof(T) == 4 && LOG_V == 4 && LO0 == 4;
  static_assert(!REGTW || LaneTw<A, LOG_N, LOG_V>::kHeld, "register twiddles need LOG_V == LOG_N - LOG_V");
  T v[V];
  if (!INVERSE) {
    // ---- phase 0: natural-order coefficients, register bits [LO0, LOG_N)
#pragma unroll
    for (int r = 0; r < V; ++r) v[r] = slot[(r << LO0) | t];
#pragma unroll
    for (int b = LOG_N - 1; b >= LO0; --b) {
      const int rb = 1 << (b - LO0);
#pragma unroll
      for (int r = 0; r < V; ++r) {
        if (r & rb) continue;
        const Tw w = tw[(1 << (LOG_N - 1 - b)) + (r >> (b + 1 - LO0))];
        if (b == LOG_N - 1)
          ar.fwd_first(v[r], v[r | rb], w);
        else
          ar.fwd(v[r], v[r | rb], w);
      }
    }
    __syncwarp();
    if constexpr (SWZ) {
#pragma unroll
      for (int r = 0; r < V; ++r) slot[swz16((r << LO0) | (int)t)] = v[r];
    } else {
#pragma unroll
      for (int r = 0; r < V; ++r) slot[SL::padded((r << LO0) | t)] = v[r];
    }
    __syncwarp();
    // ---- phase 1: register bits [0, LOG_V), levels b < LO0
    if constexpr (SWZ) {
      const uint32_t sx = (t >> 1) & 3u;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint4 q4 = *reinterpret_cast<const uint4*>(slot + (t << 4) + ((c ^ sx) << 2));
        v[4 * c] = q4.x;
        v[4 * c + 1] = q4.y;
        v[4 * c + 2] = q4.z;
        v[4 * c + 3] = q4.w;
      }
    } else {
#pragma unroll
      for (int r = 0; r < V; ++r) v[r] = slot[SL::padded((t << LOG_V) | r)];
    }
#pragma unroll
    for (int b = LO0 - 1; b >= 0; --b) {
      const int rb = 1 << b;
#pragma unroll
      for (int r = 0; r < V; ++r) {
        if (r & rb) continue;
        Tw w;
        if constexpr (REGTW) w = lt.w[((V >> (b + 1)) - 1) + (r >> (b + 1))];
        else w = tw[G::fwd_phase1_off(b) + (r >> (b + 1)) * TT + t];
        ar.fwd(v[r], v[r | rb], w);
      }
    }
    __syncwarp();
    // ---- output in natural order: LN index (t<<LOG_V)|r sits at brv of it
#pragma unroll
    for (int r = 0; r < V; ++r)
      slot[(brv_bits(r, LOG_V) << LO0) | brv_bits(t, LO0)] = ar.fwd_final(v[r]);
  } else {
    // ---- phase 0: evaluations (natural order) read at bit-reversed slots,
    //      register bits [0, LOG_V), levels b < LOG_V (per-lane twiddles)
#pragma unroll
    for (int r = 0; r < V; ++r) v[r] = slot[(brv_bits(r, LOG_V) << LO0) | brv_bits(t, LO0)];
#pragma unroll
    for (int b = 0; b < LOG_V; ++b) {
      const int rb = 1 << b;
#pragma unroll
      for (int r = 0; r < V; ++r) {
        if (r & rb) continue;
        Tw w;
        if constexpr (REGTW) w = lt.w[(V - (V >> b)) + (r >> (b + 1))];
        else w = tw[G::inv_phase0_off(b) + (r >> (b + 1)) * TT + t];
        if (b == 0)
          ar.inv_first(v[r], v[r | rb], w);
        else
          ar.inv(v[r], v[r | rb], w);
      }
    }
    __syncwarp();
    if constexpr (SWZ) {
      const uint32_t sx = (t >> 1) & 3u;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(slot + (t << 4) + ((c ^ sx) << 2)) =
            make_uint4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    } else {
#pragma unroll
      for (int r = 0; r < V; ++r) slot[SL::padded((t << LOG_V) | r)] = v[r];
    }
    __syncwarp();
    // ---- phase 1: register bits [LO0, LOG_N), levels b >= LOG_V (uniform twiddles)
    if constexpr (SWZ) {
#pragma unroll
      for (int r = 0; r < V; ++r) v[r] = slot[swz16((r << LO0) | (int)t)];
    } else {
#pragma unroll
      for (int r = 0; r < V; ++r) v[r] = slot[SL::padded((r << LO0) | t)];
    }
    constexpr int P1 = G::inv_phase1_off();
#pragma unroll
    for (int b = LOG_V; b < LOG_N; ++b) {
      const int rb = 1 << (b - LO0);
#pragma unroll
      for (int r = 0; r < V; ++r) {
        if (r & rb) continue;
        if (b == LOG_N - 1) {
          ar.inv_last(v[r], v[r | rb], tw[P1 + 0], tw[P1 + 1]);
        } else {
          const Tw w = tw[P1 + (1 << (LOG_N - 1 - b)) + (r >> (b + 1 - LO0))];
          ar.inv(v[r], v[r | rb], w);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < V; ++r) slot[(r << LO0) | t] = ar.inv_final(v[r]);
  }
}

template <class A, int LOG_N, int LOG_V, bool INVERSE>
LC_D void transform_slot(typename A::T* slot, const typename A::Tw* tw, const A& ar, uint32_t t) {
  const LaneTw<A, LOG_N, LOG_V> unused{};
  transform_slot_x<A, LOG_N, LOG_V, INVERSE, 0>(slot, tw, ar, t, unused);
}

// Persistent tile loop over a ring of STAGES shared-memory tile buffers;
// OPT: kOpt* flags of the transform.
template <class A, int LOG_N, int LOG_V, int NT, int IT, int STAGES, bool INVERSE, int OPT>
__global__ void __launch_bounds__(NT) ntt_tile_kernel(const __grid_constant__ NttParams p) {
  using C = NttKernelCfg<A, LOG_N, LOG_V, NT, IT, STAGES, INVERSE>;
  using G = typename C::G;
  using T = typename C::T;
  using Tw = typename C::Tw;
  constexpr int N = G::N, TT = G::T, S = C::SL::S, P = C::P;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // this modulus's twiddle table, then the stage ring, then the mbarriers
  Tw* tw = reinterpret_cast<Tw*>(smem_raw);
  T* data = reinterpret_cast<T*>(smem_raw + C::TW_BYTES);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + C::TW_BYTES + STAGES * C::STAGE_BYTES);

  const uint32_t mi = blockIdx.y;
  const A ar = make_arith<A>(p, mi);
  const int tid = threadIdx.x;
  const int grp = tid / TT;
  const uint32_t t = (uint32_t)(tid % TT);

  {
    const Tw* src = reinterpret_cast<const Tw*>(p.tw) + (size_t)mi * p.tw_stride;
    for (int i = tid; i < C::TW_ENTRIES; i += NT) tw[i] = src[i];
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  LaneTw<A, LOG_N, LOG_V> lt;
  if constexpr ((OPT & kOptRegTw) != 0) load_lane_tw<A, LOG_N, LOG_V, INVERSE>(lt, tw, t);

  const T* in = reinterpret_cast<const T*>(p.in) + (size_t)mi * p.count * N;
  T* out = reinterpret_cast<T*>(p.out) + (size_t)mi * p.count * N;
  const uint32_t ntiles = (uint32_t)((p.count + P - 1) / P);
  const uint32_t stride = gridDim.x;

  auto valid = [&](uint32_t tile) -> int {
    const unsigned long long first = (unsigned long long)tile * P;
    return (int)((p.count - first) < (unsigned long long)P ? (p.count - first) : P);
  };
  auto issue_load = [&](uint32_t tile, int s) {
    const T* src = in + (size_t)tile * P * N;
    const int nv = valid(tile);
    T* dst = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
    mbar_arrive_expect_tx(&bar[s], (uint32_t)(nv * N * sizeof(T)));
    for (int q = 0; q < nv; ++q) bulk_g2s(dst + q * S, src + (size_t)q * N, N * sizeof(T), &bar[s]);
  };

  // Ring of STAGES tile buffers.  Iteration i consumes stage i % STAGES; at
  // its start thread 0 refills the stage consumed by iteration i-1 with the
  // tile STAGES-1 strides ahead once that stage's stores have finished
  // reading it, so up to STAGES-1 tile loads stay in flight behind the
  // transforms.
  if (tid == 0) {
    for (int k = 0; k < STAGES - 1; ++k) {
      const unsigned long long tk = blockIdx.x + (unsigned long long)k * stride;
      if (tk < ntiles) issue_load((uint32_t)tk, k);
    }
  }
  uint32_t parity = 0;  // bit s: parity of the next completion of stage s
  bool refilled = false;  // (thread 0) whether this iteration issued a prefetch
  int failed_at = -1;     // iteration whose wait timed out
  uint32_t tile = blockIdx.x;
  for (int i = 0; tile < ntiles; ++i, tile += stride) {
    const int s = i % STAGES;
    if (tid == 0) {
      refilled = false;
      const unsigned long long ahead = tile + (unsigned long long)(STAGES - 1) * stride;
      if (ahead < ntiles) {
        bulk_wait_read<0>();  // stores of iteration i-1 (the refilled stage) are done reading
        issue_load((uint32_t)ahead, (i + STAGES - 1) % STAGES);
        refilled = true;
      }
    }
    const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
    parity ^= 1u << s;
    if (__syncthreads_or(!ok)) {
      failed_at = i;
      break;
    }

    T* stage = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
#pragma unroll 1
    for (int it = 0; it < IT; ++it)
      transform_slot_x<A, LOG_N, LOG_V, INVERSE, OPT>(stage + (it * C::GROUPS + grp) * S, tw, ar, t, lt);

    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      T* dst = out + (size_t)tile * P * N;
      const int nv = valid(tile);
      for (int q = 0; q < nv; ++q) bulk_s2g(dst + (size_t)q * N, stage + q * S, N * sizeof(T));
      bulk_commit();
    }
  }
  if (tid == 0) {
    if (failed_at >= 0) {
      record_error(p.err, LC_DEVERR_TIMEOUT);
      // Loads still in flight must land before the CTA exits: the tiles
      // 1 .. STAGES-2 strides ahead (issued earlier) and STAGES-1 ahead
      // (issued in the failed iteration when `refilled`).  Bounded waits;
      // the timed-out stage is not waited for again.
      for (int k = 1; k < STAGES; ++k) {
        const unsigned long long tk = tile + (unsigned long long)k * stride;
        const bool issued = (k < STAGES - 1) || refilled;
        if (tk >= ntiles || !issued) continue;
        const int sk = (failed_at + k) % STAGES;
        mbar_wait(&bar[sk], (parity >> sk) & 1u);
      }
    }
    bulk_wait<0>();
  }
}

// ---------------------------------------------------------------------------
// Warp-autonomous variant: every warp runs its own ring of STAGES tiles of
// 32/T * IT polynomials (its own mbarriers; lane 0 issues its bulk copies), so
// the steady-state loop has no CTA-wide barrier at all.  Warps take tiles
// strided over the whole grid.
template <class A, int LOG_N, int LOG_V, int WARPS, int IT, int STAGES, bool INVERSE>
struct NttWarpCfg {
  using G = Geo<LOG_N, LOG_V>;
  using SL = Slots<A, LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  static constexpr int NT = 32 * WARPS;
  static constexpr int GROUPS = 32 / G::T;      // polynomials per warp per pass
  static constexpr int P = GROUPS * IT;          // polynomials per warp tile
  static constexpr int TW_ENTRIES = INVERSE ? G::inv_entries() : G::fwd_entries();
  static constexpr size_t TW_BYTES = ((size_t)TW_ENTRIES * sizeof(Tw) + 15) / 16 * 16;
  static constexpr size_t STAGE_BYTES = (size_t)P * SL::S * sizeof(T);
  static constexpr size_t WARP_BYTES = STAGES * STAGE_BYTES;
  static constexpr size_t SMEM = TW_BYTES + WARPS * WARP_BYTES + 8 * STAGES * WARPS;
  static_assert(G::T <= 32 && 32 % G::T == 0, "a polynomial group lives in one warp");
  static_assert(STAGES >= 2 && STAGES <= 4, "stages");
  static_assert(STAGE_BYTES % 16 == 0, "stage alignment");
};

template <class A, int LOG_N, int LOG_V, int WARPS, int IT, int STAGES, bool INVERSE>
__global__ void __launch_bounds__(32 * WARPS) ntt_warp_kernel(const __grid_constant__ NttParams p) {
  using C = NttWarpCfg<A, LOG_N, LOG_V, WARPS, IT, STAGES, INVERSE>;
  using G = typename C::G;
  using T = typename C::T;
  using Tw = typename C::Tw;
  constexpr int N = G::N, TT = G::T, S = C::SL::S, P = C::P;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  Tw* tw = reinterpret_cast<Tw*>(smem_raw);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  T* data = reinterpret_cast<T*>(smem_raw + C::TW_BYTES + warp * C::WARP_BYTES);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + C::TW_BYTES + WARPS * C::WARP_BYTES) +
                  warp * STAGES;

  const uint32_t mi = blockIdx.y;
  const A ar = make_arith<A>(p, mi);
  const int grp = lane / TT;
  const uint32_t t = (uint32_t)(lane % TT);
  {
    const Tw* src = reinterpret_cast<const Tw*>(p.tw) + (size_t)mi * p.tw_stride;
    for (int i = tid; i < C::TW_ENTRIES; i += C::NT) tw[i] = src[i];
  }
  if (lane == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();  // twiddles and barriers ready; the only CTA-wide barrier

  const T* in = reinterpret_cast<const T*>(p.in) + (size_t)mi * p.count * N;
  T* out = reinterpret_cast<T*>(p.out) + (size_t)mi * p.count * N;
  const uint32_t ntiles = (uint32_t)((p.count + P - 1) / P);
  const uint32_t stride = gridDim.x * WARPS;
  const uint32_t first_tile = blockIdx.x * WARPS + warp;

  auto valid = [&](uint32_t tile) -> int {
    const unsigned long long first = (unsigned long long)tile * P;
    return (int)((p.count - first) < (unsigned long long)P ? (p.count - first) : P);
  };
  auto issue_load = [&](uint32_t tile, int s) {
    const T* src = in + (size_t)tile * P * N;
    const int nv = valid(tile);
    T* dst = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
    mbar_arrive_expect_tx(&bar[s], (uint32_t)(nv * N * sizeof(T)));
    for (int q = 0; q < nv; ++q) bulk_g2s(dst + q * S, src + (size_t)q * N, N * sizeof(T), &bar[s]);
  };

  if (lane == 0) {
    for (int k = 0; k < STAGES - 1; ++k) {
      const unsigned long long tk = first_tile + (unsigned long long)k * stride;
      if (tk < ntiles) issue_load((uint32_t)tk, k);
    }
  }
  uint32_t parity = 0;
  bool refilled = false;
  int failed_at = -1;
  uint32_t tile = first_tile;
  for (int i = 0; tile < ntiles; ++i, tile += stride) {
    const int s = i % STAGES;
    if (lane == 0) {
      refilled = false;
      const unsigned long long ahead = tile + (unsigned long long)(STAGES - 1) * stride;
      if (ahead < ntiles) {
        bulk_wait_read<0>();  // this warp's stores of iteration i-1 are done reading
        issue_load((uint32_t)ahead, (i + STAGES - 1) % STAGES);
        refilled = true;
      }
    }
    const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
    parity ^= 1u << s;
    if (__any_sync(0xffffffffu, !ok)) {
      failed_at = i;
      break;
    }
    T* stage = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
#pragma unroll 1
    for (int it = 0; it < IT; ++it)
      transform_slot<A, LOG_N, LOG_V, INVERSE>(stage + (it * C::GROUPS + grp) * S, tw, ar, t);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      T* dst = out + (size_t)tile * P * N;
      const int nv = valid(tile);
      for (int q = 0; q < nv; ++q) bulk_s2g(dst + (size_t)q * N, stage + q * S, N * sizeof(T));
      bulk_commit();
    }
  }
  if (lane == 0) {
    if (failed_at >= 0) {
      record_error(p.err, LC_DEVERR_TIMEOUT);
      for (int k = 1; k < STAGES; ++k) {
        const unsigned long long tk = tile + (unsigned long long)k * stride;
        const bool issued = (k < STAGES - 1) || refilled;
        if (tk >= ntiles || !issued) continue;
        const int sk = (failed_at + k) % STAGES;
        mbar_wait(&bar[sk], (parity >> sk) & 1u);
      }
    }
    bulk_wait<0>();
  }
}

// ---------------------------------------------------------------------------
// Small rings (T = 1): one thread per polynomial, all levels in registers,
// direct global loads/stores.  Twiddles: forward uses psi^brv(k) at k in
// [1,N); inverse uses entry 0 = n^{-1}, 1 = psi^-brv(1) n^{-1}, k >= 2 the
// plain inverse twiddle.
template <class A, int LOG_N, bool INVERSE>
__global__ void __launch_bounds__(128) ntt_small_kernel(const __grid_constant__ NttParams p) {
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int N = 1 << LOG_N;
  __shared__ Tw tw[N];
  const uint32_t mi = blockIdx.y;
  const A ar = make_arith<A>(p, mi);
  {
    const Tw* src = reinterpret_cast<const Tw*>(p.tw) + (size_t)mi * p.tw_stride;
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = src[i];
  }
  __syncthreads();
  const T* in = reinterpret_cast<const T*>(p.in) + (size_t)mi * p.count * N;
  T* out = reinterpret_cast<T*>(p.out) + (size_t)mi * p.count * N;
  for (unsigned long long poly = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
       poly < p.count; poly += (unsigned long long)gridDim.x * blockDim.x) {
    T v[N];
    const T* src = in + poly * N;
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = src[INVERSE ? brv_bits(i, LOG_N) : i];
    if (!INVERSE) {
#pragma unroll
      for (int b = LOG_N - 1; b >= 0; --b) {
#pragma unroll
        for (int r = 0; r < N; ++r) {
          if (r & (1 << b)) continue;
          ar.fwd(v[r], v[r | (1 << b)], tw[(1 << (LOG_N - 1 - b)) + (r >> (b + 1))]);
        }
      }
      T* dst = out + poly * N;
#pragma unroll
      for (int i = 0; i < N; ++i) dst[brv_bits(i, LOG_N)] = ar.fwd_final(v[i]);
    } else {
#pragma unroll
      for (int b = 0; b < LOG_N; ++b) {
#pragma unroll
        for (int r = 0; r < N; ++r) {
          if (r & (1 << b)) continue;
          if (b == LOG_N - 1)
            ar.inv_last(v[r], v[r | (1 << b)], tw[0], tw[1]);
          else
            ar.inv(v[r], v[r | (1 << b)], tw[(1 << (LOG_N - 1 - b)) + (r >> (b + 1))]);
        }
      }
      T* dst = out + poly * N;
#pragma unroll
      for (int i = 0; i < N; ++i) dst[i] = ar.inv_final(v[i]);
    }
  }
}

}  // namespace lc
