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
//     transposes through an XOR-swizzled copy of the slot (bank-conflict
//     free) and phase 1 runs the remaining levels.  T <= 32, so a group
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
  static constexpr int XM = (1 << (LOG_V < LO0 ? LOG_V : LO0)) - 1;
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

// Shared-memory slot geometry for a tile.
template <class A, int LOG_N, int LOG_V>
struct Slots {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  // pad so that the polynomials sharing a warp land on disjoint banks
  static constexpr int PAD = (sizeof(T) == 4) ? (G::T < 32 ? G::T : 0) : (G::T < 16 ? G::T : 0);
  static constexpr int S = G::N + PAD;
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
  static_assert(STAGES == 1 || STAGES == 2, "stages");
  static_assert((SL::S * sizeof(T)) % 16 == 0, "slot alignment for bulk copies");
  static_assert(STAGE_BYTES % 16 == 0, "stage alignment");
};

// One polynomial held by a group of T threads: the complete forward
// (natural coefficients -> natural evaluations) or inverse transform of the
// shared-memory slot, in place.
template <class A, int LOG_N, int LOG_V, bool INVERSE>
LC_D void transform_slot(typename A::T* slot, const typename A::Tw* tw, const A& ar, uint32_t t) {
  using G = Geo<LOG_N, LOG_V>;
  using T = typename A::T;
  using Tw = typename A::Tw;
  constexpr int V = G::V, LO0 = G::LO0, TT = G::T;
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
        ar.fwd(v[r], v[r | rb], w);
      }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < V; ++r) {
      const uint32_t idx = (r << LO0) | t;
      slot[idx ^ ((idx >> LOG_V) & G::XM)] = v[r];
    }
    __syncwarp();
    // ---- phase 1: register bits [0, LOG_V), levels b < LO0
#pragma unroll
    for (int r = 0; r < V; ++r) {
      const uint32_t idx = (t << LOG_V) | r;
      v[r] = slot[idx ^ ((idx >> LOG_V) & G::XM)];
    }
#pragma unroll
    for (int b = LO0 - 1; b >= 0; --b) {
      const int rb = 1 << b;
#pragma unroll
      for (int r = 0; r < V; ++r) {
        if (r & rb) continue;
        const Tw w = tw[G::fwd_phase1_off(b) + (r >> (b + 1)) * TT + t];
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
        const Tw w = tw[G::inv_phase0_off(b) + (r >> (b + 1)) * TT + t];
        ar.inv(v[r], v[r | rb], w);
      }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < V; ++r) {
      const uint32_t idx = (t << LOG_V) | r;
      slot[idx ^ ((idx >> LOG_V) & G::XM)] = v[r];
    }
    __syncwarp();
    // ---- phase 1: register bits [LO0, LOG_N), levels b >= LOG_V (uniform twiddles)
#pragma unroll
    for (int r = 0; r < V; ++r) {
      const uint32_t idx = (r << LO0) | t;
      v[r] = slot[idx ^ ((idx >> LOG_V) & G::XM)];
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

// Persistent tile loop.  STAGES == 2 double-buffers the tiles: the bulk load
// of the next tile is in flight while the current one is transformed.
template <class A, int LOG_N, int LOG_V, int NT, int IT, int STAGES, bool INVERSE>
__global__ void __launch_bounds__(NT) ntt_tile_kernel(const __grid_constant__ NttParams p) {
  using C = NttKernelCfg<A, LOG_N, LOG_V, NT, IT, STAGES, INVERSE>;
  using G = typename C::G;
  using T = typename C::T;
  using Tw = typename C::Tw;
  constexpr int N = G::N, TT = G::T, S = C::SL::S, P = C::P;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  Tw* tw = reinterpret_cast<Tw*>(smem_raw);
  T* data = reinterpret_cast<T*>(smem_raw + C::TW_BYTES);
  uint64_t* bar =
      reinterpret_cast<uint64_t*>(smem_raw + C::TW_BYTES + STAGES * C::STAGE_BYTES);

  const uint32_t mi = blockIdx.y;
  const A ar = make_arith<A>(p, mi);
  const int tid = threadIdx.x;
  const int grp = tid / TT;
  const uint32_t t = (uint32_t)(tid % TT);

  // twiddles for this modulus -> shared memory
  {
    const Tw* src = reinterpret_cast<const Tw*>(p.tw) + (size_t)mi * p.tw_stride;
    for (int i = tid; i < C::TW_ENTRIES; i += NT) tw[i] = src[i];
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  const T* in = reinterpret_cast<const T*>(p.in) + (size_t)mi * p.count * N;
  T* out = reinterpret_cast<T*>(p.out) + (size_t)mi * p.count * N;
  const unsigned long long ntiles = (p.count + P - 1) / P;

  auto tile_valid = [&](unsigned long long tile) -> int {
    const unsigned long long first = tile * P;
    return (int)((p.count - first) < (unsigned long long)P ? (p.count - first) : P);
  };
  auto issue_load = [&](unsigned long long tile, int s) {
    const unsigned long long first = tile * P;
    const int nv = tile_valid(tile);
    T* dst = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
    mbar_arrive_expect_tx(&bar[s], (uint32_t)(nv * N * sizeof(T)));
    for (int q = 0; q < nv; ++q) bulk_g2s(dst + q * S, in + (first + q) * N, N * sizeof(T), &bar[s]);
  };

  unsigned long long tile = blockIdx.x;
  if (STAGES == 2 && tid == 0 && tile < ntiles) issue_load(tile, 0);
  uint32_t parity = 0;   // bit s: parity of the next completion of stage s
  int other_inflight = -1;  // (thread 0) stage whose prefetch was issued this iteration
  bool failed = false;
  for (int i = 0; tile < ntiles; ++i, tile += gridDim.x) {
    const int s = (STAGES == 1) ? 0 : (i & 1);
    if (tid == 0) {
      other_inflight = -1;
      if (STAGES == 1) {
        bulk_wait_read<0>();  // the previous tile's stores have read the slots
        issue_load(tile, 0);
      } else if (tile + gridDim.x < ntiles) {
        bulk_wait_read<0>();  // stores of the previous iteration (stage s^1) are done reading
        issue_load(tile + gridDim.x, s ^ 1);
        other_inflight = s ^ 1;
      }
    }
    const bool ok = mbar_wait(&bar[s], (parity >> s) & 1u);
    parity ^= 1u << s;
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }

    T* stage = data + (size_t)s * (C::STAGE_BYTES / sizeof(T));
#pragma unroll 1
    for (int it = 0; it < IT; ++it)
      transform_slot<A, LOG_N, LOG_V, INVERSE>(stage + (it * C::GROUPS + grp) * S, tw, ar, t);

    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      const unsigned long long first = tile * P;
      const int nv = tile_valid(tile);
      for (int q = 0; q < nv; ++q) bulk_s2g(out + (first + q) * N, stage + q * S, N * sizeof(T));
      bulk_commit();
    }
  }
  if (tid == 0) {
    if (failed) {
      record_error(p.err, LC_DEVERR_TIMEOUT);
      // a prefetch issued into the other stage must land before the CTA exits
      // (bounded wait; the timed-out stage itself is not waited for again)
      if (other_inflight >= 0) mbar_wait(&bar[other_inflight], (parity >> other_inflight) & 1u);
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
