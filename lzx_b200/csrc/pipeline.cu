// pipeline.cu -- one folding step of the commitment path as a single
// CUDA-graph launch, and the u64 -> CRT residue split it needs.
//
// A folding step over d = 64 Goldilocks (lattice-folding/src/neo.rs): the
// witness z (m ring elements) is split into its base-2^8 digit rows
// (decomp_b, neo.rs:253-266), every digit row is committed with the cached-NTT
// key (AjtaiPublicKey::commit, lattice-commitment/src/ajtai.rs:118-153, batch
// of 8 witnesses), and z itself is mapped to a CRT set of 30-bit primes
// (Modulus32::reduce_u64, lattice-ring/src/modulus.rs:65 per prime) and
// transformed there (NttTables::forward_fast, ntt.rs:118-146).  The CRT
// branch depends only on z, so it runs on a second stream beside the
// decomposition and the commitments (forked and joined with events; in the
// graph, two parallel branches).  The object owns fixed device buffers, so
// after one eager warm-up run (which sizes the key's scratch) the stages are
// captured once into a CUDA graph and every later run is one cudaGraphLaunch.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>

#include "../../include/lattice_cuda.h"
#include "arith.cuh"
#include "common.cuh"
#include "internal.h"
#include "ntt_kernels.cuh"

namespace lc {

struct CrtParams {
  uint32_t q[8];
  uint64_t mu[8];  // floor(2^64 / q)
  uint32_t nm;
};

// out[mod][e] = z[e] mod q_mod (Barrett with floor(2^64/q): remainder < 2q,
// one correction).  4 elements per thread, 16-byte stores when aligned.
__global__ void crt_residues_kernel(const uint64_t* __restrict__ z, size_t count, uint32_t* __restrict__ out,
                                    const __grid_constant__ CrtParams p) {
  const bool vec = (count & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  const size_t groups = (count + 3) / 4;
  for (size_t gi = blockIdx.x * (size_t)blockDim.x + threadIdx.x; gi < groups;
       gi += (size_t)gridDim.x * blockDim.x) {
    const size_t e0 = gi * 4;
    uint64_t x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = e0 + u < count ? __ldg(z + e0 + u) : 0;
    for (uint32_t mi = 0; mi < p.nm; ++mi) {
      const uint32_t q = p.q[mi];
      uint32_t r[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        uint64_t t = x[u] - __umul64hi(x[u], p.mu[mi]) * q;
        r[u] = (uint32_t)(t >= q ? t - q : t);
      }
      uint32_t* dst = out + (size_t)mi * count + e0;
      if (vec) {
        *reinterpret_cast<uint4*>(dst) = make_uint4(r[0], r[1], r[2], r[3]);
      } else {
        for (int u = 0; u < 4 && e0 + u < count; ++u) dst[u] = r[u];
      }
    }
  }
}

int crt_residues(const lc_ntt_plan* plan, const uint64_t* z, size_t count, uint32_t* out, cudaStream_t st) {
  CrtParams p{};
  p.nm = plan->num_moduli;
  for (uint32_t i = 0; i < p.nm; ++i) {
    p.q[i] = plan->q[i];
    p.mu[i] = ~0ull / plan->q[i];
  }
  const int sms = std::max(device_sm_count(), 1);
  const size_t groups = (count + 3) / 4;
  const unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((groups + 255) / 256, (size_t)sms * 16));
  crt_residues_kernel<<<blocks, 256, 0, st>>>(z, count, out, p);
  return map_cuda(cudaGetLastError());
}

// The CRT branch in one pass over z: every CTA brings tiles of P ring
// elements of z (u64) into shared memory by TMA (a ring of STAGES tiles) and,
// for each prime of the set, every thread group reduces its ring element mod
// q into its own shared-memory slot (the canonical remainder, as
// crt_residues_kernel), transforms it there (the forward transform of
// ntt_tile_kernel) and stores it to out[prime][..] with 16-byte stores -- z
// is read once and the residues never go through HBM: 1.5 bytes of traffic
// per residue instead of 3.5 for the two separate launches.  A group
// synchronises only its own warp; the CTA meets once per tile.
struct CrtNttParams {
  NttParams np;  // out = [nm][count][n] residues; tw = the forward tables; q, qinv, err
  const uint64_t* z;  // [count][n]
  uint64_t mu[kMaxModuli];  // floor(2^64 / q)
};

template <class A, int LOG_N, int LOG_V, int NT, int STAGES>
struct CrtNttCfg {
  using G = Geo<LOG_N, LOG_V>;
  using SL = Slots<A, LOG_N, LOG_V>;
  static constexpr int P = NT / G::T;  // polynomials per tile, one per thread group
  static constexpr size_t ZSTAGE = (size_t)P * G::N * 8;
  static constexpr size_t RBUF = (size_t)P * SL::S * 4;
  static constexpr size_t OFF_R = STAGES * ZSTAGE;
  static constexpr size_t OFF_BAR = OFF_R + RBUF;
  static constexpr size_t OFF_TW = (OFF_BAR + 8 * STAGES + 15) / 16 * 16;
  static constexpr int TW_ENTRIES = G::fwd_entries();
  static size_t smem(uint32_t nm) { return OFF_TW + (size_t)nm * TW_ENTRIES * sizeof(typename A::Tw); }
  static_assert(ZSTAGE % 16 == 0 && (SL::S * 4) % 16 == 0, "16-byte alignment");
  static_assert(G::N % (4 * G::T) == 0, "whole 16-byte stores per thread");
};

template <class A, int LOG_N, int LOG_V, int NT, int STAGES>
__global__ void __launch_bounds__(NT) crt_ntt_kernel(const __grid_constant__ CrtNttParams p) {
  using C = CrtNttCfg<A, LOG_N, LOG_V, NT, STAGES>;
  using G = typename C::G;
  using Tw = typename A::Tw;
  constexpr int N = G::N, TT = G::T, S = C::SL::S, P = C::P;
  constexpr int PER = N / TT;  // values per thread of a group
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* zst = reinterpret_cast<uint64_t*>(smem_raw);
  uint32_t* rbuf = reinterpret_cast<uint32_t*>(smem_raw + C::OFF_R);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + C::OFF_BAR);
  Tw* tw = reinterpret_cast<Tw*>(smem_raw + C::OFF_TW);
  const uint32_t nm = p.np.num_moduli;
  const int tid = threadIdx.x;
  const int grp = tid / TT;
  const uint32_t t = (uint32_t)(tid % TT);
  {
    const Tw* src = reinterpret_cast<const Tw*>(p.np.tw);
    for (uint32_t mi = 0; mi < nm; ++mi)
      for (int i = tid; i < C::TW_ENTRIES; i += NT)
        tw[mi * C::TW_ENTRIES + i] = src[(size_t)mi * p.np.tw_stride + i];
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const unsigned long long count = p.np.count;
  uint32_t* out = static_cast<uint32_t*>(p.np.out);
  uint32_t* slot = rbuf + grp * S;  // this group's ring element
  const uint32_t ntiles = (uint32_t)((count + P - 1) / P);
  const uint32_t stride = gridDim.x;
  auto valid = [&](uint32_t tile) -> int {
    const unsigned long long first = (unsigned long long)tile * P;
    return (int)((count - first) < (unsigned long long)P ? (count - first) : P);
  };
  auto issue_load = [&](uint32_t tile, int s) {
    const uint32_t bytes = (uint32_t)(valid(tile) * N * 8);
    mbar_arrive_expect_tx(&bar[s], bytes);
    bulk_g2s(zst + (size_t)s * P * N, p.z + (size_t)tile * P * N, bytes, &bar[s]);
  };
  if (tid == 0) {
    for (int k = 0; k < STAGES - 1; ++k) {
      const unsigned long long tk = blockIdx.x + (unsigned long long)k * stride;
      if (tk < ntiles) issue_load((uint32_t)tk, k);
    }
  }
  uint32_t parity = 0;
  bool refilled = false;
  int failed_at = -1;
  uint32_t tile = blockIdx.x;
  for (int i = 0; tile < ntiles; ++i, tile += stride) {
    const int s = i % STAGES;
    if (tid == 0) {
      // the stage consumed by iteration i-1 is free: every thread passed the
      // barrier that ends each iteration
      refilled = false;
      const unsigned long long ahead = tile + (unsigned long long)(STAGES - 1) * stride;
      if (ahead < ntiles) {
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
    const uint64_t* zt = zst + (size_t)s * P * N + (size_t)grp * N;
    const bool mine = grp < valid(tile);
    for (uint32_t mi = 0; mi < nm; ++mi) {
      const uint32_t q = p.np.q[mi];
      const uint64_t mu = p.mu[mi];
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const uint64_t x = zt[t + k * TT];
        const uint64_t r = x - __umul64hi(x, mu) * q;  // < 2q
        slot[t + k * TT] = (uint32_t)(r >= q ? r - q : r);
      }
      __syncwarp();
      const A ar = make_arith<A>(p.np, mi);
      transform_slot<A, LOG_N, LOG_V, false>(slot, tw + mi * C::TW_ENTRIES, ar, t);
      __syncwarp();
      if (mine) {
        uint4* dst = reinterpret_cast<uint4*>(out + ((size_t)mi * count + (size_t)tile * P + grp) * N + t * PER);
        const uint4* src = reinterpret_cast<const uint4*>(slot + t * PER);
#pragma unroll
        for (int k = 0; k < PER / 4; ++k) dst[k] = src[k];
      }
      __syncwarp();  // the slot is read out before the next prime's residues
    }
    __syncthreads();  // the z stage is read out before its refill
  }
  if (tid == 0 && failed_at >= 0) {
    record_error(p.np.err, LC_DEVERR_TIMEOUT);
    // loads still in flight must land before the CTA exits (bounded waits;
    // the timed-out stage is not waited for again)
    for (int k = 1; k < STAGES; ++k) {
      const unsigned long long tk = tile + (unsigned long long)k * stride;
      const bool issued = (k < STAGES - 1) || refilled;
      if (tk >= ntiles || !issued) continue;
      const int sk = (failed_at + k) % STAGES;
      mbar_wait(&bar[sk], (parity >> sk) & 1u);
    }
  }
}

template <class A>
static int launch_crt_ntt(const lc_ntt_plan* plan, const uint64_t* z, size_t count, uint32_t* out,
                          cudaStream_t st) {
  constexpr int NT = 128, STAGES = 3;
  using C = CrtNttCfg<A, 6, 3, NT, STAGES>;
  auto kern = crt_ntt_kernel<A, 6, 3, NT, STAGES>;
  const size_t smem = C::smem(plan->num_moduli);
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = smem_attr_once(attr_done, kern, C::smem(kMaxModuli));
  if (e != cudaSuccess) return map_cuda(e);
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
  if (e != cudaSuccess) return map_cuda(e);
  per_sm = std::max(per_sm, 1);
  CrtNttParams p{};
  p.np.out = out;
  p.np.count = count;
  p.np.tw = plan->d_tw_fwd;
  p.np.tw_stride = plan->tw_fwd_entries;
  p.np.num_moduli = plan->num_moduli;
  p.np.err = plan->d_err;
  for (uint32_t i = 0; i < plan->num_moduli; ++i) {
    p.np.q[i] = plan->q[i];
    p.np.qinv[i] = plan->qinv[i];
    p.mu[i] = ~0ull / plan->q[i];
  }
  p.z = z;
  const unsigned long long ntiles = (count + C::P - 1) / C::P;
  const unsigned long long gx =
      std::max<unsigned long long>(1, std::min<unsigned long long>(ntiles, (unsigned long long)device_sm_count() * per_sm));
  kern<<<(unsigned)gx, NT, smem, st>>>(p);
  return map_cuda(cudaGetLastError());
}

// Residues of z under the plan's moduli, forward-transformed, in one launch:
// out[mod][count][64] = NTT(z mod q_mod).  d = 64 u32 plans only
// (LC_ERR_UNSUPPORTED otherwise: the caller runs crt_residues + the NTT).
int crt_ntt_forward(const lc_ntt_plan* plan, const uint64_t* z, size_t count, uint32_t* out, cudaStream_t st) {
  if (count == 0) return LC_OK;
  if (plan->log_n != 6 || count > ((size_t)1 << 29)) return LC_ERR_UNSUPPORTED;
  if (((uintptr_t)z & 15) || ((uintptr_t)out & 15)) return LC_ERR_UNSUPPORTED;
  if (plan->kind == PlanKind::U32Lazy) return launch_crt_ntt<ShoupLazy>(plan, z, count, out, st);
  if (plan->kind == PlanKind::U32Mont) return launch_crt_ntt<MontCanon>(plan, z, count, out, st);
  return LC_ERR_UNSUPPORTED;
}

}  // namespace lc

struct lc_fold_pipeline {
  lc_ajtai_key* key = nullptr;
  const lc_ntt_plan* crt = nullptr;
  uint32_t m = 0, kappa = 0;
  uint64_t* z = nullptr;       // [m][64] residues
  uint8_t* digits = nullptr;   // [8][m][64]
  uint64_t* commits = nullptr; // [8][kappa][64]
  uint32_t* crt_out = nullptr; // [num_moduli][m][64]
  int use_graph = 0;
  bool warmed = false;
  cudaStream_t cap = nullptr;
  cudaStream_t side = nullptr;    // the CRT branch
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t scratch_sig = 0;  // key scratch the graph was captured with
};

namespace lc {

static int fold_stages(lc_fold_pipeline* f, cudaStream_t st) {
  const size_t coeffs = (size_t)f->m * 64;
  // fork: the CRT branch starts after the caller's earlier work on st
  cudaError_t e = cudaEventRecord(f->ev_fork, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(f->side, f->ev_fork, 0);
  if (e != cudaSuccess) return map_cuda(e);
  int rc_crt = crt_ntt_forward(f->crt, f->z, f->m, f->crt_out, f->side);
  if (rc_crt == LC_ERR_UNSUPPORTED) {
    rc_crt = crt_residues(f->crt, f->z, coeffs, f->crt_out, f->side);
    if (!rc_crt) rc_crt = lc_ntt_forward(f->crt, f->crt_out, f->crt_out, f->m, f->side);
  }
  int rc = lc_decomp_b(f->z, coeffs, 8, f->digits, st);
  if (!rc) rc = lc_ajtai_commit_u8(f->key, f->digits, 8, f->commits, st);
  // join: st continues after both branches (also closes the side stream's
  // part of a capture)
  e = cudaEventRecord(f->ev_join, f->side);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, f->ev_join, 0);
  if (e != cudaSuccess) return map_cuda(e);
  return rc ? rc : rc_crt;
}

}  // namespace lc

extern "C" {

LC_API int lc_fold_pipeline_create(lc_ajtai_key* key, const lc_ntt_plan* crt_plan, int use_graph,
                                   lc_fold_pipeline** out) {
  using namespace lc;
  if (!key || !crt_plan || !out) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  uint32_t k = 0, m = 0, log_n = 0, ln = 0, nm = 0, eb = 0;
  lc_ajtai_key_info(key, &k, &m, &log_n);
  lc_ntt_plan_info(crt_plan, &ln, &nm, &eb);
  if (log_n != 6 || ln != 6 || eb != 4) return LC_ERR_UNSUPPORTED;
  if ((size_t)m > (1u << 24)) return LC_ERR_UNSUPPORTED;
  lc_fold_pipeline* f = new (std::nothrow) lc_fold_pipeline();
  if (!f) return LC_ERR_OUT_OF_MEMORY;
  f->key = key;
  f->crt = crt_plan;
  f->m = m;
  f->kappa = k;
  f->use_graph = use_graph;
  const size_t coeffs = (size_t)m * 64;
  if (cudaMalloc(&f->z, coeffs * 8) != cudaSuccess || cudaMalloc(&f->digits, coeffs * 8) != cudaSuccess ||
      cudaMalloc(&f->commits, (size_t)8 * k * 64 * 8) != cudaSuccess ||
      cudaMalloc(&f->crt_out, coeffs * nm * 4) != cudaSuccess ||
      cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&f->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&f->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    lc_fold_pipeline_destroy(f);
    return LC_ERR_OUT_OF_MEMORY;
  }
  *out = f;
  return LC_OK;
}

LC_API int lc_fold_pipeline_buffers(lc_fold_pipeline* f, uint64_t** z, uint8_t** digits, uint64_t** commits,
                                    uint32_t** crt_ntt) {
  if (!f) return LC_ERR_INVALID_ARGUMENT;
  if (z) *z = f->z;
  if (digits) *digits = f->digits;
  if (commits) *commits = f->commits;
  if (crt_ntt) *crt_ntt = f->crt_out;
  return LC_OK;
}

LC_API int lc_fold_pipeline_run(lc_fold_pipeline* f, lc_stream stream) {
  using namespace lc;
  if (!f) return LC_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (!f->use_graph || !f->warmed) {
    // eager: the first run also sizes every scratch buffer the graph will use
    const int rc = fold_stages(f, st);
    if (!rc) f->warmed = true;
    return rc;
  }
  if (f->exec && commit_scratch_signature(f->key) != f->scratch_sig) {
    // the key's scratch moved (another commit grew it): capture again
    cudaGraphExecDestroy(f->exec);
    cudaGraphDestroy(f->graph);
    f->exec = nullptr;
    f->graph = nullptr;
    const int rc = fold_stages(f, st);  // eager run re-sizes the scratch for this step
    if (rc) return rc;
  }
  if (!f->exec) {
    if (!f->cap && cudaStreamCreateWithFlags(&f->cap, cudaStreamNonBlocking) != cudaSuccess)
      return map_cuda(cudaGetLastError());
    // the captured stream starts after the caller's earlier work
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return map_cuda(cudaGetLastError());
    cudaEventRecord(ev, st);
    cudaStreamWaitEvent(f->cap, ev, 0);
    cudaEventDestroy(ev);
    cudaError_t e = cudaStreamBeginCapture(f->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return map_cuda(e);
    const int rc = fold_stages(f, f->cap);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(f->cap, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc;
    }
    if (e != cudaSuccess) return map_cuda(e);
    e = cudaGraphInstantiate(&f->exec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      f->exec = nullptr;
      return map_cuda(e);
    }
    f->graph = g;
    f->scratch_sig = commit_scratch_signature(f->key);
  }
  return map_cuda(cudaGraphLaunch(f->exec, st));
}

LC_API int lc_fold_pipeline_check(lc_fold_pipeline* f, lc_stream stream) {
  if (!f) return LC_ERR_INVALID_ARGUMENT;
  int rc = lc_ajtai_key_check(f->key, stream);
  if (!rc) rc = lc_ntt_plan_check(const_cast<lc_ntt_plan*>(f->crt), stream);
  return rc;
}

LC_API void lc_fold_pipeline_destroy(lc_fold_pipeline* f) {
  if (!f) return;
  if (f->exec) cudaGraphExecDestroy(f->exec);
  if (f->graph) cudaGraphDestroy(f->graph);
  if (f->cap) cudaStreamDestroy(f->cap);
  if (f->side) cudaStreamDestroy(f->side);
  if (f->ev_fork) cudaEventDestroy(f->ev_fork);
  if (f->ev_join) cudaEventDestroy(f->ev_join);
  for (void* p : {(void*)f->z, (void*)f->digits, (void*)f->commits, (void*)f->crt_out})
    if (p) cudaFree(p);
  delete f;
}

LC_API int lc_crt_residues(const lc_ntt_plan* plan, const uint64_t* z, size_t count, uint32_t* out,
                           lc_stream stream) {
  using namespace lc;
  if (!plan || (count && (!z || !out))) return LC_ERR_INVALID_ARGUMENT;
  uint32_t ln = 0, nm = 0, eb = 0;
  lc_ntt_plan_info(plan, &ln, &nm, &eb);
  if (eb != 4) return LC_ERR_UNSUPPORTED;
  if (count == 0) return LC_OK;
  return crt_residues(plan, z, count, out, (cudaStream_t)stream);
}

}  // extern "C"
