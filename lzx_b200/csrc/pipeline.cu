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
  int rc_crt = crt_residues(f->crt, f->z, coeffs, f->crt_out, f->side);
  if (!rc_crt) rc_crt = lc_ntt_forward(f->crt, f->crt_out, f->crt_out, f->m, f->side);
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
