// internal.h -- host-side structures shared by the lattice_cuda translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/lattice_cuda.h"

namespace lc {

enum class PlanKind : int { U32Lazy = 0, U32Mont = 1, Goldilocks = 2 };

// Two device staging buffers and two streams for the host-buffer entry
// points; chunk k uses buffer/stream k&1 so copies of one chunk overlap the
// transform of the other.
struct HostPipeline {
  // kSlots chunks in flight: while one slot's results go back over the link,
  // the next slots' inputs come in
  static constexpr int kSlots = 3;
  void* buf[kSlots] = {};
  size_t bytes = 0;
  cudaStream_t stream[kSlots] = {};

  int ensure(size_t need) {
    // any stream missing (first call, or an earlier creation that failed)
    for (int i = 0; i < kSlots; ++i) {
      if (!stream[i] && cudaStreamCreateWithFlags(&stream[i], cudaStreamNonBlocking) != cudaSuccess) {
        stream[i] = nullptr;
        cudaGetLastError();
        return LC_ERR_CUDA;
      }
    }
    if (need <= bytes) return LC_OK;
    for (int i = 0; i < kSlots; ++i) {
      if (buf[i]) cudaFree(buf[i]);
      buf[i] = nullptr;
    }
    bytes = 0;
    for (int i = 0; i < kSlots; ++i) {
      if (cudaMalloc(&buf[i], need) != cudaSuccess) {
        cudaGetLastError();
        return LC_ERR_OUT_OF_MEMORY;
      }
    }
    bytes = need;
    return LC_OK;
  }
  // first error of the slots' streams (all of them are waited for)
  cudaError_t sync() {
    cudaError_t first = cudaSuccess;
    for (int i = 0; i < kSlots; ++i) {
      if (!stream[i]) continue;
      const cudaError_t e = cudaStreamSynchronize(stream[i]);
      if (first == cudaSuccess) first = e;
    }
    return first;
  }
  void release() {
    for (int i = 0; i < kSlots; ++i) {
      if (buf[i]) cudaFree(buf[i]);
      if (stream[i]) cudaStreamDestroy(stream[i]);
      buf[i] = nullptr;
      stream[i] = nullptr;
    }
    bytes = 0;
  }
};

}  // namespace lc

struct lc_ntt_plan {
  lc::PlanKind kind = lc::PlanKind::U32Lazy;
  uint32_t log_n = 0;
  uint32_t num_moduli = 0;
  uint32_t q[8] = {};
  uint32_t qinv[8] = {};
  uint32_t two_adicity[8] = {};
  uint32_t generator[8] = {};
  // one device block: the forward table, the inverse table, the error word
  void* d_block = nullptr;
  void* d_tw_fwd = nullptr;
  void* d_tw_inv = nullptr;
  uint32_t tw_fwd_entries = 0;
  uint32_t tw_inv_entries = 0;
  uint32_t tw_bytes = 0;
  uint32_t* d_err = nullptr;
  int variant = 0;
  lc::HostPipeline staging;
  uint32_t* d_pow = nullptr;  // partial transforms: per modulus psi^i (n) then omega^k (n/2), built on first use
};

struct lc_tc_tables;  // INT8 tensor-core commit tables (tc_commit.cu)

// Ajtai key: cached NTT(A) transposed to [slot t][ring element j][row i padded
// to 16], plus the scratch a commit grows on demand (commit.cu).
struct lc_ajtai_key {
  lc_ntt_plan* plan = nullptr;  // owned copy of the ring's plan
  uint32_t k = 0, m = 0, n = 0, log_n = 0;
  bool wide = false;           // Goldilocks (u64) or u32
  void* d_ahat_t = nullptr;    // [n][a_m][16]
  uint32_t a_m = 0;            // ring elements per NTT slot of d_ahat_t (m, or the parent's m for a view)
  bool owns_ahat = true;       // false for a view (lc_ajtai_key_view)
  // scratch, grown on demand
  void* d_what_t = nullptr;
  size_t what_bytes = 0;
  void* d_partial = nullptr;
  size_t partial_bytes = 0;
  void* d_chat = nullptr;
  size_t chat_bytes = 0;
  void* d_wtmp = nullptr;  // generic witness path: converted + transformed witnesses
  size_t wtmp_bytes = 0;
  void* d_fused = nullptr;  // single-launch commit: ticket (16 B), then 128-bit accumulators
  size_t fused_bytes = 0;
  unsigned int* d_grid = nullptr;  // grid-barrier counter of the one-launch products + inverse NTT
  int fused = 1;            // one-launch forms: 0 never, 1 where faster, 2 every form (lc_ajtai_key_set_fused)
  bool last_fused = false;  // the last commit on this key ran as one launch
  int slot_products = LC_PRODUCTS_TENSOR;  // lc_ajtai_key_set_slot_products
  void* d_in = nullptr;  // host-API staging
  size_t in_bytes = 0;
  void* d_out = nullptr;
  size_t out_bytes = 0;
  void* h_stage_in = nullptr;  // pinned staging of small pageable host buffers (host API)
  size_t h_stage_in_bytes = 0;
  void* h_stage_out = nullptr;
  size_t h_stage_out_bytes = 0;
  cudaStream_t host_stream = nullptr;
  uint32_t* h_flags = nullptr;  // pinned: the key's and the plan's error words (host API)
  uint32_t* d_err = nullptr;
  lc_tc_tables* tc = nullptr;  // tensor-core engine tables (LC_KEY_TENSOR_I8)
  int engine = LC_ENGINE_NTT;
};

namespace lc {
// Sets a kernel's dynamic shared-memory limit once per device: `done` keeps
// one bit per device (the attribute is per device; devices past 63 set it on
// every call).
template <class K>
inline cudaError_t smem_attr_once(std::atomic<uint64_t>& done, K kern, size_t bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cudaGetLastError();
  const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t)1 << dev : 0;
  if (bit && (done.load(std::memory_order_relaxed) & bit)) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_relaxed);
  return e;
}

int device_sm_count();
// Ajtai key creation (commit.cu): the argument check, and the creation from a
// device buffer of the coefficient-form matrix that the call takes over.
int key_create_check(const lc_ntt_plan* plan, uint32_t k, uint32_t m, uint32_t flags);
int key_create_from(const lc_ntt_plan* plan, uint32_t k, uint32_t m, void* tmp, uint32_t flags,
                    lc_ajtai_key** out);
int map_cuda(cudaError_t e);
int run_ntt(const lc_ntt_plan* plan, const void* in, void* out, size_t count, bool inverse,
            cudaStream_t s);

// Goldilocks, d = 64: build the rotation-limb tables from the coefficient
// matrix [k][m][64] on the device (default stream); commit byte-digit
// witnesses [batch][m][64] -> residues [batch][k][64] on `st`.
int tc_tables_create(const uint64_t* matrix_dev, uint32_t k, uint32_t m, lc_tc_tables** out);
void tc_tables_destroy(lc_tc_tables* t);
size_t tc_tables_bytes(const lc_tc_tables* t);
uint64_t commit_scratch_signature(const lc_ajtai_key* key);
int crt_residues(const lc_ntt_plan* plan, const uint64_t* z, size_t count, uint32_t* out, cudaStream_t st);
// w: int8 digits (s8 = true) or unsigned byte digits (s8 = false)
int tc_commit(lc_tc_tables* t, const void* w, bool s8, size_t batch, uint64_t* out, uint32_t* err,
              cudaStream_t st);
// Goldilocks d = 64 witness NTT of byte digits on the INT8 tensor cores:
// What_T[64][m][b_pad] from w[batch][m][64]; LC_ERR_UNSUPPORTED for shapes it
// does not take (the caller then runs the CUDA-core transform).  The matrix
// image is made by tc_ntt_prepare (once per device, outside stream capture).
int tc_ntt_prepare();
int tc_witness_ntt(const void* w, bool s8, size_t batch, uint32_t m, uint32_t b_pad, uint64_t* what_t,
                   uint32_t* err, cudaStream_t st);
// Per-slot products Chat[b][i][t] = sum_j Ahat_T[t][j][i] What_T[t][j][b]
// (mod q; Goldilocks for elem_bytes 8, the u32 modulus q for elem_bytes 4) as
// exact byte-limb GEMMs on the INT8 tensor cores (n slots, m ring elements,
// a_m the key's row stride); scratch grown in *part.  LC_ERR_UNSUPPORTED
// unless a witness row of What_T (elem_bytes * b_pad bytes) is 32, 64, 128,
// 256 or a multiple of 512 bytes.
int tc_slot_products(const void* ahat_t, uint32_t a_m, const void* what_t, uint32_t elem_bytes, uint32_t q,
                     uint32_t m, uint32_t n, uint32_t kappa, size_t batch, uint32_t b_pad, void** part,
                     size_t* part_bytes, void* chat, uint32_t* err, cudaStream_t st);
}  // namespace lc
