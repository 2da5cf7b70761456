// internal.h -- host-side structures shared by the lattice_cuda translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lattice_cuda.h"

namespace lc {

enum class PlanKind : int { U32Lazy = 0, U32Mont = 1, Goldilocks = 2 };

// Two device staging buffers and two streams for the host-buffer entry
// points; chunk k uses buffer/stream k&1 so copies of one chunk overlap the
// transform of the other.
struct HostPipeline {
  void* buf[2] = {nullptr, nullptr};
  size_t bytes = 0;
  cudaStream_t stream[2] = {nullptr, nullptr};

  int ensure(size_t need) {
    if (!stream[0]) {
      if (cudaStreamCreateWithFlags(&stream[0], cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&stream[1], cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return LC_ERR_CUDA;
      }
    }
    if (need <= bytes) return LC_OK;
    for (int i = 0; i < 2; ++i) {
      if (buf[i]) cudaFree(buf[i]);
      buf[i] = nullptr;
    }
    bytes = 0;
    for (int i = 0; i < 2; ++i) {
      if (cudaMalloc(&buf[i], need) != cudaSuccess) {
        cudaGetLastError();
        return LC_ERR_OUT_OF_MEMORY;
      }
    }
    bytes = need;
    return LC_OK;
  }
  void release() {
    for (int i = 0; i < 2; ++i) {
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
  void* d_tw_fwd = nullptr;
  void* d_tw_inv = nullptr;
  uint32_t tw_fwd_entries = 0;
  uint32_t tw_inv_entries = 0;
  uint32_t tw_bytes = 0;
  uint32_t* d_err = nullptr;
  int variant = 0;
  lc::HostPipeline staging;
};

namespace lc {
int device_sm_count();
int map_cuda(cudaError_t e);
int run_ntt(const lc_ntt_plan* plan, const void* in, void* out, size_t count, bool inverse,
            cudaStream_t s);
}  // namespace lc
