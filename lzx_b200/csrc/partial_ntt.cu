// partial_ntt.cu -- the incomplete NTT of lattice-ring and its completion.
//
// NttTables::forward_partial (lattice-ring/src/ntt.rs:252-286): multiply
// coefficient i by psi^i, bit-reverse, then run only the first `levels`
// Cooley-Tukey levels (len = 2 .. 2^levels, twiddle omega^(n/len * j)).
// NttTables::complete_partial (ntt.rs:288-316) runs the levels after
// `already`.  The intermediate order is the reference's own (a mixed
// representation other code may read), so these follow its loop structure
// exactly rather than the merged-psi kernels: one CTA per polynomial, the
// polynomial in shared memory, bit reversal folded into the first store,
// canonical arithmetic mod q (Barrett with floor(2^64/q), as
// Modulus32::reduce_u64).  The composition of the two is forward_fast.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace lc {

struct PartialParams {
  const uint32_t* in;
  uint32_t* out;
  const uint32_t* pow;  // [modulus][psi^i (n), omega^k (n/2)]
  size_t count;
  uint32_t log_n, level_from, level_to;  // run levels level_from .. level_to (len = 2^level)
  uint32_t prescale;                     // forward_partial: psi scale and bit reversal first
  uint32_t q[8];
  uint64_t mu[8];
};

LC_D uint32_t pmul(uint32_t a, uint32_t b, uint32_t q, uint64_t mu) {
  const uint64_t x = (uint64_t)a * b;
  uint64_t r = x - __umul64hi(x, mu) * q;
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return (uint32_t)r;
}
LC_D uint32_t padd(uint32_t a, uint32_t b, uint32_t q) {
  const uint64_t s = (uint64_t)a + b;
  return (uint32_t)(s >= q ? s - q : s);
}
LC_D uint32_t psub(uint32_t a, uint32_t b, uint32_t q) { return a >= b ? a - b : (uint32_t)((uint64_t)a + q - b); }

__global__ void __launch_bounds__(128) ntt_partial_kernel(const __grid_constant__ PartialParams p) {
  extern __shared__ uint32_t s[];
  const uint32_t n = 1u << p.log_n, mi = blockIdx.y;
  const uint32_t q = p.q[mi];
  const uint64_t mu = p.mu[mi];
  const uint32_t* psi = p.pow + (size_t)mi * (n + n / 2);
  const uint32_t* omega = psi + n;
  for (size_t poly = blockIdx.x; poly < p.count; poly += gridDim.x) {
    const size_t base = ((size_t)mi * p.count + poly) * n;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t x = p.in[base + i];
      if (p.prescale)
        s[__brev(i) >> (32 - p.log_n)] = pmul(x, psi[i], q, mu);
      else
        s[i] = x;
    }
    __syncthreads();
    for (uint32_t lv = p.level_from; lv <= p.level_to; ++lv) {
      const uint32_t half = 1u << (lv - 1), stride = n >> lv;
      for (uint32_t bf = threadIdx.x; bf < n / 2; bf += blockDim.x) {
        const uint32_t j = bf & (half - 1), start = (bf >> (lv - 1)) << lv;
        const uint32_t u = s[start + j];
        const uint32_t v = pmul(s[start + j + half], omega[stride * j], q, mu);
        s[start + j] = padd(u, v, q);
        s[start + j + half] = psub(u, v, q);
      }
      __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) p.out[base + i] = s[i];
    __syncthreads();
  }
}

static uint64_t pw(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  while (e) {
    if (e & 1) r = (uint64_t)((unsigned __int128)r * a % q);
    a = (uint64_t)((unsigned __int128)a * a % q);
    e >>= 1;
  }
  return r;
}

static std::mutex g_pow_mu;

// psi^i and omega^k = psi^(2k) per modulus, psi = g^((q-1) >> (log_n+1))
// (Modulus32::root_of_unity_order_2n, modulus.rs:149-161).
static int partial_tables(lc_ntt_plan* plan) {
  std::lock_guard<std::mutex> lk(g_pow_mu);
  if (plan->d_pow) return LC_OK;
  const uint32_t n = 1u << plan->log_n;
  std::vector<uint32_t> t((size_t)plan->num_moduli * (n + n / 2));
  for (uint32_t m = 0; m < plan->num_moduli; ++m) {
    const uint64_t q = plan->q[m];
    const uint64_t psi = pw(plan->generator[m], (q - 1) >> (plan->log_n + 1), q);
    uint32_t* row = t.data() + (size_t)m * (n + n / 2);
    uint64_t x = 1;
    for (uint32_t i = 0; i < n; ++i, x = x * psi % q) row[i] = (uint32_t)x;
    const uint64_t omega = psi * psi % q;
    x = 1;
    for (uint32_t k = 0; k < n / 2; ++k, x = x * omega % q) row[n + k] = (uint32_t)x;
  }
  void* d = nullptr;
  if (cudaMalloc(&d, t.size() * 4) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  if (cudaMemcpy(d, t.data(), t.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return map_cuda(cudaGetLastError());
  }
  plan->d_pow = static_cast<uint32_t*>(d);
  return LC_OK;
}

static int run_partial(lc_ntt_plan* plan, const void* in, void* out, size_t count, uint32_t from, uint32_t to,
                       bool prescale, cudaStream_t st) {
  if (!plan || (count && (!in || !out))) return LC_ERR_INVALID_ARGUMENT;
  if (plan->kind == PlanKind::Goldilocks) return LC_ERR_UNSUPPORTED;
  if (count == 0) return LC_OK;
  if (count > ((size_t)1 << 29)) return LC_ERR_INVALID_ARGUMENT;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  const int rc = partial_tables(plan);
  if (rc) return rc;
  PartialParams p{};
  p.in = static_cast<const uint32_t*>(in);
  p.out = static_cast<uint32_t*>(out);
  p.pow = plan->d_pow;
  p.count = count;
  p.log_n = plan->log_n;
  p.level_from = from;
  p.level_to = to;
  p.prescale = prescale;
  for (uint32_t m = 0; m < plan->num_moduli; ++m) {
    p.q[m] = plan->q[m];
    p.mu[m] = ~0ull / plan->q[m];
  }
  const uint32_t n = 1u << plan->log_n;
  const unsigned gx = (unsigned)std::min<size_t>(count, (size_t)device_sm_count() * 32);
  ntt_partial_kernel<<<dim3(gx, plan->num_moduli), 128, n * 4, st>>>(p);
  return map_cuda(cudaGetLastError());
}

}  // namespace lc

extern "C" {

LC_API int lc_ntt_forward_partial(lc_ntt_plan* plan, const void* in, void* out, size_t count, uint32_t levels,
                                  lc_stream stream) {
  if (!plan) return LC_ERR_INVALID_ARGUMENT;
  if (levels > plan->log_n) return LC_ERR_LENGTH_MISMATCH;  // ntt.rs:258-260
  return lc::run_partial(plan, in, out, count, 1, levels, true, (cudaStream_t)stream);
}

LC_API int lc_ntt_complete_partial(lc_ntt_plan* plan, const void* in, void* out, size_t count, uint32_t already,
                                   lc_stream stream) {
  if (!plan) return LC_ERR_INVALID_ARGUMENT;
  if (already > plan->log_n) return LC_ERR_LENGTH_MISMATCH;  // ntt.rs:292-294
  return lc::run_partial(plan, in, out, count, already + 1, plan->log_n, false, (cudaStream_t)stream);
}

}  // extern "C"
