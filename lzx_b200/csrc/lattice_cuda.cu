// lattice_cuda.cu -- host side of the lattice_cuda C ABI: NTT plans, twiddle
// tables, kernel dispatch, host-buffer pipelines.
//
// Plan construction restates NttTables::new (lattice-ring/src/ntt.rs:46-106):
// psi = g^((q-1) >> (log_n+1)), psi^-1, n^-1, with the twiddles reordered for
// the merged-psi kernels (see ntt_kernels.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "internal.h"
#include "ntt_kernels.cuh"

using namespace lc;

namespace lc {

// Largest batch (polynomials per modulus) of one call; keeps the kernels' tile
// counters in 32 bits.
constexpr size_t kMaxBatch = (size_t)1 << 29;

// --------------------------------------------------------------- host modular arithmetic

typedef unsigned __int128 u128;

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  while (e) {
    if (e & 1) r = mulmod(r, a, q);
    a = mulmod(a, a, q);
    e >>= 1;
  }
  return r;
}

static uint32_t brv(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// ---------------------------------------------------------------- geometry choice

// Values per thread (log2) used for each ring degree; the dispatch below and
// the table generator must agree.  0 = small-ring kernel (one thread per
// polynomial).
static int choose_log_v(PlanKind kind, int log_n) {
  const bool wide = (kind == PlanKind::Goldilocks);
  if (log_n <= (wide ? 4 : 5)) return 0;
  switch (log_n) {
    case 5: return 3;
    case 6: return 3;
    case 7: return 4;
    case 8: return 4;
    case 9: return 5;
    case 10: return 5;
    case 11: return 6;
    default: return -1;
  }
}

// Raw twiddle residues in the order the kernels read them.
static void make_tables(int log_n, int log_v, uint64_t q, uint64_t psi, std::vector<uint64_t>& fwd,
                        std::vector<uint64_t>& inv) {
  const uint32_t n = 1u << log_n;
  const uint64_t psi_inv = powmod(psi, q - 2, q);
  const uint64_t ninv = powmod(n, q - 2, q);
  std::vector<uint64_t> Psi(n), PsiI(n);
  for (uint32_t k = 0; k < n; ++k) {
    Psi[k] = powmod(psi, brv(k, log_n), q);
    PsiI[k] = powmod(psi_inv, brv(k, log_n), q);
  }
  auto special = [&](uint32_t k) -> uint64_t {
    if (k == 0) return ninv;
    if (k == 1) return mulmod(PsiI[1], ninv, q);
    return PsiI[k];
  };
  fwd.clear();
  inv.clear();
  if (log_v == 0) {
    fwd = Psi;
    for (uint32_t k = 0; k < n; ++k) inv.push_back(special(k));
    return;
  }
  const int lo0 = log_n - log_v;
  const uint32_t T = 1u << lo0;
  for (uint32_t k = 0; k < (1u << log_v); ++k) fwd.push_back(Psi[k]);
  for (int b = lo0 - 1; b >= 0; --b)
    for (uint32_t rr = 0; rr < (1u << (log_v - b - 1)); ++rr)
      for (uint32_t t = 0; t < T; ++t)
        fwd.push_back(Psi[(1u << (log_n - 1 - b)) + (t << (log_v - b - 1)) + rr]);
  for (int b = 0; b < log_v; ++b)
    for (uint32_t rr = 0; rr < (1u << (log_v - b - 1)); ++rr)
      for (uint32_t t = 0; t < T; ++t)
        inv.push_back(PsiI[(1u << (log_n - 1 - b)) + (t << (log_v - b - 1)) + rr]);
  for (uint32_t k = 0; k < T; ++k) inv.push_back(special(k));
}

// ---------------------------------------------------------------- device state

static int g_num_sms = -1;
static std::mutex g_mu;

int device_sm_count() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_num_sms < 0) {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    g_num_sms = prop.major == 10 ? prop.multiProcessorCount : 0;
  }
  return g_num_sms;
}

int map_cuda(cudaError_t e) {
  if (e == cudaSuccess) return LC_OK;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return LC_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LC_ERR_NO_DEVICE;
  return LC_ERR_CUDA;
}

// ---------------------------------------------------------------- launch

template <class A, int LOG_N, int LOG_V, int NT, int IT, int STAGES, bool INV, int OPT = 0>
static int launch_tile_cfg(const NttParams& p, cudaStream_t s) {
  using C = NttKernelCfg<A, LOG_N, LOG_V, NT, IT, STAGES, INV>;
  auto kern = ntt_tile_kernel<A, LOG_N, LOG_V, NT, IT, STAGES, INV, OPT>;
  constexpr size_t smem = C::SMEM;
  static std::atomic<uint64_t> attr_done{0};
  {
    const cudaError_t e = smem_attr_once(attr_done, kern, smem);
    if (e != cudaSuccess) return e == cudaErrorInvalidValue ? LC_ERR_UNSUPPORTED : map_cuda(e);
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
  if (e != cudaSuccess) return map_cuda(e);
  per_sm = std::max(per_sm, 1);
  const unsigned long long ntiles = (p.count + C::P - 1) / C::P;
  const int sms = device_sm_count();
  unsigned long long gx = std::min<unsigned long long>(ntiles, (unsigned long long)sms * per_sm);
  gx = std::max<unsigned long long>(gx, 1);
  kern<<<dim3((unsigned)gx, p.num_moduli), NT, smem, s>>>(p);
  return map_cuda(cudaGetLastError());
}

template <class A, int LOG_N, int LOG_V, int WARPS, int IT, int STAGES, bool INV>
static int launch_warp_cfg(const NttParams& p, cudaStream_t s) {
  using C = NttWarpCfg<A, LOG_N, LOG_V, WARPS, IT, STAGES, INV>;
  auto kern = ntt_warp_kernel<A, LOG_N, LOG_V, WARPS, IT, STAGES, INV>;
  constexpr size_t smem = C::SMEM;
  static std::atomic<uint64_t> attr_done{0};
  {
    const cudaError_t e = smem_attr_once(attr_done, kern, smem);
    if (e != cudaSuccess) return e == cudaErrorInvalidValue ? LC_ERR_UNSUPPORTED : map_cuda(e);
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, smem);
  if (e != cudaSuccess) return map_cuda(e);
  per_sm = std::max(per_sm, 1);
  const unsigned long long wtiles = (p.count + C::P - 1) / C::P;
  const unsigned long long need = (wtiles + WARPS - 1) / WARPS;
  const int sms = device_sm_count();
  unsigned long long gx = std::min<unsigned long long>(need, (unsigned long long)sms * per_sm);
  gx = std::max<unsigned long long>(gx, 1);
  kern<<<dim3((unsigned)gx, p.num_moduli), C::NT, smem, s>>>(p);
  return map_cuda(cudaGetLastError());
}

// Tile size: about 36 KB of polynomials per stage by default.
template <class A, int LOG_N, int LOG_V, int NT>
constexpr int default_it() {
  using G = Geo<LOG_N, LOG_V>;
  using SL = Slots<A, LOG_N, LOG_V>;
  constexpr size_t per_it = (size_t)(NT / G::T) * SL::S * sizeof(typename A::T);
  return per_it >= 4 * 1024 ? 1 : (int)((4 * 1024) / per_it);
}

// Ring degrees whose tile kernels are instantiated in several shapes for the
// tuner: the CRT batch (u32, d = 256) and the commit witnesses (Goldilocks, d = 64).
template <class A, int LOG_N>
constexpr bool tunable() {
  return (LOG_N == 8 && std::is_same<A, ShoupLazy>::value) ||
         (LOG_N == 6 && std::is_same<A, Goldilocks>::value);
}

template <class A, int LOG_N, int LOG_V, bool INV>
static int launch_tile(const NttParams& p, int variant, cudaStream_t s) {
  if constexpr (!tunable<A, LOG_N>()) {
    (void)variant;
    return launch_tile_cfg<A, LOG_N, LOG_V, 128, default_it<A, LOG_N, LOG_V, 128>(), 2, INV>(p, s);
  } else {
  // variant 0 is the default; 1..6 are alternatives kept for the tuner
  constexpr int IT1 = default_it<A, LOG_N, LOG_V, 128>();
  switch (variant) {
    case 1: return launch_tile_cfg<A, LOG_N, LOG_V, 128, IT1, 3, INV>(p, s);
    case 2: return launch_tile_cfg<A, LOG_N, LOG_V, 256, default_it<A, LOG_N, LOG_V, 256>(), 2, INV>(p, s);
    case 3: return launch_warp_cfg<A, LOG_N, LOG_V, 4, 1, 2, INV>(p, s);
    case 4: return launch_warp_cfg<A, LOG_N, LOG_V, 4, 1, 3, INV>(p, s);
    case 5: return launch_tile_cfg<A, LOG_N, LOG_V, 128, IT1, 2, INV, kOptSwz>(p, s);
    case 6: return launch_tile_cfg<A, LOG_N, LOG_V, 128, IT1, 2, INV, kOptSwz | kOptRegTw>(p, s);
    default: return launch_tile_cfg<A, LOG_N, LOG_V, 128, IT1, 2, INV>(p, s);
  }
  }
}

template <class A, int LOG_N, bool INV>
static int launch_small(const NttParams& p, cudaStream_t s) {
  const int sms = device_sm_count();
  unsigned long long blocks = (p.count + 127) / 128;
  blocks = std::min<unsigned long long>(blocks, (unsigned long long)sms * 16);
  blocks = std::max<unsigned long long>(blocks, 1);
  ntt_small_kernel<A, LOG_N, INV><<<dim3((unsigned)blocks, p.num_moduli), 128, 0, s>>>(p);
  return map_cuda(cudaGetLastError());
}

template <class A, bool INV>
static int dispatch(int log_n, const NttParams& p, int variant, cudaStream_t s) {
  constexpr bool wide = sizeof(typename A::T) == 8;
  switch (log_n) {
    case 1: return launch_small<A, 1, INV>(p, s);
    case 2: return launch_small<A, 2, INV>(p, s);
    case 3: return launch_small<A, 3, INV>(p, s);
    case 4: return launch_small<A, 4, INV>(p, s);
    case 5:
      if constexpr (wide) return launch_tile<A, 5, 3, INV>(p, variant, s);
      else return launch_small<A, 5, INV>(p, s);
    case 6: return launch_tile<A, 6, 3, INV>(p, variant, s);
    case 7: return launch_tile<A, 7, 4, INV>(p, variant, s);
    case 8: return launch_tile<A, 8, 4, INV>(p, variant, s);
    case 9: return launch_tile<A, 9, 5, INV>(p, variant, s);
    case 10: return launch_tile<A, 10, 5, INV>(p, variant, s);
    case 11:
      if constexpr (wide) return LC_ERR_UNSUPPORTED;
      else return launch_tile<A, 11, 6, INV>(p, variant, s);
    default: return LC_ERR_UNSUPPORTED;
  }
}

// Transforms of `count` polynomials under each of the plan's moduli
// m0 .. m0 + nm - 1, laid out [modulus][count][n] at `in` / `out`.
static int run_ntt_moduli(const lc_ntt_plan* plan, uint32_t m0, uint32_t nm, const void* in, void* out,
                          size_t count, bool inverse, cudaStream_t s) {
  if (count == 0) return LC_OK;
  if (count > kMaxBatch || m0 + nm > plan->num_moduli) return LC_ERR_INVALID_ARGUMENT;
  NttParams p{};
  p.in = in;
  p.out = out;
  p.count = count;
  p.tw_stride = inverse ? plan->tw_inv_entries : plan->tw_fwd_entries;
  // every table entry is 8 bytes ({w, w'} pairs or Goldilocks residues)
  p.tw = static_cast<const char*>(inverse ? plan->d_tw_inv : plan->d_tw_fwd) + (size_t)m0 * p.tw_stride * 8;
  p.num_moduli = nm;
  for (uint32_t i = 0; i < nm; ++i) {
    p.q[i] = plan->q[m0 + i];
    p.qinv[i] = plan->qinv[m0 + i];
  }
  p.err = plan->d_err;
  const int ln = (int)plan->log_n;
  const int v = plan->variant;
  switch (plan->kind) {
    case PlanKind::U32Lazy:
      return inverse ? dispatch<ShoupLazy, true>(ln, p, v, s) : dispatch<ShoupLazy, false>(ln, p, v, s);
    case PlanKind::U32Mont:
      return inverse ? dispatch<MontCanon, true>(ln, p, v, s) : dispatch<MontCanon, false>(ln, p, v, s);
    case PlanKind::Goldilocks:
      return inverse ? dispatch<Goldilocks, true>(ln, p, v, s) : dispatch<Goldilocks, false>(ln, p, v, s);
  }
  return LC_ERR_INVALID_ARGUMENT;
}

int run_ntt(const lc_ntt_plan* plan, const void* in, void* out, size_t count, bool inverse,
            cudaStream_t s) {
  return run_ntt_moduli(plan, 0, plan->num_moduli, in, out, count, inverse, s);
}

}  // namespace lc

// ====================================================================== C ABI

extern "C" {

LC_API const char* lc_version(void) { return "0.1.0"; }

LC_API const char* lc_status_string(int s) {
  switch (s) {
    case LC_OK: return "ok";
    case LC_ERR_LENGTH_MISMATCH: return "length mismatch";
    case LC_ERR_ADICITY_TOO_SMALL: return "adicity too small";
    case LC_ERR_DIMENSION_MISMATCH: return "dimension mismatch";
    case LC_ERR_NORM_EXCEEDED: return "norm exceeded";
    case LC_ERR_COMMITMENT_MISMATCH: return "commitment mismatch";
    case LC_ERR_NON_CANONICAL: return "non-canonical residue";
    case LC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LC_ERR_UNSUPPORTED: return "unsupported";
    case LC_ERR_CUDA: return "cuda error";
    case LC_ERR_OUT_OF_MEMORY: return "out of memory";
    case LC_ERR_TIMEOUT: return "device wait timed out";
    case LC_ERR_NO_DEVICE: return "no sm_100 device";
    case LC_ERR_LOG_N_OUT_OF_RANGE: return "log_n out of range";
    case LC_ERR_GENERATOR_INVALID: return "generator invalid";
    default: return "unknown status";
  }
}

LC_API int lc_device_available(void) { return device_sm_count() > 0 ? 1 : 0; }

static int finish_plan(lc_ntt_plan* plan, const std::vector<uint64_t>& fwd_raw_all,
                       const std::vector<uint64_t>& inv_raw_all) {
  // convert raw residues into kernel twiddle entries (8 bytes each): the
  // forward table, the inverse table and the zeroed error word go to the
  // device as one block in one copy
  const uint32_t M = plan->num_moduli;
  const uint32_t ef = plan->tw_fwd_entries, ei = plan->tw_inv_entries;
  plan->tw_bytes = 8;
  const size_t nf = fwd_raw_all.size(), ni = inv_raw_all.size();
  std::vector<uint64_t> img(nf + ni + 2, 0);  // + 16 bytes: the error word, zero
  if (plan->kind == PlanKind::Goldilocks) {
    std::copy(fwd_raw_all.begin(), fwd_raw_all.end(), img.begin());
    std::copy(inv_raw_all.begin(), inv_raw_all.end(), img.begin() + nf);
  } else {
    uint2* f = reinterpret_cast<uint2*>(img.data());
    uint2* i = f + nf;
    for (uint32_t m = 0; m < M; ++m) {
      const uint64_t q = plan->q[m];
      auto conv = [&](uint64_t w) -> uint2 {
        if (plan->kind == PlanKind::U32Lazy)
          return make_uint2((uint32_t)w, (uint32_t)(((u128)w << 32) / q));
        return make_uint2((uint32_t)(((u128)w << 32) % q), 0u);
      };
      for (uint32_t k = 0; k < ef; ++k) f[m * ef + k] = conv(fwd_raw_all[m * ef + k]);
      for (uint32_t k = 0; k < ei; ++k) i[m * ei + k] = conv(inv_raw_all[m * ei + k]);
    }
  }
  if (cudaMalloc(&plan->d_block, img.size() * 8) != cudaSuccess) {
    cudaGetLastError();
    plan->d_block = nullptr;
    return LC_ERR_OUT_OF_MEMORY;
  }
  plan->d_tw_fwd = plan->d_block;
  plan->d_tw_inv = static_cast<uint64_t*>(plan->d_block) + nf;
  plan->d_err = reinterpret_cast<uint32_t*>(static_cast<uint64_t*>(plan->d_block) + nf + ni);
  return map_cuda(cudaMemcpy(plan->d_block, img.data(), img.size() * 8, cudaMemcpyHostToDevice));
}

LC_API int lc_ntt_plan_create_u32(uint32_t log_n, const uint32_t* q, const uint32_t* two_adicity,
                                  const uint32_t* generator, uint32_t num_moduli,
                                  lc_ntt_plan** out) {
  if (!out || !q || !two_adicity || !generator || num_moduli == 0 || num_moduli > kMaxModuli)
    return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (log_n < 1) return LC_ERR_INVALID_ARGUMENT;
  bool lazy = true;
  for (uint32_t m = 0; m < num_moduli; ++m) {
    if (q[m] < 3 || (q[m] & 1u) == 0) return LC_ERR_INVALID_ARGUMENT;
    if (log_n + 1 > two_adicity[m]) return LC_ERR_ADICITY_TOO_SMALL;  // ntt.rs:47-50
    if (q[m] >= (1u << 30)) lazy = false;
  }
  const PlanKind kind = lazy ? PlanKind::U32Lazy : PlanKind::U32Mont;
  const int log_v = choose_log_v(kind, (int)log_n);
  if (log_v < 0) return LC_ERR_UNSUPPORTED;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  lc_ntt_plan* plan = new (std::nothrow) lc_ntt_plan();
  if (!plan) return LC_ERR_OUT_OF_MEMORY;
  plan->kind = kind;
  plan->log_n = log_n;
  plan->num_moduli = num_moduli;
  const uint32_t n = 1u << log_n;
  std::vector<uint64_t> fwd_all, inv_all;
  for (uint32_t m = 0; m < num_moduli; ++m) {
    const uint64_t qq = q[m];
    // Modulus32::root_of_unity(log_n + 1), modulus.rs:149-156
    const uint64_t psi = powmod(generator[m], (qq - 1) >> (log_n + 1), qq);
    if (powmod(psi, n, qq) != qq - 1) {  // psi must have order exactly 2n
      delete plan;
      return LC_ERR_INVALID_ARGUMENT;
    }
    std::vector<uint64_t> f, i;
    make_tables((int)log_n, log_v, qq, psi, f, i);
    plan->tw_fwd_entries = (uint32_t)f.size();
    plan->tw_inv_entries = (uint32_t)i.size();
    fwd_all.insert(fwd_all.end(), f.begin(), f.end());
    inv_all.insert(inv_all.end(), i.begin(), i.end());
    plan->q[m] = q[m];
    plan->two_adicity[m] = two_adicity[m];
    plan->generator[m] = generator[m];
    uint32_t inv = 1;  // q^-1 mod 2^32 by Newton iteration
    for (int k = 0; k < 5; ++k) inv *= 2u - q[m] * inv;
    plan->qinv[m] = inv;
  }
  int rc = finish_plan(plan, fwd_all, inv_all);
  if (rc != LC_OK) {
    lc_ntt_plan_destroy(plan);
    return rc;
  }
  *out = plan;
  return LC_OK;
}

LC_API int lc_ntt_plan_create_goldilocks(uint32_t log_n, lc_ntt_plan** out) {
  if (!out) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (log_n < 1) return LC_ERR_INVALID_ARGUMENT;
  if (log_n + 1 > 32) return LC_ERR_ADICITY_TOO_SMALL;
  const int log_v = choose_log_v(PlanKind::Goldilocks, (int)log_n);
  if (log_v < 0 || log_n > 10) return LC_ERR_UNSUPPORTED;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  lc_ntt_plan* plan = new (std::nothrow) lc_ntt_plan();
  if (!plan) return LC_ERR_OUT_OF_MEMORY;
  plan->kind = PlanKind::Goldilocks;
  plan->log_n = log_n;
  plan->num_moduli = 1;
  const uint64_t P = 0xFFFFFFFF00000001ull;
  const uint64_t psi = powmod(7, (P - 1) >> (log_n + 1), P);  // field.rs:195-200
  std::vector<uint64_t> f, i;
  make_tables((int)log_n, log_v, P, psi, f, i);
  plan->tw_fwd_entries = (uint32_t)f.size();
  plan->tw_inv_entries = (uint32_t)i.size();
  int rc = finish_plan(plan, f, i);
  if (rc != LC_OK) {
    lc_ntt_plan_destroy(plan);
    return rc;
  }
  *out = plan;
  return LC_OK;
}

LC_API void lc_ntt_plan_destroy(lc_ntt_plan* plan) {
  if (!plan) return;
  if (plan->d_block) cudaFree(plan->d_block);  // both tables and the error word
  if (plan->d_pow) cudaFree(plan->d_pow);
  plan->staging.release();
  delete plan;
}

LC_API int lc_ntt_plan_set_variant(lc_ntt_plan* plan, int variant) {
  if (!plan || variant < 0 || variant >= LC_NTT_NUM_VARIANTS) return LC_ERR_INVALID_ARGUMENT;
  plan->variant = variant;
  return LC_OK;
}

LC_API int lc_ntt_plan_info(const lc_ntt_plan* plan, uint32_t* log_n, uint32_t* num_moduli,
                            uint32_t* elem_bytes) {
  if (!plan) return LC_ERR_INVALID_ARGUMENT;
  if (log_n) *log_n = plan->log_n;
  if (num_moduli) *num_moduli = plan->num_moduli;
  if (elem_bytes) *elem_bytes = plan->kind == PlanKind::Goldilocks ? 8 : 4;
  return LC_OK;
}

static int check_dev_args(const lc_ntt_plan* plan, const void* in, const void* out) {
  if (!plan || !in || !out) return LC_ERR_INVALID_ARGUMENT;
  if (((uintptr_t)in | (uintptr_t)out) & 15) return LC_ERR_INVALID_ARGUMENT;
  return LC_OK;
}

LC_API int lc_ntt_forward(const lc_ntt_plan* plan, const void* in, void* out, size_t count,
                          lc_stream stream) {
  int rc = check_dev_args(plan, in, out);
  if (rc) return rc;
  return run_ntt(plan, in, out, count, false, (cudaStream_t)stream);
}

LC_API int lc_ntt_inverse(const lc_ntt_plan* plan, const void* in, void* out, size_t count,
                          lc_stream stream) {
  int rc = check_dev_args(plan, in, out);
  if (rc) return rc;
  return run_ntt(plan, in, out, count, true, (cudaStream_t)stream);
}

LC_API int lc_ntt_plan_check(lc_ntt_plan* plan, lc_stream stream) {
  if (!plan) return LC_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return map_cuda(e);
  uint32_t flag = 0;
  e = cudaMemcpy(&flag, plan->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return map_cuda(e);
  if (flag) {
    cudaMemset(plan->d_err, 0, 4);
    return LC_ERR_TIMEOUT;
  }
  return LC_OK;
}

static int ntt_host(lc_ntt_plan* plan, const void* in, void* out, size_t count, bool inverse) {
  if (!plan || (!in && count) || (!out && count)) return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  const size_t eb = plan->kind == PlanKind::Goldilocks ? 8 : 4;
  const size_t poly_bytes = ((size_t)1 << plan->log_n) * eb;
  // chunks of about 16 MiB, each a contiguous run of polynomials under one
  // modulus (the host layout is [modulus][count][n]): one upload, one
  // transform and one download per chunk (measured: 8 and 32 MiB chunks, or
  // one copy per modulus per 16 MiB chunk, ran slower end to end)
  size_t chunk = std::max<size_t>(1, ((size_t)16 << 20) / poly_bytes);
  chunk = std::min(chunk, count);
  HostPipeline& hp = plan->staging;
  int rc = hp.ensure(chunk * poly_bytes);
  if (rc) return rc;
  const char* src = static_cast<const char*>(in);
  char* dst = static_cast<char*>(out);
  int k = 0;
  for (uint32_t m = 0; m < plan->num_moduli && rc == LC_OK; ++m) {
    for (size_t done = 0; done < count; done += chunk, ++k) {
      const size_t c = std::min(chunk, count - done);
      const size_t off = (m * count + done) * poly_bytes;
      cudaStream_t s = hp.stream[k % HostPipeline::kSlots];
      char* dbuf = static_cast<char*>(hp.buf[k % HostPipeline::kSlots]);
      // the buffer of this stream is free once its previous download has
      // finished (stream order)
      cudaMemcpyAsync(dbuf, src + off, c * poly_bytes, cudaMemcpyHostToDevice, s);
      rc = run_ntt_moduli(plan, m, 1, dbuf, dbuf, c, inverse, s);
      if (rc) break;
      cudaMemcpyAsync(dst + off, dbuf, c * poly_bytes, cudaMemcpyDeviceToHost, s);
    }
  }
  const cudaError_t e = hp.sync();
  if (rc) return rc;
  if (e != cudaSuccess) return map_cuda(e);
  return lc_ntt_plan_check(plan, nullptr);
}

LC_API int lc_ntt_forward_host(lc_ntt_plan* plan, const void* in, void* out, size_t count) {
  return ntt_host(plan, in, out, count, false);
}

LC_API int lc_ntt_inverse_host(lc_ntt_plan* plan, const void* in, void* out, size_t count) {
  return ntt_host(plan, in, out, count, true);
}

}  // extern "C"
