// quad50.cu -- the ~2^50 modulus class and its quadratic-slot incomplete NTT.
//
// Modulus50 / QuadSlotTables / RingConfig50 (lattice-ring/src/modulus50.rs):
// q = 2^50 - 2687 (or another two-adicity-7 prime in (2^49, 2^50)), n = 2^k
// with k in [1, 7].  X^n + 1 splits into n/2 quadratics X^2 - gamma_p; the
// forward transform is k-1 DIF levels (lo' = lo + w*hi, hi' = lo - w*hi, one
// twiddle per block), the inverse undoes each butterfly exactly
// (lo = (lo'+hi')/2, hi = (lo'-hi')/(2w)), and a ring product is the slotwise
// Karatsuba (u0 + u1 X)(v0 + v1 X) mod (X^2 - gamma) between two transforms.
//
// GPU layout: polynomials are contiguous [count][n] u64 residues.  A warp
// owns 32/G polynomials (G = min(32, n/2) lanes per polynomial) staged in
// shared memory; every level is one butterfly (or one slot) per lane per
// n/(2G), separated by __syncwarp.
//
// Arithmetic: residues below q < 2^50 are exact doubles, so a modular
// product runs on the FP64 pipe -- h = RN(ab), the exact remainder
// l = fma(a, b, -h), a quotient c = the integer nearest h*(1/q) (one fma
// into the 1.5*2^52 rounding constant), and r = fma(-c, q, h) + l, which is
// exact and lies in (-q, q): |c - ab/q| <= 1/2 + 1/8 + 1/8 because
// |l| <= 2^46 and q > 2^49.  One conditional add of q makes it canonical, so
// every output equals the reference's u64 arithmetic bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>

#include "../../include/lattice_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace lc {

// Table layout (entries): forward twiddles of level d (2^d blocks) at
// 2^d - 1, then the inverse constants inv2 * w^-1 at kQ50Inv + 2^d - 1, the
// leaf gammas at kQ50Gamma, and inv2 at kQ50Inv2.
constexpr int kQ50Inv = 64, kQ50Gamma = 128, kQ50Inv2 = 192, kQ50Tab = 193;

}  // namespace lc

struct lc_quad50_plan {
  uint64_t q = 0, zeta = 0, generator = 0;
  uint32_t two_adicity = 0, log_n = 0;
  uint64_t tab[lc::kQ50Tab] = {};
  double* d_tab = nullptr;
  lc::HostPipeline staging;
};

namespace lc {

using u128 = unsigned __int128;

enum Q50Op : int { kQ50Fwd = 0, kQ50Inv_ = 1, kQ50Slot = 2, kQ50Mul = 3 };

struct Q50Params {
  const uint64_t* a;
  const uint64_t* b;
  uint64_t* out;
  size_t count;
  double q, qinv;  // qinv = RN(1/q)
  const double* tab;
};

constexpr double kRound52 = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds [0, 2^51) to integers

LC_D double q50_add(double a, double b, double q) {
  const double s = __dadd_rn(a, b);
  return s >= q ? __dadd_rn(s, -q) : s;
}

LC_D double q50_sub(double a, double b, double q) {
  const double d = __dadd_rn(a, -b);
  return d < 0.0 ? __dadd_rn(d, q) : d;
}

// a * b mod q for residues a, b < q, 2^49 < q < 2^50
LC_D double q50_mul(double a, double b, double q, double qinv) {
  const double h = __dmul_rn(a, b);
  const double l = __fma_rn(a, b, -h);
  const double c = __dadd_rn(__fma_rn(h, qinv, kRound52), -kRound52);
  const double r = __dadd_rn(__fma_rn(-c, q, h), l);
  return r < 0.0 ? __dadd_rn(r, q) : r;
}

template <int LOG_N>
struct Q50Geo {
  static constexpr int N = 1 << LOG_N;
  static constexpr int HALF = N / 2;                // butterflies per level = quadratic slots
  static constexpr int G = HALF < 32 ? HALF : 32;   // lanes per polynomial
  static constexpr int PW = 32 / G;                 // polynomials per warp
  static constexpr int BPT = HALF / G;              // butterflies (slots) per lane
  static constexpr int WE = PW * N;                 // elements per warp
};

// Register levels: lane l holds elements l + 32 r (r < E) of its warp's
// region.  For n >= 64 the DIF levels whose half span is at least 32 pair
// elements of one lane, with a twiddle that depends on r only.
template <int LOG_N>
struct Q50Reg {
  static constexpr int E = Q50Geo<LOG_N>::WE / 32;         // elements per lane
  static constexpr int LEVELS = LOG_N >= 6 ? LOG_N - 5 : 0;  // forward d < LEVELS, inverse likewise
};

template <int LOG_N>
LC_D void q50_forward_regs(double (&v)[Q50Reg<LOG_N>::E], const double* tab, double q, double qinv) {
  constexpr int E = Q50Reg<LOG_N>::E;
#pragma unroll
  for (int d = 0; d < Q50Reg<LOG_N>::LEVELS; ++d) {
    const int hr = (1 << (LOG_N - 1 - d)) / 32;  // register distance of the pair
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (r & hr) continue;
      const double t = q50_mul(v[r + hr], tab[(1 << d) - 1 + r / (2 * hr)], q, qinv);
      const double L = v[r];
      v[r] = q50_add(L, t, q);
      v[r + hr] = q50_sub(L, t, q);
    }
  }
}

template <int LOG_N>
LC_D void q50_inverse_regs(double (&v)[Q50Reg<LOG_N>::E], const double* tab, double q, double qinv) {
  constexpr int E = Q50Reg<LOG_N>::E;
  const double inv2 = tab[kQ50Inv2];
#pragma unroll
  for (int d = Q50Reg<LOG_N>::LEVELS - 1; d >= 0; --d) {
    const int hr = (1 << (LOG_N - 1 - d)) / 32;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      if (r & hr) continue;
      const double L = v[r], H = v[r + hr];
      v[r] = q50_mul(q50_add(L, H, q), inv2, q, qinv);
      v[r + hr] = q50_mul(q50_sub(L, H, q), tab[kQ50Inv + (1 << d) - 1 + r / (2 * hr)], q, qinv);
    }
  }
}

// Shared-memory levels d in [Q50Reg::LEVELS, LOG_N - 1) of NX polynomials
// (one per operand) of this lane's group, interleaved for independent work.
template <int LOG_N, int NX>
LC_D void q50_forward_smem(double* const (&x)[NX], const double* tab, uint32_t g, double q, double qinv) {
  using Q = Q50Geo<LOG_N>;
#pragma unroll
  for (int d = Q50Reg<LOG_N>::LEVELS; d + 1 < LOG_N; ++d) {
    const int hb = LOG_N - 1 - d;  // log2 of the half span
#pragma unroll
    for (int r = 0; r < Q::BPT; ++r) {
      const uint32_t u = g + Q::G * r;
      const uint32_t i = u >> hb, j = u & ((1u << hb) - 1);
      const uint32_t lo = (i << (hb + 1)) + j, hi = lo + (1u << hb);
      const double w = tab[(1u << d) - 1 + i];
#pragma unroll
      for (int k = 0; k < NX; ++k) {
        const double L = x[k][lo];
        const double t = q50_mul(x[k][hi], w, q, qinv);
        x[k][lo] = q50_add(L, t, q);
        x[k][hi] = q50_sub(L, t, q);
      }
    }
    __syncwarp();
  }
}

template <int LOG_N>
LC_D void q50_inverse_smem(double* x, const double* tab, uint32_t g, double q, double qinv) {
  using Q = Q50Geo<LOG_N>;
  const double inv2 = tab[kQ50Inv2];
#pragma unroll
  for (int d = LOG_N - 2; d >= Q50Reg<LOG_N>::LEVELS; --d) {
    const int hb = LOG_N - 1 - d;
#pragma unroll
    for (int r = 0; r < Q::BPT; ++r) {
      const uint32_t u = g + Q::G * r;
      const uint32_t i = u >> hb, j = u & ((1u << hb) - 1);
      const uint32_t lo = (i << (hb + 1)) + j, hi = lo + (1u << hb);
      const double L = x[lo], H = x[hi];
      x[lo] = q50_mul(q50_add(L, H, q), inv2, q, qinv);
      x[hi] = q50_mul(q50_sub(L, H, q), tab[kQ50Inv + (1u << d) - 1 + i], q, qinv);
    }
    __syncwarp();
  }
}

// x <- x (*) y slotwise: (u0 + u1 X)(v0 + v1 X) mod (X^2 - gamma_p)
template <int LOG_N>
LC_D void q50_slotwise(double* x, const double* y, const double* tab, uint32_t g, double q, double qinv) {
  using Q = Q50Geo<LOG_N>;
#pragma unroll
  for (int r = 0; r < Q::BPT; ++r) {
    const uint32_t p = g + Q::G * r;
    const double u0 = x[2 * p], u1 = x[2 * p + 1], v0 = y[2 * p], v1 = y[2 * p + 1];
    const double p0 = q50_mul(u0, v0, q, qinv);
    const double p1 = q50_mul(u1, v1, q, qinv);
    const double cross = q50_mul(q50_add(u0, u1, q), q50_add(v0, v1, q), q, qinv);
    x[2 * p] = q50_add(p0, q50_mul(p1, tab[kQ50Gamma + p], q, qinv), q);
    x[2 * p + 1] = q50_sub(cross, q50_add(p0, p1, q), q);
  }
  __syncwarp();
}

constexpr int kQ50Warps = 8;

// five CTAs per SM (48 registers, no spills): the kernel is latency-bound at four
template <int LOG_N, int OP>
__global__ void __launch_bounds__(kQ50Warps * 32, 5) quad50_kernel(const __grid_constant__ Q50Params p) {
  using Q = Q50Geo<LOG_N>;
  constexpr int E = Q50Reg<LOG_N>::E;
  constexpr bool TWO = OP == kQ50Slot || OP == kQ50Mul;
  __shared__ double s_tab[kQ50Tab];
  __shared__ __align__(16) double s_a[kQ50Warps][Q::WE];
  __shared__ __align__(16) double s_b[kQ50Warps][TWO ? Q::WE : 1];
  for (int e = threadIdx.x; e < kQ50Tab; e += blockDim.x) s_tab[e] = p.tab[e];
  __syncthreads();
  const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t g = lane % Q::G, poly = lane / Q::G;
  const size_t total = p.count * Q::N;
  const size_t tasks = (p.count + Q::PW - 1) / Q::PW;
  double* xa = s_a[warp];
  double* xb = s_b[warp];
  const double q = p.q, qinv = p.qinv;
  for (size_t task = (size_t)blockIdx.x * kQ50Warps + warp; task < tasks; task += (size_t)gridDim.x * kQ50Warps) {
    const size_t base = task * Q::WE;
    const uint32_t valid = total - base < (size_t)Q::WE ? (uint32_t)(total - base) : (uint32_t)Q::WE;
    double va[E], vb[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
      // plain loads (out may alias a or b); residues < 2^50 convert exactly
      const uint32_t e = lane + 32 * r;
      va[r] = e < valid ? __ull2double_rn(p.a[base + e]) : 0.0;
      if (TWO) vb[r] = e < valid ? __ull2double_rn(p.b[base + e]) : 0.0;
    }
    if (OP == kQ50Fwd || OP == kQ50Mul) q50_forward_regs<LOG_N>(va, s_tab, q, qinv);
    if (OP == kQ50Mul) q50_forward_regs<LOG_N>(vb, s_tab, q, qinv);
#pragma unroll
    for (int r = 0; r < E; ++r) {
      xa[lane + 32 * r] = va[r];
      if (TWO) xb[lane + 32 * r] = vb[r];
    }
    __syncwarp();
    double* x = xa + poly * Q::N;
    double* y = xb + poly * Q::N;
    if (OP == kQ50Fwd) {
      double* const xs[1] = {x};
      q50_forward_smem<LOG_N, 1>(xs, s_tab, g, q, qinv);
    }
    if (OP == kQ50Inv_) q50_inverse_smem<LOG_N>(x, s_tab, g, q, qinv);
    if (OP == kQ50Slot) q50_slotwise<LOG_N>(x, y, s_tab, g, q, qinv);
    if (OP == kQ50Mul) {
      double* const xs[2] = {x, y};
      q50_forward_smem<LOG_N, 2>(xs, s_tab, g, q, qinv);
      q50_slotwise<LOG_N>(x, y, s_tab, g, q, qinv);
      q50_inverse_smem<LOG_N>(x, s_tab, g, q, qinv);
    }
#pragma unroll
    for (int r = 0; r < E; ++r) va[r] = xa[lane + 32 * r];
    if (OP == kQ50Inv_ || OP == kQ50Mul) q50_inverse_regs<LOG_N>(va, s_tab, q, qinv);
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const uint32_t e = lane + 32 * r;
      if (e < valid) p.out[base + e] = __double2ull_rn(va[r]);
    }
    __syncwarp();
  }
}

template <int LOG_N, int OP>
static int q50_launch(const lc_quad50_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* out,
                      size_t count, cudaStream_t st) {
  using Q = Q50Geo<LOG_N>;
  Q50Params p{a, b, out, count, (double)plan->q, 1.0 / (double)plan->q, plan->d_tab};
  const size_t tasks = (count + Q::PW - 1) / Q::PW;
  const size_t want = (tasks + kQ50Warps - 1) / kQ50Warps;
  const size_t cap = (size_t)std::max(1, device_sm_count()) * 8;
  quad50_kernel<LOG_N, OP><<<(unsigned)std::min(want, cap), kQ50Warps * 32, 0, st>>>(p);
  return map_cuda(cudaGetLastError());
}

template <int OP>
static int q50_dispatch(const lc_quad50_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* out,
                        size_t count, cudaStream_t st) {
  switch (plan->log_n) {
    case 1: return q50_launch<1, OP>(plan, a, b, out, count, st);
    case 2: return q50_launch<2, OP>(plan, a, b, out, count, st);
    case 3: return q50_launch<3, OP>(plan, a, b, out, count, st);
    case 4: return q50_launch<4, OP>(plan, a, b, out, count, st);
    case 5: return q50_launch<5, OP>(plan, a, b, out, count, st);
    case 6: return q50_launch<6, OP>(plan, a, b, out, count, st);
    case 7: return q50_launch<7, OP>(plan, a, b, out, count, st);
    default: return LC_ERR_INVALID_ARGUMENT;
  }
}

static int q50_run(const lc_quad50_plan* plan, int op, const uint64_t* a, const uint64_t* b, uint64_t* out,
                   size_t count, cudaStream_t st) {
  if (!plan || ((!a || !out || (op >= kQ50Slot && !b)) && count)) return LC_ERR_INVALID_ARGUMENT;
  if (count > ((size_t)1 << 36)) return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  switch (op) {
    case kQ50Fwd: return q50_dispatch<kQ50Fwd>(plan, a, b, out, count, st);
    case kQ50Inv_: return q50_dispatch<kQ50Inv_>(plan, a, b, out, count, st);
    case kQ50Slot: return q50_dispatch<kQ50Slot>(plan, a, b, out, count, st);
    default: return q50_dispatch<kQ50Mul>(plan, a, b, out, count, st);
  }
}

// host-side exact arithmetic for the tables
static uint64_t hmul(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }

static uint64_t hpow(uint64_t b, uint64_t e, uint64_t q) {
  uint64_t acc = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) acc = hmul(acc, b, q);
    b = hmul(b, b, q);
    e >>= 1;
  }
  return acc;
}

static uint32_t rev_bits(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t b = 0; b < bits; ++b) r |= ((x >> b) & 1u) << (bits - 1 - b);
  return r;
}

}  // namespace lc

extern "C" {

LC_API int lc_quad50_plan_create(uint64_t q, uint32_t two_adicity, uint64_t generator, uint32_t log_n,
                                 lc_quad50_plan** out) {
  using namespace lc;
  if (!out) return LC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (q <= ((uint64_t)1 << 49) || q >= ((uint64_t)1 << 50) || !(q & 1)) return LC_ERR_INVALID_ARGUMENT;
  if (log_n == 0 || log_n > 7) return LC_ERR_LOG_N_OUT_OF_RANGE;  // modulus50.rs:252-254
  if (two_adicity < 7) return LC_ERR_ADICITY_TOO_SMALL;           // :255-259
  const uint64_t zeta = hpow(generator, (q - 1) >> 7, q);          // root_of_unity(7), :191-197
  if (hpow(zeta, 64, q) != q - 1) return LC_ERR_GENERATOR_INVALID;  // :266-268
  lc_quad50_plan* p = new (std::nothrow) lc_quad50_plan();
  if (!p) return LC_ERR_OUT_OF_MEMORY;
  p->q = q;
  p->zeta = zeta;
  p->generator = generator;
  p->two_adicity = two_adicity;
  p->log_n = log_n;
  const uint64_t inv2 = hpow(2, q - 2, q);
  for (uint32_t d = 0; d + 1 < log_n; ++d) {  // :272-289
    for (uint32_t i = 0; i < (1u << d); ++i) {
      const uint64_t e = ((2 * (uint64_t)rev_bits(i, d) + 1) << (5 - d)) % 128;
      const uint64_t w = hpow(zeta, e, q);
      p->tab[(1u << d) - 1 + i] = w;
      p->tab[kQ50Inv + (1u << d) - 1 + i] = hmul(inv2, hpow(w, q - 2, q), q);
    }
  }
  for (uint32_t s = 0; s < (1u << (log_n - 1)); ++s) {  // :291-296
    const uint64_t e = ((2 * (uint64_t)rev_bits(s, log_n - 1) + 1) << (7 - log_n)) % 128;
    p->tab[kQ50Gamma + s] = hpow(zeta, e, q);
  }
  p->tab[kQ50Inv2] = inv2;
  double dtab[kQ50Tab];
  for (int i = 0; i < kQ50Tab; ++i) dtab[i] = (double)p->tab[i];  // < 2^50: exact
  if (device_sm_count() <= 0) {
    delete p;
    return LC_ERR_NO_DEVICE;
  }
  if (cudaMalloc(&p->d_tab, sizeof(p->tab)) != cudaSuccess) {
    cudaGetLastError();
    delete p;
    return LC_ERR_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaMemcpy(p->d_tab, dtab, sizeof(dtab), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p->d_tab);
    delete p;
    return map_cuda(e);
  }
  *out = p;
  return LC_OK;
}

LC_API void lc_quad50_plan_destroy(lc_quad50_plan* plan) {
  if (!plan) return;
  if (plan->d_tab) cudaFree(plan->d_tab);
  plan->staging.release();
  delete plan;
}

LC_API int lc_quad50_plan_info(const lc_quad50_plan* plan, uint64_t* zeta, uint64_t* slot_constants) {
  if (!plan) return LC_ERR_INVALID_ARGUMENT;
  if (zeta) *zeta = plan->zeta;
  if (slot_constants)
    for (uint32_t s = 0; s < (1u << (plan->log_n - 1)); ++s) slot_constants[s] = plan->tab[lc::kQ50Gamma + s];
  return LC_OK;
}

LC_API int lc_quad50_forward(const lc_quad50_plan* plan, const uint64_t* in, uint64_t* out, size_t count,
                             lc_stream stream) {
  return lc::q50_run(plan, lc::kQ50Fwd, in, nullptr, out, count, (cudaStream_t)stream);
}

LC_API int lc_quad50_inverse(const lc_quad50_plan* plan, const uint64_t* in, uint64_t* out, size_t count,
                             lc_stream stream) {
  return lc::q50_run(plan, lc::kQ50Inv_, in, nullptr, out, count, (cudaStream_t)stream);
}

LC_API int lc_quad50_slotwise_mul(const lc_quad50_plan* plan, const uint64_t* a, const uint64_t* b,
                                  uint64_t* out, size_t count, lc_stream stream) {
  return lc::q50_run(plan, lc::kQ50Slot, a, b, out, count, (cudaStream_t)stream);
}

LC_API int lc_quad50_mul(const lc_quad50_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* out,
                         size_t count, lc_stream stream) {
  return lc::q50_run(plan, lc::kQ50Mul, a, b, out, count, (cudaStream_t)stream);
}

// Host buffers: chunks of about 8 MiB per operand alternate between two
// staging buffers and streams, so copies of one chunk overlap the other's kernel.
LC_API int lc_quad50_mul_host(lc_quad50_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* out,
                              size_t count) {
  using namespace lc;
  if (!plan || ((!a || !b || !out) && count)) return LC_ERR_INVALID_ARGUMENT;
  if (count == 0) return LC_OK;
  if (device_sm_count() <= 0) return LC_ERR_NO_DEVICE;
  const size_t n = (size_t)1 << plan->log_n, pb = n * 8;
  const size_t chunk = std::min(count, std::max<size_t>(1, ((size_t)8 << 20) / pb));
  HostPipeline& hp = plan->staging;
  int rc = hp.ensure(3 * chunk * pb);
  if (rc) return rc;
  size_t done = 0;
  int k = 0;
  while (done < count) {
    const size_t c = std::min(chunk, count - done);
    cudaStream_t s = hp.stream[k % HostPipeline::kSlots];
    uint64_t* da = static_cast<uint64_t*>(hp.buf[k % HostPipeline::kSlots]);
    uint64_t* db = da + chunk * n;
    uint64_t* dout = db + chunk * n;
    cudaMemcpyAsync(da, a + done * n, c * pb, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(db, b + done * n, c * pb, cudaMemcpyHostToDevice, s);
    rc = q50_run(plan, kQ50Mul, da, db, dout, c, s);
    if (rc) break;
    cudaMemcpyAsync(out + done * n, dout, c * pb, cudaMemcpyDeviceToHost, s);
    done += c;
    ++k;
  }
  const cudaError_t e = hp.sync();
  if (rc) return rc;
  return map_cuda(e);
}

}  // extern "C"
