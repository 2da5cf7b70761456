// tc_commit.cu -- Ajtai commitment over Goldilocks (d = 64) on the INT8
// tensor cores (tcgen05.mma .kind::i8, sm_100a), exact.
//
// Coefficient-domain form of the commitment (lattice-folding/src/neo.rs:
// 138-158 and 419-441; the same map as AjtaiPublicKey::commit, ajtai.rs:
// 118-153):
//   c_{b,i}[r] = sum_j sum_s R_ij[r][s] * w_{b,j}[s]   (mod p),
//   R_ij = rot(a_ij),  R[r][s] = a[r-s] (r >= s),  p - a[r-s+64] (r < s),
// with witness digits w in [-128, 127].  Every residue R[r][s] in [0, p) is
// split into 8 byte limbs, R = sum_l 2^(8l) R_l, so each limb is an exact
// integer GEMM
//   D_l[b][(i,r)] = sum_(j,s) W[b][(j,s)] * R_l[(i,r)][(j,s)]   (s8 x u8 -> s32)
// with K = 64 per ring element.  A CTA sums at most 1024 ring elements
// (K <= 65536), so |D_l| <= 65536 * 128 * 255 < 2^31 and the int32
// accumulator is exact.  Unsigned byte digits (decomp_b rows,
// lattice-folding/src/neo.rs:253-266) run the same kernel as u8 x u8 with
// at most 512 ring elements per CTA: 32768 * 255 * 255 < 2^31.  The reduction kernel forms sum_l 2^(8l) D_l over all
// K-splits in 128-bit integers and reduces mod p.
//
// CTA tile: 128 witnesses (MMA M; the W tile comes from HBM by TMA with the
// 128-byte swizzle), 4 rows i x 64 coefficients r (MMA N = 256, built in
// shared memory), two limbs (two 128 x 256 int32 accumulators = all 512 TMEM
// columns).  The rotation tiles are Toeplitz: row r of the 64-byte K block of
// ring element j is the window F[63-r .. 126-r] of the 127-byte source
//   F[v] = limb(a[63-v]) (v < 64),  limb(p - a[127-v]) (64 <= v < 127),
// so the key is stored as F rows (128 bytes, zero tail).  With the operand
// rows in reversed coefficient order r' = 63 - r, the 8-row x 16-byte block
// (g, c) of a tile depends on u = g + 2c only: C_u, row x = F[8u + x ..
// 8u + x + 16).  The builders store the 14 blocks C_u of each row i (7 KB per
// limb and ring element instead of a 16 KB tile) and the MMA reads the tile
// through a no-swizzle K-major descriptor that revisits them (8-row group
// 4g + i at 128 (4g + i), next K chunk at +1024); one thread loads 5 aligned
// words and emits 4 rows of a block with funnel shifts.
//
// Warp roles: 0-7 build rotation blocks (and drain TMEM at the end), 8 issues
// the TMA loads, 9 owns TMEM and issues the MMAs.  Rings: 4 slots of
// (W tile + F rows), 4 slots of rotation blocks; mbarrier hand-offs, every
// wait bounded (on expiry the kernel records LC_DEVERR_TIMEOUT, waits --
// again bounded -- for its copies and MMAs in flight, frees TMEM, returns).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/lattice_cuda.h"
#include "arith.cuh"
#include "common.cuh"
#include "internal.h"
#include "tcgen05.cuh"

namespace lc {

// ring elements per CTA (K = 64 each): the int32 bound above
template <bool S8>
struct TcJPer {
  static constexpr int value = S8 ? 1024 : 512;
};
constexpr int kTcFRow = 128;             // bytes per F row
constexpr int kTcWBytes = 128 * 128;     // W tile: 128 witnesses x 128 bytes (2 ring elements)
// One limb's rotation operand for one ring element, compact: with the
// coefficient order reversed (r' = 63 - r) the 8-row x 16-byte block (g, c)
// of the Toeplitz tile is C_u, u = g + 2c, row x = F[8u + x .. 8u + x + 16);
// C_u of row i sits at (4u + i) * 128, so the no-swizzle K-major descriptor
// with SBO = 128 (8-row group 4g + i) and LBO = 1024 (next 16-byte K chunk)
// walks the full 256 x 64 tile over 14 x 4 blocks.
constexpr int kTcRotBytes = 14 * 4 * 128;  // 7 KB
constexpr int kTcFHalf = 8 * kTcFRow + 64;  // rows of one ring element; +64 B skews banks
constexpr int kTcFSlot = 2 * kTcFHalf;
// (at most 4 rotation slots: the builders wait on the 4-slot mma_done ring)
constexpr int kTcWSlots = 4, kTcRotSlots = 4;
constexpr int kTcOffRot = kTcWSlots * kTcWBytes;
constexpr int kTcOffF = kTcOffRot + kTcRotSlots * 4 * kTcRotBytes;  // slot: 2 limbs x 2 ring elements
constexpr int kTcOffBar = kTcOffF + kTcWSlots * kTcFSlot;
constexpr size_t kTcSmem = 1024 + kTcOffBar + 256;
constexpr int kTcThreads = 320;
constexpr uint32_t kTcLoadBytes = kTcWBytes + 2 * 8 * kTcFRow;
static_assert(kTcOffRot % 1024 == 0 && kTcOffF % 16 == 0 && kTcFHalf % 16 == 0, "alignment");
static_assert(kTcSmem <= 227 * 1024, "shared memory");

// ------------------------------------------------------------------ device helpers

// D = s32 (4), A = s8 or u8 (7), B = u8 (10), both K-major, N = 256 (17), M = 128 (24)
template <bool S8>
struct TcIdesc {
  static constexpr uint32_t value =
      (2u << 4) | ((S8 ? 1u : 0u) << 7) | (0u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);
};

// ------------------------------------------------------------------ key tables

// fkey[g][lp][j][ll][ii][128]: F row of limb 2*lp+ll of A[4g+ii][j] (zero for
// i >= k or j >= m).  One thread writes 16 bytes.
__global__ void tc_key_tables_kernel(const uint64_t* __restrict__ a, uint8_t* __restrict__ fkey, uint32_t k,
                                     uint32_t m, uint32_t m_pad, uint32_t groups) {
  const size_t total16 = (size_t)groups * 4 * m_pad * 8 * (kTcFRow / 16);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total16;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t v0 = (uint32_t)(e % 8) * 16;
    size_t rest = e / 8;
    const uint32_t ii = rest % 4;
    rest /= 4;
    const uint32_t ll = rest % 2;
    rest /= 2;
    const uint32_t j = rest % m_pad;
    rest /= m_pad;
    const uint32_t lp = rest % 4;
    const uint32_t g = (uint32_t)(rest / 4);
    const uint32_t i = 4 * g + ii, shift = 8 * (2 * lp + ll);
    uint32_t wv[4] = {0, 0, 0, 0};
    if (i < k && j < m) {
      const uint64_t* ae = a + ((size_t)i * m + j) * 64;
      for (int t = 0; t < 16; ++t) {
        const uint32_t v = v0 + t;
        uint64_t x = 0;
        if (v < 64) {
          x = ae[63 - v];
        } else if (v < 127) {
          x = ae[127 - v];
          x = x == 0 ? 0 : kGlP - x;
        }
        wv[t >> 2] |= (uint32_t)((x >> shift) & 0xFF) << (8 * (t & 3));
      }
    }
    reinterpret_cast<uint4*>(fkey)[e] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
  }
}

// ------------------------------------------------------------------ the product kernel

struct TcParams {
  const uint8_t* fkey;
  int64_t* partial;  // [split][lp][g][bt][256][128]
  uint32_t m_pad, groups, splits, btiles;
  uint32_t* err;
};

template <bool S8>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_commit_kernel(const __grid_constant__ CUtensorMap wmap, const __grid_constant__ TcParams p) {
  constexpr int kTcJPer = TcJPer<S8>::value;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kTcOffBar);
  uint64_t* loaded = bars;         // [4] W + F of a stage landed (tx bytes)
  uint64_t* mma_done = bars + 4;   // [4] tcgen05.commit of a stage
  uint64_t* built = bars + 8;      // [kTcRotSlots] 8 builder-warp arrivals
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 8 + kTcRotSlots);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 9 + kTcRotSlots);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t lp = blockIdx.x, g = blockIdx.y;
  const uint32_t split = blockIdx.z % p.splits, bt = blockIdx.z / p.splits;
  const uint32_t j0 = split * kTcJPer;
  const uint32_t j1 = min(p.m_pad, j0 + kTcJPer);
  const int nst = (int)((j1 - j0) / 2);  // stages of two ring elements; m_pad is even

  if (tid == 0) {
    for (int s = 0; s < 4; ++s) {
      mbar_init(&loaded[s], 1);
      mbar_init(&mma_done[s], 1);
    }
    for (int r = 0; r < kTcRotSlots; ++r) mbar_init(&built[r], 8);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 9) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  auto w_slot = [&](int s) { return base + (s & 3) * kTcWBytes; };
  auto rot_slot = [&](int s, int ll, int jj) {
    return base + kTcOffRot + (((s % kTcRotSlots) * 2 + ll) * 2 + jj) * kTcRotBytes;
  };
  auto f_slot = [&](int s) { return base + kTcOffF + (s & 3) * kTcFSlot; };
  auto fail = [&]() {
    record_error(p.err, LC_DEVERR_TIMEOUT);
    *abort_flag = 1;
  };

  int last_loaded = -1;  // TMA thread: last stage whose load was issued
  int last_mma = -1;     // MMA thread: last stage whose MMAs were committed

  if (warp == 8) {
    // ---------------- TMA producer
    if (lane == 0) {
      const uint8_t* fsrc = p.fkey + (((size_t)g * 4 + lp) * p.m_pad) * 8 * kTcFRow;
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (s >= 4 && !mbar_wait(&mma_done[s & 3], ((s - 4) >> 2) & 1)) {  // slot free again
          fail();
          break;
        }
        const uint32_t j = j0 + 2 * s;
        mbar_arrive_expect_tx(&loaded[s & 3], kTcLoadBytes);
        tma_load_2d(w_slot(s), &wmap, (int)(j * 64), (int)(bt * 128), &loaded[s & 3]);
        bulk_g2s(f_slot(s), fsrc + (size_t)j * 8 * kTcFRow, 8 * kTcFRow, &loaded[s & 3]);
        bulk_g2s(f_slot(s) + kTcFHalf, fsrc + (size_t)(j + 1) * 8 * kTcFRow, 8 * kTcFRow, &loaded[s & 3]);
        last_loaded = s;
      }
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer
    if (lane == 0) {
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (!mbar_wait(&loaded[s & 3], (s >> 2) & 1) ||
            !mbar_wait(&built[s % kTcRotSlots], (uint32_t)((s / kTcRotSlots) & 1))) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t wa = smem_u32(w_slot(s));
#pragma unroll
        for (int ll = 0; ll < 2; ++ll) {
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            // K step ks: ring element ks / 2, its 16-byte chunks 2 (ks % 2) and 2 (ks % 2) + 1
            const uint32_t ra = smem_u32(rot_slot(s, ll, ks >> 1)) + 2 * (ks & 1) * 1024;
            mma_i8(tmem + ll * 256, umma_desc_sw128(wa + 32 * ks), umma_desc_noswz(ra, 1024, 128),
                   TcIdesc<S8>::value, (s > 0 || ks > 0) ? 1u : 0u);
          }
        }
        mma_commit(&mma_done[s & 3]);
        last_mma = s;
      }
    }
  } else {
    // ---------------- builders
    // Warp-round (2 per stage) = one (limb ll, ring element jj, row i); lane
    // 2u + h (< 28) writes rows 4h .. 4h + 3 of C_u from 5 aligned words of
    // the F row.  Row order rho = (t + u) & 3 per store keeps the 8 lanes of a
    // quarter-warp on 8 distinct 16-byte bank groups; the loads (one F row per
    // warp, 28 distinct words) are conflict free.
    const uint32_t u = lane >> 1, h = lane & 1;
    for (int s = 0; s < nst; ++s) {
      bool ok = true;
      if (s >= kTcRotSlots)  // rotation slot free: the MMAs of stage s - kTcRotSlots are done
        ok = mbar_wait(&mma_done[(s - kTcRotSlots) & 3], (uint32_t)(((s - kTcRotSlots) >> 2) & 1));
      ok = ok && mbar_wait(&loaded[s & 3], (s >> 2) & 1);
      if (!ok) fail();
      // warp-uniform: the loop below synchronises the warp
      if (__any_sync(0xffffffffu, *abort_flag)) break;
#pragma unroll
      for (int rd = 0; rd < 2; ++rd) {
        const uint32_t combo = 2 * warp + rd;  // bits: 0-1 row i, 2 ring element jj, 3 limb ll
        const uint32_t ii = combo & 3, jj = (combo >> 2) & 1, ll = combo >> 3;
        if (lane < 28) {
          const uint32_t* frow =
              reinterpret_cast<const uint32_t*>(f_slot(s) + jj * kTcFHalf + (ll * 4 + ii) * kTcFRow);
          uint32_t w[5];
#pragma unroll
          for (int e = 0; e < 5; ++e) w[e] = frow[2 * u + h + e];  // word 2u + h + 4 <= 31
          unsigned char* blk = rot_slot(s, (int)ll, (int)jj) + (4 * u + ii) * 128;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const uint32_t rho = (t + u) & 3, x = 4 * h + rho;
            uint32_t o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) o[q] = __funnelshift_r(w[q], w[q + 1], 8 * rho);
            *reinterpret_cast<uint4*>(blk + 16 * x) = make_uint4(o[0], o[1], o[2], o[3]);
          }
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&built[s % kTcRotSlots]);
    }
  }

  // ---------------- drain the accumulators (builder warps)
  __syncthreads();
  if (nst > 0 && warp < 8 && !__any_sync(0xffffffffu, *abort_flag)) {
    const int ls = nst - 1;
    // warp-uniform decision: the TMEM loads below are .sync.aligned
    if (!__all_sync(0xffffffffu, mbar_wait(&mma_done[ls & 3], (ls >> 2) & 1))) {
      fail();
    } else {
      tc_fence_after();
      const uint32_t lane_base = 32 * (warp & 3), col_half = warp >> 2;
      const uint32_t b_local = lane_base + lane;
      int64_t* out = p.partial + ((((size_t)split * 4 + lp) * p.groups + g) * p.btiles + bt) * 256 * 128;
#pragma unroll 1
      for (int cc = 0; cc < 8; ++cc) {
        const uint32_t col = col_half * 128 + cc * 16;
        uint32_t d0[16], d1[16];
        tmem_ld16(tmem + (lane_base << 16) + col, d0);
        tmem_ld16(tmem + (lane_base << 16) + 256 + col, d1);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          // operand row n = 8 (4g + i) + x holds row i, coefficient r = 63 - (8g + x)
          const uint32_t n = col + u;
          const uint32_t nr = ((n >> 3) & 3) * 64 + 63 - (8 * (n >> 5) + (n & 7));
          out[(size_t)nr * 128 + b_local] = (int64_t)(int32_t)d0[u] + 256 * (int64_t)(int32_t)d1[u];
        }
      }
    }
  }
  // ---------------- nothing may be in flight when TMEM and shared memory go
  // (these waits return at once on the normal path)
  if (warp == 8 && lane == 0) {
    for (int s = max(0, last_loaded - 3); s <= last_loaded; ++s) mbar_wait(&loaded[s & 3], (s >> 2) & 1);
  }
  if (warp == 9 && lane == 0 && last_mma >= 0) mbar_wait(&mma_done[last_mma & 3], (last_mma >> 2) & 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 9) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// out[b][i][r] = sum_split sum_lp 2^(16 lp) partial[split][lp][g][bt][n][bl]  mod p,
// i = 4g + n/64, r = n%64, b = 128 bt + bl.  Threads run along bl (coalesced reads).
__global__ void tc_reduce_kernel(const int64_t* __restrict__ partial, uint64_t* __restrict__ out,
                                 uint32_t batch, uint32_t k, uint32_t groups, uint32_t splits,
                                 uint32_t btiles) {
  const size_t total = (size_t)groups * btiles * 256 * 128;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const uint32_t bl = idx % 128;
    const uint32_t n = (idx / 128) % 256;
    const uint32_t bt = (uint32_t)((idx / (128 * 256)) % btiles);
    const uint32_t g = (uint32_t)(idx / ((size_t)128 * 256 * btiles));
    const uint32_t b = bt * 128 + bl, i = 4 * g + n / 64;
    if (b >= batch || i >= k) continue;
    __int128 acc = 0;
    for (uint32_t lp = 0; lp < 4; ++lp) {
      int64_t s = 0;
      for (uint32_t sp = 0; sp < splits; ++sp) s += partial[((size_t)sp * 4 + lp) * total + idx];
      acc += (__int128)s << (16 * lp);
    }
    const bool neg = acc < 0;
    const unsigned __int128 u = neg ? (unsigned __int128)(-acc) : (unsigned __int128)acc;
    uint64_t res = gl_canon(gl_reduce128_lazy((uint64_t)(u >> 64), (uint64_t)u));
    if (neg && res) res = kGlP - res;
    out[((size_t)b * k + i) * 64 + n % 64] = res;
  }
}

// ------------------------------------------------------------------ witness NTT on the tensor cores
//
// For d = 64 the forward transform of a digit vector w is a fixed matrix
// product, What[t] = sum_c V[t][c] w[c] (mod p) with V[t][c] = psi^((2t+1)c)
// (the natural-order negacyclic NTT, out[t] = w(psi^(2t+1))).  With the
// residues V split into 8 byte limbs, D_l[r][t] = sum_c W[r][c] V_l[t][c] is
// exact in int32 (64 * 128 * 255 < 2^21, u8 digits 64 * 255 * 255 < 2^22) and
// What = sum_l 2^(8l) D_l (mod p).  An M = 128 tile holds R consecutive ring
// elements x BB witnesses (R * BB = 128; rows ordered witness fastest, one
// 64-byte ring element each, read by a 3-D TMA view of w[b][j][64] -- x the
// digit, y the witness, z the ring element -- with the 64-byte swizzle); a
// tile is four MMAs (two limb groups N = 256, K = 64 as two K-steps) into all
// 512 TMEM columns.  Sixteen epilogue warps read the limbs back, fold them
// mod p and write What_T[t][j][b]: a warp's 32 rows are 32 consecutive
// entries of one slot.
constexpr int kTnSlots = 4;
constexpr int kTnATile = 128 * 64;  // 128 rows (ring element, witness) x 64 digit bytes
constexpr int kTnVTile = 256 * 128;
constexpr int kTnOffV = kTnSlots * kTnATile;
constexpr int kTnOffBar = kTnOffV + 2 * kTnVTile;
constexpr size_t kTnSmem = 1024 + kTnOffBar + 256;
constexpr int kTnEpiWarps = 16;  // 4 per TMEM lane quarter, 16 slots each
constexpr int kTnThreads = (kTnEpiWarps + 2) * 32;
static_assert(kTnSmem <= 227 * 1024, "shared memory");

struct TnParams {
  const uint4* vimg;  // [2][256][128] bytes: the limb tiles in their swizzled shared-memory image
  uint64_t* what_t;   // [64][m][b_pad]
  uint32_t m, b_pad, batch, BB, R, nblk;  // tile: R ring elements x BB witnesses; nblk ring-element blocks
  uint64_t items;
  uint32_t* err;
};

// sum_l 2^(8l) D_l mod p for one output (|D_l| < 2^22), as a 64-bit value
// congruent mod p but not necessarily canonical (it may lie in [p, 2^64)):
// every reader of the witness transforms -- the byte-limb slot products and
// the 160-bit integer products -- takes any 64-bit representative.  A = D0 +
// 2^8 D1 + 2^16 D2 + 2^24 D3 and B (limbs 4..7) are exact in int64 (|A|,
// |B| < 2^47); the value is A + 2^32 B == S + 2^32 lo(B) with
// S = A + hi(B) (2^32 - 1) (2^64 == 2^32 - 1 mod p), |S| < 2^48.  With
// U = S + 2^32 lo(B) in (-2^48, 2^64 + 2^48), R = U mod 2^64 and
// U = R + k 2^64, k = carry - [S < 0] in {-1, 0, 1}: the value is
// R + k (2^32 - 1), which stays inside [0, 2^64) in each case (k = 1 only
// when R < 2^48, k = -1 only when R > 2^64 - 2^48).
LC_D uint64_t tn_fold(const uint32_t (&d)[8][8], int u) {
  // limb pairs in 32 bits: |D| < 2^21 (s8 digits) or 0 <= D < 2^22 (u8), so
  // D_l + 2^8 D_(l+1) stays inside int32
  const int32_t p01 = (int32_t)d[0][u] + (int32_t)d[1][u] * 256;
  const int32_t p23 = (int32_t)d[2][u] + (int32_t)d[3][u] * 256;
  const int32_t p45 = (int32_t)d[4][u] + (int32_t)d[5][u] * 256;
  const int32_t p67 = (int32_t)d[6][u] + (int32_t)d[7][u] * 256;
  const int64_t A = (int64_t)p01 + (int64_t)p23 * 65536;
  const int64_t B = (int64_t)p45 + (int64_t)p67 * 65536;
  const int64_t S = A + (B >> 32) * (int64_t)kGlEps;
  const uint64_t lo = (uint64_t)(uint32_t)B << 32;
  const uint64_t R = (uint64_t)S + lo;
  const int k = (int)(R < lo) - (int)(S < 0);
  return R + (uint64_t)(int64_t)k * kGlEps;
}

template <bool S8>
__global__ void __launch_bounds__(kTnThreads, 1)
    tc_ntt_kernel(const __grid_constant__ CUtensorMap wmap, const __grid_constant__ TnParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kTnOffBar);
  uint64_t* loaded = bars;        // [4] A tile of a slot landed (tx bytes)
  uint64_t* freed = bars + 4;     // [4] the MMAs that read a slot finished
  uint64_t* acc_full = bars + 8;  // MMAs of a ring element finished
  uint64_t* acc_empty = bars + 9; // the epilogue warps read TMEM
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 10);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 11);
  uint64_t* all_done = bars + 12;  // final commit: every MMA issued has finished
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int s = 0; s < kTnSlots; ++s) {
      mbar_init(&loaded[s], 1);
      mbar_init(&freed[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kTnEpiWarps);
    mbar_init(all_done, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  constexpr int kTmaWarp = kTnEpiWarps, kMmaWarp = kTnEpiWarps + 1;
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // the two limb-group tiles, already in their swizzled layout
  uint4* vs = reinterpret_cast<uint4*>(base + kTnOffV);
  for (int i = tid; i < 2 * kTnVTile / 16; i += kTnThreads) vs[i] = __ldg(p.vimg + i);
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const uint64_t n_my = p.items > blockIdx.x ? (p.items - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto a_slot = [&](uint64_t i) { return base + (i % kTnSlots) * kTnATile; };
  auto fail = [&]() {
    record_error(p.err, LC_DEVERR_TIMEOUT);
    *abort_flag = 1;
  };
  int64_t last_loaded = -1;

  if (warp == kTmaWarp) {
    // ---------------- TMA producer
    if (lane == 0) {
      for (uint64_t i = 0; i < n_my && !*abort_flag; ++i) {
        if (i >= kTnSlots && !mbar_wait(&freed[i % kTnSlots], (uint32_t)(((i - kTnSlots) / kTnSlots) & 1))) {
          fail();
          break;
        }
        const uint64_t item = blockIdx.x + i * gridDim.x;
        const uint32_t jb = (uint32_t)(item % p.nblk), bt = (uint32_t)(item / p.nblk);
        mbar_arrive_expect_tx(&loaded[i % kTnSlots], kTnATile);
        tma_load_3d(a_slot(i), &wmap, 0, (int)(bt * p.BB), (int)(jb * p.R), &loaded[i % kTnSlots]);
        last_loaded = (int64_t)i;
      }
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issuer
    if (lane == 0) {
      for (uint64_t i = 0; i < n_my && !*abort_flag; ++i) {
        if (!mbar_wait(&loaded[i % kTnSlots], (uint32_t)((i / kTnSlots) & 1))) {
          fail();
          break;
        }
        if (i >= 1 && !mbar_wait(acc_empty, (uint32_t)((i - 1) & 1))) {  // the epilogue read the last item
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t aa = smem_u32(a_slot(i));
#pragma unroll
        for (int g = 0; g < 2; ++g) {
          const uint32_t va = smem_u32(base + kTnOffV + g * kTnVTile);
#pragma unroll
          for (int ks = 0; ks < 2; ++ks)
            mma_i8(tmem + g * 256, umma_desc_sw64(aa + 32 * ks), umma_desc_sw128(va + 32 * ks),
                   TcIdesc<S8>::value, ks > 0 ? 1u : 0u);
        }
        mma_commit(acc_full);
        mma_commit(&freed[i % kTnSlots]);
      }
      mma_commit(all_done);
      if (!mbar_wait(all_done, 0)) fail();
    }
  } else {
    // ---------------- epilogue: warp w reads TMEM lanes 32 (w % 4).., slots 16 (w / 4)..
    // row = (ring element jl, witness bb), witness fastest: a warp's 32 rows
    // are 32 consecutive What_T entries of one slot
    const uint32_t q = warp & 3, part = warp >> 2;
    const uint32_t row = 32 * q + lane;
    const uint32_t jl = row / p.BB, bb = row % p.BB;
    for (uint64_t i = 0; i < n_my; ++i) {
      const uint64_t item = blockIdx.x + i * gridDim.x;
      const uint32_t jb = (uint32_t)(item % p.nblk), bt = (uint32_t)(item / p.nblk);
      const uint32_t b = bt * p.BB + bb;
      {
        // warp-uniform decision: the TMEM loads below are .sync.aligned
        const bool ok = !*abort_flag && mbar_wait(acc_full, (uint32_t)(i & 1));
        if (!__all_sync(0xffffffffu, ok)) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t j = jb * p.R + jl;
        const bool valid = b < p.b_pad && j < p.m;
        const size_t stride = (size_t)p.m * p.b_pad;  // one slot t
        uint64_t* dst = p.what_t + (size_t)(16 * part) * stride + (size_t)j * p.b_pad + b;
#pragma unroll 1
        for (int tb = 0; tb < 2; ++tb) {
          const uint32_t t0 = 16 * part + 8 * tb;
          uint32_t d[8][8];
#pragma unroll
          for (int l = 0; l < 8; ++l) tmem_ld8(tmem + ((32 * q) << 16) + (l >> 2) * 256 + (l & 3) * 64 + t0, d[l]);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (tb == 1) {
            // this warp's accumulator columns are all in registers: the next
            // item's MMAs may overwrite them while the fold runs
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (valid) *dst = tn_fold(d, u);
            dst += stride;
          }
        }
      }
    }
  }
  // ---------------- nothing in flight when TMEM and shared memory go
  __syncthreads();
  if (warp == kTmaWarp && lane == 0) {
    for (int64_t i = last_loaded >= kTnSlots - 1 ? last_loaded - (kTnSlots - 1) : 0; i <= last_loaded; ++i)
      mbar_wait(&loaded[i % kTnSlots], (uint32_t)((i / kTnSlots) & 1));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ------------------------------------------------------------------ host side

}  // namespace lc

struct lc_tc_tables {
  uint8_t* fkey = nullptr;
  uint32_t k = 0, m = 0, m_pad = 0, groups = 0;
  int64_t* partial = nullptr;
  size_t partial_bytes = 0;
};

namespace lc {

void tc_tables_destroy(lc_tc_tables* t) {
  if (!t) return;
  if (t->fkey) cudaFree(t->fkey);
  if (t->partial) cudaFree(t->partial);
  delete t;
}

int tc_tables_create(const uint64_t* matrix_dev, uint32_t k, uint32_t m, lc_tc_tables** out) {
  lc_tc_tables* t = new (std::nothrow) lc_tc_tables();
  if (!t) return LC_ERR_OUT_OF_MEMORY;
  t->k = k;
  t->m = m;
  t->m_pad = (m + 1) & ~1u;
  t->groups = (k + 3) / 4;
  const size_t bytes = (size_t)t->groups * 4 * t->m_pad * 8 * kTcFRow;
  if (cudaMalloc(&t->fkey, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete t;
    return LC_ERR_OUT_OF_MEMORY;
  }
  const int sms = device_sm_count();
  tc_key_tables_kernel<<<std::max(sms, 1) * 8, 256>>>(matrix_dev, t->fkey, k, m, t->m_pad, t->groups);
  const int rc = map_cuda(cudaGetLastError());
  if (rc) {
    tc_tables_destroy(t);
    return rc;
  }
  *out = t;
  return LC_OK;
}

size_t tc_tables_bytes(const lc_tc_tables* t) {
  return t ? (size_t)t->groups * 4 * t->m_pad * 8 * kTcFRow : 0;
}

int tc_commit(lc_tc_tables* t, const void* w, bool s8, size_t batch, uint64_t* out, uint32_t* err,
              cudaStream_t st) {
  if (batch == 0) return LC_OK;
  const int jper = s8 ? TcJPer<true>::value : TcJPer<false>::value;
  if (reinterpret_cast<uintptr_t>(w) & 15) return LC_ERR_INVALID_ARGUMENT;
  if (batch > (1u << 24)) return LC_ERR_INVALID_ARGUMENT;
  EncodeTiledFn enc = encode_fn();
  if (!enc) return LC_ERR_UNSUPPORTED;
  const uint32_t btiles = (uint32_t)((batch + 127) / 128);
  const uint32_t splits = (t->m_pad + jper - 1) / jper;
  // grid z = splits * btiles; TMA x coordinate j*64 is a signed 32-bit int
  if ((size_t)splits * btiles > 65535 || (size_t)t->m_pad * 64 > 0x7FFFFFFF) return LC_ERR_UNSUPPORTED;
  const size_t pbytes = (size_t)splits * 4 * t->groups * btiles * 256 * 128 * sizeof(int64_t);
  if (pbytes > t->partial_bytes) {
    if (t->partial) cudaFree(t->partial);
    t->partial = nullptr;
    t->partial_bytes = 0;
    if (cudaMalloc(&t->partial, pbytes) != cudaSuccess) {
      cudaGetLastError();
      return LC_ERR_OUT_OF_MEMORY;
    }
    t->partial_bytes = pbytes;
  }
  // W as a 2-D byte array [batch][m*64]; box 128 bytes x 128 rows, 128-byte
  // swizzle; columns past m*64 (odd m) and rows past batch read as zero.
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)t->m * 64, (cuuint64_t)batch};
  const cuuint64_t strides[1] = {(cuuint64_t)t->m * 64};
  const cuuint32_t box[2] = {128, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(w), dims, strides, box,
                          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return LC_ERR_INVALID_ARGUMENT;
  auto kern = s8 ? tc_commit_kernel<true> : tc_commit_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return map_cuda(e);
  const TcParams prm{t->fkey, t->partial, t->m_pad, t->groups, splits, btiles, err};
  kern<<<dim3(4, t->groups, splits * btiles), kTcThreads, kTcSmem, st>>>(map, prm);
  int rc = map_cuda(cudaGetLastError());
  if (rc) return rc;
  const size_t total = (size_t)t->groups * btiles * 256 * 128;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, (size_t)device_sm_count() * 16);
  tc_reduce_kernel<<<blocks, 256, 0, st>>>(t->partial, out, (uint32_t)batch, t->k, t->groups, splits, btiles);
  return map_cuda(cudaGetLastError());
}


// The limb tiles of V in their shared-memory image: tile g, row n = 64 (l - 4g) + t,
// 16-byte chunk c16 of the 128-byte row at n*128 + ((c16 ^ (n & 7)) << 4);
// bytes 0..63 hold limb l of V[t][c], bytes 64..127 are zero.
static void tn_build_image(std::vector<uint8_t>& img) {
  img.assign(2 * kTnVTile, 0);
  auto mulp = [](uint64_t a, uint64_t b) { return (uint64_t)((unsigned __int128)a * b % kGlP); };
  auto powp = [&](uint64_t x, uint64_t e) {
    uint64_t r = 1;
    while (e) {
      if (e & 1) r = mulp(r, x);
      x = mulp(x, x);
      e >>= 1;
    }
    return r;
  };
  const uint64_t psi = powp(7, (kGlP - 1) >> 7);  // primitive 128th root (generator 7)
  for (int g = 0; g < 2; ++g)
    for (int n = 0; n < 256; ++n) {
      const int l = 4 * g + n / 64, t = n % 64;
      for (int c = 0; c < 64; ++c) {
        const uint64_t v = powp(psi, (uint64_t)((2 * t + 1) * c) % 128);
        const int c16 = c / 16;
        img[(size_t)g * kTnVTile + n * 128 + ((c16 ^ (n & 7)) << 4) + c % 16] = (uint8_t)(v >> (8 * l));
      }
    }
}

static std::mutex g_tn_mu;
static uint4* g_tn_img[64] = {};

int tc_ntt_prepare() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return LC_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(g_tn_mu);
  if (g_tn_img[dev]) return LC_OK;
  std::vector<uint8_t> img;
  tn_build_image(img);
  uint4* d = nullptr;
  if (cudaMalloc(&d, img.size()) != cudaSuccess) {
    cudaGetLastError();
    return LC_ERR_OUT_OF_MEMORY;
  }
  if (cudaMemcpy(d, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d);
    return LC_ERR_CUDA;
  }
  g_tn_img[dev] = d;
  return LC_OK;
}

int tc_witness_ntt(const void* w, bool s8, size_t batch, uint32_t m, uint32_t b_pad, uint64_t* what_t,
                   uint32_t* err, cudaStream_t st) {
  if (batch == 0) return LC_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return LC_ERR_UNSUPPORTED;
  }
  const uint4* img = g_tn_img[dev];
  EncodeTiledFn enc = encode_fn();
  if (!img || !enc || (reinterpret_cast<uintptr_t>(w) & 15)) return LC_ERR_UNSUPPORTED;
  if ((size_t)m * b_pad < ((size_t)1 << 16) || (size_t)m * 64 > 0x7FFFFFFF) return LC_ERR_UNSUPPORTED;
  // M tile: R consecutive ring elements x BB witnesses, witness fastest
  uint32_t BB;
  if (b_pad % 128 == 0)
    BB = 128;
  else if (b_pad < 128 && (b_pad & (b_pad - 1)) == 0)
    BB = b_pad;
  else
    return LC_ERR_UNSUPPORTED;
  const uint32_t R = 128 / BB;
  const uint32_t nblk = (m + R - 1) / R;
  const uint64_t items = (uint64_t)(b_pad / BB) * nblk;
  // w[b][j][64] as a 3-D byte array: x = digit c, y = witness b, z = ring
  // element j; rows past batch or past m read as zero
  CUtensorMap map;
  const cuuint64_t dims[3] = {64, (cuuint64_t)batch, (cuuint64_t)m};
  const cuuint64_t strides[2] = {(cuuint64_t)m * 64, 64};
  const cuuint32_t box[3] = {64, BB, R};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(w), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return LC_ERR_UNSUPPORTED;
  auto kern = s8 ? tc_ntt_kernel<true> : tc_ntt_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTnSmem);
  if (e != cudaSuccess) return map_cuda(e);
  const TnParams prm{img, what_t, m, b_pad, (uint32_t)batch, BB, R, nblk, items, err};
  const unsigned grid = (unsigned)std::min<uint64_t>(items, (uint64_t)std::max(1, device_sm_count()));
  kern<<<grid, kTnThreads, kTnSmem, st>>>(map, prm);
  return map_cuda(cudaGetLastError());
}

}  // namespace lc

namespace lc {

// ------------------------------------------------------------------ slot products on the tensor cores
//
// The NTT engine's per-slot products C_t[i][b] = sum_j Ahat[i][j][t] What[b][j][t]
// (mod q) as exact unsigned byte GEMMs.  With both residues split into L byte
// limbs (L = 8 for Goldilocks, 4 for u32 moduli),
// C_t = sum_{la,lw} 2^(8 (la + lw)) D_t[(i,la)][(b,lw)] and
//   D_t[(i,la)][(b,lw)] = sum_j Ahat_la[i][j][t] * What_lw[b][j][t]   (u8 x u8 -> s32),
// exact for at most 32768 ring elements j per sum (32768 * 255^2 < 2^31).
// The cached key Ahat_T[t][j][16] is, read as bytes, the A operand of slot t
// in MN-major form: row j (the K index) holds the 16 L bytes (i, la), la
// fastest; What_T[t][j][b_pad] is the B operand the same way, L b_pad bytes
// (b, lw) per row.  3-D TMA maps (x = bytes of a row, y = j < m, z = slot)
// load 64-row stages with the swizzle of the row width (128, 64 or 32 bytes),
// the MN-major canonical layout of the MMA descriptors (SBO = 8 rows, LBO =
// next atom along M/N); rows past m read as zero.  For u32 keys the 64-byte A
// rows fill half of M = 128: the descriptor's second A atom is a zero tile.
// CTA (slot, N tile of up to 512 bytes, K split): one TMA thread, one MMA
// thread (M = 128, N <= 256 per accumulator, K = 32), four epilogue warps
// writing D transposed so that the lanes (rows (i, la)) store contiguously;
// a second kernel sums the splits and limbs and reduces into Chat[b][i][t].
constexpr int kSpStages = 4;
constexpr int kSpRows = 64;          // K rows (ring elements j) per stage
constexpr uint32_t kSpKSplit = 32768;  // ring elements per exact int32 sum
constexpr int kSpThreads = 192;      // warp 0 TMA, 1 MMA + TMEM, 2..5 epilogue

template <int NCTA, int AW>
struct SpCfg {
  static constexpr int SW = NCTA >= 128 ? 128 : NCTA;  // B swizzle atom (bytes of a row): 128, 64 or 32
  static constexpr int ATOMS = NCTA / SW;
  static constexpr int MMA_N = NCTA > 256 ? 256 : NCTA;
  static constexpr int ACCS = NCTA / MMA_N;
  static constexpr int A_LOAD = kSpRows * AW;    // bytes TMA writes per stage (AW = 128 or 64)
  static constexpr int A_BYTES = kSpRows * 128;  // A region: for AW = 64 the zero atom follows
  static constexpr int B_ATOM = kSpRows * SW;
  static constexpr int STAGE = A_BYTES + ATOMS * B_ATOM;
  static constexpr size_t SMEM = 1024 + (size_t)kSpStages * STAGE + 128;
  static constexpr uint32_t A_LAYOUT = AW == 128 ? 2u : 4u;
  static constexpr uint32_t B_LAYOUT = SW == 128 ? 2u : SW == 64 ? 4u : 6u;
  static_assert(AW == 128 || AW == 64, "row bytes of the key");
  static_assert(SW == 128 || SW == 64 || SW == 32, "swizzle atom");
  static_assert(STAGE % 1024 == 0 && B_ATOM % 256 == 0, "swizzle atoms stay aligned");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// D = s32, A = B = u8, both MN-major (bits 15, 16), M = 128
template <int N>
struct SpIdesc {
  static constexpr uint32_t value =
      (2u << 4) | (1u << 15) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
};

struct SpParams {
  int32_t* partial;  // [split][t][ntile][NCTA][128]
  uint32_t m, nslots, ntiles, splits;
  uint32_t* err;
};

template <int NCTA, int AW>
__global__ void __launch_bounds__(kSpThreads, 1)
    slot_products_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap wmap,
                         const __grid_constant__ SpParams p) {
  using C = SpCfg<NCTA, AW>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kSpStages * C::STAGE);
  uint64_t* full = bars;                   // [4] stage landed (tx bytes)
  uint64_t* empty = bars + kSpStages;      // [4] its MMAs finished
  uint64_t* done = bars + 2 * kSpStages;   // every MMA finished
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kSpStages + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 2 * kSpStages + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t t = blockIdx.x, nt = blockIdx.y, split = blockIdx.z;
  const uint32_t j0 = split * kSpKSplit;
  const uint32_t j1 = min(p.m, j0 + kSpKSplit);
  const int nst = (int)((j1 - j0 + kSpRows - 1) / kSpRows);

  if (tid == 0) {
    for (int s = 0; s < kSpStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if constexpr (AW == 64) {
    // the second A atom of every stage: rows (i, la) 64..127 are zero
    for (int s = 0; s < kSpStages; ++s) {
      uint4* z = reinterpret_cast<uint4*>(base + s * C::STAGE + C::A_LOAD);
      for (int e = tid; e < (C::A_BYTES - C::A_LOAD) / 16; e += kSpThreads) z[e] = make_uint4(0, 0, 0, 0);
    }
    fence_proxy_async_smem();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(NCTA < 32 ? 32 : NCTA));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto stage = [&](int s) { return base + (s % kSpStages) * C::STAGE; };
  auto fail = [&]() {
    record_error(p.err, LC_DEVERR_TIMEOUT);
    *abort_flag = 1;
  };
  int last_loaded = -1, last_mma = -1;

  if (warp == 0) {
    // ---------------- TMA: A rows (i, la) and the B atoms of this N tile
    if (lane == 0) {
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (s >= kSpStages && !mbar_wait(&empty[s % kSpStages], (uint32_t)(((s - kSpStages) / kSpStages) & 1))) {
          fail();
          break;
        }
        unsigned char* st = stage(s);
        const int y = (int)(j0 + kSpRows * s);
        mbar_arrive_expect_tx(&full[s % kSpStages], (uint32_t)(C::A_LOAD + C::ATOMS * C::B_ATOM));
        tma_load_3d(st, &amap, 0, y, (int)t, &full[s % kSpStages]);
#pragma unroll
        for (int a = 0; a < C::ATOMS; ++a)
          tma_load_3d(st + C::A_BYTES + a * C::B_ATOM, &wmap, (int)(nt * NCTA + a * C::SW), y, (int)t,
                      &full[s % kSpStages]);
        last_loaded = s;
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      for (int s = 0; s < nst && !*abort_flag; ++s) {
        if (!mbar_wait(&full[s % kSpStages], (uint32_t)((s / kSpStages) & 1))) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(stage(s)), sb = sa + C::A_BYTES;
#pragma unroll
        for (int ks = 0; ks < kSpRows / 32; ++ks) {
#pragma unroll
          for (int acc = 0; acc < C::ACCS; ++acc) {
            // A: one 128-byte atom, or (AW = 64) the key's atom and the zero atom C::A_LOAD later
            const uint64_t ad = umma_desc_mn(sa + ks * 32 * AW, C::A_LOAD, 8 * AW, C::A_LAYOUT);
            const uint64_t bd = umma_desc_mn(sb + acc * (C::MMA_N / C::SW) * C::B_ATOM + ks * 32 * C::SW,
                                             C::B_ATOM, 8 * C::SW, C::B_LAYOUT);
            mma_i8(tmem + acc * C::MMA_N, ad, bd, SpIdesc<C::MMA_N>::value, (s > 0 || ks > 0) ? 1u : 0u);
          }
        }
        mma_commit(&empty[s % kSpStages]);
        last_mma = s;
      }
      if (last_mma >= 0) mma_commit(done);
    }
  } else {
    // ---------------- epilogue: lane = row (i, la); column = (b, lw)
    const bool ok = nst > 0 && !*abort_flag && mbar_wait(done, 0);
    if (__all_sync(0xffffffffu, ok)) {
      tc_fence_after();
      const uint32_t lq = warp & 3, row = 32 * lq + lane;
      int32_t* out = p.partial + (((size_t)split * p.nslots + t) * p.ntiles + nt) * (size_t)NCTA * 128;
#pragma unroll 1
      for (int c0 = 0; c0 < NCTA; c0 += 16) {
        uint32_t d[16];
        tmem_ld16(tmem + ((32 * lq) << 16) + c0, d);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int u = 0; u < 16; ++u) out[(size_t)(c0 + u) * 128 + row] = (int32_t)d[u];
      }
    } else if (nst > 0 && lane == 0) {
      fail();
    }
  }
  // ---------------- nothing in flight when TMEM and shared memory go
  __syncthreads();
  if (warp == 0 && lane == 0) {
    for (int s = max(0, last_loaded - (kSpStages - 1)); s <= last_loaded; ++s)
      mbar_wait(&full[s % kSpStages], (uint32_t)((s / kSpStages) & 1));
  }
  if (warp == 1 && lane == 0 && last_mma >= 0) mbar_wait(done, 0);
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCTA < 32 ? 32 : NCTA));
  }
}

// Chat[b][i][t] = sum_{la,lw} 2^(8 (la + lw)) sum_split D[split][t][nt][(bl, lw)][(i, la)]  mod q.
// Pair sums over the splits fit 64 bits (< 2^31 * splits); the 2L - 1 sums of
// equal la + lw = k are folded with 2^(8k) mod q (128 bits for Goldilocks,
// 64-bit remainders for u32 q).
template <class E>
__global__ void slot_products_reduce_kernel(const int32_t* __restrict__ part, E* __restrict__ chat, uint32_t n,
                                            uint32_t kappa, uint32_t batch, uint32_t ncta, uint32_t ntiles,
                                            uint32_t splits, uint32_t q) {
  constexpr int L = sizeof(E);
  const size_t total = (size_t)n * batch * kappa;
  const uint32_t wpt = ncta / L;  // witnesses per N tile
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = idx % kappa;
    const uint32_t b = (uint32_t)((idx / kappa) % batch);
    const uint32_t t = (uint32_t)(idx / ((size_t)kappa * batch));
    const uint32_t nt = b / wpt, bl = b % wpt;
    uint64_t tk[2 * L - 1];
#pragma unroll
    for (int k = 0; k < 2 * L - 1; ++k) tk[k] = 0;
    for (uint32_t sp = 0; sp < splits; ++sp) {
      const int32_t* d = part + (((size_t)sp * n + t) * ntiles + nt) * (size_t)ncta * 128;
#pragma unroll
      for (int lw = 0; lw < L; ++lw) {
        const int32_t* col = d + (size_t)(bl * L + lw) * 128 + i * L;
#pragma unroll
        for (int la = 0; la < L; ++la) tk[la + lw] += (uint64_t)(uint32_t)col[la];
      }
    }
    E res;
    if constexpr (L == 8) {
      unsigned __int128 v = 0;
      uint64_t c = 1;  // 2^(8k) mod p
#pragma unroll
      for (int k = 0; k < 2 * L - 1; ++k) {
        v += (unsigned __int128)tk[k] * c;
        c = gl_mul(c, 256);
      }
      res = gl_canon(gl_reduce128_lazy((uint64_t)(v >> 64), (uint64_t)v));
    } else {
      uint64_t v = 0, c = 1 % q;  // 2^(8k) mod q
#pragma unroll
      for (int k = 0; k < 2 * L - 1; ++k) {
        v = (v + (tk[k] % q) * c % q) % q;  // each term < q < 2^32 before the sum
        c = (c << 8) % q;
      }
      res = (E)v;
    }
    chat[((size_t)b * kappa + i) * n + t] = res;
  }
}

template <int NCTA, int AW>
static int launch_slot_products(const CUtensorMap& amap, const CUtensorMap& wmap, const SpParams& prm,
                                cudaStream_t st) {
  auto kern = slot_products_kernel<NCTA, AW>;
  using C = SpCfg<NCTA, AW>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return map_cuda(e);
  kern<<<dim3(prm.nslots, prm.ntiles, prm.splits), kSpThreads, C::SMEM, st>>>(amap, wmap, prm);
  return map_cuda(cudaGetLastError());
}

template <int AW>
static int launch_slot_products_n(uint32_t ncta, const CUtensorMap& amap, const CUtensorMap& wmap,
                                  const SpParams& prm, cudaStream_t st) {
  switch (ncta) {
    case 512: return launch_slot_products<512, AW>(amap, wmap, prm, st);
    case 256: return launch_slot_products<256, AW>(amap, wmap, prm, st);
    case 128: return launch_slot_products<128, AW>(amap, wmap, prm, st);
    case 64: return launch_slot_products<64, AW>(amap, wmap, prm, st);
    case 32: return launch_slot_products<32, AW>(amap, wmap, prm, st);
    default: return LC_ERR_UNSUPPORTED;
  }
}

int tc_slot_products(const void* ahat_t, uint32_t a_m, const void* what_t, uint32_t elem_bytes, uint32_t q,
                     uint32_t m, uint32_t n, uint32_t kappa, size_t batch, uint32_t b_pad, void** part,
                     size_t* part_bytes, void* chat, uint32_t* err, cudaStream_t st) {
  if (batch == 0) return LC_OK;
  EncodeTiledFn enc = encode_fn();
  if (!enc || kappa > 16 || m == 0 || (elem_bytes != 8 && elem_bytes != 4)) return LC_ERR_UNSUPPORTED;
  // N tile: 512 bytes, or the whole row when it is 32, 64, 128 or 256 bytes
  const uint64_t row = (uint64_t)elem_bytes * b_pad;
  uint32_t ncta;
  if (row % 512 == 0)
    ncta = 512;
  else if (row == 256 || row == 128 || row == 64 || row == 32)
    ncta = (uint32_t)row;
  else
    return LC_ERR_UNSUPPORTED;
  const uint64_t ntiles = row / ncta;
  const uint32_t splits = (m + kSpKSplit - 1) / kSpKSplit;
  if (ntiles > 65535 || splits > 65535) return LC_ERR_UNSUPPORTED;  // grid y, z
  const size_t need = (size_t)splits * n * ntiles * ncta * 128 * sizeof(int32_t);
  if (need > *part_bytes) {
    if (*part) cudaFree(*part);
    *part = nullptr;
    *part_bytes = 0;
    if (cudaMalloc(part, need) != cudaSuccess) {
      cudaGetLastError();
      return LC_ERR_OUT_OF_MEMORY;
    }
    *part_bytes = need;
  }
  // A: bytes (i, la) of Ahat_T[t][j][16]; B: bytes (b, lw) of What_T[t][j][b_pad]
  const uint32_t aw = 16 * elem_bytes;
  CUtensorMap amap, wmap;
  const cuuint32_t estr[3] = {1, 1, 1};
  {
    const cuuint64_t dims[3] = {aw, (cuuint64_t)m, (cuuint64_t)n};
    const cuuint64_t strides[2] = {aw, (cuuint64_t)a_m * aw};
    const cuuint32_t box[3] = {aw, (cuuint32_t)kSpRows, 1};
    if (enc(&amap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(ahat_t), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, aw == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return LC_ERR_UNSUPPORTED;
  }
  {
    const cuuint64_t dims[3] = {row, (cuuint64_t)m, (cuuint64_t)n};
    const cuuint64_t strides[2] = {row, (cuuint64_t)m * row};
    const cuuint32_t sw = ncta >= 128 ? 128 : ncta;
    const cuuint32_t box[3] = {sw, (cuuint32_t)kSpRows, 1};
    const CUtensorMapSwizzle swz = sw == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : sw == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    if (enc(&wmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(what_t), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return LC_ERR_UNSUPPORTED;
  }
  const SpParams prm{static_cast<int32_t*>(*part), m, n, (uint32_t)ntiles, splits, err};
  int rc = aw == 128 ? launch_slot_products_n<128>(ncta, amap, wmap, prm, st)
                     : launch_slot_products_n<64>(ncta, amap, wmap, prm, st);
  if (rc) return rc;
  const size_t total = (size_t)n * batch * kappa;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, (size_t)device_sm_count() * 16);
  if (elem_bytes == 8)
    slot_products_reduce_kernel<uint64_t><<<blocks, 256, 0, st>>>(
        static_cast<const int32_t*>(*part), static_cast<uint64_t*>(chat), n, kappa, (uint32_t)batch, ncta,
        (uint32_t)ntiles, splits, q);
  else
    slot_products_reduce_kernel<uint32_t><<<blocks, 256, 0, st>>>(
        static_cast<const int32_t*>(*part), static_cast<uint32_t*>(chat), n, kappa, (uint32_t)batch, ncta,
        (uint32_t)ntiles, splits, q);
  return map_cuda(cudaGetLastError());
}

}  // namespace lc

// ------------------------------------------------------------------ INT8 tensor rate
//
// Measurement kernel for the INT8 tensor roofline: one CTA per SM keeps its
// tensor pipe busy with tcgen05.mma.kind::i8 of the commit engines' shape
// (M = 128, N = 256, K = 32, int32 accumulators in TMEM) on operands that
// stay in shared memory, with no global traffic.  One MMA is 2*128*256*32
// integer operations; the products are discarded.
namespace lc {

constexpr int kRateThreads = 128;
constexpr int kRateOperandBytes = 128 * 128 + 256 * 128;  // A tile, B tile (K = 128 bytes each)
// more shared memory than two CTAs could hold: one CTA per SM
constexpr size_t kRateSmem = 116 * 1024;
static_assert(1024 + kRateOperandBytes + 64 <= (int)kRateSmem, "rate kernel layout");

static __device__ uint32_t g_rate_err;

template <bool S8>
__global__ void __launch_bounds__(kRateThreads, 1) tc_rate_kernel(uint32_t iters) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* done = reinterpret_cast<uint64_t*>(base + kRateOperandBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  uint32_t* words = reinterpret_cast<uint32_t*>(base);
  for (int i = tid; i < kRateOperandBytes / 4; i += kRateThreads) words[i] = 0x9E3779B9u * (uint32_t)(i + 1);
  if (tid == 0) {
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (tid == 0) {
    const uint32_t sa = smem_u32(base), sb = smem_u32(base + 128 * 128);
    for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        mma_i8(tmem, umma_desc_sw128(sa + 32 * ks), umma_desc_sw128(sb + 32 * ks), TcIdesc<S8>::value,
               (it | (uint32_t)ks) ? 1u : 0u);
    }
    mma_commit(done);
    if (!mbar_wait(done, 0)) record_error(&g_rate_err, LC_DEVERR_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
  }
}

}  // namespace lc

extern "C" {

LC_API int lc_tc_i8_rate(uint32_t iters, int s8, double* ops_per_s, float* ms) {
  if (!ops_per_s || iters == 0 || iters > (1u << 24)) return LC_ERR_INVALID_ARGUMENT;
  const int sms = lc::device_sm_count();
  if (sms <= 0) return LC_ERR_NO_DEVICE;
  auto kern = s8 ? lc::tc_rate_kernel<true> : lc::tc_rate_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lc::kRateSmem);
  if (e != cudaSuccess) return lc::map_cuda(e);
  uint32_t* err = nullptr;
  e = cudaGetSymbolAddress(reinterpret_cast<void**>(&err), lc::g_rate_err);
  if (e != cudaSuccess) return lc::map_cuda(e);
  cudaStream_t st = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  float t = 0.f;
  uint32_t flag = 0;
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 4, st);
  if (e == cudaSuccess) {
    kern<<<sms, lc::kRateThreads, lc::kRateSmem, st>>>(iters / 8 + 1);  // warm-up
    cudaEventRecord(a, st);
    kern<<<sms, lc::kRateThreads, lc::kRateSmem, st>>>(iters);
    cudaEventRecord(b, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  if (e == cudaSuccess) e = cudaMemcpy(&flag, err, 4, cudaMemcpyDeviceToHost);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) return lc::map_cuda(e);
  if (flag) return LC_ERR_TIMEOUT;
  *ops_per_s = 2.0 * 128 * 256 * 32 * 4 * (double)iters * sms / (t * 1e-3);
  if (ms) *ms = t;
  return LC_OK;
}

}  // extern "C"
