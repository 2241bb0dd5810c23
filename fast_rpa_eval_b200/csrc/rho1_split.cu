// Split-precision rho1: the contraction work1 = P1c * phi on the 5th-generation
// tensor cores (tcgen05, BF16 in, FP32 accumulate in TMEM) at FP64-grade
// accuracy, with the per-point dot products in FP64.
//
// Same semantics as the plain FP64 path (rho1_fp64.cu,
// fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho.cpp:116-209).
//
// Numerics.  Every FP64 operand element x of a row with power-of-two scale
// 2^e >= max|x| is written as y = x 2^-e in [-1, 1] and split into five BF16
// slices, y ~ 2^-7 (S0 + S1 + S2 + S3 + S4), S_s = a_s 2^(-8 s), with integer
// digits |a_0| <= 128 (7 bits) and |a_s| <= 128 (8 bits, round to nearest) --
// 39 bits in all, each slice exact in BF16.  The product of two split rows is
// summed as 15 slice products (s + t <= 4) in four FP32 TMEM accumulators, one
// per slice level s + t:
//   acc0 = S0 S0,  acc1 = S0 S1 + S1 S0,  acc2 = S0 S2 + S1 S1 + S2 S0   (exact)
//   acc3 = the levels 3 and 4                                           (rounded)
// and recombined in FP64: work1(i, p) = 2^(eA_p + eB_i - 14) (acc0 + acc1 + acc2 + acc3).
// The three exact levels are integer sums (in units of their level) of at most
// 2^14, 2^15 and 3 2^14 per K step, so they cannot leave the FP32 integer range
// for K <= 1024, 512 and 341; past those bounds they stay exact unless the sums
// of residual digits (which behave like random signs) grow ~100x beyond their
// typical size.  Only levels 3-4, 2^-24 below the result, see the tensor core's
// FP32 truncation.  The benchmark recipes give normwise errors of ~2e-11.
//
// Data flow (one persistent CTA per SM, warp-specialised, 512 threads):
//   * a work item is one batch's tile of <= 128 points; the MMA computes
//     D[p, i] = sum_k Phi^T[p, k] P1c^T[k, i] (M = 128 points, N = 128 rows i,
//     K = 16 per instruction), so each TMEM lane is one grid point and the
//     epilogue's per-point sums need no cross-thread reduction;
//   * 8 producer warps read phi (FP64) and gather P1c (FP64), scale, split and
//     store the 10 slice tiles of a 32-wide K chunk in shared memory
//     (canonical K-major layout, no swizzle) -- a two-stage ring;
//   * epilogue warp 0 owns TMEM (512 columns = 4 accumulators x 128) and its
//     lane 0 issues the 15 x 2 tcgen05.mma per stage, committing to mbarriers
//     (with one accumulator set, a tile's MMAs and its epilogue never overlap);
//   * 8 epilogue warps (two per TMEM lane quarter, each taking half of the
//     columns) read the accumulators (tcgen05.ld), recombine in FP64 and
//     contract with phi and grad phi (FP64, global memory, loads issued a
//     chunk ahead).
// Every mbarrier wait is bounded in time; on a timeout the kernel records an
// error flag, lets in-flight MMAs finish (bounded), frees TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "frpa_internal.cuh"
#include "sm100_sync.cuh"

namespace frpa {
namespace {

constexpr int SP_M = 128;         // points per work item (TMEM lanes)
constexpr int SP_N = 128;         // rows i per N tile (accumulator columns)
constexpr int SP_KC = 32;         // K per pipeline stage
constexpr int SP_STAGES = 2;
constexpr int SP_SLICES = 5;
constexpr int SP_EPI_WARPS = 8;   // warps 0..7: epilogue (lane quarter w % 4, column half w / 4);
                                  // warp 0 owns TMEM and its lane 0 issues the MMAs
constexpr int SP_PROD_WARPS = 8;  // warps 8..15: producers
constexpr int SP_PROD0 = SP_EPI_WARPS;
constexpr int SP_THREADS = 32 * (SP_EPI_WARPS + SP_PROD_WARPS);
constexpr int SP_PROD_THREADS = 32 * SP_PROD_WARPS;
constexpr int SP_MAX_K = 1024;    // exactness bound of the FP32 levels 0 and 1
constexpr int SP_TILE_ELEMS = SP_M * SP_KC;           // one slice tile (bf16 elements)
constexpr uint32_t SP_LBO = 128;                      // bytes between K-adjacent core matrices
constexpr uint32_t SP_SBO = (SP_KC / 8) * 128;        // bytes between 8-row groups

static_assert(SP_M == 128 && SP_N == 128, "instruction shape");

struct SplitSmem {
  __nv_bfloat16 A[SP_STAGES][SP_SLICES][SP_TILE_ELEMS];
  __nv_bfloat16 B[SP_STAGES][SP_SLICES][SP_TILE_ELEMS];
  double scaleA[2][SP_M];  // 2^(eA - 7) per point, by item parity
  double scaleB[2][SP_N];  // 2^(eB - 7) per row i, by tile parity
  double partial[2][4][SP_M];  // upper column half's per-point sums
  unsigned long long full[SP_STAGES];
  unsigned long long empty[SP_STAGES];
  unsigned long long acc_full;
  unsigned long long acc_empty;
  unsigned long long drain;
  unsigned long long sa_full[2];  // per-point scales of an item published (by item parity)
  unsigned long long sb_full[2];  // per-row scales of a tile published (by tile parity)
  unsigned long long sa_free[2];  // per-point scales released by the epilogue
  unsigned long long sb_free[2];  // per-row scales released by the epilogue
  unsigned long long ep_sum[2];   // partial sums published by the upper column half
  unsigned long long ep_free[2];  // partial-sum buffer released by the lower half
  uint32_t tmem_base;
  int abort_flag;
};

// ---------------------------------------------------------------- PTX glue

using sm100::fence_proxy_async_smem;
using sm100::global_ns;
using sm100::mbar_arrive;
using sm100::mbar_init;
using sm100::mbar_try_wait;
using sm100::mbar_wait;
using sm100::smem_u32;
using sm100::tc_fence_after;
using sm100::tc_fence_before;
using sm100::tmem_wait_ld;
using sm100::umma_commit;
using sm100::warp_wait;

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) { return sm100::smem_desc<SP_LBO, SP_SBO>(addr); }

// Instruction descriptor: kind::f16, D = F32, A = B = BF16, both K-major,
// N = 128, M = 128.
constexpr uint32_t SP_IDESC = (1u << 4)                       // D format F32
                              | (1u << 7)                     // A format BF16
                              | (1u << 10)                    // B format BF16
                              | ((uint32_t)(SP_N >> 3) << 17)  // N
                              | ((uint32_t)(SP_M >> 4) << 24); // M

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(SP_IDESC), "r"(accumulate));
}

// Byte offset of element (row r, k) in a K-major no-swizzle tile of SP_KC columns.
__device__ __forceinline__ int tile_off(int r, int k) {
  return (r >> 3) * SP_SBO + (k >> 3) * SP_LBO + (r & 7) * 16 + (k & 7) * 2;
}

// Five slices of 8 consecutive raw values x (row scale folded into
// sc39 = 2^(39 - e)) written as 16-byte rows into the slice tiles at byte
// offset `off`.  Integer digit extraction, no FP64 rounding or conversion:
//   t = fma(x, sc39, 1.5 2^52) rounds X = rint(y 2^39) into the mantissa:
//       lo word = X mod 2^32, hi word & 0xFFFFF = 2^19 + floor(X / 2^32);
//   X + 0x80808080 = a0 2^32 + sum_i c_i 2^(8 i), c_i bytes in [0, 255], so
//       X = a0 2^32 + sum_i (c_i - 128) 2^(8 i): balanced digits d = c - 128;
//   a digit c becomes the float (c - 128) 2^(-8 s) exactly as
//       fma(bits(0x4B000000 | c), 2^(-8 s), -(2^23 + 128) 2^(-8 s)),
//   and a float with <= 8 significant bits is exact in BF16: its top 16 bits.
__device__ __forceinline__ void split8_store(const double (&x)[8], double sc39,
                                             __nv_bfloat16 (*tiles)[SP_TILE_ELEMS], int off) {
  uint32_t lo[8], f0[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double t = fma(x[j], sc39, 6755399441055744.0);  // 1.5 * 2^52
    const uint32_t l = (uint32_t)__double2loint(t), h = (uint32_t)__double2hiint(t);
    const uint32_t lp = l + 0x80808080u;
    const uint32_t carry = lp < l ? 1u : 0u;
    lo[j] = lp;
    // bits of the float 2^23 + (a0 + 128), a0 = (h & 0xFFFFF) - 2^19 + carry
    f0[j] = (h & 0xFFFFFu) + carry + (0x4B000000u + 128u - 0x80000u);
  }
  {
    uint32_t packed[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const float v0 = __int_as_float((int)f0[j]) - 8388736.0f;  // 2^23 + 128
      const float v1 = __int_as_float((int)f0[j + 1]) - 8388736.0f;
      packed[j / 2] = __byte_perm(__float_as_uint(v0), __float_as_uint(v1), 0x7632);
    }
    *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(tiles[0]) + off) =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
  }
#pragma unroll
  for (int s = 1; s < SP_SLICES; ++s) {
    const float sc = __int_as_float((127 - 8 * s) << 23);  // 2^(-8 s)
    const float bias = -8388736.0f * sc;
    const uint32_t sel = 0x7540u + (uint32_t)(4 - s);     // byte 4 - s of lp, then 0x00, 0x00, 0x4B
    uint32_t packed[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const float v0 = fmaf(__uint_as_float(__byte_perm(lo[j], 0x4B000000u, sel)), sc, bias);
      const float v1 = fmaf(__uint_as_float(__byte_perm(lo[j + 1], 0x4B000000u, sel)), sc, bias);
      packed[j / 2] = __byte_perm(__float_as_uint(v0), __float_as_uint(v1), 0x7632);
    }
    *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(tiles[s]) + off) =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
  }
}

// 2^e >= |m| with e from frexp (e = 0 for m = 0, e >= -960 so that the
// fixed-point factor stays finite); returns {2^(e - 7), 2^(39 - e)}.
__device__ __forceinline__ void pow2_scale(double m, double *scale, double *sc39) {
  int e = 0;
  if (m > 0.0) frexp(m, &e);
  e = max(e, -960);
  *scale = ldexp(1.0, e - 7);
  *sc39 = ldexp(1.0, 39 - e);
}

struct SplitParams {
  const Rho1WorkItem *items;
  int n_items;
  const int *ib_all;
  const int *map;
  int T, n_active, n_basis, n_full_points, n_max_batch_size, n_batches;
  const double *wave, *gwave, *P1, *bias, *gbias;
  const double *rowmax;  // (n_basis, T): max_c |P1(r, c, t)|
  double *rho, *grad;
  int *err;
};

// Producer thread mapping: segment q in [0, 512) of a 128 x 32 tile is
// (row, kseg) = ((q & 7) + 8 (q >> 5), (q >> 3) & 3): a quarter warp stores
// eight rows' 16-byte chunks of one core-matrix column (conflict-free), and
// the four lanes sharing a row are lanes l, l^8, l^16, l^24 of one warp.
// Each producer thread owns segments ptid and ptid + 256 (rows r and r + 64,
// same kseg) of both operand tiles.
__device__ __forceinline__ void seg_of(int q, int *row, int *kseg) {
  *row = (q & 7) + 8 * (q >> 5);
  *kseg = (q >> 3) & 3;
}

// Raw FP64 operands of one stage for one producer thread (2 rows x 8 k).
struct StageRegs {
  double a[2][8];
  double b[2][8];
};

__device__ __forceinline__ void load_a(StageRegs &R, const double *__restrict__ phi, int ncp, int nc, int pn,
                                       const int (&rows)[2], int k) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int j = 0; j < 8; ++j)
      R.a[h][j] = (rows[h] < pn && k + j < nc) ? __ldg(phi + k + j + (long long)rows[h] * ncp) : 0.0;
}

__device__ __forceinline__ void load_b(StageRegs &R, const double *__restrict__ P1t, int n_basis, int nc,
                                       const int (&ibrow)[2], const bool (&rok)[2], const int (&ibk)[8]) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int j = 0; j < 8; ++j)
      R.b[h][j] = (rok[h] && ibk[j] >= 0) ? __ldg(P1t + ibrow[h] + (long long)ibk[j] * n_basis) : 0.0;
}

__device__ __forceinline__ void load_ibk(int (&ibk)[8], const int *__restrict__ ib, int nc, int k) {
#pragma unroll
  for (int j = 0; j < 8; ++j) ibk[j] = (k + j < nc) ? __ldg(ib + k + j) - 1 : -1;
}

__device__ void producer_role(const SplitParams &P, SplitSmem &S, int ptid, int lane) {
  int *err = P.err;
  volatile int *abort_flag = &S.abort_flag;
  const long long nb2 = (long long)P.n_basis * P.n_basis;
  uint32_t fill = 0, tile_ctr = 0, item_ctr = 0;
  int rows[2], kseg;
  seg_of(ptid, &rows[0], &kseg);
  rows[1] = rows[0] + 64;
  for (int it = blockIdx.x; it < P.n_items; it += gridDim.x, ++item_ctr) {
    const Rho1WorkItem W = P.items[it];
    const int nc = W.nc, pn = W.pn, ncp = (nc + 3) & ~3;
    const double *phi = P.wave + W.wave_off + (long long)W.p0 * ncp;
    const int *ib = P.ib_all + W.ib_off;
    const int ip = item_ctr & 1;
    // the epilogue is done with this parity's scales of two items ago
    if (!warp_wait(&S.sa_free[ip], ((item_ctr >> 1) & 1) ^ 1, abort_flag, err, lane)) return;
    // per-point scales: the four lanes sharing a row split its column
    double invA[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = rows[h];
      double m = 0.0;
      if (r < pn) {
        const double *c = phi + (long long)r * ncp;
#pragma unroll 4
        for (int k = kseg; k < nc; k += 4) m = fmax(m, fabs(__ldg(c + k)));
      }
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 8));
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 16));
      double sc;
      pow2_scale(m, &sc, &invA[h]);
      if (kseg == 0) S.scaleA[ip][r] = sc;
    }
    if (kseg == 0) mbar_arrive(&S.sa_full[ip]);
    const int n_nt = (nc + SP_N - 1) / SP_N, n_kc = (nc + SP_KC - 1) / SP_KC;
    const int n_stages = P.T * n_nt * n_kc;  // flattened (t, jn, kc)
    StageRegs R;
    int ibk[8], ibrow[2];
    bool rok[2];
    double invB[2];
    // prologue: operands of the item's first stage
    load_ibk(ibk, ib, nc, 8 * kseg);
    load_a(R, phi, ncp, nc, pn, rows, 8 * kseg);
    for (int st = 0; st < n_stages; ++st, ++fill) {
      const int kc = st % n_kc, jn = (st / n_kc) % n_nt, t = st / (n_kc * n_nt);
      const double *P1t = P.P1 + t * nb2;
      if (kc == 0) {
        // a new N tile: its per-row scales (buffer released by the epilogue)
        const int n0 = jn * SP_N, tp = tile_ctr & 1;
        if (!warp_wait(&S.sb_free[tp], ((tile_ctr >> 1) & 1) ^ 1, abort_flag, err, lane)) return;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = n0 + rows[h];
          rok[h] = i < nc;
          ibrow[h] = rok[h] ? __ldg(ib + i) - 1 : 0;
          const double m = rok[h] ? __ldg(P.rowmax + ibrow[h] + (long long)P.n_basis * t) : 0.0;
          double sc;
          pow2_scale(m, &sc, &invB[h]);
          if (kseg == 0) S.scaleB[tp][rows[h]] = sc;
        }
        if (kseg == 0) mbar_arrive(&S.sb_full[tp]);
        ++tile_ctr;
      }
      load_b(R, P1t, P.n_basis, nc, ibrow, rok, ibk);
      const int stage = fill & 1;
      if (!warp_wait(&S.empty[stage], ((fill >> 1) & 1) ^ 1, abort_flag, err, lane)) return;
      // A half: convert, then start the next stage's A loads
      const int koff = 8 * kseg;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        split8_store(R.a[h], invA[h], S.A[stage], tile_off(rows[h], koff));
      }
      const bool more = st + 1 < n_stages;
      if (more) {
        const int k1 = ((st + 1) % n_kc) * SP_KC + koff;
        load_ibk(ibk, ib, nc, k1);
        load_a(R, phi, ncp, nc, pn, rows, k1);
      }
      // B half
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        split8_store(R.b[h], invB[h], S.B[stage], tile_off(rows[h], koff));
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.full[stage]);
    }
  }
}

// Issues one N tile's MMAs (all K stages) from a single thread.  With one
// accumulator set in TMEM the MMAs of a tile never overlap that tile's
// epilogue, so the issuing thread is lane 0 of epilogue warp 0.
__device__ bool mma_tile(SplitSmem &S, uint32_t tmem, int n_kc, uint32_t &fill, uint32_t tile_ctr,
                         volatile int *abort_flag, int *err) {
  if (!mbar_wait(&S.acc_empty, (tile_ctr & 1) ^ 1, abort_flag, err)) return false;
  tc_fence_after();
  for (int kc = 0; kc < n_kc; ++kc, ++fill) {
    const int stage = fill & 1;
    if (!mbar_wait(&S.full[stage], (fill >> 1) & 1, abort_flag, err)) return false;
    tc_fence_after();
#pragma unroll
    for (int ks = 0; ks < SP_KC / 16; ++ks) {
      uint64_t a[SP_SLICES], b[SP_SLICES];
#pragma unroll
      for (int s = 0; s < SP_SLICES; ++s) {
        a[s] = smem_desc(smem_u32(S.A[stage][s]) + ks * 2 * SP_LBO);
        b[s] = smem_desc(smem_u32(S.B[stage][s]) + ks * 2 * SP_LBO);
      }
      const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
      // accumulator q holds slice level s + u = q (q < 3, exact) and the
      // levels 3 and 4 (q = 3, rounded)
      uint32_t first[4] = {acc, acc, acc, acc};
#pragma unroll
      for (int s = 0; s < SP_SLICES; ++s)
#pragma unroll
        for (int u = 0; u < SP_SLICES; ++u)
          if (s + u <= 4) {
            const int q = s + u < 3 ? s + u : 3;
            umma_bf16(tmem + q * SP_N, a[s], b[u], first[q]);
            first[q] = 1u;
          }
    }
    umma_commit(&S.empty[stage]);
  }
  umma_commit(&S.acc_full);
  return true;
}

// Waits (bounded) until every MMA issued so far by this thread has completed.
__device__ void mma_drain(SplitSmem &S, int *err) {
  umma_commit(&S.drain);
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(&S.drain, 0)) {
    if (global_ns() - t0 > sm100::WAIT_NS) {
      atomicOr(err, 4);
      break;
    }
  }
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = __uint_as_float(r[j]);
}

// FP64 operands of one 8-column chunk of the epilogue: phi and grad phi at
// rows i = i0..i0+7 of one point's column (zero past n_compute).
struct EpiRegs {
  double f[8], gx[8], gy[8], gz[8];
};

__device__ __forceinline__ void epi_load(EpiRegs &E, const double *__restrict__ phi, const double *__restrict__ gph,
                                         int ncp, int nc, int i0, bool live) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const bool ok = live && i0 + j < nc;
    E.f[j] = ok ? __ldg(phi + i0 + j) : 0.0;
    E.gx[j] = ok ? __ldg(gph + i0 + j) : 0.0;
    E.gy[j] = ok ? __ldg(gph + i0 + j + ncp) : 0.0;
    E.gz[j] = ok ? __ldg(gph + i0 + j + 2 * ncp) : 0.0;
  }
}

// Epilogue warp w reads TMEM lanes 32 (w % 4).. (its points) and accumulator
// columns 64 (w / 4)..+63 of every N tile; the two warps sharing a lane
// quarter add their partial sums through shared memory at each perturbation's
// end (the upper half publishes through ep_sum, the lower half writes the
// outputs and releases the buffer through ep_free).
__device__ void epilogue_body(const SplitParams &P, SplitSmem &S, uint32_t tmem, int warp, int lane, bool &issued) {
  int *err = P.err;
  volatile int *abort_flag = &S.abort_flag;
  const int quarter = warp & 3, half = warp >> 2;
  const int p = quarter * 32 + lane;  // TMEM lane = point within the tile
  const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
  const int cbase = half * (SP_N / 2);
  uint32_t tile_ctr = 0, item_ctr = 0, sum_ctr = 0, fill = 0;
  const bool issuer = warp == 0 && lane == 0;
  for (int it = blockIdx.x; it < P.n_items; it += gridDim.x, ++item_ctr) {
    const Rho1WorkItem W = P.items[it];
    const int nc = W.nc, pn = W.pn, ncp = (nc + 3) & ~3;
    const int ip = item_ctr & 1;
    const bool live = p < pn;
    const int n_kc = (nc + SP_KC - 1) / SP_KC;
    const double *phi = P.wave + W.wave_off + (long long)(W.p0 + p) * ncp;
    const double *gph = P.gwave + 3 * W.wave_off + 3LL * (W.p0 + p) * ncp;
    if (!warp_wait(&S.sa_full[ip], (item_ctr >> 1) & 1, abort_flag, err, lane)) return;
    const double sA = S.scaleA[ip][p];
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.sa_free[ip]);
    const int n_nt = (nc + SP_N - 1) / SP_N;
    for (int t = 0; t < P.T; ++t) {
      double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
      for (int jn = 0; jn < n_nt; ++jn, ++tile_ctr) {
        const int tp = tile_ctr & 1;
        const int ibase = jn * SP_N + cbase;
        EpiRegs E;
        epi_load(E, phi, gph, ncp, nc, ibase, live);  // independent of the MMA: before the wait
        if (issuer) {
          issued = true;
          mma_tile(S, tmem, n_kc, fill, tile_ctr, abort_flag, err);  // a failure sets abort_flag
        }
        __syncwarp();
        if (*abort_flag) return;
        if (!warp_wait(&S.sb_full[tp], (tile_ctr >> 1) & 1, abort_flag, err, lane)) return;
        if (!warp_wait(&S.acc_full, tile_ctr & 1, abort_flag, err, lane)) return;
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < SP_N / 2; c += 8) {
          float v0[8], v1[8], v2[8], v3[8];
          tmem_ld8(lane_base + 0 * SP_N + cbase + c, v0);
          tmem_ld8(lane_base + 1 * SP_N + cbase + c, v1);
          tmem_ld8(lane_base + 2 * SP_N + cbase + c, v2);
          tmem_ld8(lane_base + 3 * SP_N + cbase + c, v3);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double w = sA * S.scaleB[tp][cbase + c + j] *
                             (((double)v0[j] + (double)v1[j] + (double)v2[j]) + (double)v3[j]);
            r += E.f[j] * w;
            gx += E.gx[j] * w;
            gy += E.gy[j] * w;
            gz += E.gz[j] * w;
          }
          if (c + 8 < SP_N / 2) epi_load(E, phi, gph, ncp, nc, ibase + c + 8, live);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&S.sb_free[tp]);
          mbar_arrive(&S.acc_empty);
        }
      }
      // combine the two column halves of this point and write
      const int sp = sum_ctr & 1;
      if (half == 1) {
        if (!warp_wait(&S.ep_free[sp], ((sum_ctr >> 1) & 1) ^ 1, abort_flag, err, lane)) return;
        S.partial[sp][0][p] = r;
        S.partial[sp][1][p] = gx;
        S.partial[sp][2][p] = gy;
        S.partial[sp][3][p] = gz;
        mbar_arrive(&S.ep_sum[sp]);
      } else {
        if (!warp_wait(&S.ep_sum[sp], (sum_ctr >> 1) & 1, abort_flag, err, lane)) return;
        r += S.partial[sp][0][p];
        gx += S.partial[sp][1][p];
        gy += S.partial[sp][2][p];
        gz += S.partial[sp][3][p];
        mbar_arrive(&S.ep_free[sp]);
        if (live) {
          const int pp = W.p0 + p;
          const long long bidx = pp + (long long)P.n_max_batch_size * (W.batch + (long long)P.n_batches * t);
          P.grad[3 * bidx + 0] = gx * 2 - P.gbias[3 * bidx + 0];
          P.grad[3 * bidx + 1] = gy * 2 - P.gbias[3 * bidx + 1];
          P.grad[3 * bidx + 2] = gz * 2 - P.gbias[3 * bidx + 2];
          if (t < P.n_active) P.rho[P.map[W.prefix + pp] + (long long)P.n_full_points * t] = r + P.bias[bidx];
        }
      }
      ++sum_ctr;
    }
  }
}

__device__ void epilogue_role(const SplitParams &P, SplitSmem &S, uint32_t tmem, int warp, int lane) {
  bool issued = false;
  epilogue_body(P, S, tmem, warp, lane, issued);
  // no MMA may be in flight when TMEM is released
  if (issued) mma_drain(S, P.err);
}

__global__ void __launch_bounds__(SP_THREADS, 1) rho1_split_kernel(const SplitParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  SplitSmem &S = *reinterpret_cast<SplitSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < SP_STAGES; ++s) {
      mbar_init(&S.full[s], SP_PROD_WARPS);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    mbar_init(&S.acc_empty, SP_EPI_WARPS);
    mbar_init(&S.drain, 1);
    for (int h = 0; h < 2; ++h) {
      mbar_init(&S.sa_full[h], SP_PROD_THREADS / 4);
      mbar_init(&S.sb_full[h], SP_PROD_THREADS / 4);
      mbar_init(&S.sa_free[h], SP_EPI_WARPS);
      mbar_init(&S.sb_free[h], SP_EPI_WARPS);
      mbar_init(&S.ep_sum[h], SP_M);
      mbar_init(&S.ep_free[h], SP_M);
    }
    S.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(4 * SP_N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;

  if (warp < SP_EPI_WARPS) {
    epilogue_role(P, S, tmem, warp, lane);
    __syncwarp();
  } else {
    producer_role(P, S, tid - SP_PROD0 * 32, lane);
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(4 * SP_N));
  }
}

// rowmax[r + n_basis t] = max_c |P1(r, c, t)|, the per-row scale of P1c
// (an upper bound of the batch-local row maximum).
__global__ void p1_rowmax_kernel(const double *__restrict__ P1, int n_basis, int cols_per_block,
                                 unsigned long long *__restrict__ rowmax) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.z;
  if (r >= n_basis) return;
  const int c0 = blockIdx.y * cols_per_block, c1 = min(n_basis, c0 + cols_per_block);
  const double *col = P1 + (long long)n_basis * n_basis * t + r;
  double m = 0.0;
  for (int c = c0; c < c1; ++c) m = fmax(m, fabs(col[(long long)c * n_basis]));
  atomicMax(rowmax + r + (long long)n_basis * t, (unsigned long long)__double_as_longlong(m));
}

}  // namespace

int rho1_split_smem_bytes() { return (int)sizeof(SplitSmem) + 1024; }

// plan.d_rowmax[r + n_basis t] = max_c |P1(r, c, t)|: the per-row scales of
// P1c used by both split paths.
int p1_rowmax_launch(const Rho1Plan &plan, const double *P1, cudaStream_t stream) {
  FRPA_CUDA_TRY(cudaMemsetAsync(plan.d_rowmax, 0, sizeof(double) * (size_t)plan.n_basis * plan.T, stream));
  const int cols = 256;
  dim3 rg((plan.n_basis + 255) / 256, (plan.n_basis + cols - 1) / cols, plan.T);
  p1_rowmax_kernel<<<rg, 256, 0, stream>>>(P1, plan.n_basis, cols,
                                           reinterpret_cast<unsigned long long *>(plan.d_rowmax));
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

int rho1_split_launch(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave,
                      const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                      cudaStream_t stream) {
  if (plan.n_max_compute > SP_MAX_K)
    return fail(FRPA_ERR_UNSUPPORTED,
                "rho1 split-BF16: n_compute_c up to %d exceeds %d, the bound under which its exact FP32 levels "
                "stay exact; use the FP64 mode",
                plan.n_max_compute, SP_MAX_K);
  FRPA_CUDA_TRY(cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)plan.n_full_points * plan.T, stream));
  FRPA_CUDA_TRY(cudaMemsetAsync(
      grad, 0, sizeof(double) * 3 * (size_t)plan.n_max_batch_size * plan.n_batches * plan.T, stream));
  if (plan.n_items_split == 0) return FRPA_OK;
  FRPA_TRY(p1_rowmax_launch(plan, P1, stream));
  static PerDeviceOnce configured;
  const int smem = rho1_split_smem_bytes();
  FRPA_TRY(configured.run(plan.device, [smem]() -> int {
    FRPA_CUDA_TRY(cudaFuncSetAttribute(rho1_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return FRPA_OK;
  }));
  int n_sm = 148;
  FRPA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, plan.device));
  SplitParams P;
  P.items = plan.d_items_split;
  P.n_items = plan.n_items_split;
  P.ib_all = plan.d_ib;
  P.map = plan.d_map;
  P.T = plan.T;
  P.n_active = n_active;
  P.n_basis = plan.n_basis;
  P.n_full_points = plan.n_full_points;
  P.n_max_batch_size = plan.n_max_batch_size;
  P.n_batches = plan.n_batches;
  P.wave = wave;
  P.gwave = gwave;
  P.P1 = P1;
  P.bias = bias;
  P.gbias = gbias;
  P.rowmax = plan.d_rowmax;
  P.rho = rho;
  P.grad = grad;
  P.err = plan.d_err;
  const int grid = std::min(n_sm, plan.n_items_split);
  rho1_split_kernel<<<grid, SP_THREADS, smem, stream>>>(P);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

// Work items of the split path: point tiles of <= tile_points (<= 128)
// points, a batch's points split evenly; largest first or in batch order.
void rho1_split_build_items(const std::vector<Rho1WorkItem> &batches, int tile_points, int order,
                            std::vector<Rho1WorkItem> *out) {
  out->clear();
  const int tp = std::max(1, std::min(tile_points, SP_M));
  for (const Rho1WorkItem &w : batches) {
    const int np = w.np;
    if (np == 0) continue;
    const int tiles = (np + tp - 1) / tp;
    const int width = (np + tiles - 1) / tiles;
    for (int p0 = 0; p0 < np; p0 += width)
      out->push_back(Rho1WorkItem{w.batch, w.nc, w.np, p0, std::min(width, np - p0), w.ib_off, w.prefix, w.key,
                                  w.wave_off});
  }
  rho1_order_items(out, order);
}

}  // namespace frpa
