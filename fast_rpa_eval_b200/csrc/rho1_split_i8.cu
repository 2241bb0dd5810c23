// Split-precision rho1 on the integer tensor cores (tcgen05 kind::i8):
// work1 = P1c * phi at FP64-grade accuracy from exact int32 sums of 8-bit
// digit products, with the per-point dot products in FP64.
//
// Same semantics as the plain FP64 path (rho1_fp64.cu,
// fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho.cpp:116-209).
//
// Numerics.  Each FP64 operand x of a row (one grid point's phi over the
// batch's compute functions, or one row of P1) with scale 2^e,
// max|x| < 0.9921875 2^e, is rounded to the integer X = rint(x 2^(39 - e))
// and written in balanced base 256, X = a0 2^32 + a1 2^24 + a2 2^16 +
// a3 2^8 + a4, every digit a signed byte (|a0| <= 127 since
// |X| < 2^39 - 2^31 - 2^23 - 2^15 - 2^7).  The product of two rows is the sum
// of the 19 digit products with s + u <= 5, accumulated per level L = s + u
// in six int32 TMEM accumulators; |a_s b_u| <= 2^14, so every level stays
// exact for K < 26,000 (at most five products per level).  Recombined in FP64:
//   work1(i, p) = 2^(eA + eB - 54) (L0 2^40 + L1 2^32 + L2 2^24 + L3 2^16 + L4 2^8 + L5).
// What remains is the rounding of the operands to 2^-40 of their row scale
// and the dropped levels 6..8 (2^-48 per product); keeping level 5 removes
// the error term that dominated with levels 0..4 only (3.5x larger than the
// operand rounding in a CPU emulation of these steps).
//
// Data flow, three launches per group of batches:
//   1. pack A: one CTA per work item (<= 128 points of one batch) finds the
//      per-point scales and writes phi's five digit planes in the tcgen05
//      shared-memory tile image (K-major, no swizzle, 8 x 16-byte core
//      matrices), one 32-wide K chunk after another, 16 points at a time;
//   2. pack B: one CTA per (batch, perturbation, N tile of 32 rows, the last
//      one zero-padded) gathers P1c = P1[ib, ib] (lanes along P1's contiguous
//      rows) and writes its digit planes the same way;
//   3. contract: one persistent CTA per SM.  A loader thread moves each
//      stage's A and B chunks into a 4-stage shared-memory ring with bulk
//      copies; an MMA thread issues a stage's 19 digit products as five
//      tcgen05.mma.kind::i8 (M = 128 points, K = 32; the digit levels run
//      along N: A plane s times B planes 0..5-s, N = 32 (6 - s) rows, into
//      the six level accumulators from level s on) in one of two sets
//      (2 x 192 of 512 TMEM columns); 8 epilogue warps read a
//      finished set (tcgen05.ld), recombine in FP64 and contract with phi and
//      grad phi (FP64, 256-bit loads from global memory issued a chunk ahead)
//      while the MMAs of the next tile fill the other set.
// The packed operands cost a write and a read of ~5 bytes per P1c and phi
// element, in exchange the contraction has no gathers, no conversions and
// no register-staged loads on its critical path.  Every mbarrier wait is
// bounded in time; on a timeout the kernel records an error flag, waits
// (bounded) for its copies and MMAs in flight, frees TMEM and returns.
#include <algorithm>
#include <vector>

#include "frpa_internal.cuh"
#include "sm100_sync.cuh"

namespace frpa {
namespace {

using namespace sm100;

constexpr int I8_M = 128;      // points per work item (TMEM lanes)
constexpr int I8_N = 32;       // rows i per N tile (accumulator columns per level)
constexpr int I8_KC = 32;      // K per stage: one kind::i8 instruction
constexpr int I8_LEVELS = 6;   // digit levels s + u = 0..5
constexpr int I8_SLICES = 5;   // digit planes per operand
constexpr int I8_SETS = 2;     // accumulator sets: a tile's epilogue overlaps the next tile's MMAs
constexpr int I8_STAGES = 4;
constexpr int I8_EPI_WARPS = 8;  // warps 0..7: lane quarter w % 4, column half w / 4; warp 0 owns TMEM
constexpr int I8_COLS = I8_N / 2;  // 16 accumulator columns per epilogue warp
constexpr int I8_LOAD_WARP = 8;  // lane 0 issues the bulk copies
constexpr int I8_MMA_WARP = 9;   // lane 0 issues the MMAs
constexpr int I8_THREADS = 32 * 10;
constexpr int I8_ROWB = I8_KC;                         // bytes per tile row of one plane
constexpr int I8_A_PLANE = I8_M * I8_ROWB;             // 4096
constexpr int I8_B_STAGE = I8_SLICES * I8_N * I8_ROWB;  // 5120: the five planes of a stage's B chunk
constexpr int I8_B_SLOT = I8_B_STAGE + I8_N * I8_ROWB;  // 6144: plus a zero plane (see mma_role)
constexpr uint32_t I8_LBO = 128;                       // K-adjacent core matrices
constexpr uint32_t I8_SBO = 256;                       // 8-row groups
constexpr int I8_TMEM_COLS = 512;
constexpr int I8_SET_COLS = I8_LEVELS * I8_N;          // 192

static_assert(I8_SETS * I8_SET_COLS <= I8_TMEM_COLS, "accumulators fit TMEM");

// Instruction descriptor: kind::i8, D = S32, A = B = signed 8-bit, both
// K-major, M = 128; N is or-ed in per tile.
constexpr uint32_t I8_IDESC = (2u << 4)                         // D format S32
                              | (1u << 7)                       // A signed 8-bit
                              | (1u << 10)                      // B signed 8-bit
                              | ((uint32_t)(I8_M >> 4) << 24);  // M
__device__ __forceinline__ uint32_t idesc_n(int n) { return I8_IDESC | ((uint32_t)(n >> 3) << 17); }

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// Every N tile has 32 rows; the last one of a batch is padded with zero rows
// (the B planes of all tiles then share one layout: plane u at rows 32 u).
__host__ __device__ __forceinline__ int tile_rows(int, int, int) { return I8_N; }

// Byte offset of (row r, K half kg) inside one plane of a tile.
__device__ __forceinline__ int plane_off(int r, int kg) { return (r >> 3) * (int)I8_SBO + kg * 128 + (r & 7) * 16; }

// Row scale: 2^e with max|x| < 0.9921875 2^e (e >= -960 so that 2^(39 - e)
// stays finite); sc39 = 2^(39 - e) for the digits, s23 = 2^(e - 23) for the
// recombination.
__device__ __forceinline__ void digit_scale(double m, double *sc39, double *s23) {
  int e = 0;
  if (m > 0.0) {
    const double f = frexp(m, &e);
    if (f >= 0.9921875) ++e;
  }
  e = max(e, -960);
  *sc39 = ldexp(1.0, 39 - e);
  *s23 = ldexp(1.0, e - 23);
}

// Sixteen consecutive values of one row as five 16-byte digit planes.
//   t = fma(x, sc39, 1.5 2^52) holds X = rint(x sc39) in its mantissa, so
//   bits(t) - 0x4338000000000000 = X exactly; X + 0x80808080 = a0 2^32 + sum
//   c_s 2^(8 (4 - s)) with bytes c_s in [0, 255], i.e. the balanced digits
//   a_s = c_s - 128 (= c_s ^ 0x80 as a signed byte) and a0 the high word.
__device__ __forceinline__ void digits16(const double (&x)[16], double sc39, uint4 (&plane)[I8_SLICES]) {
  int hi[16];
  uint32_t lo[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const double t = fma(x[j], sc39, 6755399441055744.0);
    const long long xp = __double_as_longlong(t) + (0x80808080LL - 0x4338000000000000LL);
    hi[j] = (int)(xp >> 32);
    lo[j] = (uint32_t)xp;
  }
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t t1 = __byte_perm((uint32_t)hi[4 * q], (uint32_t)hi[4 * q + 1], 0x40);
    const uint32_t t2 = __byte_perm((uint32_t)hi[4 * q + 2], (uint32_t)hi[4 * q + 3], 0x40);
    w[q] = __byte_perm(t1, t2, 0x5410);
  }
  plane[0] = make_uint4(w[0], w[1], w[2], w[3]);
#pragma unroll
  for (int s = 1; s < I8_SLICES; ++s) {
    const uint32_t b = (uint32_t)(4 - s), sel = b | ((b + 4) << 4);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t t1 = __byte_perm(lo[4 * q], lo[4 * q + 1], sel);
      const uint32_t t2 = __byte_perm(lo[4 * q + 2], lo[4 * q + 3], sel);
      w[q] = __byte_perm(t1, t2, 0x5410) ^ 0x80808080u;
    }
    plane[s] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// ------------------------------------------------------------ pack kernels

// Four doubles from a 32-byte aligned address, not kept in L1.
__device__ __forceinline__ void ld4(const double *p, double *v) {
  asm volatile("ld.global.nc.L1::no_allocate.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
               : "l"(p));
}

constexpr int PA_THREADS = 256;
constexpr int PA_GROUP = 16;  // points per pass: their rows are re-read from L2, not DRAM

// phi of one work item -> A scratch: chunk kc, plane s at
// a_off + (5 kc + s) rows8 32 bytes; rows pn..rows8-1 and k >= nc are zero.
// Sixteen points at a time: their scales (one warp per point, lanes along the
// row), then their digits (one thread per row and 16-wide K group; a warp's
// stores cover 512 contiguous bytes of a plane).
__global__ void __launch_bounds__(PA_THREADS) i8_pack_a_kernel(const I8Item *__restrict__ items,
                                                               const double *__restrict__ wave,
                                                               unsigned char *__restrict__ a_scr,
                                                               double *__restrict__ sa, int vec) {
  __shared__ double s_sc[PA_GROUP];
  const I8Item W = items[blockIdx.x];
  const int nc = W.nc, pn = W.pn, rows8 = W.rows8, ncp = (nc + 3) & ~3;
  const double *phi = wave + W.wave_off + (long long)W.p0 * ncp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long chunk = (long long)I8_SLICES * rows8 * I8_ROWB;
  for (int g0 = 0; g0 < rows8; g0 += PA_GROUP) {
    const int gn = min(PA_GROUP, rows8 - g0);  // 8 or 16
    for (int r = warp; r < gn; r += PA_THREADS / 32) {
      const int p = g0 + r;
      double m = 0.0;
      if (p < pn) {
        const double *row = phi + (long long)p * ncp;
        for (int k = lane; k < nc; k += 32) m = fmax(m, fabs(__ldg(row + k)));
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) {
        double sc39, s23;
        digit_scale(m, &sc39, &s23);
        s_sc[r] = sc39;
        sa[W.sa_off + p] = s23;
      }
    }
    __syncthreads();
    const int units = W.n_kc * 2 * gn;
    for (int u = threadIdx.x; u < units; u += PA_THREADS) {
      const int r = u % gn, kg = (u / gn) & 1, kc = u / (2 * gn), p = g0 + r;
      const int k0 = kc * I8_KC + kg * 16;
      const double *row = phi + (long long)(p < pn ? p : 0) * ncp;
      double x[16];
      if (vec) {  // rows start on 32-byte boundaries; a vector that starts below nc ends by ncp
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          if (p < pn && k0 + 4 * v < nc) {
            ld4(row + k0 + 4 * v, &x[4 * v]);
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) x[4 * v + e] = 0.0;
          }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = k0 + j < nc ? x[j] : 0.0;  // the row padding
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = (p < pn && k0 + j < nc) ? __ldg(row + k0 + j) : 0.0;
      }
      uint4 plane[I8_SLICES];
      digits16(x, s_sc[r], plane);
      unsigned char *dst = a_scr + W.a_off + kc * chunk + plane_off(p, kg);
#pragma unroll
      for (int s = 0; s < I8_SLICES; ++s) *reinterpret_cast<uint4 *>(dst + s * rows8 * I8_ROWB) = plane[s];
    }
    __syncthreads();  // s_sc is rewritten by the next group
  }
}

constexpr int PB_THREADS = 2 * I8_N;  // 32 rows x two 16-wide halves of a K chunk

// P1c rows of one N tile -> B scratch: chunk kc, plane s at
// b_off + kc 5 n_rows 32 + s n_rows 32; rows >= nc and k >= nc are zero.
__global__ void __launch_bounds__(PB_THREADS) i8_pack_b_kernel(const I8BTile *__restrict__ tiles,
                                                               const int *__restrict__ ib_all,
                                                               const double *__restrict__ P1,
                                                               const double *__restrict__ rowmax, int n_basis,
                                                               unsigned char *__restrict__ b_scr,
                                                               double *__restrict__ sb) {
  __shared__ int s_ib[FRPA_MAX_N_COMPUTE];
  const I8BTile B = tiles[blockIdx.x];
  const int nc = B.nc, N = B.n_rows;
  for (int i = threadIdx.x; i < nc; i += PB_THREADS) s_ib[i] = __ldg(ib_all + B.ib_off + i) - 1;
  __syncthreads();
  const int r = threadIdx.x % I8_N, kg = threadIdx.x / I8_N;
  if (r >= N) return;
  const int i = B.jn * I8_N + r;
  const bool rok = i < nc;
  const int ibr = rok ? s_ib[i] : 0;
  const double *P1t = P1 + (long long)n_basis * n_basis * B.t;
  double sc39, s23;
  digit_scale(rok ? __ldg(rowmax + ibr + (long long)n_basis * B.t) : 0.0, &sc39, &s23);
  if (kg == 0) sb[B.sb_off + r] = rok ? s23 * 0.00390625 : 0.0;  // 2^(e - 31): the recombination sums 256 S
  const long long chunk = (long long)I8_SLICES * N * I8_ROWB;
  for (int kc = 0; kc < B.n_kc; ++kc) {
    const int k0 = kc * I8_KC + kg * 16;
    double x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
      x[j] = (rok && k0 + j < nc) ? __ldg(P1t + ibr + (long long)s_ib[k0 + j] * n_basis) : 0.0;
    uint4 plane[I8_SLICES];
    digits16(x, sc39, plane);
    unsigned char *dst = b_scr + B.b_off + kc * chunk + plane_off(r, kg);
#pragma unroll
    for (int s = 0; s < I8_SLICES; ++s) *reinterpret_cast<uint4 *>(dst + s * N * I8_ROWB) = plane[s];
  }
}

// ------------------------------------------------------ contraction kernel

struct I8Smem {
  unsigned char A[I8_STAGES][I8_SLICES][I8_A_PLANE];
  unsigned char B[I8_STAGES][I8_B_SLOT];  // planes 0..4 (32 rows each), then a zero plane
  double partial[2][4][I8_M];              // upper column half's per-point sums
  unsigned long long full[I8_STAGES];
  unsigned long long empty[I8_STAGES];
  unsigned long long acc_full[I8_SETS];
  unsigned long long acc_empty[I8_SETS];
  unsigned long long drain;
  unsigned long long ep_sum[2];   // partial sums published by the upper column half
  unsigned long long ep_free[2];  // partial-sum buffer released by the lower half
  uint32_t tmem_base;
  int abort_flag;
};

struct I8Params {
  const I8Item *items;
  int n_items;
  const int *map;
  int T, n_active, n_full_points, n_max_batch_size, n_batches;
  const double *wave, *gwave, *bias, *gbias;
  const unsigned char *a_scr, *b_scr;
  const double *sa, *sb;
  double *rho, *grad;
  int *err;
  int wave_vec;  // every phi / grad phi row starts on a 32-byte boundary: 256-bit loads
};

// Lane 0 of the loader warp: every stage's A planes (5 copies of rows8 x 32
// bytes) and B planes (one copy of 5 x n_rows x 32 bytes) into the ring.
__device__ void loader_role(const I8Params &P, I8Smem &S) {
  volatile int *abort_flag = &S.abort_flag;
  uint32_t fill = 0;
  for (int it = blockIdx.x; it < P.n_items; it += gridDim.x) {
    const I8Item W = P.items[it];
    const uint32_t a_bytes = (uint32_t)W.rows8 * I8_ROWB;
    for (int t = 0; t < P.T; ++t)
      for (int jn = 0; jn < W.n_nt; ++jn) {
        const int N = tile_rows(W.nc, jn, W.n_nt);
        const uint32_t b_bytes = (uint32_t)(I8_SLICES * N * I8_ROWB);
        const unsigned char *bsrc = P.b_scr + W.b_off + t * W.b_tstride + (long long)jn * W.n_kc * I8_B_STAGE;
        for (int kc = 0; kc < W.n_kc; ++kc, ++fill) {
          const int st = fill % I8_STAGES;
          if (!mbar_wait(&S.empty[st], ((fill / I8_STAGES) & 1) ^ 1, abort_flag, P.err)) goto out;
          mbar_arrive_expect_tx(&S.full[st], I8_SLICES * a_bytes + b_bytes);
          const unsigned char *a = P.a_scr + W.a_off + (long long)kc * I8_SLICES * a_bytes;
#pragma unroll
          for (int s = 0; s < I8_SLICES; ++s) bulk_g2s(S.A[st][s], a + s * a_bytes, a_bytes, &S.full[st]);
          bulk_g2s(S.B[st], bsrc + (long long)kc * b_bytes, b_bytes, &S.full[st]);
        }
      }
  }
out:
  // the copies of the last (up to) I8_STAGES fills land before the CTA exits
  const uint32_t n = fill < (uint32_t)I8_STAGES ? fill : (uint32_t)I8_STAGES;
  for (uint32_t f = fill - n; f < fill; ++f)
    if (!mbar_wait_quiet(&S.full[f % I8_STAGES], (f / I8_STAGES) & 1)) atomicOr(P.err, 4);
}

// Lane 0 of the MMA warp: per N tile, all K chunks' 19 digit products into
// the six level accumulators of the tile's set (sets alternate by tile), five
// MMA instructions per stage (one ~50-cycle issue each, so that issuing no
// longer outlasts the tensor work of a stage).
__device__ void mma_role(const I8Params &P, I8Smem &S, uint32_t tmem) {
  volatile int *abort_flag = &S.abort_flag;
  uint32_t fill = 0, tile_ctr = 0;
  bool issued = false;
  for (int it = blockIdx.x; it < P.n_items; it += gridDim.x) {
    const I8Item W = P.items[it];
    for (int t = 0; t < P.T; ++t)
      for (int jn = 0; jn < W.n_nt; ++jn, ++tile_ctr) {
        const int set = tile_ctr & 1;
        const uint32_t dcol = tmem + (uint32_t)(set * I8_SET_COLS);
        if (!mbar_wait(&S.acc_empty[set], ((tile_ctr >> 1) & 1) ^ 1, abort_flag, P.err)) goto out;
        tc_fence_after();
        for (int kc = 0; kc < W.n_kc; ++kc, ++fill) {
          const int st = fill % I8_STAGES;
          if (!mbar_wait(&S.full[st], (fill / I8_STAGES) & 1, abort_flag, P.err)) goto out;
          tc_fence_after();
          // Digit levels along N: B planes 0..m of a stage are one contiguous
          // matrix of 32 (m + 1) rows, so A plane s times planes 0..5-s, written
          // from accumulator column 32 s on, puts product (s, u) into the
          // columns of level s + u.  Plane s = 0 also multiplies the zero plane
          // (rows 160..191), so its MMA covers all six levels and alone starts
          // the accumulation of a tile; the other four always accumulate.
          const uint64_t bdesc = smem_desc<I8_LBO, I8_SBO>(smem_u32(S.B[st]));
#pragma unroll
          for (int s = 0; s < I8_SLICES; ++s) {
            const int n_mma = I8_N * (s == 0 ? I8_LEVELS : I8_LEVELS - s);  // 192, 160, 128, 96, 64
            umma_i8(dcol + (uint32_t)(s * I8_N), smem_desc<I8_LBO, I8_SBO>(smem_u32(S.A[st][s])), bdesc,
                    idesc_n(n_mma), (s > 0 || kc > 0) ? 1u : 0u);
          }
          umma_commit(&S.empty[st]);
          issued = true;
        }
        umma_commit(&S.acc_full[set]);
      }
  }
out:
  // no MMA may be in flight when TMEM is released
  if (issued) {
    umma_commit(&S.drain);
    if (!mbar_wait_quiet(&S.drain, 0)) atomicOr(P.err, 4);
  }
}

// FP64 operands of one 8-column chunk of the epilogue: phi and grad phi at
// rows i0..i0+7 of one point's column.  Values at rows >= n_compute (the
// row padding, possibly garbage) are masked where they are used.
struct EpiRegs {
  double f[8], gx[8], gy[8], gz[8];
};

__device__ __forceinline__ void epi_load(EpiRegs &E, const double *__restrict__ phi, const double *__restrict__ gph,
                                         int ncp, int nc, int i0, bool live, bool vec) {
  if (vec) {  // 32-byte loads: i0 and the row starts are multiples of 4, rows end at ncp >= i0 + 4
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = i0 + 4 * h;
      if (live && c < nc) {
        ld4(phi + c, &E.f[4 * h]);
        ld4(gph + c, &E.gx[4 * h]);
        ld4(gph + ncp + c, &E.gy[4 * h]);
        ld4(gph + 2 * ncp + c, &E.gz[4 * h]);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) E.f[4 * h + e] = E.gx[4 * h + e] = E.gy[4 * h + e] = E.gz[4 * h + e] = 0.0;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const bool ok = live && i0 + j < nc;
      E.f[j] = ok ? __ldg(phi + i0 + j) : 0.0;
      E.gx[j] = ok ? __ldg(gph + i0 + j) : 0.0;
      E.gy[j] = ok ? __ldg(gph + i0 + j + ncp) : 0.0;
      E.gz[j] = ok ? __ldg(gph + i0 + j + 2 * ncp) : 0.0;
    }
  }
}

// Epilogue warp w reads TMEM lanes 32 (w % 4).. (its points) and columns
// 16 (w / 4)..+15 of each level accumulator of the tile's set, recombines the
// six levels in FP64 and contracts with phi and grad phi; the loads of each
// 8-column chunk are issued one chunk ahead (the first chunk of a tile
// before its accumulators are waited for).  The set is released after the
// last chunk; meanwhile the MMAs of the next tile fill the other set.  The
// two warps of a lane quarter add their partial sums through shared memory
// at each perturbation's end.
__device__ void epilogue_role(const I8Params &P, I8Smem &S, uint32_t tmem, int warp, int lane) {
  int *err = P.err;
  volatile int *abort_flag = &S.abort_flag;
  const int quarter = warp & 3, half = warp >> 2;
  const int p = quarter * 32 + lane;  // TMEM lane = point within the tile
  const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
  const int cbase = half * I8_COLS;
  const bool vec = P.wave_vec != 0;
  uint32_t tile_ctr = 0, sum_ctr = 0;
  for (int it = blockIdx.x; it < P.n_items; it += gridDim.x) {
    const I8Item W = P.items[it];
    const int nc = W.nc, ncp = (nc + 3) & ~3;
    const bool live = p < W.pn;
    const long long pt = W.p0 + (live ? p : 0);
    const double *phi = P.wave + W.wave_off + pt * ncp;
    const double *gph = P.gwave + 3 * W.wave_off + 3 * pt * ncp;
    for (int t = 0; t < P.T; ++t) {
      double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
      const double *sbt = P.sb + W.sb_off + (long long)t * W.sb_tstride;
      for (int jn = 0; jn < W.n_nt; ++jn, ++tile_ctr) {
        const int N = tile_rows(nc, jn, W.n_nt);
        const int ncols = min(I8_COLS, N - cbase);  // warp-uniform, a multiple of 8 (or <= 0)
        const int ibase = jn * I8_N + cbase;
        const int set = tile_ctr & 1;
        const uint32_t acc = lane_base + (uint32_t)(set * I8_SET_COLS + cbase);
        const double *sbv = sbt + ibase;
        EpiRegs E;
        if (ncols > 0) epi_load(E, phi, gph, ncp, nc, ibase, live, vec);  // before the wait
        if (!warp_wait(&S.acc_full[set], (tile_ctr >> 1) & 1, abort_flag, err, lane)) return;
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < ncols; c += 8) {
          const int lim = live ? nc - (ibase + c) : 0;  // rows of this chunk inside n_compute
#pragma unroll
          for (int hq = 0; hq < 8; hq += 4) {
            uint32_t v[I8_LEVELS][4];
#pragma unroll
            for (int l = 0; l < I8_LEVELS; ++l) tmem_ld4(acc + (uint32_t)(l * I8_N + c + hq), v[l]);
            tmem_wait_ld();
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int j = hq + e;
              // 256 S = (L0 256 + L1) 2^32 + (L2 256 + L3) 2^16 + (L4 256 + L5), each pair exact in int64
              const long long hi = (long long)(int)v[0][e] * 256 + (int)v[1][e];
              const long long mid = (long long)(int)v[2][e] * 256 + (int)v[3][e];
              const long long lo = (long long)(int)v[4][e] * 256 + (int)v[5][e];
              const double w = fma((double)hi, 4294967296.0, fma((double)mid, 65536.0, (double)lo)) *
                               __ldg(sbv + c + j);
              const bool ok = j < lim;
              r = fma(ok ? E.f[j] : 0.0, w, r);
              gx = fma(ok ? E.gx[j] : 0.0, w, gx);
              gy = fma(ok ? E.gy[j] : 0.0, w, gy);
              gz = fma(ok ? E.gz[j] : 0.0, w, gz);
            }
          }
          if (c + 8 < ncols) epi_load(E, phi, gph, ncp, nc, ibase + c + 8, live, vec);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.acc_empty[set]);
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
          const double sA = P.sa[W.sa_off + p];
          const int pp = W.p0 + p;
          const long long bidx = pp + (long long)P.n_max_batch_size * (W.batch + (long long)P.n_batches * t);
          P.grad[3 * bidx + 0] = (gx * sA) * 2 - P.gbias[3 * bidx + 0];
          P.grad[3 * bidx + 1] = (gy * sA) * 2 - P.gbias[3 * bidx + 1];
          P.grad[3 * bidx + 2] = (gz * sA) * 2 - P.gbias[3 * bidx + 2];
          if (t < P.n_active) P.rho[P.map[W.prefix + pp] + (long long)P.n_full_points * t] = r * sA + P.bias[bidx];
        }
      }
      ++sum_ctr;
    }
  }
}

__global__ void __launch_bounds__(I8_THREADS, 1) rho1_i8_kernel(const I8Params P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  I8Smem &S = *reinterpret_cast<I8Smem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < I8_STAGES; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    for (int s = 0; s < I8_SETS; ++s) {
      mbar_init(&S.acc_full[s], 1);
      mbar_init(&S.acc_empty[s], I8_EPI_WARPS);
    }
    mbar_init(&S.drain, 1);
    for (int h = 0; h < 2; ++h) {
      mbar_init(&S.ep_sum[h], I8_M);
      mbar_init(&S.ep_free[h], I8_M);
    }
    S.abort_flag = 0;
    mbar_init_fence();
  }
  // the zero B plane of every stage (never written by the copies), made
  // visible to the tensor core's (async proxy) reads
  for (int e = tid; e < I8_STAGES * I8_N * I8_ROWB / 16; e += I8_THREADS) {
    const int st = e / (I8_N * I8_ROWB / 16), o = e % (I8_N * I8_ROWB / 16);
    reinterpret_cast<uint4 *>(S.B[st] + I8_B_STAGE)[o] = make_uint4(0u, 0u, 0u, 0u);
  }
  fence_proxy_async_smem();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(I8_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;

  if (warp < I8_EPI_WARPS) {
    epilogue_role(P, S, tmem, warp, lane);
    __syncwarp();
  } else if (warp == I8_LOAD_WARP) {
    if (lane == 0) loader_role(P, S);
    __syncwarp();
  } else if (warp == I8_MMA_WARP) {
    if (lane == 0) mma_role(P, S, tmem);
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(I8_TMEM_COLS));
  }
}

int i8_smem_bytes() { return (int)sizeof(I8Smem) + 128; }

}  // namespace

// Work lists and groups from the plan's valid batches: batches by decreasing
// cost (nc^2 np), each split into point tiles of <= 128 points (evenly), the
// tiles of a batch adjacent; consecutive batches form a group while its A + B
// scratch stays within plan->i8_budget (a batch larger than that is a group
// of its own).
int rho1_i8_build(Rho1Plan *plan) {
  // Groups follow the lexicographic order of the batches' (ascending) basis
  // lists, so that batches over the same atoms are packed together and
  // their P1c gathers meet in L2; inside a group the contraction takes the
  // batches by decreasing cost (nc^2 np), a batch's point tiles adjacent.
  std::vector<Rho1WorkItem> batches = plan->h_batches;
  const int *ibh = plan->h_ib.data();
  std::stable_sort(batches.begin(), batches.end(), [ibh](const Rho1WorkItem &a, const Rho1WorkItem &b) {
    return std::lexicographical_compare(ibh + a.ib_off, ibh + a.ib_off + a.nc, ibh + b.ib_off, ibh + b.ib_off + b.nc);
  });
  const int T = plan->T;
  std::vector<I8Item> items;
  std::vector<I8BTile> tiles;
  std::vector<I8Group> groups;
  I8Group g{0, 0, 0, 0, 0, 0, 0, 0};
  for (const Rho1WorkItem &bt : batches) {
    if (bt.np == 0) continue;
    const int nc = bt.nc, n_nt = ceil_div(nc, I8_N), n_kc = ceil_div(nc, I8_KC);
    const int n_last = tile_rows(nc, n_nt - 1, n_nt);
    const long long b_t = (long long)(n_nt - 1) * n_kc * I8_B_STAGE + (long long)n_kc * I8_SLICES * n_last * I8_ROWB;
    const int ntiles = ceil_div(bt.np, I8_M), width = ceil_div(bt.np, ntiles);
    long long a_need = 0;
    for (int p0 = 0; p0 < bt.np; p0 += width) {
      const int pn = std::min(width, bt.np - p0);
      a_need += (long long)n_kc * I8_SLICES * (((pn + 7) / 8) * 8) * I8_ROWB;
    }
    const long long need = a_need + b_t * T;
    if (g.item1 > g.item0 && g.a_bytes + g.b_bytes + need > plan->i8_budget) {
      groups.push_back(g);
      g = I8Group{(int)items.size(), (int)items.size(), (int)tiles.size(), (int)tiles.size(), 0, 0, 0, 0};
    }
    const long long b_off = g.b_bytes;
    const int sb_off = g.sb_len;
    for (int t = 0; t < T; ++t)
      for (int jn = 0; jn < n_nt; ++jn)
        tiles.push_back(I8BTile{bt.ib_off, nc, jn, t, tile_rows(nc, jn, n_nt), n_kc,
                                sb_off + t * n_nt * I8_N + jn * I8_N, 0,
                                b_off + t * b_t + (long long)jn * n_kc * I8_B_STAGE});
    for (int p0 = 0; p0 < bt.np; p0 += width) {
      const int pn = std::min(width, bt.np - p0), rows8 = ((pn + 7) / 8) * 8;
      I8Item it{};
      it.batch = bt.batch;
      it.nc = nc;
      it.p0 = p0;
      it.pn = pn;
      it.prefix = bt.prefix;
      it.rows8 = rows8;
      it.n_nt = n_nt;
      it.n_kc = n_kc;
      it.wave_off = bt.wave_off;
      it.a_off = g.a_bytes;
      it.b_off = b_off;
      it.b_tstride = b_t;
      it.sa_off = g.sa_len;
      it.sb_off = sb_off;
      it.sb_tstride = n_nt * I8_N;
      items.push_back(it);
      g.a_bytes += (long long)n_kc * I8_SLICES * rows8 * I8_ROWB;
      g.sa_len += I8_M;
    }
    g.b_bytes += b_t * T;
    g.sb_len += T * n_nt * I8_N;
    g.item1 = (int)items.size();
    g.tile1 = (int)tiles.size();
  }
  if (g.item1 > g.item0) groups.push_back(g);
  for (const I8Group &q : groups)  // cost order inside each group (siblings stay adjacent)
    std::stable_sort(items.begin() + q.item0, items.begin() + q.item1, [](const I8Item &a, const I8Item &b) {
      return a.nc != b.nc ? a.nc > b.nc : a.batch < b.batch;
    });
  plan->i8_wave4 = 1;
  for (const Rho1WorkItem &bt : batches)
    if (bt.wave_off & 3) plan->i8_wave4 = 0;
  cudaFree(plan->d_i8_items);
  cudaFree(plan->d_i8_tiles);
  plan->d_i8_items = nullptr;
  plan->d_i8_tiles = nullptr;
  plan->i8_groups = groups;
  if (items.empty()) return FRPA_OK;
  if (cudaMalloc((void **)&plan->d_i8_items, sizeof(I8Item) * items.size()) != cudaSuccess ||
      cudaMalloc((void **)&plan->d_i8_tiles, sizeof(I8BTile) * tiles.size()) != cudaSuccess)
    return fail(FRPA_ERR_OOM, "rho1 split-int8: work list allocation failed");
  FRPA_CUDA_TRY(cudaMemcpy(plan->d_i8_items, items.data(), sizeof(I8Item) * items.size(), cudaMemcpyHostToDevice));
  FRPA_CUDA_TRY(cudaMemcpy(plan->d_i8_tiles, tiles.data(), sizeof(I8BTile) * tiles.size(), cudaMemcpyHostToDevice));
  return FRPA_OK;
}

static void i8_free_scratch(Rho1Plan *plan) {
  for (int k = 0; k < 2; ++k) {
    cudaFree(plan->d_i8_a[k]);
    cudaFree(plan->d_i8_b[k]);
    cudaFree(plan->d_i8_sa[k]);
    cudaFree(plan->d_i8_sb[k]);
    plan->d_i8_a[k] = plan->d_i8_b[k] = nullptr;
    plan->d_i8_sa[k] = plan->d_i8_sb[k] = nullptr;
  }
}

void rho1_i8_free(Rho1Plan *plan) {
  cudaFree(plan->d_i8_items);
  cudaFree(plan->d_i8_tiles);
  plan->d_i8_items = nullptr;
  plan->d_i8_tiles = nullptr;
  i8_free_scratch(plan);
  if (plan->i8_side) cudaStreamDestroy(plan->i8_side);
  if (plan->i8_ev_start) cudaEventDestroy(plan->i8_ev_start);
  for (int k = 0; k < 2; ++k) {
    if (plan->i8_ev_packed[k]) cudaEventDestroy(plan->i8_ev_packed[k]);
    if (plan->i8_ev_done[k]) cudaEventDestroy(plan->i8_ev_done[k]);
    plan->i8_ev_packed[k] = plan->i8_ev_done[k] = nullptr;
  }
  plan->i8_side = nullptr;
  plan->i8_ev_start = nullptr;
}

// Scratch sets sized for the largest group (two when there are several
// groups) and the side stream, created on first use (not while the stream is
// being captured into a graph).
static int i8_scratch(Rho1Plan &plan, cudaStream_t stream) {
  if (plan.d_i8_a[0]) return FRPA_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  FRPA_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(FRPA_ERR_INVALID,
                "rho1 split-int8: the packed-operand scratch is allocated by the first execution; execute once "
                "before capturing a graph");
  long long a = 16, b = 16;
  int sa = 1, sb = 1;
  for (const I8Group &g : plan.i8_groups) {
    a = std::max(a, g.a_bytes);
    b = std::max(b, g.b_bytes);
    sa = std::max(sa, g.sa_len);
    sb = std::max(sb, g.sb_len);
  }
  const int sets = plan.i8_groups.size() > 1 ? 2 : 1;
  for (int k = 0; k < sets; ++k)
    if (cudaMalloc((void **)&plan.d_i8_a[k], a) != cudaSuccess ||
        cudaMalloc((void **)&plan.d_i8_b[k], b) != cudaSuccess ||
        cudaMalloc((void **)&plan.d_i8_sa[k], sizeof(double) * sa) != cudaSuccess ||
        cudaMalloc((void **)&plan.d_i8_sb[k], sizeof(double) * sb) != cudaSuccess) {
      i8_free_scratch(&plan);
      return fail(FRPA_ERR_OOM, "rho1 split-int8: %d scratch sets of %lld + %lld bytes could not be allocated",
                  sets, a, b);
    }
  if (!plan.i8_side) {
    FRPA_CUDA_TRY(cudaStreamCreateWithFlags(&plan.i8_side, cudaStreamNonBlocking));
    FRPA_CUDA_TRY(cudaEventCreateWithFlags(&plan.i8_ev_start, cudaEventDisableTiming));
    for (int k = 0; k < 2; ++k) {
      FRPA_CUDA_TRY(cudaEventCreateWithFlags(&plan.i8_ev_packed[k], cudaEventDisableTiming));
      FRPA_CUDA_TRY(cudaEventCreateWithFlags(&plan.i8_ev_done[k], cudaEventDisableTiming));
    }
  }
  return FRPA_OK;
}

int rho1_i8_launch(Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *P1,
                   const double *bias, const double *gbias, double *rho, double *grad, cudaStream_t stream) {
  FRPA_CUDA_TRY(cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)plan.n_full_points * plan.T, stream));
  FRPA_CUDA_TRY(cudaMemsetAsync(
      grad, 0, sizeof(double) * 3 * (size_t)plan.n_max_batch_size * plan.n_batches * plan.T, stream));
  if (plan.i8_groups.empty()) return FRPA_OK;
  FRPA_TRY(i8_scratch(plan, stream));
  FRPA_TRY(p1_rowmax_launch(plan, P1, stream));
  static PerDeviceOnce configured;
  const int smem = i8_smem_bytes();
  FRPA_TRY(configured.run(plan.device, [smem]() -> int {
    FRPA_CUDA_TRY(cudaFuncSetAttribute(rho1_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return FRPA_OK;
  }));
  int n_sm = 148;
  FRPA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, plan.device));
  I8Params P;
  P.map = plan.d_map;
  P.T = plan.T;
  P.n_active = n_active;
  P.n_full_points = plan.n_full_points;
  P.n_max_batch_size = plan.n_max_batch_size;
  P.n_batches = plan.n_batches;
  P.wave = wave;
  P.gwave = gwave;
  P.bias = bias;
  P.gbias = gbias;
  P.rho = rho;
  P.grad = grad;
  P.err = plan.d_err;
  P.wave_vec = (plan.i8_wave4 && !(((uintptr_t)wave | (uintptr_t)gwave) & 31)) ? 1 : 0;
  // group g: packed on the side stream into scratch set g % 2 (after the
  // contraction of group g - 2 released it), contracted on the caller's
  // stream; the side stream joins back before the last contraction
  const int sets = plan.d_i8_a[1] ? 2 : 1;
  FRPA_CUDA_TRY(cudaEventRecord(plan.i8_ev_start, stream));
  FRPA_CUDA_TRY(cudaStreamWaitEvent(plan.i8_side, plan.i8_ev_start, 0));
  const int n_groups = (int)plan.i8_groups.size();
  for (int gi = 0; gi < n_groups; ++gi) {
    const I8Group &g = plan.i8_groups[gi];
    const int k = gi % sets, ni = g.item1 - g.item0, nt = g.tile1 - g.tile0;
    if (gi >= sets) FRPA_CUDA_TRY(cudaStreamWaitEvent(plan.i8_side, plan.i8_ev_done[k], 0));
    i8_pack_a_kernel<<<ni, PA_THREADS, 0, plan.i8_side>>>(plan.d_i8_items + g.item0, wave, plan.d_i8_a[k],
                                                          plan.d_i8_sa[k], P.wave_vec);
    FRPA_LAUNCH_CHECK();
    i8_pack_b_kernel<<<nt, PB_THREADS, 0, plan.i8_side>>>(plan.d_i8_tiles + g.tile0, plan.d_ib, P1, plan.d_rowmax,
                                                          plan.n_basis, plan.d_i8_b[k], plan.d_i8_sb[k]);
    FRPA_LAUNCH_CHECK();
    FRPA_CUDA_TRY(cudaEventRecord(plan.i8_ev_packed[k], plan.i8_side));
    FRPA_CUDA_TRY(cudaStreamWaitEvent(stream, plan.i8_ev_packed[k], 0));
    P.items = plan.d_i8_items + g.item0;
    P.n_items = ni;
    P.a_scr = plan.d_i8_a[k];
    P.b_scr = plan.d_i8_b[k];
    P.sa = plan.d_i8_sa[k];
    P.sb = plan.d_i8_sb[k];
    rho1_i8_kernel<<<std::min(n_sm, ni), I8_THREADS, smem, stream>>>(P);
    FRPA_LAUNCH_CHECK();
    if (gi + sets < n_groups) FRPA_CUDA_TRY(cudaEventRecord(plan.i8_ev_done[k], stream));
  }
  return FRPA_OK;
}

}  // namespace frpa
