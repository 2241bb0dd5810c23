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
// Data flow, two launches per group of batches:
//   1. pack A: one CTA per work item (<= 128 points of one batch) finds the
//      per-point scales and writes phi's five digit planes in the tcgen05
//      shared-memory tile image (K-major, no swizzle, 8 x 16-byte core
//      matrices), one 32-wide K chunk after another, 16 points at a time;
//   2. contract: one persistent CTA per SM takes units (up to three point
//      tiles of one batch, one perturbation) in turn.  Four producer warps
//      gather P1c = P1[ib, ib] straight from P1 (lanes along P1's contiguous
//      rows) and write its digit planes, chunk by chunk, into a 20-slot
//      shared-memory ring, once per (unit, N tile) for all of the unit's
//      point tiles; a loader thread moves each stage's phi planes into a
//      4-stage ring with bulk copies; an MMA thread issues a stage's 19 digit
//      products as five tcgen05.mma.kind::i8 (M = 128 points, K = 32; the
//      digit levels run along N: A plane s times B planes 0..5-s, into the
//      six level accumulators from level s on) in one of two sets (2 x 192 of
//      512 TMEM columns); 8 epilogue warps read a finished set (tcgen05.ld),
//      recombine in FP64 and contract with phi and grad phi (FP64, 256-bit
//      loads issued a chunk ahead) while the MMAs of the next tile fill the
//      other set; per-point sums stay in shared memory until the unit ends.
// P1c never goes through global memory: of the packed operands only phi's
// planes do (a write and ~n_compute/32 L2 reads of 5 bytes per element).
// Every mbarrier wait is bounded in time; on a timeout the kernel records an
// error flag, waits (bounded) for its copies and MMAs in flight, frees TMEM
// and returns.
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
constexpr int I8_STAGES = 4;     // A ring
constexpr int I8_SLOTS = 20;     // B chunk ring: a unit's P1c stays resident for n_compute <= 640
constexpr int I8_MAX_ITEMS = 3;  // point tiles per unit
constexpr int I8_EPI_WARPS = 8;  // warps 0..7: lane quarter w % 4, column half w / 4; warp 0 owns TMEM
constexpr int I8_COLS = I8_N / 2;  // 16 accumulator columns per epilogue warp
constexpr int I8_LOAD_WARP = 8;  // lane 0 issues the bulk copies
constexpr int I8_MMA_WARP = 9;   // lane 0 issues the MMAs
constexpr int I8_PROD_WARP0 = 10;
constexpr int I8_PROD_WARPS = 4;  // warps 10..13 build the B chunks
constexpr int I8_THREADS = 32 * (I8_PROD_WARP0 + I8_PROD_WARPS);
static_assert(I8_SLOTS % I8_PROD_WARPS == 0, "a slot is always built by the same producer warp");
constexpr int I8_ROWB = I8_KC;                         // bytes per tile row of one plane
constexpr int I8_A_PLANE = I8_M * I8_ROWB;             // 4096
constexpr int I8_B_CHUNK = I8_SLICES * I8_N * I8_ROWB;  // 5120: the five planes of one B chunk
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
constexpr int PA_GROUP = 8;  // points per pass: one 8-row group of the tile image

// Shared-memory row layout of pack A: 16-value pieces padded to 17 doubles
// and rows padded to 4 (mod 16) doubles, so that the 32 threads of a warp
// reading one value of 8 rows x 4 pieces hit distinct bank pairs.
__host__ __device__ __forceinline__ int pa_row_stride(int kpad) {
  const int ldr = (kpad / 16) * 17;
  return ldr + ((4 - ldr) % 16 + 16) % 16;
}

// phi of one work item -> A scratch: chunk kc, plane s at
// a_off + (5 kc + s) rows8 32 bytes; rows pn..rows8-1 and k >= nc are zero.
// Eight points at a time: one warp per point copies its row into shared
// memory (lanes along the row, 256-bit loads when rows are 32-byte aligned)
// and finds its scale on the way, then every thread turns 16-wide K pieces of
// the staged rows into five 16-byte digit planes (a warp's stores cover whole
// 128-byte core-matrix rows).  phi crosses HBM once.
__global__ void __launch_bounds__(PA_THREADS) i8_pack_a_kernel(const I8Item *__restrict__ items,
                                                               const double *__restrict__ wave,
                                                               unsigned char *__restrict__ a_scr,
                                                               double *__restrict__ sa, int vec) {
  extern __shared__ __align__(32) double s_rows[];  // PA_GROUP rows, pa_row_stride(kpad) doubles each
  __shared__ double s_sc[PA_GROUP];
  const I8Item W = items[blockIdx.x];
  const int nc = W.nc, pn = W.pn, rows8 = W.rows8, ncp = (nc + 3) & ~3, kpad = W.n_kc * I8_KC;
  const int ld = pa_row_stride(kpad);
  const double *phi = wave + W.wave_off + (long long)W.p0 * ncp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long chunk = (long long)I8_SLICES * rows8 * I8_ROWB;
  for (int g0 = 0; g0 < rows8; g0 += PA_GROUP) {
    {  // warp r stages row g0 + r (zeros past n_compute and for padding rows)
      const int r = warp, p = g0 + r;
      double *dst = s_rows + r * ld;
      auto at = [](int k) { return (k >> 4) * 17 + (k & 15); };
      double m = 0.0;
      if (p < pn) {
        const double *row = phi + (long long)p * ncp;
        if (vec) {  // rows start on 32-byte boundaries; a vector that starts below nc ends by ncp
          for (int k = 4 * lane; k < nc; k += 128) {
            double v[4];
            ld4(row + k, v);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const double x = k + e < nc ? v[e] : 0.0;
              dst[at(k) + e] = x;
              m = fmax(m, fabs(x));
            }
          }
          for (int k = ((nc + 3) & ~3) + lane; k < kpad; k += 32) dst[at(k)] = 0.0;
        } else {
          for (int k = lane; k < kpad; k += 32) {
            const double x = k < nc ? __ldg(row + k) : 0.0;
            dst[at(k)] = x;
            m = fmax(m, fabs(x));
          }
        }
      } else {
        for (int k = lane; k < kpad; k += 32) dst[at(k)] = 0.0;
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) {
        double sc39, s23;
        digit_scale(m, &sc39, &s23);
        s_sc[r] = sc39;
        if (p < pn) sa[W.sa_off + p] = s23;
      }
    }
    __syncthreads();
    const int units = W.n_kc * 2 * PA_GROUP;
    for (int u = threadIdx.x; u < units; u += PA_THREADS) {
      const int r = u % PA_GROUP, kg = (u / PA_GROUP) & 1, kc = u / (2 * PA_GROUP), p = g0 + r;
      const double *src = s_rows + r * ld + (2 * kc + kg) * 17;
      double x[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) x[j] = src[j];
      uint4 plane[I8_SLICES];
      digits16(x, s_sc[r], plane);
      unsigned char *dst = a_scr + W.a_off + kc * chunk + plane_off(p, kg);
#pragma unroll
      for (int s = 0; s < I8_SLICES; ++s) *reinterpret_cast<uint4 *>(dst + s * rows8 * I8_ROWB) = plane[s];
    }
    __syncthreads();  // the rows and scales are rewritten by the next group
  }
}

// ------------------------------------------------------ contraction kernel

struct I8Smem {
  unsigned char A[I8_STAGES][I8_SLICES][I8_A_PLANE];  // phi planes of a stage
  unsigned char B[I8_SLOTS][I8_B_CHUNK];              // P1c chunks: plane u at rows 32 u
  double sums[2][I8_MAX_ITEMS * I8_M][4];             // per column half and point: rho, grad x, y, z
  unsigned long long a_full[I8_STAGES];
  unsigned long long a_empty[I8_STAGES];
  unsigned long long b_full[I8_SLOTS];
  unsigned long long b_empty[I8_SLOTS];
  unsigned long long acc_full[I8_SETS];
  unsigned long long acc_empty[I8_SETS];
  unsigned long long drain;
  uint32_t tmem_base;
  int abort_flag;
};

struct I8Params {
  const I8Item *items;
  const I8Unit *units;
  int n_units;
  const int *map;
  const int *ib_all;
  const double *P1, *rowmax;
  int n_basis;
  int T, n_active, n_full_points, n_max_batch_size, n_batches;
  const double *wave, *gwave, *bias, *gbias;
  const unsigned char *a_scr;
  const double *sa;
  double *rho, *grad;
  int *err;
  int wave_vec;  // every phi / grad phi row starts on a 32-byte boundary: 256-bit loads
};

// The B chunks of a unit: with n_kc <= I8_SLOTS the chunks of an N tile are
// built once and serve all of the unit's point tiles; beyond that they are
// built again for every point tile.  Chunk productions are numbered in one
// sequence shared by all roles; production q goes to slot q % I8_SLOTS and is
// that slot's (q / I8_SLOTS)-th, which gives the phase of its barriers.
__device__ __forceinline__ bool unit_slab(const I8Unit &U) { return U.n_kc <= I8_SLOTS; }
__device__ __forceinline__ int unit_productions(const I8Unit &U) {
  return U.n_nt * U.n_kc * (unit_slab(U) ? 1 : U.n_items);
}

// Producer warp pw: the productions q with q % I8_PROD_WARPS == pw.  Lane r
// builds row 32 jn + r of the chunk: 32 values of P1c (two 16-wide K halves,
// lanes along P1's contiguous rows, the column indices broadcast by shuffle),
// their digits at the row's P1 scale, 5 x 16 bytes per half into the slot.
__device__ void producer_role(const I8Params &P, I8Smem &S, int pw, int lane) {
  volatile int *abort_flag = &S.abort_flag;
  uint32_t q0 = 0;
  for (int u = blockIdx.x; u < P.n_units; u += gridDim.x) {
    const I8Unit U = P.units[u];
    const int nc = U.nc, reps = unit_slab(U) ? 1 : U.n_items;
    const int *ib = P.ib_all + U.ib_off;
    const double *P1t = P.P1 + (long long)P.n_basis * P.n_basis * U.t;
    const uint32_t nq = (uint32_t)unit_productions(U);
    for (uint32_t k = (pw - q0 % I8_PROD_WARPS + I8_PROD_WARPS) % I8_PROD_WARPS; k < nq; k += I8_PROD_WARPS) {
      const uint32_t q = q0 + k;
      const int kc = (int)(k % U.n_kc), jn = (int)(k / (U.n_kc * reps));
      const int slot = (int)(q % I8_SLOTS);
      const uint32_t round = q / I8_SLOTS;
      if (round > 0 && !warp_wait(&S.b_empty[slot], (round - 1) & 1, abort_flag, P.err, lane)) return;
      const int i = jn * I8_N + lane;
      const bool rok = i < nc;
      const int ibr = rok ? __ldg(ib + i) - 1 : 0;
      double sc39, s23;
      digit_scale(rok ? __ldg(P.rowmax + ibr + (long long)P.n_basis * U.t) : 0.0, &sc39, &s23);
      const int kcol = kc * I8_KC + lane;
      const int my_col = kcol < nc ? __ldg(ib + kcol) - 1 : -1;
      unsigned char *dst = S.B[slot];
      // all 32 gathers of the row are issued before any is used: one memory
      // round trip per chunk
      double x[2][16];
#pragma unroll
      for (int kg = 0; kg < 2; ++kg)
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = __shfl_sync(0xffffffffu, my_col, kg * 16 + j);
          x[kg][j] = (rok && col >= 0) ? __ldg(P1t + ibr + (long long)col * P.n_basis) : 0.0;
        }
#pragma unroll
      for (int kg = 0; kg < 2; ++kg) {
        uint4 plane[I8_SLICES];
        digits16(x[kg], sc39, plane);
#pragma unroll
        for (int s = 0; s < I8_SLICES; ++s)
          *reinterpret_cast<uint4 *>(dst + s * I8_N * I8_ROWB + plane_off(lane, kg)) = plane[s];
      }
      fence_proxy_async_smem();  // the tensor core (async proxy) reads these bytes next
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.b_full[slot]);
    }
    q0 += nq;
  }
}

// Lane 0 of the loader warp: every stage's A planes (5 copies of rows8 x 32
// bytes), in the order the MMA thread consumes them: per unit, N tile, point
// tile, K chunk.
__device__ void loader_role(const I8Params &P, I8Smem &S) {
  volatile int *abort_flag = &S.abort_flag;
  uint32_t fill = 0;
  for (int u = blockIdx.x; u < P.n_units; u += gridDim.x) {
    const I8Unit U = P.units[u];
    for (int jn = 0; jn < U.n_nt; ++jn)
      for (int m = 0; m < U.n_items; ++m) {
        const I8Item W = P.items[U.item0 + m];
        const uint32_t a_bytes = (uint32_t)W.rows8 * I8_ROWB;
        for (int kc = 0; kc < U.n_kc; ++kc, ++fill) {
          const int st = fill % I8_STAGES;
          if (!mbar_wait(&S.a_empty[st], ((fill / I8_STAGES) & 1) ^ 1, abort_flag, P.err)) goto out;
          mbar_arrive_expect_tx(&S.a_full[st], I8_SLICES * a_bytes);
          const unsigned char *a = P.a_scr + W.a_off + (long long)kc * I8_SLICES * a_bytes;
#pragma unroll
          for (int s = 0; s < I8_SLICES; ++s) bulk_g2s(S.A[st][s], a + s * a_bytes, a_bytes, &S.a_full[st]);
        }
      }
  }
out:
  // the copies of the last (up to) I8_STAGES fills land before the CTA exits
  const uint32_t n = fill < (uint32_t)I8_STAGES ? fill : (uint32_t)I8_STAGES;
  for (uint32_t f = fill - n; f < fill; ++f)
    if (!mbar_wait_quiet(&S.a_full[f % I8_STAGES], (f / I8_STAGES) & 1)) atomicOr(P.err, 4);
}

// Lane 0 of the MMA warp: per N tile and point tile, all K chunks' 19 digit
// products into the six level accumulators of the tile's set (sets alternate
// by tile).  The digit levels run along N: the B planes of a chunk are one
// contiguous matrix of 32 x 5 rows, so A plane s times planes 0..m, written
// from accumulator column 32 s on, puts product (s, u) into the columns of
// level s + u.  A tile's first chunk starts its accumulators with two MMAs
// that write (not add): plane 1 times B planes 0..4 (levels 1..5) and plane 0
// times B plane 0 (level 0); plane 0 times B planes 1..4 then adds to levels
// 1..4.  Every later chunk issues five MMAs that add (N = 160, 160, 128, 96, 64).
__device__ void mma_role(const I8Params &P, I8Smem &S, uint32_t tmem) {
  volatile int *abort_flag = &S.abort_flag;
  uint32_t fill = 0, tile_ctr = 0, q0 = 0;
  bool issued = false;
  for (int u = blockIdx.x; u < P.n_units; u += gridDim.x) {
    const I8Unit U = P.units[u];
    const bool slab = unit_slab(U);
    for (int jn = 0; jn < U.n_nt; ++jn)
      for (int m = 0; m < U.n_items; ++m, ++tile_ctr) {
        const int set = tile_ctr & 1;
        const uint32_t dcol = tmem + (uint32_t)(set * I8_SET_COLS);
        if (!mbar_wait(&S.acc_empty[set], ((tile_ctr >> 1) & 1) ^ 1, abort_flag, P.err)) goto out;
        tc_fence_after();
        for (int kc = 0; kc < U.n_kc; ++kc, ++fill) {
          const int st = fill % I8_STAGES;
          const uint32_t q = q0 + (uint32_t)(slab ? jn * U.n_kc + kc : (jn * U.n_items + m) * U.n_kc + kc);
          const int slot = (int)(q % I8_SLOTS);
          const bool first = !slab || m == 0, last = !slab || m == U.n_items - 1;
          if (first && !mbar_wait(&S.b_full[slot], (q / I8_SLOTS) & 1, abort_flag, P.err)) goto out;
          if (!mbar_wait(&S.a_full[st], (fill / I8_STAGES) & 1, abort_flag, P.err)) goto out;
          tc_fence_after();
          const uint32_t bslot = smem_u32(S.B[slot]);
          const uint64_t b0 = smem_desc<I8_LBO, I8_SBO>(bslot);
          const uint64_t a0 = smem_desc<I8_LBO, I8_SBO>(smem_u32(S.A[st][0]));
          if (kc == 0) {
            umma_i8(dcol + I8_N, smem_desc<I8_LBO, I8_SBO>(smem_u32(S.A[st][1])), b0, idesc_n(5 * I8_N), 0u);
            umma_i8(dcol, a0, b0, idesc_n(I8_N), 0u);
            umma_i8(dcol + I8_N, a0, smem_desc<I8_LBO, I8_SBO>(bslot + I8_N * I8_ROWB), idesc_n(4 * I8_N), 1u);
          } else {
            umma_i8(dcol, a0, b0, idesc_n(5 * I8_N), 1u);
            umma_i8(dcol + I8_N, smem_desc<I8_LBO, I8_SBO>(smem_u32(S.A[st][1])), b0, idesc_n(5 * I8_N), 1u);
          }
#pragma unroll
          for (int s = 2; s < I8_SLICES; ++s)  // N = 128, 96, 64
            umma_i8(dcol + (uint32_t)(s * I8_N), smem_desc<I8_LBO, I8_SBO>(smem_u32(S.A[st][s])), b0,
                    idesc_n(I8_N * (I8_LEVELS - s)), 1u);
          umma_commit(&S.a_empty[st]);
          if (last) umma_commit(&S.b_empty[slot]);
          issued = true;
        }
        umma_commit(&S.acc_full[set]);
      }
    q0 += (uint32_t)unit_productions(U);
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

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(32 * I8_EPI_WARPS) : "memory"); }

// Epilogue warp w reads TMEM lanes 32 (w % 4).. (the points of the tile) and
// columns 16 (w / 4)..+15 of each level accumulator of the tile's set,
// recombines the six levels in FP64 and contracts with phi and grad phi; the
// loads of each 8-column chunk are issued one chunk ahead (the first chunk of
// a tile before its accumulators are waited for).  The set is released after
// the last chunk; meanwhile the MMAs of the next tile fill the other set.  A
// tile's sums are added to the point's shared-memory sums of this column
// half; at the unit's end the halves are combined and written.
__device__ void epilogue_role(const I8Params &P, I8Smem &S, uint32_t tmem, int warp, int lane) {
  int *err = P.err;
  volatile int *abort_flag = &S.abort_flag;
  const int quarter = warp & 3, half = warp >> 2;
  const int p = quarter * 32 + lane;  // TMEM lane = point within the tile
  const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
  const int cbase = half * I8_COLS;
  const bool vec = P.wave_vec != 0;
  uint32_t tile_ctr = 0;
  // after a wait gave up, the warp skips all further work but still takes
  // part in every epilogue barrier (bar.sync has no time limit)
  bool dead = false;
  for (int u = blockIdx.x; u < P.n_units; u += gridDim.x) {
    const I8Unit U = P.units[u];
    const int nc = U.nc, ncp = (nc + 3) & ~3, t = U.t;
    const int *ib = P.ib_all + U.ib_off;
    for (int jn = 0; jn < U.n_nt; ++jn) {
      const int ibase = jn * I8_N + cbase;
      const int ncols = min(I8_COLS, nc - ibase);  // warp-uniform (<= 0: this half has no rows)
      // the recombination scale 2^(e - 31) of row ibase + lane (lanes < 16)
      double sb_mine = 0.0;
      if (!dead && lane < I8_COLS && ibase + lane < nc) {
        double sc39, s23;
        digit_scale(__ldg(P.rowmax + (__ldg(ib + ibase + lane) - 1) + (long long)P.n_basis * t), &sc39, &s23);
        sb_mine = s23 * 0.00390625;
      }
      for (int m = 0; m < U.n_items && !dead; ++m, ++tile_ctr) {
        const I8Item W = P.items[U.item0 + m];
        const bool live = p < W.pn;
        const long long pt = W.p0 + (live ? p : 0);
        const double *phi = P.wave + W.wave_off + pt * ncp;
        const double *gph = P.gwave + 3 * W.wave_off + 3 * pt * ncp;
        const int set = tile_ctr & 1;
        const uint32_t acc = lane_base + (uint32_t)(set * I8_SET_COLS + cbase);
        double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        EpiRegs E;
        if (ncols > 0) epi_load(E, phi, gph, ncp, nc, ibase, live, vec);  // before the wait
        if (!warp_wait(&S.acc_full[set], (tile_ctr >> 1) & 1, abort_flag, err, lane)) {
          dead = true;
          break;
        }
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
                               __shfl_sync(0xffffffffu, sb_mine, c + j);
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
        double *sm = S.sums[half][m * I8_M + p];
        sm[0] += r;
        sm[1] += gx;
        sm[2] += gy;
        sm[3] += gz;
      }
    }
    // combine the two column halves of every point of the unit and write
    epi_bar();
    if (half == 0 && !dead) {
      for (int m = 0; m < U.n_items; ++m) {
        const I8Item W = P.items[U.item0 + m];
        double *s0 = S.sums[0][m * I8_M + p], *s1 = S.sums[1][m * I8_M + p];
        if (p < W.pn) {
          const double sA = P.sa[W.sa_off + p];
          const int pp = W.p0 + p;
          const long long bidx = pp + (long long)P.n_max_batch_size * (W.batch + (long long)P.n_batches * t);
          P.grad[3 * bidx + 0] = ((s0[1] + s1[1]) * sA) * 2 - P.gbias[3 * bidx + 0];
          P.grad[3 * bidx + 1] = ((s0[2] + s1[2]) * sA) * 2 - P.gbias[3 * bidx + 1];
          P.grad[3 * bidx + 2] = ((s0[3] + s1[3]) * sA) * 2 - P.gbias[3 * bidx + 2];
          if (t < P.n_active)
            P.rho[P.map[W.prefix + pp] + (long long)P.n_full_points * t] = (s0[0] + s1[0]) * sA + P.bias[bidx];
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) s0[e] = s1[e] = 0.0;
      }
    }
    epi_bar();
  }
}

__global__ void __launch_bounds__(I8_THREADS, 1) rho1_i8_kernel(const I8Params P) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  I8Smem &S = *reinterpret_cast<I8Smem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < I8_STAGES; ++s) {
      mbar_init(&S.a_full[s], 1);
      mbar_init(&S.a_empty[s], 1);
    }
    for (int s = 0; s < I8_SLOTS; ++s) {
      mbar_init(&S.b_full[s], 1);
      mbar_init(&S.b_empty[s], 1);
    }
    for (int s = 0; s < I8_SETS; ++s) {
      mbar_init(&S.acc_full[s], 1);
      mbar_init(&S.acc_empty[s], I8_EPI_WARPS);
    }
    mbar_init(&S.drain, 1);
    S.abort_flag = 0;
    mbar_init_fence();
  }
  for (int e = tid; e < 2 * I8_MAX_ITEMS * I8_M * 4; e += I8_THREADS) (&S.sums[0][0][0])[e] = 0.0;
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
  } else {
    producer_role(P, S, warp - I8_PROD_WARP0, lane);
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

// Work lists and groups from the plan's valid batches: each batch split into
// point tiles of <= 128 points (evenly), consecutive tiles of a batch forming
// units of <= 3 (one per perturbation); consecutive batches form a group
// while its A scratch stays within plan->i8_budget (a batch larger than that
// is a group of its own).
int rho1_i8_build(Rho1Plan *plan) {
  // Groups follow the lexicographic order of the batches' (ascending) basis
  // lists, so that batches over the same atoms are contracted close in time
  // and their P1 rows meet in L2; inside a group the units go by decreasing
  // cost (nc^2 np).
  std::vector<Rho1WorkItem> batches = plan->h_batches;
  const int *ibh = plan->h_ib.data();
  std::stable_sort(batches.begin(), batches.end(), [ibh](const Rho1WorkItem &a, const Rho1WorkItem &b) {
    return std::lexicographical_compare(ibh + a.ib_off, ibh + a.ib_off + a.nc, ibh + b.ib_off, ibh + b.ib_off + b.nc);
  });
  const int T = plan->T;
  std::vector<I8Item> items;
  std::vector<I8Unit> units;
  std::vector<long long> unit_cost;
  std::vector<I8Group> groups;
  I8Group g{0, 0, 0, 0, 0, 0, 0};
  for (const Rho1WorkItem &bt : batches) {
    if (bt.np == 0) continue;
    const int nc = bt.nc, n_nt = ceil_div(nc, I8_N), n_kc = ceil_div(nc, I8_KC);
    const int ntiles = ceil_div(bt.np, I8_M), width = ceil_div(bt.np, ntiles);
    long long a_need = 0;
    for (int p0 = 0; p0 < bt.np; p0 += width) {
      const int pn = std::min(width, bt.np - p0);
      a_need += (long long)n_kc * I8_SLICES * (((pn + 7) / 8) * 8) * I8_ROWB;
    }
    if (g.item1 > g.item0 && g.a_bytes + a_need > plan->i8_budget) {
      groups.push_back(g);
      g = I8Group{(int)items.size(), (int)items.size(), (int)units.size(), (int)units.size(), 0, 0, 0};
    }
    const int first = (int)items.size();
    for (int p0 = 0; p0 < bt.np; p0 += width) {
      const int pn = std::min(width, bt.np - p0), rows8 = ((pn + 7) / 8) * 8;
      I8Item it{};
      it.batch = bt.batch;
      it.nc = nc;
      it.p0 = p0;
      it.pn = pn;
      it.prefix = bt.prefix;
      it.rows8 = rows8;
      it.n_kc = n_kc;
      it.sa_off = g.sa_len;
      it.wave_off = bt.wave_off;
      it.a_off = g.a_bytes;
      items.push_back(it);
      g.a_bytes += (long long)n_kc * I8_SLICES * rows8 * I8_ROWB;
      g.sa_len += I8_M;
    }
    const int last = (int)items.size();
    for (int t = 0; t < T; ++t)
      for (int i0 = first; i0 < last; i0 += I8_MAX_ITEMS) {
        const int n = std::min(I8_MAX_ITEMS, last - i0);
        units.push_back(I8Unit{i0, n, bt.batch, nc, bt.ib_off, t, n_nt, n_kc});
        long long pts = 0;
        for (int k = i0; k < i0 + n; ++k) pts += items[k].pn;
        unit_cost.push_back((long long)nc * nc * pts);
      }
    g.item1 = (int)items.size();
    g.unit1 = (int)units.size();
  }
  if (g.item1 > g.item0) groups.push_back(g);
  for (const I8Group &q : groups) {  // cost order inside each group
    std::vector<int> order(q.unit1 - q.unit0);
    for (size_t k = 0; k < order.size(); ++k) order[k] = q.unit0 + (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return unit_cost[a] > unit_cost[b]; });
    std::vector<I8Unit> sorted;
    for (int k : order) sorted.push_back(units[k]);
    std::copy(sorted.begin(), sorted.end(), units.begin() + q.unit0);
  }
  plan->i8_wave4 = 1;
  for (const Rho1WorkItem &bt : batches)
    if (bt.wave_off & 3) plan->i8_wave4 = 0;
  cudaFree(plan->d_i8_items);
  cudaFree(plan->d_i8_units);
  plan->d_i8_items = nullptr;
  plan->d_i8_units = nullptr;
  plan->i8_groups = groups;
  if (items.empty()) return FRPA_OK;
  if (cudaMalloc((void **)&plan->d_i8_items, sizeof(I8Item) * items.size()) != cudaSuccess ||
      cudaMalloc((void **)&plan->d_i8_units, sizeof(I8Unit) * units.size()) != cudaSuccess)
    return fail(FRPA_ERR_OOM, "rho1 split-int8: work list allocation failed");
  FRPA_CUDA_TRY(cudaMemcpy(plan->d_i8_items, items.data(), sizeof(I8Item) * items.size(), cudaMemcpyHostToDevice));
  FRPA_CUDA_TRY(cudaMemcpy(plan->d_i8_units, units.data(), sizeof(I8Unit) * units.size(), cudaMemcpyHostToDevice));
  return FRPA_OK;
}

static void i8_free_scratch(Rho1Plan *plan) {
  cudaFree(plan->d_i8_a);
  cudaFree(plan->d_i8_sa);
  plan->d_i8_a = nullptr;
  plan->d_i8_sa = nullptr;
}

void rho1_i8_free(Rho1Plan *plan) {
  cudaFree(plan->d_i8_items);
  cudaFree(plan->d_i8_units);
  plan->d_i8_items = nullptr;
  plan->d_i8_units = nullptr;
  i8_free_scratch(plan);
}

// Packed-phi scratch sized for the largest group, allocated on first use
// (not while the stream is being captured into a graph).
static int i8_scratch(Rho1Plan &plan, cudaStream_t stream) {
  if (plan.d_i8_a) return FRPA_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  FRPA_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(FRPA_ERR_INVALID,
                "rho1 split-int8: the packed-operand scratch is allocated by the first execution; execute once "
                "before capturing a graph");
  long long a = 16;
  int sa = 1;
  for (const I8Group &g : plan.i8_groups) {
    a = std::max(a, g.a_bytes);
    sa = std::max(sa, g.sa_len);
  }
  if (cudaMalloc((void **)&plan.d_i8_a, a) != cudaSuccess ||
      cudaMalloc((void **)&plan.d_i8_sa, sizeof(double) * sa) != cudaSuccess) {
    i8_free_scratch(&plan);
    return fail(FRPA_ERR_OOM, "rho1 split-int8: %lld bytes of packed-phi scratch could not be allocated", a);
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
  // pack A stages PA_GROUP rows of up to n_compute (rounded to a K chunk) doubles
  const int pa_smem =
      (int)sizeof(double) * PA_GROUP * pa_row_stride(ceil_div(std::max(1, plan.n_max_compute), I8_KC) * I8_KC);
  const int PA_SMEM_MAX = (int)sizeof(double) * PA_GROUP * pa_row_stride(FRPA_MAX_N_COMPUTE);
  FRPA_TRY(configured.run(plan.device, [smem, PA_SMEM_MAX]() -> int {
    FRPA_CUDA_TRY(cudaFuncSetAttribute(rho1_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    FRPA_CUDA_TRY(cudaFuncSetAttribute(i8_pack_a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PA_SMEM_MAX));
    return FRPA_OK;
  }));
  int n_sm = 148;
  FRPA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, plan.device));
  I8Params P;
  P.map = plan.d_map;
  P.ib_all = plan.d_ib;
  P.P1 = P1;
  P.rowmax = plan.d_rowmax;
  P.n_basis = plan.n_basis;
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
  P.a_scr = plan.d_i8_a;
  P.sa = plan.d_i8_sa;
  for (const I8Group &g : plan.i8_groups) {
    const int ni = g.item1 - g.item0, nu = g.unit1 - g.unit0;
    i8_pack_a_kernel<<<ni, PA_THREADS, pa_smem, stream>>>(plan.d_i8_items + g.item0, wave, plan.d_i8_a,
                                                          plan.d_i8_sa, P.wave_vec);
    FRPA_LAUNCH_CHECK();
    P.items = plan.d_i8_items;
    P.units = plan.d_i8_units + g.unit0;
    P.n_units = nu;
    rho1_i8_kernel<<<std::min(n_sm, nu), I8_THREADS, smem, stream>>>(P);
    FRPA_LAUNCH_CHECK();
  }
  return FRPA_OK;
}

}  // namespace frpa
