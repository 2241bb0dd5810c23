// Plain FP64 first-order density (rho1) and its gradient, one persistent
// grouped launch over the plan's work list.
//
// Reference semantics (fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho.cpp:116-209):
//   per non-empty grid batch b, perturbation t:
//     P1c(i, j)   = P1(ib[i], ib[j], t)                       (gather, :149-159)
//     work1       = P1c * phi                                 (GEMM,   :161-175)
//     rho1(map p) = sum_i phi(i, p) work1(i, p) + bias(p, b, t)           (:177-207)
//     grad(:,p,b,t) = 2 sum_i grad_phi(i, :, p) work1(i, p) - gbias(:, p, b, t)
// The reference GPU path runs gather, a MAGMA vbatched DGEMM and a ddot kernel
// as three launches with P1c and work1 round-tripping through HBM
// (evaluate_first_order_rho.cu:282-360).  Here one CTA owns a (batch, point
// tile) work item and fuses all three: P1c tiles are gathered straight into
// shared memory, the contraction runs on the FP64 tensor-core MMA
// (mma.sync m8n8k4 f64) with the accumulators in registers, and the epilogue
// contracts each finished work1 tile against phi / grad phi, so work1 never
// leaves the SM: the tile is staged in the shared-memory stage its last K
// chunk used, and each warp then reads whole point rows of phi / grad phi
// with 16-byte loads.  Per-point sums are reduced in a fixed order (lane
// pairs -> recursive halving over the warp -> row tiles in order), so results
// are deterministic.
//
// Optionally the same launch also computes the ground-state density-matrix
// part of the rho1 bias (what generate_first_order_rho_bias_part2.cpp:84-150
// produces as a separate pass; the reference's fused form is
// task1_atom_tiling/version3_rho_with_bias/evaluate_first_order_rho.cu.hpp:93-254):
// for perturbation t = atom j_atom_begin + t with compute range R,
//   bias(p) = sum_i phi_i(p) sum_{k in R} (D(ib_i, ib_k) + D(ib_k, ib_i)) (-d phi_k / d x_jcoord)(p),
// as extra K chunks after each row tile's main chunks (A: the symmetrised
// gather D(ib_i, ib_k) + D(ib_k, ib_i), B: the gradient of phi along j_coord),
// added to rho1 only.
#include <algorithm>
#include <vector>

#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int BM = 64;       // rows (i_compute) per tile
constexpr int KC = 32;       // contraction chunk
constexpr int STAGES = 2;    // cp.async pipeline depth (double buffering)
constexpr int LDA = BM + 4;  // As[k][m]: stride = 4 (mod 16) doubles -> conflict-free fragment loads
constexpr int LDB = KC + 4;  // Bs[n][k]: stride = 4 (mod 16) doubles, rows 16-byte aligned
constexpr int MAX_NC = FRPA_MAX_N_COMPUTE;
constexpr int WM = BM / 32;  // warps along M (warp tile 32 x 16)
// Epilogue staging: a finished 64-row work1 tile is written to the stage that
// its last K chunk used (rows 0-31 in A's buffer, rows 32-63 in B's), 64
// points per round, each point's 32 rows at a stride of LDW doubles
// (LDW = 2 mod 8: the fragment stores are conflict-free, rows 16-byte aligned).
constexpr int LDW = 34;
static_assert(BM == 64, "the epilogue staging assumes 64-row tiles");
static_assert(64 * LDW <= KC * LDA && 64 * LDW <= 64 * LDB, "a 64-point work1 half-tile fits a stage buffer");

// Tile shapes: BN points per work item, 2 warps along M x BN / 16 along N,
// warp tile 32 x 16, 32-wide K chunks.  BN = 64: 256 threads, 2 CTAs per SM
// (84 KB of shared memory each, up to 128 registers); BN = 128: 512 threads,
// one CTA per SM, each gathered P1c tile serving twice the points.
// The loop is issue-bound, not MMA-bound, when its bookkeeping is heavy: every
// step advances its (t, row tile, K chunk) position by increments (no integer
// division), and warps whose 32 x 16 tile and K chunk are complete run an
// unpredicated MMA loop.
template <int BN, bool BIAS>
struct Fp64Shape {
  static constexpr int WN = BN / 16;
  static constexpr int THREADS = 32 * WM * WN;
  static constexpr int MIN_BLOCKS = (BN == 64 && BM == 64) ? 2 : 1;
};

template <int BN>
struct Smem {
  double A[STAGES][KC * LDA];
  double B[STAGES][BN * LDB];
  double red[WM][4][BN];
  int ib[MAX_NC];
  int rs[FRPA_MAX_ATOM_TILE], re[FRPA_MAX_ATOM_TILE];  // fused bias: each perturbation's compute range
  int nkb;                                             // fused bias: K chunks per row tile
  int next;
};

// The in-kernel bias inputs (null dm: no fused bias).
struct FusedBias {
  const double *dm;       // ground-state density matrix (n_basis, n_basis)
  const int *atom_valid;  // (n_atoms + 1, n_batches), 0-based compute ranges
  int n_atoms, j_atom_begin, j_coord;
  int *err;               // device flags: bit 3 = a range leaves its batch (clipped)
};

// (K chunk, row tile, t) of one step, advanced by one step
__device__ __forceinline__ void step_advance(int &kk, int &mt, int &t, int nKs, int nMt) {
  if (++kk == nKs) {
    kk = 0;
    if (++mt == nMt) {
      mt = 0;
      ++t;
    }
  }
}

template <int BN, bool BIAS>
__global__ void __launch_bounds__(Fp64Shape<BN, BIAS>::THREADS, Fp64Shape<BN, BIAS>::MIN_BLOCKS)
    rho1_fp64_kernel(const Rho1WorkItem *__restrict__ items, int n_items, int *__restrict__ counter,
                     const int *__restrict__ ib_all, const int *__restrict__ map, int T, int n_active, int n_basis,
                     int n_full_points, int n_max_batch_size, int n_batches, const double *__restrict__ wave,
                     const double *__restrict__ gwave, const double *__restrict__ P1,
                     const double *__restrict__ bias, const double *__restrict__ gbias, double *__restrict__ rho,
                     double *__restrict__ grad, int aligned16, FusedBias fb) {
  constexpr int THREADS = Fp64Shape<BN, BIAS>::THREADS, WN = Fp64Shape<BN, BIAS>::WN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<BN> &S = *reinterpret_cast<Smem<BN> *>(smem_raw);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm = warp / WN, wn = warp % WN;
  const int col_w = wn * 16;  // this warp's first point in the tile
  const int g = lane >> 2, q = lane & 3;
  const long long nb2 = (long long)n_basis * n_basis;

  for (;;) {
    if (tid == 0) S.next = atomicAdd(counter, 1);
    __syncthreads();
    const int it = S.next;
    if (it >= n_items) break;
    const Rho1WorkItem W = items[it];
    const int nc = W.nc, pn = W.pn;
    const int ncp = (nc + 3) & ~3;
    for (int i = tid; i < nc; i += THREADS) S.ib[i] = ib_all[W.ib_off + i] - 1;
    if (BIAS && tid == 0) {
      int rmax = 0;
      for (int t = 0; t < T; ++t) {
        int r0 = 0, r1 = 0;
        if (fb.dm && t < n_active) {  // the bias of perturbation t belongs to atom j_atom_begin + t
          const int atom = fb.j_atom_begin + t;
          const int s0 = fb.atom_valid[(atom - 1) + (long long)(fb.n_atoms + 1) * W.batch];
          const int s1 = fb.atom_valid[atom + (long long)(fb.n_atoms + 1) * W.batch];
          r0 = min(max(s0, 0), nc);
          r1 = min(max(s1, r0), nc);
          if (r0 != s0 || r1 != s1) atomicOr(fb.err, 8);
        }
        S.rs[t] = r0;
        S.re[t] = r1;
        rmax = max(rmax, r1 - r0);
      }
      S.nkb = (rmax + KC - 1) / KC;
    }
    __syncthreads();

    const double *phi = wave + W.wave_off + (long long)W.p0 * ncp;
    const double *gph = gwave + 3 * W.wave_off + 3LL * W.p0 * ncp;
    const int nMt = (nc + BM - 1) / BM;
    const int nKc = (nc + KC - 1) / KC;
    const int nKb = BIAS ? S.nkb : 0, nKs = nKc + nKb;  // K chunks per (t, row tile): main, then the bias's
    const int steps = T * nMt * nKs;

    // position of the next chunk to load (runs STAGES - 1 steps ahead)
    int ld_kk = 0, ld_mt = 0, ld_t = 0;
    auto load = [&](int stage) {
      const int kk = ld_kk, mt = ld_mt, t = ld_t;
      step_advance(ld_kk, ld_mt, ld_t, nKs, nMt);
      const int m0 = mt * BM;
      double *As = S.A[stage];
      double *Bs = S.B[stage];
      if (BIAS && kk >= nKc) {
        // bias chunk over k in the perturbation's range: A = D(ib_i, ib_k) +
        // D(ib_k, ib_i), gathered with plain loads (the sum is formed on the
        // way into shared memory); B = d phi_k / d x_jcoord
        const int k0 = S.rs[t] + (kk - nKc) * KC, kend = S.re[t];
#pragma unroll
        for (int j = 0; j < (BM * KC) / THREADS; ++j) {
          const int e = tid + THREADS * j;
          const int m = e & (BM - 1), k = e / BM;
          const int gm = m0 + m, gk = k0 + k;
          double d = 0.0;
          if (gm < nc && gk < kend) {
            const long long bi = S.ib[gm], bk = S.ib[gk];
            d = __ldg(fb.dm + bi + bk * n_basis) + __ldg(fb.dm + bk + bi * n_basis);
          }
          As[k * LDA + m] = d;
        }
#pragma unroll
        for (int j = 0; j < (BN * KC) / THREADS; ++j) {
          const int e = tid + THREADS * j;
          const int k = e & (KC - 1), n = e / KC;
          const int gk = k0 + k;
          const bool ok = n < pn && gk < kend;
          cp_async_8(&Bs[n * LDB + k], ok ? gph + gk + (long long)ncp * ((fb.j_coord - 1) + 3LL * n) : gph,
                     ok ? 8 : 0);
        }
        return;
      }
      const int k0 = kk * KC;
      const double *P = P1 + t * nb2;
      // A: this thread's row is fixed (THREADS is a multiple of BM); its
      // columns step by THREADS / BM
      const int m = tid & (BM - 1), gm = m0 + m;
      const bool row_ok = gm < nc;
      const double *Prow = P + (row_ok ? S.ib[gm] : 0);
#pragma unroll
      for (int j = 0; j < (BM * KC) / THREADS; ++j) {
        const int k = tid / BM + (THREADS / BM) * j;
        const int gk = k0 + k;
        const bool ok = row_ok && gk < nc;
        cp_async_8(&As[k * LDA + m], ok ? Prow + (long long)S.ib[gk] * n_basis : P, ok ? 8 : 0);
      }
      if (aligned16) {
#pragma unroll
        for (int j = 0; j < (BN * KC / 2) / THREADS; ++j) {
          const int e = tid + THREADS * j;
          const int kp = e & (KC / 2 - 1), n = e / (KC / 2);
          const int gk = k0 + 2 * kp;
          int bytes = 0;
          if (n < pn) bytes = (gk + 1 < nc) ? 16 : (gk < nc ? 8 : 0);
          const double *src = bytes ? phi + gk + (long long)n * ncp : phi;
          cp_async_16(&Bs[n * LDB + 2 * kp], src, bytes);
        }
      } else {
#pragma unroll
        for (int j = 0; j < (BN * KC) / THREADS; ++j) {
          const int e = tid + THREADS * j;
          const int k = e & (KC - 1), n = e / KC;
          const int gk = k0 + k;
          const bool ok = n < pn && gk < nc;
          cp_async_8(&Bs[n * LDB + k], ok ? phi + gk + (long long)n * ncp : phi, ok ? 8 : 0);
        }
      }
    };

    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    // per-point sums: after each row tile's epilogue lane l of warp w holds the
    // sum (over rows so far) of component c = (l % NV) / PPW (rho1, d/dx, d/dy,
    // d/dz) of point w PPW + (l % NV) % PPW of each 64-point round
    constexpr int ROUNDS = BN / 64, NWARP = THREADS / 32, PPW = 64 / NWARP, NV = 4 * PPW;
    static_assert(NV == 16 || NV == 32, "per-lane reduction shape");
    double tot[ROUNDS];
#pragma unroll
    for (int r = 0; r < ROUNDS; ++r) tot[r] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < steps) load(s);
      cp_async_commit();
    }

    // all rows of perturbation t done: gather the per-lane sums by point, write
    // rho1 and grad rho1, clear the sums
    auto finish = [&](int t) {
      if (lane < NV) {
#pragma unroll
        for (int r = 0; r < ROUNDS; ++r) {
          const int idx = lane & (NV - 1);
          S.red[0][idx / PPW][r * 64 + warp * PPW + idx % PPW] = tot[r];
          tot[r] = 0.0;
        }
      }
      __syncthreads();
      if (tid < pn) {
        const int p = W.p0 + tid;
        const double r = S.red[0][0][tid], gx = S.red[0][1][tid], gy = S.red[0][2][tid], gz = S.red[0][3][tid];
        const long long bidx = p + (long long)n_max_batch_size * (W.batch + (long long)n_batches * t);
        const long long gi = 3 * bidx;
        grad[gi + 0] = gx * 2 - gbias[gi + 0];
        grad[gi + 1] = gy * 2 - gbias[gi + 1];
        grad[gi + 2] = gz * 2 - gbias[gi + 2];
        if (t < n_active) rho[map[W.prefix + p] + (long long)n_full_points * t] = r + bias[bidx];
      }
      __syncthreads();
    };

    // Epilogue of one finished tile (acc = work1 rows m0.., or the bias tile):
    // acc goes to this step's stage buffers, then each warp contracts PPW
    // points with phi (and grad phi): lane l takes rows 2l, 2l + 1 of a point
    // (16-byte loads, 512 contiguous bytes per warp and array), and the NV
    // per-lane products are summed over the 32 lanes by recursive halving
    // (31 shuffles), lane l keeping value l % NV.  Main tiles add all four
    // components; bias tiles subtract from rho1 only.
    auto tile_epilogue = [&](int stage, int m0, bool bias_tile) {
      double *Wa = S.A[stage], *Wb = S.B[stage];
      __syncthreads();  // every warp's MMAs are done with this stage's operands
#pragma unroll
      for (int round = 0; round < ROUNDS; ++round) {
        if (col_w / 64 == round) {
          double *Wh = wm == 0 ? Wa : Wb;
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
#pragma unroll
              for (int h = 0; h < 2; ++h)
                Wh[((col_w & 63) + ni * 8 + 2 * q + h) * LDW + mi * 8 + g] = acc[mi][ni][h];
        }
        __syncthreads();
        double v[NV];
        const int r0 = m0 + 2 * lane;
        const bool in_block = r0 < ncp, ok0 = r0 < nc, ok1 = r0 + 1 < nc;
#pragma unroll
        for (int j = 0; j < PPW; ++j) {
          const int pl = warp * PPW + j, p = round * 64 + pl;
#pragma unroll
          for (int c = 0; c < 4; ++c) v[c * PPW + j] = 0.0;
          if (p < pn && in_block) {
            const double2 w = *reinterpret_cast<const double2 *>((lane < 16 ? Wa : Wb) + pl * LDW + 2 * (lane & 15));
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              if (bias_tile && c > 0) continue;
              const double *src =
                  c == 0 ? phi + r0 + (long long)p * ncp : gph + r0 + (long long)ncp * (3LL * p + (c - 1));
              double x0, x1;
              if (aligned16) {
                const double2 x = __ldg(reinterpret_cast<const double2 *>(src));
                x0 = x.x;
                x1 = x.y;
              } else {
                x0 = __ldg(src);
                x1 = __ldg(src + 1);
              }
              v[c * PPW + j] = fma(ok1 ? x1 : 0.0, w.y, (ok0 ? x0 : 0.0) * w.x);
            }
          }
        }
        // sum over the 32 lanes: fold the offsets >= NV, then halve
#pragma unroll
        for (int o = 16; o >= NV; o >>= 1)
#pragma unroll
          for (int i = 0; i < NV; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
#pragma unroll
        for (int o = NV / 2; o >= 1; o >>= 1) {
          const bool upper = (lane & o) != 0;
#pragma unroll
          for (int i = 0; i < o; ++i) {
            const double keep = upper ? v[i + o] : v[i], give = upper ? v[i] : v[i + o];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, give, o);
          }
        }
        if (bias_tile)
          tot[round] -= v[0];
        else
          tot[round] += v[0];
        if (round + 1 < ROUNDS) __syncthreads();  // the next round rewrites the staging
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    };

    int kk = 0, mt = 0, t = 0;
    for (int s = 0; s < steps; ++s) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      if (s + STAGES - 1 < steps) load((s + STAGES - 1) % STAGES);
      cp_async_commit();

      const int m0 = mt * BM;
      const double *As = S.A[s % STAGES];
      const double *Bs = S.B[s % STAGES];
      const int row_w = m0 + wm * 32;
      // valid K extent of this chunk: the compute functions, or the bias range
      const int klim = (!BIAS || kk < nKc) ? nc - kk * KC : (S.re[t] - S.rs[t]) - (kk - nKc) * KC;
      if (row_w + 32 <= nc && col_w + 16 <= pn && klim >= KC) {
        // complete warp tile and chunk: no predicates
#pragma unroll
        for (int ks = 0; ks < KC / 4; ++ks) {
          double a[4], b[2];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) a[mi] = As[(ks * 4 + q) * LDA + wm * 32 + mi * 8 + g];
#pragma unroll
          for (int ni = 0; ni < 2; ++ni) b[ni] = Bs[(col_w + ni * 8 + g) * LDB + ks * 4 + q];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
      } else if (row_w < nc && col_w < pn) {
        const int nmi = min(4, (nc - row_w + 7) / 8), nni = min(2, (pn - col_w + 7) / 8);
#pragma unroll
        for (int ks = 0; ks < KC / 4; ++ks) {
          if (ks * 4 < klim) {
            double a[4], b[2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) a[mi] = As[(ks * 4 + q) * LDA + wm * 32 + mi * 8 + g];
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) b[ni] = Bs[(col_w + ni * 8 + g) * LDB + ks * 4 + q];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
              for (int ni = 0; ni < 2; ++ni)
                if (mi < nmi && ni < nni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
          }
        }
      }

      if (kk == nKc - 1) {
        tile_epilogue(s % STAGES, m0, false);  // work1 tile: contract with phi and grad phi
        if (!BIAS && mt == nMt - 1) finish(t);
      }
      // the bias of this row tile: rho1 -= sum_i phi_i (S d phi / d x_jcoord)_i
      if (BIAS && nKb > 0 && kk == nKs - 1) tile_epilogue(s % STAGES, m0, true);
      if (BIAS && kk == nKs - 1 && mt == nMt - 1) finish(t);
      step_advance(kk, mt, t, nKs, nMt);
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

template <int BN, bool BIAS>
int fp64_grid(int device, int ctas_per_sm) {
  static int cached[64] = {0};
  const int smem = (int)sizeof(Smem<BN>);
  if (device < 0 || device >= 64 || !cached[device]) {
    if (cudaFuncSetAttribute(rho1_fp64_kernel<BN, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rho1_fp64_kernel<BN, BIAS>, Fp64Shape<BN, BIAS>::THREADS, smem) !=
        cudaSuccess)
      return 0;
    if (device >= 0 && device < 64) cached[device] = per_sm > 0 ? per_sm : 1;
    if (device < 0 || device >= 64) return 0;
  }
  int n_sm = 0;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  const int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, cached[device]) : cached[device];
  return per_sm * n_sm;
}

// items [item0, item0 + n_items) of the plan's list; the cursor must be zero
template <int BN, bool BIAS>
int fp64_launch(const Rho1Plan &plan, int item0, int n_items, int n_active, const double *wave, const double *gwave,
                const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                const FusedBias *fused, cudaStream_t stream) {
  int grid = fp64_grid<BN, BIAS>(plan.device, plan.fp64_ctas_per_sm);
  if (grid <= 0) return fail(FRPA_ERR_CUDA, "rho1_fp64: occupancy query failed");
  if (grid > n_items) grid = n_items;
  if (grid <= 0) return FRPA_OK;
  FusedBias fb{};
  if (fused) fb = *fused;
  // 16-byte loads need even batch offsets (the plan) and 16-byte aligned arrays
  const int aligned16 = plan.wave_aligned16 && !(((uintptr_t)wave | (uintptr_t)gwave) & 15);
  rho1_fp64_kernel<BN, BIAS><<<grid, Fp64Shape<BN, BIAS>::THREADS, sizeof(Smem<BN>), stream>>>(
      plan.d_items + item0, n_items, plan.d_counter, plan.d_ib, plan.d_map, plan.T, n_active, plan.n_basis,
      plan.n_full_points, plan.n_max_batch_size, plan.n_batches, wave, gwave, P1, bias, gbias, rho, grad,
      aligned16, fb);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

}  // namespace

// Sets the kernels' shared-memory attributes once per device (outside any
// stream capture); 0 on failure.
int rho1_fp64_grid(int device) {
  return fp64_grid<64, false>(device, 0) > 0 && fp64_grid<128, false>(device, 0) > 0 &&
                 fp64_grid<64, true>(device, 0) > 0 && fp64_grid<128, true>(device, 0) > 0
             ? fp64_grid<64, false>(device, 0)
             : 0;
}

static int fp64_run(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *P1,
                    const double *bias, const double *gbias, double *rho, double *grad, const FusedBias *fused,
                    cudaStream_t stream) {
  // evaluate_first_order_rho.cpp:113-114 zeroes both outputs before the batch loop
  FRPA_CUDA_TRY(cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)plan.n_full_points * plan.T, stream));
  FRPA_CUDA_TRY(cudaMemsetAsync(
      grad, 0, sizeof(double) * 3 * (size_t)plan.n_max_batch_size * plan.n_batches * plan.T, stream));
  if (plan.n_items == 0) return FRPA_OK;
  FRPA_CUDA_TRY(cudaMemsetAsync(plan.d_counter, 0, sizeof(int), stream));
  if (fused) {
    if (plan.fp64_tile_points == 128)
      return fp64_launch<128, true>(plan, 0, plan.n_items, n_active, wave, gwave, P1, bias, gbias, rho, grad, fused,
                                    stream);
    return fp64_launch<64, true>(plan, 0, plan.n_items, n_active, wave, gwave, P1, bias, gbias, rho, grad, fused,
                                 stream);
  }
  if (plan.fp64_tile_points == 128)
    return fp64_launch<128, false>(plan, 0, plan.n_items, n_active, wave, gwave, P1, bias, gbias, rho, grad, nullptr,
                                   stream);
  return fp64_launch<64, false>(plan, 0, plan.n_items, n_active, wave, gwave, P1, bias, gbias, rho, grad, nullptr,
                                stream);
}

int rho1_fp64_launch_chunk(const Rho1Plan &plan, int chunk, int n_active, const double *wave, const double *gwave,
                           const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                           cudaStream_t stream) {
  if (chunk < 0 || chunk + 1 >= (int)plan.fp64_chunk_items.size())
    return fail(FRPA_ERR_INVALID, "rho1_fp64: chunk %d outside the plan's %d", chunk,
                (int)plan.fp64_chunk_items.size() - 1);
  const int i0 = plan.fp64_chunk_items[chunk], n = plan.fp64_chunk_items[chunk + 1] - i0;
  if (n <= 0) return FRPA_OK;
  FRPA_CUDA_TRY(cudaMemsetAsync(plan.d_counter, 0, sizeof(int), stream));
  if (plan.fp64_tile_points == 128)
    return fp64_launch<128, false>(plan, i0, n, n_active, wave, gwave, P1, bias, gbias, rho, grad, nullptr, stream);
  return fp64_launch<64, false>(plan, i0, n, n_active, wave, gwave, P1, bias, gbias, rho, grad, nullptr, stream);
}

int rho1_fp64_launch(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *P1,
                     const double *bias, const double *gbias, double *rho, double *grad, cudaStream_t stream) {
  return fp64_run(plan, n_active, wave, gwave, P1, bias, gbias, rho, grad, nullptr, stream);
}

int rho1_fp64_fused_bias_launch(const Rho1Plan &plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                                const int *atom_valid, const double *density_matrix, const double *wave,
                                const double *gwave, const double *P1, const double *bias, const double *gbias,
                                double *rho, double *grad, cudaStream_t stream) {
  FusedBias fb{density_matrix, atom_valid, n_atoms, j_atom_begin, j_coord, plan.d_err};
  return fp64_run(plan, n_active, wave, gwave, P1, bias, gbias, rho, grad, &fb, stream);
}

// Orders a work list: 0 largest nc^2 x points first, 1 batch order, 2 by the
// batches' locality key (batches sharing basis functions run together, so
// the density-matrix blocks they gather stay in L2), largest first within a key.
void rho1_order_items(std::vector<Rho1WorkItem> *items, int order) {
  auto cost = [](const Rho1WorkItem &a) { return (long long)a.nc * a.nc * a.pn; };
  if (order == 0)
    std::stable_sort(items->begin(), items->end(),
                     [&](const Rho1WorkItem &a, const Rho1WorkItem &b) { return cost(a) > cost(b); });
  else if (order == 2)
    std::stable_sort(items->begin(), items->end(), [&](const Rho1WorkItem &a, const Rho1WorkItem &b) {
      if (a.key != b.key) return (unsigned)a.key < (unsigned)b.key;
      return cost(a) > cost(b);
    });
}

// MinHash of a batch's basis list (1-based indices): the smallest 32-bit
// integer hash over its functions (Wellons' lowbias32 mixer).  Batches whose
// lists overlap a lot share it with high probability.
int rho1_locality_key(const int *ib, int nc) {
  unsigned best = 0xffffffffu;
  for (int i = 0; i < nc; ++i) {
    unsigned x = (unsigned)ib[i];
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    best = std::min(best, x);
  }
  return (int)best;
}

// Work items of <= tile_points points (a batch's points split evenly, widths a
// multiple of 8), grouped into FP64_CHUNKS ranges of consecutive batches, each
// range in the given order.  The ranges hold 6%, 44%, 44% and 6% of the cost
// (nc^2 np): the host-buffer entry waits for the first range's biases before
// any compute and for the last range's outputs after it, so those are small.
void rho1_fp64_build_items(const std::vector<Rho1WorkItem> &batches, int tile_points, int order, int n_batches,
                           std::vector<Rho1WorkItem> *out, std::vector<int> *chunk_items,
                           std::vector<int> *chunk_batches) {
  // chunk boundaries in the caller's batch indices (batches are in that order)
  double total = 0.0;
  for (const Rho1WorkItem &b : batches) total += (double)b.nc * b.nc * b.np;
  static_assert(FP64_CHUNKS == 4, "cost split of the chunks");
  const double split[FP64_CHUNKS + 1] = {0.0, 0.06, 0.50, 0.94, 1.0};
  std::vector<int> bounds(FP64_CHUNKS + 1, n_batches);
  bounds[0] = 0;
  {
    double run = 0.0;
    int c = 1;
    for (const Rho1WorkItem &b : batches) {
      while (c < FP64_CHUNKS && run >= total * split[c]) bounds[c++] = b.batch;
      run += (double)b.nc * b.nc * b.np;
    }
    for (; c < FP64_CHUNKS; ++c) bounds[c] = n_batches;
  }
  out->clear();
  std::vector<int> item_bounds(FP64_CHUNKS + 1, 0);
  for (int c = 0; c < FP64_CHUNKS; ++c) {
    std::vector<Rho1WorkItem> part;
    for (const Rho1WorkItem &b : batches) {
      if (b.np == 0 || b.batch < bounds[c] || b.batch >= bounds[c + 1]) continue;
      const int tiles = (b.np + tile_points - 1) / tile_points;
      int w = (b.np + tiles - 1) / tiles;
      w = std::min(tile_points, (w + 7) & ~7);
      for (int p0 = 0; p0 < b.np; p0 += w)
        part.push_back(Rho1WorkItem{b.batch, b.nc, b.np, p0, std::min(w, b.np - p0), b.ib_off, b.prefix, b.key,
                                    b.wave_off});
    }
    rho1_order_items(&part, order);
    out->insert(out->end(), part.begin(), part.end());
    item_bounds[c + 1] = (int)out->size();
  }
  if (chunk_items) *chunk_items = item_bounds;
  if (chunk_batches) *chunk_batches = bounds;
}

}  // namespace frpa
