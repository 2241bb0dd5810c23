// The first-order H integration and the adjoint of rho1 with respect to P1,
// one engine for both: per batch and perturbation t, a contraction over the
// batch's points of a per-point combination A(i, p) of phi, grad phi and the
// Hessian of phi with phi itself, scattered into an (n_basis, n_basis, T)
// matrix through the batch's compute-function list.
//
// First-order H (fast_rap_src_dfpt_gpu_eval/evaluate_first_order_H.cpp:77-215):
//   A(i, p) = cs1(i, p) = c_phi(p) phi_i + sum_k c_grad_k(p) d_k phi_i
//             + [i in atom j's range] sum_k c_hess_k(p) hess_i(k, j_coord),
//   c_phi = (H_prefactor1 + pf3) / 2, c_grad = pf2, c_hess = -pf5 with the
//   reference's per-point prefactors (:144-168), and
//   H(ib_i, ib_j, t) += sum_p A(i, p) phi_j(p) + phi_i(p) A(j, p)
//   (its rank-2k update and symmetric scatter, :192-215).
// Adjoint of rho1 (evaluate_first_order_rho.cpp:149-207):
//   A(i, p) = g_rho(map p, t) phi_i + 2 sum_d g_grad(d, p, b, t) d_d phi_i,
//   dP1(ib_i, ib_j, t) += sum_p A(i, p) phi_j(p).
// With g_rho = w v and no g_grad the adjoint is the first-order H with every
// exchange-correlation term zero.
//
// Work: one CTA per 64 x 64 (i, j) tile of one batch and perturbation on the
// FP64 MMA (mma.sync m8n8k4, the only FP64 tensor instruction of sm_100a),
// A and phi staged in shared memory as the point dimension streams; the
// symmetric H computes the tiles with j >= i only, each from both products.
//
// Determinism.  Batches overlap in the output, so tiles of different batches
// add into the same entries.  Every contribution is added as a 128-bit
// fixed-point integer (two 64-bit words, the low word's carry propagated by
// the thread that produced it), and integer addition does not depend on the
// order: two runs give bit-identical results.  The fixed-point scale 2^s is
// fixed per call before any addition from a bound of the inputs (a pass over
// phi, grad phi, Hessian and the per-point coefficients): every single
// contribution is below 2^emax, at most 2 n_batches contributions meet in one
// entry, so with s = 100 - emax - ceil(log2(2 n_batches)) every partial sum
// stays below 2^100 and each contribution is represented to 2^-s, about 2^-80
// of the largest one.  A last pass converts each entry to FP64 (one rounding)
// and adds it to the output.
#include <climits>
#include <cstring>
#include <vector>

#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int BM = 64, BN = 64, KC = 16, THREADS = 256;
constexpr int COEF_PTS = 128;  // points whose coefficients are staged together (a multiple of KC)
static_assert(COEF_PTS % KC == 0, "coefficient stage holds whole K chunks");
constexpr int LDA = BM + 4;  // As[k = point][m = i]
constexpr int LDB = KC + 4;  // Bs[n = j][k = point]
constexpr int EMAX_EMPTY = -2139062144;  // 0x80808080: no non-zero bound seen
constexpr int H1_FLAG_NONFINITE = 16;    // device flag: a non-finite input reached the accumulation

struct H1Item {
  int batch, nc, np, ib_off, prefix, m0, n0, t;
  long long wave_off;
};

// Per-point inputs of the first-order H, reference layouts
// (evaluate_first_order_H.cpp:13-53); nullptr members mean "adjoint mode".
struct H1Inputs {
  const double *vsigma, *gradient_rho, *hessian, *H_prefactor1, *fogr, *vhg, *rho1, *v2rho2, *v2rhosigma,
      *v2sigma2, *partition_tab;
  const int *atom_valid;  // (n_atoms + 1, n_batches), 0-based compute ranges
  int n_atoms, j_atom_begin, j_coord;
};

struct H1Args {
  int mode;  // 0: adjoint, 1: first-order H
  int n_active, n_basis, n_full_points, n_max_batch_size, n_batches;
  const int *ib_all, *map;
  const double *wave, *gwave;
  const double *g_rho, *g_grad;  // adjoint mode
  H1Inputs h;                     // first-order H mode
  unsigned long long *acc;        // (2, n_basis, n_basis, T): low words, then high words
  long long n_entries;            // n_basis^2 T
  int *emax;
  int *err;
};

// Coefficients of A(i, p) for one point of batch b, perturbation t.
struct PointCoef {
  double c_phi, c_grad[3], c_hess[3];
};

__device__ __forceinline__ PointCoef point_coef(const H1Args &a, int b, int p, int prefix, int t) {
  PointCoef c;
  const long long f = a.map[prefix + p];
  const long long bp = p + (long long)a.n_max_batch_size * (b + (long long)a.n_batches * t);
  if (a.mode == 0) {
    c.c_phi = (a.g_rho != nullptr && t < a.n_active) ? a.g_rho[f + (long long)a.n_full_points * t] : 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      c.c_grad[k] = a.g_grad ? 2.0 * a.g_grad[3 * bp + k] : 0.0;
      c.c_hess[k] = 0.0;
    }
    return c;
  }
  // evaluate_first_order_H.cpp:144-168, same operation order
  const H1Inputs &h = a.h;
  const long long nmb = a.n_max_batch_size;
  const double pf1 = h.H_prefactor1[bp];
  const double *fog = h.fogr + 3 * bp;
  const double *gr = h.gradient_rho + 3 * f;
  const double vsig = h.vsigma[3 * nmb * b + 3 * p];
  const double v2r2 = h.v2rho2[3 * nmb * b + 3 * p];
  const double v2rs = h.v2rhosigma[6 * nmb * b + 6 * p];
  const double v2s2 = h.v2sigma2[6 * nmb * b + 6 * p];
  const double w = h.partition_tab[f];
  const double r1 = h.rho1[f + (long long)a.n_full_points * t];
  double lfos = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) lfos = __dadd_rn(lfos, __dmul_rn(fog[k], gr[k]));
  lfos = __dmul_rn(lfos, 2.0);
  const double inner = __dadd_rn(__dmul_rn(v2rs, r1), __dmul_rn(v2s2, lfos));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c.c_grad[k] = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, w), gr[k]), inner),
                            __dmul_rn(__dmul_rn(__dmul_rn(2.0, w), vsig), fog[k]));
    c.c_hess[k] = -__dmul_rn(__dmul_rn(__dmul_rn(2.0, vsig), w), gr[k]);
  }
  const double pf3 = __dmul_rn(w, __dadd_rn(__dadd_rn(h.vhg[f + (long long)a.n_full_points * t], __dmul_rn(v2r2, r1)),
                                            __dmul_rn(v2rs, lfos)));
  c.c_phi = __dmul_rn(0.5, __dadd_rn(pf1, pf3));
  return c;
}

// Hessian component of hess_i(k, j_coord) (evaluate_first_order_H.cpp:6-10,185).
__device__ __forceinline__ int hess_component(int k, int j_coord) {
  const int r = j_coord - 1;
  return k == 0 ? r : (k == 1 ? (r == 0 ? 1 : (r == 1 ? 3 : 4)) : (r == 0 ? 2 : (r == 1 ? 4 : 5)));
}

// A(i, p) from the point's coefficients; i < nc.
__device__ __forceinline__ double a_value(const PointCoef &c, const double *phi, const double *gph,
                                          const double *hph, int i, int ncp, bool in_range, int j_coord) {
  double v = c.c_phi * phi[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) v = fma(c.c_grad[k], gph[i + k * ncp], v);
  if (in_range) {
#pragma unroll
    for (int k = 0; k < 3; ++k) v = fma(c.c_hess[k], hph[i + hess_component(k, j_coord) * ncp], v);
  }
  return v;
}

// Compute-function range [vs, ve) of atom j_atom_begin + t in batch b
// (atom_valid_n_compute_c_batches, evaluate_first_order_H.cpp:131-133),
// clipped to the batch's compute functions; a range that leaves them sets
// device flag bit 3 (once, from the bound pass) and is clipped, never read
// outside the batch.
__device__ __forceinline__ void atom_range(const H1Args &a, int b, int t, int nc, int *vs, int *ve, bool flag) {
  const int atom = a.h.j_atom_begin + t;  // 1-based
  int s0 = 0, s1 = 0;
  if (atom >= 1 && atom <= a.h.n_atoms) {
    s0 = a.h.atom_valid[(atom - 1) + (long long)(a.h.n_atoms + 1) * b];
    s1 = a.h.atom_valid[atom + (long long)(a.h.n_atoms + 1) * b];
  }
  const int c0 = min(max(s0, 0), nc), c1 = min(max(s1, c0), nc);
  if (flag && (c0 != s0 || c1 != s1)) atomicOr(a.err, 8);
  *vs = c0;
  *ve = c1;
}

// ---------------------------------------------------------------- bound

// One block per (batch, t): bound_b = sum_p max_i |A(i, p)| max_j |phi_j(p)|
// (twice that for the symmetric H), then atomicMax of its binary exponent.
__global__ void __launch_bounds__(THREADS) h1_bound_kernel(const H1Item *__restrict__ items, int n_items,
                                                           H1Args a) {
  __shared__ double red[THREADS / 32];
  const int it = blockIdx.x;
  const H1Item W = items[it];
  if (W.m0 != 0 || W.n0 != 0) return;  // one block per (batch, t): its first tile
  const int t = W.t;
  if (a.mode == 1 && t >= a.n_active) return;
  const int nc = W.nc, np = W.np, ncp = (nc + 3) & ~3;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int vs = 0, ve = 0;
  if (a.mode == 1) atom_range(a, W.batch, t, nc, &vs, &ve, true);
  double sum = 0.0;
  bool finite = true;
  for (int p = warp; p < np; p += THREADS / 32) {
    const PointCoef c = point_coef(a, W.batch, p, W.prefix, t);
    const double *phi = a.wave + W.wave_off + (long long)p * ncp;
    const double *gph = a.gwave + 3 * W.wave_off + 3LL * p * ncp;
    const double *hph = a.mode == 1 ? a.h.hessian + 6 * W.wave_off + 6LL * p * ncp : nullptr;
    double mp = 0.0, mg = 0.0, mh = 0.0;
    for (int i = lane; i < nc; i += 32) {
      mp = fmax(mp, fabs(phi[i]));
#pragma unroll
      for (int k = 0; k < 3; ++k) mg = fmax(mg, fabs(gph[i + k * ncp]));
      if (hph && i >= vs && i < ve) {
#pragma unroll
        for (int k = 0; k < 3; ++k) mh = fmax(mh, fabs(hph[i + hess_component(k, a.h.j_coord) * ncp]));
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      mp = fmax(mp, __shfl_xor_sync(0xffffffffu, mp, o));
      mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
      mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
    }
    const double ca = fabs(c.c_phi) * mp +
                      (fabs(c.c_grad[0]) + fabs(c.c_grad[1]) + fabs(c.c_grad[2])) * mg +
                      (fabs(c.c_hess[0]) + fabs(c.c_hess[1]) + fabs(c.c_hess[2])) * mh;
    const double term = ca * mp;
    if (!(term <= 1.0e300)) finite = false;  // NaN, Inf or beyond what the bound can carry
    if (lane == 0) sum += term;
  }
  if (lane == 0) red[warp] = finite ? sum : -1.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    bool ok = true;
    for (int w = 0; w < THREADS / 32; ++w) {
      if (red[w] < 0.0) ok = false;
      s += red[w];
    }
    if (!ok || !(s <= 1.0e300)) {
      atomicOr(a.err, H1_FLAG_NONFINITE);
      return;
    }
    if (a.mode == 1) s *= 2.0;
    if (s > 0.0) {
      int e = 0;
      frexp(s, &e);  // s < 2^e
      atomicMax(a.emax, e);
    }
  }
}

__device__ __forceinline__ int ceil_log2(long long n) {
  int k = 0;
  while ((1LL << k) < n) ++k;
  return k;
}

// The fixed-point exponent of this call (see the file comment).
__device__ __forceinline__ int fixed_scale(int emax, int n_batches) {
  return 100 - emax - ceil_log2(2LL * (n_batches > 0 ? n_batches : 1));
}

// v 2^s (|v 2^s| < 2^100) rounded to an integer, added to the 128-bit entry
// (lo, hi).  Modular two's-complement arithmetic: the carry out of the low
// word is exactly the one of this addition, whatever other threads add.
__device__ __forceinline__ void add_fixed(unsigned long long *lo, unsigned long long *hi, double v, int s) {
  if (v == 0.0) return;
  const double V = rint(ldexp(v, s));
  const double A = trunc(ldexp(V, -52));
  const double B = V - ldexp(A, 52);  // exact, |B| < 2^52
  const __int128 x = ((__int128)(long long)A << 52) + (__int128)(long long)B;
  const unsigned long long xl = (unsigned long long)x;
  const unsigned long long xh = (unsigned long long)(x >> 64);
  const unsigned long long old = atomicAdd(lo, xl);
  const unsigned long long carry = (old + xl < old) ? 1ull : 0ull;
  atomicAdd(hi, xh + carry);
}

// ----------------------------------------------------------------- tiles

template <bool SYM>
__global__ void __launch_bounds__(THREADS, 2) h1_tile_kernel(const H1Item *__restrict__ items, int n_items, H1Args a) {
  __shared__ __align__(16) double As[KC * LDA];  // A(m0 + m, k)
  __shared__ __align__(16) double Bs[BN * LDB];  // phi(n0 + n, k)
  __shared__ __align__(16) double Ps[SYM ? KC * LDA : 1];  // phi(m0 + m, k)
  __shared__ __align__(16) double Qs[SYM ? BN * LDB : 1];  // A(n0 + n, k)
  __shared__ PointCoef coef[COEF_PTS];  // the per-point coefficients of COEF_PTS points at a time
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3, g = lane >> 2, q = lane & 3;
  const long long nb2 = (long long)a.n_basis * a.n_basis;
  const int emax = *a.emax;
  if (emax == EMAX_EMPTY) return;  // every contribution is zero
  const int s = fixed_scale(emax, a.n_batches);
  unsigned long long *acc_lo = a.acc, *acc_hi = a.acc + a.n_entries;

  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const H1Item W = items[it];
    const int nc = W.nc, np = W.np, t = W.t, ncp = (nc + 3) & ~3;
    if (a.mode == 1 && t >= a.n_active) continue;
    const double *phi = a.wave + W.wave_off;
    const double *gph = a.gwave + 3 * W.wave_off;
    const double *hph = a.mode == 1 ? a.h.hessian + 6 * W.wave_off : nullptr;
    int vs = 0, ve = 0;
    if (a.mode == 1) atom_range(a, W.batch, t, nc, &vs, &ve, false);
    double acc[4][2][2];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 2; ++y) acc[x][y][0] = acc[x][y][1] = 0.0;

    for (int k0 = 0; k0 < np; k0 += KC) {
      if (k0 % COEF_PTS == 0) {  // every thread, one point each (the loads of many points in flight)
        for (int e = tid; e < COEF_PTS && k0 + e < np; e += THREADS) coef[e] = point_coef(a, W.batch, k0 + e, W.prefix, t);
      }
      __syncthreads();
      {
        // thread -> one point k of the chunk and four consecutive rows: the
        // point's coefficients are read once, the rows' loads coalesce
        constexpr int RPT = (BM * KC) / THREADS;  // rows per thread (4)
        const int k = tid / (BM / RPT), r0 = (tid % (BM / RPT)) * RPT, p = k0 + k;
        const bool pok = p < np;
        const long long pc = (long long)(pok ? p : 0) * ncp;
        const PointCoef c = coef[(k0 % COEF_PTS) + k];
        const int jc = a.mode == 1 ? a.h.j_coord : 1;
        const double *ph = phi + pc, *gp = gph + 3 * pc, *hp = hph ? hph + 6 * pc : nullptr;
#pragma unroll
        for (int rr = 0; rr < RPT; ++rr) {
          const int i = W.m0 + r0 + rr;
          double va = 0.0, vp = 0.0;
          if (pok && i < nc) {
            va = a_value(c, ph, gp, hp, i, ncp, hp != nullptr && i >= vs && i < ve, jc);
            if (SYM) vp = ph[i];
          }
          As[k * LDA + r0 + rr] = va;
          if (SYM) Ps[k * LDA + r0 + rr] = vp;
        }
#pragma unroll
        for (int rr = 0; rr < RPT; ++rr) {
          const int jj = W.n0 + r0 + rr;
          double vb = 0.0, vq = 0.0;
          if (pok && jj < nc) {
            vb = ph[jj];
            if (SYM) vq = a_value(c, ph, gp, hp, jj, ncp, hp != nullptr && jj >= vs && jj < ve, jc);
          }
          Bs[(r0 + rr) * LDB + k] = vb;
          if (SYM) Qs[(r0 + rr) * LDB + k] = vq;
        }
      }
      __syncthreads();
#pragma unroll
      for (int ks = 0; ks < KC / 4; ++ks) {
        double fa[4], fb[2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) fa[mi] = As[(ks * 4 + q) * LDA + wm * 32 + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) fb[ni] = Bs[(wn * 16 + ni * 8 + g) * LDB + ks * 4 + q];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int ni = 0; ni < 2; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], fa[mi], fb[ni]);
        if (SYM) {
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) fa[mi] = Ps[(ks * 4 + q) * LDA + wm * 32 + mi * 8 + g];
#pragma unroll
          for (int ni = 0; ni < 2; ++ni) fb[ni] = Qs[(wn * 16 + ni * 8 + g) * LDB + ks * 4 + q];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], fa[mi], fb[ni]);
        }
      }
      __syncthreads();
    }
    // add the tile (and, for an off-diagonal symmetric tile, its transpose)
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int i = W.m0 + wm * 32 + mi * 8 + g;
      if (i >= nc) continue;
      const long long row = a.ib_all[W.ib_off + i] - 1;
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int jj = W.n0 + wn * 16 + ni * 8 + 2 * q + hh;
          if (jj >= nc) continue;
          const long long col = a.ib_all[W.ib_off + jj] - 1;
          const double v = acc[mi][ni][hh];
          const long long e1 = row + col * a.n_basis + t * nb2;
          add_fixed(acc_lo + e1, acc_hi + e1, v, s);
          if (SYM && W.n0 != W.m0) {
            const long long e2 = col + row * a.n_basis + t * nb2;
            add_fixed(acc_lo + e2, acc_hi + e2, v, s);
          }
        }
    }
  }
}

// out(e) += (the 128-bit entry) 2^-s, one rounding; entries no tile touched add 0.
__global__ void h1_finalize_kernel(long long n, const unsigned long long *__restrict__ acc, const int *emax_p,
                                   int n_batches, double *__restrict__ out) {
  const int emax = *emax_p;
  if (emax == EMAX_EMPTY) return;
  const int s = fixed_scale(emax, n_batches);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const __int128 x = (__int128)(((unsigned __int128)acc[n + e] << 64) | acc[e]);
    if (x == 0) continue;
    // magnitude as two unsigned words of one sign: no cancellation, the
    // result within 2 ulp, and the same bits on every run
    const unsigned __int128 m = x < 0 ? (unsigned __int128)(-x) : (unsigned __int128)x;
    const double v = ldexp((double)(unsigned long long)(m >> 64), 64) + (double)(unsigned long long)m;
    out[e] += ldexp(x < 0 ? -v : v, -s);
  }
}

}  // namespace

size_t rho1_h1_item_size() { return sizeof(H1Item); }

// Packs (batch, i tile, j tile, t) items; `sym` keeps the tiles with j >= i.
void rho1_h1_build_items(const int *nc_b, const int *np_b, const int *ib_off, const int *prefix,
                         const long long *wave_off, int n_batches, int T, bool sym,
                         std::vector<unsigned char> *host) {
  std::vector<H1Item> v;
  for (int b = 0; b < n_batches; ++b) {
    if (nc_b[b] <= 0 || np_b[b] <= 0) continue;
    for (int t = 0; t < T; ++t)
      for (int m0 = 0; m0 < nc_b[b]; m0 += BM)
        for (int n0 = sym ? m0 : 0; n0 < nc_b[b]; n0 += BN)
          v.push_back(H1Item{b, nc_b[b], np_b[b], ib_off[b], prefix[b], m0, n0, t, wave_off[b]});
  }
  host->resize(v.size() * sizeof(H1Item));
  if (!v.empty()) memcpy(host->data(), v.data(), host->size());
}

// Accumulator scratch: two words per entry of (n_basis, n_basis, T), plus the
// exponent word; allocated by the first call (outside stream capture).
static int h1_scratch(Rho1Plan &plan, cudaStream_t stream) {
  if (plan.d_h1_acc) return FRPA_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  FRPA_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(FRPA_ERR_INVALID,
                "first-order H / adjoint: the accumulator is allocated by the first call; call once before "
                "capturing a graph");
  const size_t n = (size_t)plan.n_basis * plan.n_basis * plan.T;
  if (cudaMalloc((void **)&plan.d_h1_acc, 2 * n * sizeof(unsigned long long) + 256) != cudaSuccess) {
    plan.d_h1_acc = nullptr;
    return fail(FRPA_ERR_OOM, "first-order H / adjoint: %zu bytes of accumulator could not be allocated",
                2 * n * sizeof(unsigned long long) + 256);
  }
  return FRPA_OK;
}

// mode 0: the adjoint over the full tile list; mode 1: the first-order H over
// the symmetric one.  `out` (n_basis, n_basis, T) is accumulated into.
static int h1_run(Rho1Plan &plan, int mode, int n_active, const double *wave, const double *gwave,
                  const double *g_rho, const double *g_grad, const H1Inputs *h, double *out, cudaStream_t stream) {
  const void *items = mode == 1 ? plan.d_h1_items_sym : plan.d_adj_items;
  const int n_items = mode == 1 ? plan.n_h1_items_sym : plan.n_adj_items;
  if (n_items == 0) return FRPA_OK;
  FRPA_TRY(h1_scratch(plan, stream));
  const size_t n = (size_t)plan.n_basis * plan.n_basis * plan.T;
  unsigned long long *acc = plan.d_h1_acc;
  int *emax = reinterpret_cast<int *>(acc + 2 * n);
  FRPA_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * n * sizeof(unsigned long long), stream));
  FRPA_CUDA_TRY(cudaMemsetAsync(emax, 0x80, sizeof(int), stream));
  H1Args a{};
  a.mode = mode;
  a.n_active = n_active;
  a.n_basis = plan.n_basis;
  a.n_full_points = plan.n_full_points;
  a.n_max_batch_size = plan.n_max_batch_size;
  a.n_batches = plan.n_batches;
  a.ib_all = plan.d_ib;
  a.map = plan.d_map;
  a.wave = wave;
  a.gwave = gwave;
  a.g_rho = g_rho;
  a.g_grad = g_grad;
  if (h) a.h = *h;
  a.acc = acc;
  a.n_entries = (long long)n;
  a.emax = emax;
  a.err = plan.d_err;
  const H1Item *it = static_cast<const H1Item *>(items);
  h1_bound_kernel<<<n_items, THREADS, 0, stream>>>(it, n_items, a);
  FRPA_LAUNCH_CHECK();
  int n_sm = 148;
  FRPA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, plan.device));
  const int grid = std::min(n_items, n_sm * 4);
  if (mode == 1)
    h1_tile_kernel<true><<<grid, THREADS, 0, stream>>>(it, n_items, a);
  else
    h1_tile_kernel<false><<<grid, THREADS, 0, stream>>>(it, n_items, a);
  FRPA_LAUNCH_CHECK();
  h1_finalize_kernel<<<n_sm * 8, 256, 0, stream>>>((long long)n, acc, emax, plan.n_batches, out);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

int rho1_adjoint_run(Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *g_rho,
                     const double *g_grad, double *dP1, cudaStream_t stream) {
  return h1_run(plan, 0, n_active, wave, gwave, g_rho, g_grad, nullptr, dP1, stream);
}

int rho1_first_order_h_run(Rho1Plan &plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                           const int *atom_valid, const double *wave, const double *gwave, const double *hwave,
                           const double *vsigma, const double *gradient_rho, const double *H_prefactor1,
                           const double *fogr, const double *vhg, const double *rho1, const double *v2rho2,
                           const double *v2rhosigma, const double *v2sigma2, const double *partition_tab,
                           double *first_order_H, cudaStream_t stream) {
  H1Inputs h{vsigma, gradient_rho, hwave, H_prefactor1, fogr, vhg, rho1, v2rho2, v2rhosigma, v2sigma2,
             partition_tab, atom_valid, n_atoms, j_atom_begin, j_coord};
  return h1_run(plan, 1, n_active, wave, gwave, nullptr, nullptr, &h, first_order_H, stream);
}

}  // namespace frpa
