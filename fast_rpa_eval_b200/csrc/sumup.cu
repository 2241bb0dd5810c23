// Hartree potential sum-up from atomic multipoles (near-field spline + far-field
// analytic multipoles), FP64.
//
// Reference: fast_rap_src_dfpt_gpu_eval/sum_up_whole_potential.cpp:195-503 (CPU),
// .../sum_up_whole_potential.cu:548-769 (GPU: four launches, near and far field
// in separate kernels).  Per valid point p, perturbation t and centre slot ic
// (in the order of centers_hartree_potential):
//   d = p - R_centre, d2 = d.d               (rounded op by op, :395-402)
//   lam = l_hartree[species]; while (outer_potential_radius(lam) < d2 && lam > 0) lam--
//   d2 <  multipole_radius_sq:  near field  = sum_{lm <= lam} spline_lm(i_r_log) Y_lm(d_hat)
//   d2 <  1e8:                  far field   = sum_{n < n_cc(lam)} x^i y^j z^k Fp[nn] cc[n] Q[l,m]
//   delta_v(p, t) += contribution, in slot order.
//
// This file keeps every branch decision bit-identical to the reference (d2 and
// the comparisons use exactly rounded products and sums) and re-designs the
// arithmetic for the FP64 pipe:
//
// * Far field (fast path).  The caller's (index_cc, cc) table is converted once,
//   exactly, into a polynomial in the Kelvin-inverted coordinates u = d / r^2:
//   every table term x^i y^j z^k Fp[nn] is multiplied through by
//   (x^2+y^2+z^2)^(l-nn) / r^(2(l-nn)), which turns it into u^(a,b,c) / r with
//   a+b+c = l.  Per (centre, t) the multipole moments are folded in by a
//   prepare kernel, so one (point, centre) pair costs one Horner evaluation of
//   C(lam+3, 3) fused multiply-adds (84 at l = 6) instead of the 176-term table
//   loop.  The Horner degree is lam, specialised at compile time per warp-
//   uniform lam (the l_max-specialised AOT kernels of the reference's
//   task3_jit/version5, but derived from the runtime table rather than baked in).
// * Near field.  Real Y_lm by the associated-Legendre recursion fused with the
//   Hermite spline dot, read straight from the caller's
//   (L^2, 2, n_hartree_grid, atom, t) table (the two grid nodes needed are one
//   contiguous 4 L^2 run), so the reference's per-call transpose is not needed.
// * Generic path.  When the fast path's preconditions do not hold (a
//   centers_hartree_potential list that is not the identity, whose far field
//   the reference evaluates with the loop slot as centre, :161-162/:183; or a
//   table whose rows are not homogeneous multipole terms), a kernel that mirrors
//   the reference table loop exactly is used instead.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "frpa_internal.cuh"
#include "kelvin_horner.cuh"

namespace frpa {

constexpr int SU_LMAX = FRPA_SUMUP_MAX_L;  // 8
constexpr int SU_THREADS = 128;  // fast kernel: 5 CTAs per SM, 96 registers (no spills; measured against
                                 // 3, 4 and 6 CTAs per SM and two centres per thread)
constexpr int SU_PPT = 2;                  // points per thread (share coefficient loads)
constexpr int SU_CHUNK = 16;               // centre records staged per shared-memory chunk

// Near-field constants: Y_lm = K[l][m] Q_l^m(z) {C_m, S_m}; recursion
// Q_l^m = RA[l][m] z Q_{l-1}^m - RB[l][m] Q_{l-2}^m; DF[m] = (2m-1)!!.
__constant__ double c_K[SU_LMAX + 1][SU_LMAX + 1];
__constant__ double c_Kcos[SU_LMAX + 1][SU_LMAX + 1];
__constant__ double c_RA[SU_LMAX + 1][SU_LMAX + 1];
__constant__ double c_RB[SU_LMAX + 1][SU_LMAX + 1];
__constant__ double c_DF[SU_LMAX + 1];
__host__ __device__ constexpr int n_kelvin(int L) { return kelvin_count(L); }

// record layout (doubles) for one (centre slot, t)
enum : int {
  R_X = 0, R_Y, R_Z, R_MRS, R_LAM0, R_ATOM, R_RGM, R_LINC, R_NGRID, R_OPR  // R_OPR .. R_OPR+L
};
__host__ __device__ constexpr int rec_coef_off(int L) { return R_OPR + L + 1; }
__host__ __device__ constexpr int rec_stride(int L) { return ((rec_coef_off(L) + n_kelvin(L)) + 1) & ~1; }

struct SumupPlan {
  int device = 0;
  int T = 1, L = 0, L2 = 1, lma = 0, icc_dim0 = 0, mc_dim = 0, hfla = 0;
  int n_full_points = 0, n_valid_points = 0, n_centers = 0, n_chp = 0, n_atoms = 0, n_species = 0;
  int n_hartree_grid = 0;
  int fast = 0;
  int n_coef = 0, rs = 0;
  // device const arrays
  int *d_map = nullptr;
  int *d_order = nullptr;  // valid points in spatial (Morton) order, for warp-uniform branches
  double *d_coord = nullptr;
  int *d_species = nullptr, *d_species_center = nullptr, *d_l_hartree = nullptr, *d_n_grid = nullptr;
  int *d_c2a = nullptr, *d_chp = nullptr, *d_icc = nullptr, *d_ncc = nullptr, *d_ijkmax = nullptr;
  int *d_icc_packed = nullptr;  // (i | j<<8 | k<<16 | nn<<24) per row
  double *d_cc = nullptr, *d_cc_xyz = nullptr, *d_rgm = nullptr, *d_linc = nullptr;
  int *d_conv_ptr = nullptr, *d_conv_n = nullptr;
  double *d_conv_f = nullptr;
  int n_conv = 0;
  // workspaces
  double *d_mc = nullptr;    // (mc_dim, n_atoms, T)
  double *d_recs = nullptr;  // (rs, n_chp, T)
  int *d_err = nullptr;      // device-side input error flags
  // adjoint: transpose of the Kelvin conversion (by table row) and workspaces
  int *d_convT_ptr = nullptr, *d_convT_k = nullptr;
  double *d_convT_f = nullptr;
  double *d_dcoef = nullptr;  // (n_coef, n_chp, T)
  double *d_dmc = nullptr;    // (mc_dim, n_atoms, T)
  // deterministic adjoint: per point-block partial sums (n_coef, n_chp, T,
  // adj_nz), reduced in block order; slots of each atom (CSR, ascending)
  double *d_dcoef_part = nullptr;
  int adj_nz = 1, adj_pts = 4096;
  int *d_atom_slot_ptr = nullptr, *d_atom_slots = nullptr;
};

namespace {

// ------------------------------------------------------------ prepare ---

// multipole_c = cc * Q with the l cap and the 1e-10 threshold
// (sum_up_whole_potential.cpp:357-378); rows past n_cc(l_hartree_max_far_distance)
// are zero (the reference leaves them uninitialised).
__global__ void sumup_multipole_c_kernel(int n_atoms, int L, int L2, int mc_dim, int icc_dim0, int lma,
                                         const int *__restrict__ icc, const int *__restrict__ ncc,
                                         const double *__restrict__ cc, const int *__restrict__ lhmfd,
                                         const double *__restrict__ Q, double *__restrict__ mc,
                                         int *__restrict__ err) {
  const int a = blockIdx.x, t = blockIdx.y;
  int lh = lhmfd[a + n_atoms * t];
  if (lh < 0 || lh > L || lh > lma) {
    if (threadIdx.x == 0) atomicOr(err, 1);
    lh = lh < 0 ? 0 : (lh > L ? L : lh);
  }
  const int nmax = ncc[lh];
  for (int n = threadIdx.x; n < mc_dim; n += blockDim.x) {
    double v = 0.0;
    if (n < nmax) {
      const int l = icc[n], m = icc[n + icc_dim0];
      const double q = Q[(l * l + l + m) + (long long)L2 * (a + (long long)n_atoms * t)];
      v = (l <= lh && fabs(q) > 1e-10) ? cc[n] * q : 0.0;
    }
    mc[n + (long long)mc_dim * (a + (long long)n_atoms * t)] = v;
  }
}

// Per (slot, t) record for the fast kernels: centre, radii, l_hartree, near
// field parameters and the Kelvin coefficients (CSR contraction of multipole_c).
__global__ void sumup_records_kernel(int L, int n_atoms, int n_chp, int mc_dim, int n_coef, int rs,
                                     const int *__restrict__ chp, const int *__restrict__ c2a,
                                     const int *__restrict__ species, const int *__restrict__ species_center,
                                     const int *__restrict__ l_hartree, const int *__restrict__ n_grid,
                                     const double *__restrict__ rgm, const double *__restrict__ linc,
                                     const double *__restrict__ cc_xyz, const double *__restrict__ mrs,
                                     const double *__restrict__ opr, const double *__restrict__ mc,
                                     const int *__restrict__ conv_ptr, const int *__restrict__ conv_n,
                                     const double *__restrict__ conv_f, double *__restrict__ recs) {
  const int slot = blockIdx.x, t = blockIdx.y;
  const int cur = chp[slot] - 1;
  const int atom = c2a[cur] - 1;
  double *r = recs + (long long)rs * (slot + (long long)n_chp * t);
  const double *m = mc + (long long)mc_dim * (atom + (long long)n_atoms * t);
  if (threadIdx.x == 0) {
    const int sp = species_center[cur] - 1;
    r[R_X] = cc_xyz[3 * cur + 0];
    r[R_Y] = cc_xyz[3 * cur + 1];
    r[R_Z] = cc_xyz[3 * cur + 2];
    r[R_MRS] = mrs[atom + (long long)n_atoms * t];
    r[R_LAM0] = (double)l_hartree[species[atom] - 1];
    r[R_ATOM] = (double)atom;
    r[R_RGM] = rgm[sp];
    r[R_LINC] = linc[sp];
    r[R_NGRID] = (double)n_grid[sp];
  }
  for (int l = threadIdx.x; l <= L; l += blockDim.x)
    r[R_OPR + l] = opr[l + (long long)(L + 1) * (atom + (long long)n_atoms * t)];
  for (int k = threadIdx.x; k < n_coef; k += blockDim.x) {
    double s = 0.0;
    for (int e = conv_ptr[k]; e < conv_ptr[k + 1]; ++e) s += conv_f[e] * m[conv_n[e]];
    r[rec_coef_off(L) + k] = s;
  }
}

// ------------------------------------------------------- device pieces ---

// Near field for one pair (sum_up_whole_potential.cpp:411-477, spline :12-52):
// trig values exactly as the reference forms them, then Y_lm by recursion
// fused with the Hermite spline dot.
__device__ double near_field(int lam, int L2, double dx, double dy, double dz, double d2, double rgm, double linc,
                             int ngrid, const double *__restrict__ spl) {
  const double dist = sqrt(d2);
  const double din0 = dx / dist, din1 = dy / dist, din2 = dz / dist;
  const double r_log = 1.0 + log(dist / rgm) / linc;
  double cph, sph, ab;
  const double abmax = fmax(fabs(din0), fabs(din1));
  if (abmax > 1.0e-36) {
    ab = sqrt(add_rn(mul_rn(din0, din0), mul_rn(din1, din1)));
    cph = din0 / ab;
    sph = din1 / ab;
  } else {
    cph = 1.0;
    sph = 0.0;
    ab = 0.0;
  }
  double ct, st;
  const double abcmax = fmax(abmax, fabs(din2));
  if (abcmax > 1.0e-36) {
    const double abc = sqrt(add_rn(mul_rn(ab, ab), mul_rn(din2, din2)));
    ct = din2 / abc;
    st = ab / abc;
  } else {
    ct = 0.0;
    st = 1.0;
  }
  const double x = st * cph, y = st * sph, z = ct;
  int i_spl = (int)r_log;
  i_spl = i_spl < 1 ? 1 : i_spl;
  i_spl = i_spl > ngrid - 1 ? ngrid - 1 : i_spl;
  const double u = r_log - i_spl;
  const double ta = (u - 1) * (u - 1) * (1 + 2 * u);
  const double tb = (u - 1) * (u - 1) * u;
  const double tc = u * u * (3 - 2 * u);
  const double td = u * u * (u - 1);
  const double *g0 = spl + (long long)2 * L2 * (i_spl - 1);
  const double *g1 = g0 + 2 * L2;
  auto S = [&](int i) { return g0[i] * ta + g0[i + L2] * tb + g1[i] * tc + g1[i + L2] * td; };
  double acc = 0.0;
  double C = 1.0, Sm = 0.0;
  for (int m = 0; m <= lam; ++m) {
    if (m > 0) {
      const double c2 = x * C - y * Sm;
      Sm = x * Sm + y * C;
      C = c2;
    }
    double q_prev = 0.0, q_prev2 = 0.0;  // Q_{l-1}^m, Q_{l-2}^m
    for (int l = m; l <= lam; ++l) {
      const double ql = (l == m) ? c_DF[m] : c_RA[l][m] * z * q_prev - c_RB[l][m] * q_prev2;
      q_prev2 = q_prev;
      q_prev = ql;
      const int base = l * l + l;
      if (m == 0) {
        acc += c_K[l][0] * ql * S(base);
      } else {
        acc += c_Kcos[l][m] * ql * C * S(base + m);
        acc += c_K[l][m] * ql * Sm * S(base - m);
      }
    }
  }
  return acc;
}

// 1/sqrt(x) for x > 0: the PTX approximation (relative error below 1e-6)
// refined by two Newton-Raphson steps y <- y + y/2 (1 - x y^2), within about
// one ulp of 1 / sqrt(x) (measured over x in [1e-4, 1e10]); cheaper than the
// library's correctly rounded form.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double e = fma(-(x * y), y, 1.0);
    y = fma(0.5 * y, e, y);
  }
  return y;
}

// --------------------------------------------------------- fast kernel ---

__global__ void __launch_bounds__(SU_THREADS, 5)
    sumup_fast_kernel(int n_valid, int n_full, const int *__restrict__ map, const int *__restrict__ order,
                      const double *__restrict__ coord, int n_active, int n_chp, int n_atoms, int L,
                      int n_hartree_grid, const double *__restrict__ recs, const double *__restrict__ spline,
                      double *__restrict__ dv, unsigned char *__restrict__ codes) {
  const int RS = rec_stride(L);
  const int CO = rec_coef_off(L);
  const int L2 = (L + 1) * (L + 1);
  __shared__ __align__(16) double srec[SU_CHUNK * rec_stride(SU_LMAX)];
  const int tid = threadIdx.x;
  const unsigned FULL = 0xffffffffu;

  int vidx[SU_PPT], full[SU_PPT];
  double px[SU_PPT], py[SU_PPT], pz[SU_PPT];
  bool valid[SU_PPT];
#pragma unroll
  for (int j = 0; j < SU_PPT; ++j) {
    // a warp's points are neighbours in space when the plan gives an order,
    // so its near / far / skip decisions for an atom mostly agree
    const int slot = blockIdx.x * (SU_THREADS * SU_PPT) + j * SU_THREADS + tid;
    valid[j] = slot < n_valid;
    vidx[j] = valid[j] ? (order ? order[slot] : slot) : 0;
    full[j] = valid[j] ? map[vidx[j]] : 0;
    px[j] = valid[j] ? coord[3LL * full[j] + 0] : 0.0;
    py[j] = valid[j] ? coord[3LL * full[j] + 1] : 0.0;
    pz[j] = valid[j] ? coord[3LL * full[j] + 2] : 0.0;
  }

  for (int t = 0; t < n_active; ++t) {
    double v[SU_PPT];
#pragma unroll
    for (int j = 0; j < SU_PPT; ++j) v[j] = valid[j] ? dv[full[j] + (long long)n_full * t] : 0.0;

    for (int c0 = 0; c0 < n_chp; c0 += SU_CHUNK) {
      const int nch = min(SU_CHUNK, n_chp - c0);
      __syncthreads();
      const double *src = recs + (long long)RS * (c0 + (long long)n_chp * t);
      for (int e = tid; e < nch * RS; e += SU_THREADS) srec[e] = src[e];
      __syncthreads();

      for (int s = 0; s < nch; ++s) {
        const double *rec = srec + s * RS;
        const double cx = rec[R_X], cy = rec[R_Y], cz = rec[R_Z], mrs = rec[R_MRS];
        const int lam0 = (int)rec[R_LAM0];
        double dx[SU_PPT], dy[SU_PPT], dz[SU_PPT], d2[SU_PPT];
        int lam[SU_PPT], br[SU_PPT];  // br: 0 skip, 1 near, 2 far
#pragma unroll
        for (int j = 0; j < SU_PPT; ++j) {
          dx[j] = sub_rn(px[j], cx);
          dy[j] = sub_rn(py[j], cy);
          dz[j] = sub_rn(pz[j], cz);
          d2[j] = add_rn(add_rn(mul_rn(dx[j], dx[j]), mul_rn(dy[j], dy[j])), mul_rn(dz[j], dz[j]));
          int l = lam0;
          while (rec[R_OPR + l] < d2[j] && l > 0) --l;
          lam[j] = l;
          br[j] = !valid[j] ? 0 : (d2[j] < mrs ? 1 : (d2[j] < 1e8 ? 2 : 0));
        }
        if (codes) {
#pragma unroll
          for (int j = 0; j < SU_PPT; ++j)
            if (valid[j])
              codes[vidx[j] + (long long)n_valid * ((c0 + s) + (long long)n_chp * t)] =
                  (unsigned char)(br[j] == 1 ? 1 + lam[j] : (br[j] == 2 ? 16 + lam[j] : 0));
        }

        // far field
        bool mine = true;
#pragma unroll
        for (int j = 0; j < SU_PPT; ++j) mine = mine && br[j] == 2 && lam[j] == lam[0];
        const int lam_lane0 = __shfl_sync(FULL, lam[0], 0);  // every lane, before the vote
        const bool all_far_same = __all_sync(FULL, mine && lam[0] == lam_lane0);
        if (all_far_same) {
          double ux[SU_PPT], uy[SU_PPT], uz[SU_PPT], P[SU_PPT], rinv[SU_PPT];
#pragma unroll
          for (int j = 0; j < SU_PPT; ++j) {
            rinv[j] = rsqrt_nr(d2[j]);
            const double ir2 = rinv[j] * rinv[j];
            ux[j] = dx[j] * ir2;
            uy[j] = dy[j] * ir2;
            uz[j] = dz[j] * ir2;
          }
          kelvin_eval<SU_PPT>(lam[0], rec + CO, ux, uy, uz, P);
#pragma unroll
          for (int j = 0; j < SU_PPT; ++j) v[j] += P[j] * rinv[j];
        } else {
#pragma unroll
          for (int j = 0; j < SU_PPT; ++j) {
            bool pend = br[j] == 2;
            while (__any_sync(FULL, pend)) {
              const int sel = __reduce_max_sync(FULL, pend ? lam[j] : -1);
              if (pend && lam[j] == sel) {
                double ux[1], uy[1], uz[1], P[1];
                const double ri = rsqrt_nr(d2[j]);
                const double ir2 = ri * ri;
                ux[0] = dx[j] * ir2;
                uy[0] = dy[j] * ir2;
                uz[0] = dz[j] * ir2;
                kelvin_eval_1(sel, rec + CO, ux, uy, uz, P);
                v[j] += P[0] * ri;
                pend = false;
              }
            }
          }
        }
        // near field (rare)
#pragma unroll
        for (int j = 0; j < SU_PPT; ++j) {
          if (br[j] == 1) {
            const long long atom = (long long)rec[R_ATOM];
            const double *spl = spline + (long long)2 * L2 * n_hartree_grid * (atom + (long long)n_atoms * t);
            v[j] += near_field(lam[j], L2, dx[j], dy[j], dz[j], d2[j], rec[R_RGM], rec[R_LINC], (int)rec[R_NGRID], spl);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < SU_PPT; ++j)
      if (valid[j]) dv[full[j] + (long long)n_full * t] = v[j];
  }
}

// ------------------------------------------------------ generic kernel ---

// Mirrors the reference loop exactly, including the far field's use of the
// loop slot as centre (sum_up_whole_potential.cpp:91-187 called with i_center + 1).
__global__ void __launch_bounds__(SU_THREADS)
    sumup_generic_kernel(int n_valid, int n_full, const int *__restrict__ map, const double *__restrict__ coord,
                         int n_active, int n_chp, int n_atoms, int L, int L2, int n_hartree_grid, int hfla,
                         const int *__restrict__ chp, const int *__restrict__ c2a, const int *__restrict__ species,
                         const int *__restrict__ species_center, const int *__restrict__ l_hartree,
                         const int *__restrict__ n_grid, const double *__restrict__ rgm,
                         const double *__restrict__ linc, const double *__restrict__ cc_xyz,
                         const double *__restrict__ mrs, const double *__restrict__ opr,
                         const int *__restrict__ ncc, const int *__restrict__ icc_packed,
                         const int *__restrict__ ijkmax, int mc_dim, const double *__restrict__ mc,
                         const double *__restrict__ spline, double *__restrict__ dv, unsigned char *__restrict__ codes) {
  const int iv = blockIdx.x * SU_THREADS + threadIdx.x;
  if (iv >= n_valid) return;
  const int f = map[iv];
  const double px = coord[3LL * f], py = coord[3LL * f + 1], pz = coord[3LL * f + 2];
  for (int t = 0; t < n_active; ++t) {
    double v = dv[f + (long long)n_full * t];
    for (int ic = 0; ic < n_chp; ++ic) {
      const int cur = chp[ic] - 1;
      const int atom = c2a[cur] - 1;
      const double dx = sub_rn(px, cc_xyz[3 * cur]), dy = sub_rn(py, cc_xyz[3 * cur + 1]),
                   dz = sub_rn(pz, cc_xyz[3 * cur + 2]);
      const double d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
      int lam = l_hartree[species[atom] - 1];
      const double *o = opr + (long long)(L + 1) * (atom + (long long)n_atoms * t);
      while (o[lam] < d2 && lam > 0) --lam;
      unsigned char code = 0;
      if (d2 < mrs[atom + (long long)n_atoms * t]) {
        const int sp = species_center[cur] - 1;
        const double *spl = spline + (long long)2 * L2 * n_hartree_grid * (atom + (long long)n_atoms * t);
        v += near_field(lam, L2, dx, dy, dz, d2, rgm[sp], linc[sp], n_grid[sp], spl);
        code = (unsigned char)(1 + lam);
      } else if (d2 < 1e8) {
        const double dist = sqrt(d2);
        double Fp[2 * SU_LMAX + 4];
        const double dsq = dist * dist;
        int k = 1;
        Fp[0] = 1.0 / dist;
        for (int l = 1; l <= lam + hfla; ++l) {
          k -= 2;
          Fp[l] = Fp[l - 1] * k / dsq;
        }
        const double ex = px - cc_xyz[3 * ic], ey = py - cc_xyz[3 * ic + 1], ez = pz - cc_xyz[3 * ic + 2];
        int maxp = ijkmax[3 * lam];
        maxp = max(maxp, ijkmax[3 * lam + 1]);
        maxp = max(maxp, ijkmax[3 * lam + 2]);
        double pw[3][2 * SU_LMAX + 2];
        pw[0][0] = pw[1][0] = pw[2][0] = 1.0;
        for (int i = 1; i <= maxp; ++i) {
          pw[0][i] = ex * pw[0][i - 1];
          pw[1][i] = ey * pw[1][i - 1];
          pw[2][i] = ez * pw[2][i - 1];
        }
        const double *m = mc + (long long)mc_dim * ((c2a[ic] - 1) + (long long)n_atoms * t);
        double dpot = 0.0;
        const int nend = ncc[lam];
        for (int n = 0; n < nend; ++n) {
          const int pk = icc_packed[n];
          const int ii = pk & 255, jj = (pk >> 8) & 255, kk = (pk >> 16) & 255, nn = (pk >> 24) & 255;
          dpot += pw[0][ii] * pw[1][jj] * pw[2][kk] * Fp[nn] * m[n];
        }
        v += dpot;
        code = (unsigned char)(16 + lam);
      }
      if (codes) codes[iv + (long long)n_valid * (ic + (long long)n_chp * t)] = code;
    }
    dv[f + (long long)n_full * t] = v;
  }
}

int launch_fast(const SumupPlan &P, int n_active, const double *spline, double *dv, unsigned char *codes,
                cudaStream_t stream) {
  const int per_block = SU_THREADS * SU_PPT;
  const int grid = (P.n_valid_points + per_block - 1) / per_block;
  sumup_fast_kernel<<<grid, SU_THREADS, 0, stream>>>(P.n_valid_points, P.n_full_points, P.d_map, P.d_order,
                                                     P.d_coord,
                                                     n_active, P.n_chp, P.n_atoms, P.L, P.n_hartree_grid, P.d_recs,
                                                     spline, dv, codes);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}


// -------------------------------------------------------- adjoint (dQ) ---

constexpr int ADJ_KCH = 32;

// Exponents (a, b, c) of coefficient slot k in the degree-graded packing
// (the inverse of kelvin_index), for compile-time use.
struct Abc {
  int a, b, c;
};
__host__ __device__ constexpr Abc kelvin_abc(int k) {
  int d = 0;
  while ((d + 1) * (d + 2) * (d + 3) / 6 <= k) ++d;
  int r = k - d * (d + 1) * (d + 2) / 6, a = 0;
  while (r >= d + 1 - a) {
    r -= d + 1 - a;
    ++a;
  }
  return Abc{a, r, d - a - r};
}
__host__ __device__ constexpr bool kelvin_abc_inverts_index() {
  for (int k = 0; k < kelvin_count(SU_LMAX); ++k) {
    const Abc m = kelvin_abc(k);
    if (kelvin_index(m.a, m.b, m.c) != k) return false;
  }
  return true;
}
static_assert(kelvin_abc_inverts_index(), "kelvin_abc is the inverse of kelvin_index");

// acc[I] += w ux^a uy^b uz^c for the chunk's slots K0 + I of degree <= lam
// (exponents are compile-time constants: the power arrays stay in registers)
template <int L, int K0, int... I>
__device__ __forceinline__ void dcoef_terms(std::integer_sequence<int, I...>, double *acc, double w, const double *pa,
                                            const double *pb, const double *pc, int lam) {
  auto term = [&](auto ic) {
    constexpr int k = K0 + decltype(ic)::value;
    if constexpr (k < kelvin_count(L)) {
      constexpr Abc m = kelvin_abc(k);
      if (m.a + m.b + m.c <= lam) acc[decltype(ic)::value] += w * pa[m.a] * pb[m.b] * pc[m.c];
    }
  };
  (term(std::integral_constant<int, I>{}), ...);
}

// One chunk of ADJ_KCH coefficient slots starting at K0: every point of the
// block once, then the block's partial sums (warp shuffles, then the warps in
// order) to part[k, slot, t, z].
template <int L, int K0>
__device__ __forceinline__ void dcoef_chunk(int n_full, const int *__restrict__ map,
                                            const double *__restrict__ coord, const double *__restrict__ rec,
                                            const double *__restrict__ g, int t, int p_begin, int p_end,
                                            double (&red)[SU_THREADS / 32][ADJ_KCH], double *__restrict__ part) {
  const double cx = rec[R_X], cy = rec[R_Y], cz = rec[R_Z], mrs = rec[R_MRS];
  const int lam0 = (int)rec[R_LAM0];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[ADJ_KCH];
#pragma unroll
  for (int kk = 0; kk < ADJ_KCH; ++kk) acc[kk] = 0.0;
  for (int iv = p_begin + threadIdx.x; iv < p_end; iv += SU_THREADS) {
    const int f = map[iv];
    const double dx = sub_rn(coord[3LL * f], cx), dy = sub_rn(coord[3LL * f + 1], cy),
                 dz = sub_rn(coord[3LL * f + 2], cz);
    const double d2 = add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
    if (d2 < mrs || !(d2 < 1e8)) continue;
    int lam = lam0;
    while (rec[R_OPR + lam] < d2 && lam > 0) --lam;
    const double ri = rsqrt(d2), ir2 = ri * ri;
    const double ux = dx * ir2, uy = dy * ir2, uz = dz * ir2;
    double pa[L + 1], pb[L + 1], pc[L + 1];
    pa[0] = pb[0] = pc[0] = 1.0;
#pragma unroll
    for (int e = 1; e <= L; ++e) {
      pa[e] = pa[e - 1] * ux;
      pb[e] = pb[e - 1] * uy;
      pc[e] = pc[e - 1] * uz;
    }
    const double w = g[f + (long long)n_full * t] * ri;
    dcoef_terms<L, K0>(std::make_integer_sequence<int, ADJ_KCH>{}, acc, w, pa, pb, pc, lam);
  }
#pragma unroll
  for (int kk = 0; kk < ADJ_KCH; ++kk) {
    double v = acc[kk];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][kk] = v;
  }
  __syncthreads();
  constexpr int NK = kelvin_count(L);
  if (threadIdx.x < ADJ_KCH && K0 + (int)threadIdx.x < NK) {
    double v = 0.0;
    for (int w = 0; w < SU_THREADS / 32; ++w) v += red[w][threadIdx.x];
    part[K0 + threadIdx.x] = v;  // this point block's partial, summed over the blocks in order later
  }
  __syncthreads();
}

template <int L, int... C>
__device__ __forceinline__ void dcoef_chunks(std::integer_sequence<int, C...>, int n_full, const int *map,
                                             const double *coord, const double *rec, const double *g, int t,
                                             int p_begin, int p_end, double (&red)[SU_THREADS / 32][ADJ_KCH],
                                             double *part) {
  (dcoef_chunk<L, C * ADJ_KCH>(n_full, map, coord, rec, g, t, p_begin, p_end, red, part), ...);
}

// part[k, slot, t, z] = sum over point block z's points of g(p, t) u^k / r
// for far-field pairs with deg(k) <= lam (the derivative of the fast path's
// Horner sum with respect to its coefficients), one instance per l_max; each
// block sums its points in a fixed order, and sumup_dcoef_reduce_kernel adds
// the blocks in order, so the result is the same on every run.
template <int L>
__global__ void __launch_bounds__(SU_THREADS)
    sumup_dcoef_kernel(int n_valid, int n_full, const int *__restrict__ map, const double *__restrict__ coord,
                       int n_chp, const double *__restrict__ recs, const double *__restrict__ g, int pts_per_block,
                       double *__restrict__ dcoef) {
  constexpr int NK = kelvin_count(L), NCH = (NK + ADJ_KCH - 1) / ADJ_KCH;
  __shared__ double red[SU_THREADS / 32][ADJ_KCH];
  const int slot = blockIdx.x, t = blockIdx.y;
  const int p_begin = blockIdx.z * pts_per_block;
  const int p_end = min(n_valid, p_begin + pts_per_block);
  const double *rec = recs + (long long)rec_stride(L) * (slot + (long long)n_chp * t);
  double *part = dcoef + (long long)NK * (slot + (long long)n_chp * (t + (long long)gridDim.y * blockIdx.z));
  dcoef_chunks<L>(std::make_integer_sequence<int, NCH>{}, n_full, map, coord, rec, g, t, p_begin, p_end, red, part);
}

// dcoef[k, slot, t] = sum over the point blocks z, in order, of part[k, slot, t, z]
__global__ void sumup_dcoef_reduce_kernel(long long n, int nz, const double *__restrict__ part,
                                          double *__restrict__ dcoef) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < nz; ++z) s += part[e + n * z];
    dcoef[e] = s;
  }
}

// dmc[n, atom, t] = sum over the atom's slots, in ascending order, of
// sum_k conv[k, n] dcoef[k, slot, t] (a gather: no two threads add into one
// entry, so the result is the same on every run)
__global__ void sumup_dmc_kernel(int n_chp, int n_atoms, int mc_dim, int n_coef, const int *__restrict__ slot_ptr,
                                 const int *__restrict__ slots, const int *__restrict__ convT_ptr,
                                 const int *__restrict__ convT_k, const double *__restrict__ convT_f,
                                 const double *__restrict__ dcoef, double *__restrict__ dmc) {
  const int atom = blockIdx.x, t = blockIdx.y;
  for (int n = threadIdx.x; n < mc_dim; n += blockDim.x) {
    double s = 0.0;
    for (int q = slot_ptr[atom]; q < slot_ptr[atom + 1]; ++q) {
      const double *dc = dcoef + (long long)n_coef * (slots[q] + (long long)n_chp * t);
      for (int e = convT_ptr[n]; e < convT_ptr[n + 1]; ++e) s += convT_f[e] * dc[convT_k[e]];
    }
    dmc[n + (long long)mc_dim * (atom + (long long)n_atoms * t)] = s;
  }
}

// dQ[lm, atom, t] = sum over rows n with (l, m) of cc[n] dmc[n] where the
// forward kept the moment (l <= l_hartree_max_far_distance, |Q| > 1e-10).
__global__ void sumup_dq_kernel(int n_atoms, int L, int L2, int mc_dim, int icc_dim0, const int *__restrict__ icc,
                                const int *__restrict__ ncc, const double *__restrict__ cc,
                                const int *__restrict__ lhmfd, const double *__restrict__ Q,
                                const double *__restrict__ dmc, double *__restrict__ dQ) {
  const int a = blockIdx.x, t = blockIdx.y;
  int lh = lhmfd[a + n_atoms * t];
  lh = lh < 0 ? 0 : (lh > L ? L : lh);
  const int nmax = ncc[lh];
  const double *dm = dmc + (long long)mc_dim * (a + (long long)n_atoms * t);
  for (int lm = threadIdx.x; lm < L2; lm += blockDim.x) {
    const long long qi = lm + (long long)L2 * (a + (long long)n_atoms * t);
    const double q = Q[qi];
    double s = 0.0;
    for (int n = 0; n < nmax; ++n) {
      const int l = icc[n], m = icc[n + icc_dim0];
      if (l * l + l + m == lm && l <= lh && fabs(q) > 1e-10) s += cc[n] * dm[n];
    }
    dQ[qi] = s;
  }
}

int launch_dcoef(const SumupPlan &P, int n_active, const double *g, cudaStream_t stream) {
  const dim3 grid(P.n_chp, n_active, P.adj_nz);
  switch (P.L) {
#define FRPA_DCOEF_CASE(LL)                                                                                  \
  case LL:                                                                                                   \
    sumup_dcoef_kernel<LL><<<grid, SU_THREADS, 0, stream>>>(P.n_valid_points, P.n_full_points, P.d_map,       \
                                                             P.d_coord, P.n_chp, P.d_recs, g, P.adj_pts,       \
                                                             P.d_dcoef_part);                                  \
    break;
    FRPA_DCOEF_CASE(0) FRPA_DCOEF_CASE(1) FRPA_DCOEF_CASE(2) FRPA_DCOEF_CASE(3) FRPA_DCOEF_CASE(4)
    FRPA_DCOEF_CASE(5) FRPA_DCOEF_CASE(6) FRPA_DCOEF_CASE(7) FRPA_DCOEF_CASE(8)
#undef FRPA_DCOEF_CASE
    default:
      return fail(FRPA_ERR_UNSUPPORTED, "sum-up adjoint: l_pot_max %d above %d", P.L, SU_LMAX);
  }
  FRPA_LAUNCH_CHECK();
  const long long n = (long long)P.n_coef * P.n_chp * n_active;
  sumup_dcoef_reduce_kernel<<<(int)std::min<long long>(4096, (n + 255) / 256), 256, 0, stream>>>(
      n, P.adj_nz, P.d_dcoef_part, P.d_dcoef);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

}  // namespace

// ------------------------------------------------------------ host side ---

static int upload(void **dst, const void *src, size_t bytes) {
  FRPA_CUDA_TRY(cudaMalloc(dst, bytes > 0 ? bytes : 8));
  if (bytes) FRPA_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return FRPA_OK;
}

static int sumup_upload_constants_once() {
  double K[SU_LMAX + 1][SU_LMAX + 1] = {}, Kc[SU_LMAX + 1][SU_LMAX + 1] = {};
  double RA[SU_LMAX + 1][SU_LMAX + 1] = {}, RB[SU_LMAX + 1][SU_LMAX + 1] = {}, DF[SU_LMAX + 1] = {};
  const double four_pi = 12.566370614359172953850573533118;
  for (int m = 0; m <= SU_LMAX; ++m) {
    double d = 1.0;
    for (int k = 1; k <= 2 * m - 1; k += 2) d *= k;
    DF[m] = d;
  }
  for (int l = 0; l <= SU_LMAX; ++l)
    for (int m = 0; m <= l; ++m) {
      double ratio = 1.0;
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= k;
      double k0 = std::sqrt((2 * l + 1) / four_pi * ratio);
      if (m > 0) k0 *= std::sqrt(2.0);
      K[l][m] = k0;
      Kc[l][m] = (m & 1) ? -k0 : k0;
      if (l > m) {
        RA[l][m] = (double)(2 * l - 1) / (l - m);
        RB[l][m] = (double)(l + m - 1) / (l - m);
      }
    }
  FRPA_CUDA_TRY(cudaMemcpyToSymbol(c_K, K, sizeof(K)));
  FRPA_CUDA_TRY(cudaMemcpyToSymbol(c_Kcos, Kc, sizeof(Kc)));
  FRPA_CUDA_TRY(cudaMemcpyToSymbol(c_RA, RA, sizeof(RA)));
  FRPA_CUDA_TRY(cudaMemcpyToSymbol(c_RB, RB, sizeof(RB)));
  FRPA_CUDA_TRY(cudaMemcpyToSymbol(c_DF, DF, sizeof(DF)));
  return FRPA_OK;
}

// The constant tables, uploaded once per device (plan creation and the
// allocation-free entry point may reach this from several host threads).
int sumup_upload_constants(int device) {
  static PerDeviceOnce uploaded;
  return uploaded.run(device, sumup_upload_constants_once);
}

void sumup_plan_free(SumupPlan *P) {
  if (!P) return;
  void *ptrs[] = {P->d_map, P->d_order, P->d_coord, P->d_species, P->d_species_center, P->d_l_hartree, P->d_n_grid,
                  P->d_c2a, P->d_chp, P->d_icc, P->d_ncc, P->d_ijkmax, P->d_icc_packed, P->d_cc, P->d_cc_xyz,
                  P->d_rgm, P->d_linc, P->d_conv_ptr, P->d_conv_n, P->d_conv_f, P->d_mc, P->d_recs, P->d_err,
                  P->d_convT_ptr, P->d_convT_k, P->d_convT_f, P->d_dcoef, P->d_dmc, P->d_dcoef_part,
                  P->d_atom_slot_ptr, P->d_atom_slots};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete P;
}

// Validates the constant inputs (every device access stays in bounds for any
// per-call data once these hold) and uploads them.
int sumup_plan_create(SumupPlan **out, const frpa_sumup_desc *D) {
  *out = nullptr;
  FRPA_CHECK_ARG(D != nullptr, "sumup: null descriptor");
  const int L = D->l_pot_max, lma = D->l_max_analytic_multipole, T = D->atom_tile_size;
  FRPA_CHECK_ARG(T >= 1 && T <= FRPA_MAX_ATOM_TILE, "sumup: atom tile size %d out of range", T);
  FRPA_CHECK_ARG(L >= 0 && L <= SU_LMAX, "sumup: l_pot_max %d unsupported (0..%d)", L, SU_LMAX);
  FRPA_CHECK_ARG(lma >= 0 && lma <= 2 * SU_LMAX, "sumup: l_max_analytic_multipole %d out of range", lma);
  FRPA_CHECK_ARG(D->hartree_force_l_add >= 0 && L + D->hartree_force_l_add <= 2 * SU_LMAX + 3,
                 "sumup: hartree_force_l_add %d out of range", D->hartree_force_l_add);
  FRPA_CHECK_ARG(D->n_full_points >= 0 && D->n_valid_points >= 0 && D->n_atoms > 0 && D->n_centers > 0 &&
                     D->n_centers_hartree_potential >= 0 && D->n_species > 0 && D->n_hartree_grid >= 2 &&
                     D->index_cc_dim_0 > 0,
                 "sumup: bad sizes");
  FRPA_CHECK_ARG(D->n_full_points < (1 << 30) && D->n_valid_points <= D->n_full_points,
                 "sumup: n_valid_points %d > n_full_points %d", D->n_valid_points, D->n_full_points);
  const int *ncc = D->n_cc_lm_ijk;
  FRPA_CHECK_ARG(lma >= L, "sumup: l_max_analytic_multipole %d < l_pot_max %d", lma, L);
  for (int l = 0; l <= lma; ++l)
    FRPA_CHECK_ARG(ncc[l] >= 0 && ncc[l] <= D->index_cc_dim_0 && (l == 0 || ncc[l] >= ncc[l - 1]),
                   "sumup: n_cc_lm_ijk not a cumulative count within index_cc_dim_0");
  const int icc_dim0 = D->index_cc_dim_0;
  const int mc_dim = ncc[L];
  for (int n = 0; n < ncc[L]; ++n) {
    const int l = D->index_cc[n], m = D->index_cc[n + icc_dim0];
    FRPA_CHECK_ARG(l >= 0 && l <= L && m >= -l && m <= l, "sumup: index_cc row %d has bad (l, m)", n);
    for (int c = 2; c <= 4; ++c)
      FRPA_CHECK_ARG(D->index_cc[n + c * icc_dim0] >= 0 && D->index_cc[n + c * icc_dim0] <= 2 * SU_LMAX + 1,
                     "sumup: index_cc row %d power out of range", n);
    const int nn = D->index_cc[n + 5 * icc_dim0];
    FRPA_CHECK_ARG(nn >= 0 && nn <= L + D->hartree_force_l_add, "sumup: index_cc row %d Fp index %d", n, nn);
  }
  for (int l = 0; l <= L; ++l)
    for (int c = 0; c < 3; ++c)
      FRPA_CHECK_ARG(D->index_ijk_max_cc[c + 3 * l] >= -1 && D->index_ijk_max_cc[c + 3 * l] <= 2 * SU_LMAX + 1,
                     "sumup: index_ijk_max_cc out of range");
  for (int i = 0; i < D->n_valid_points; ++i)
    FRPA_CHECK_ARG(D->i_valid_point_2_i_full_points_map[i] >= 0 &&
                       D->i_valid_point_2_i_full_points_map[i] < D->n_full_points,
                   "sumup: valid-point map entry %d out of range", i);
  for (int i = 0; i < D->n_centers_hartree_potential; ++i) {
    const int c = D->centers_hartree_potential[i];
    FRPA_CHECK_ARG(c >= 1 && c <= D->n_centers, "sumup: centers_hartree_potential[%d] = %d", i, c);
    FRPA_CHECK_ARG(i < D->n_centers, "sumup: more centre slots than centres");
  }
  for (int c = 0; c < D->n_centers; ++c) {
    FRPA_CHECK_ARG(D->center_to_atom[c] >= 1 && D->center_to_atom[c] <= D->n_atoms, "sumup: center_to_atom[%d]", c);
    FRPA_CHECK_ARG(D->species_center[c] >= 1 && D->species_center[c] <= D->n_species, "sumup: species_center[%d]", c);
  }
  for (int a = 0; a < D->n_atoms; ++a)
    FRPA_CHECK_ARG(D->species[a] >= 1 && D->species[a] <= D->n_species, "sumup: species[%d]", a);
  for (int s = 0; s < D->n_species; ++s) {
    FRPA_CHECK_ARG(D->l_hartree[s] >= 0 && D->l_hartree[s] <= L, "sumup: l_hartree[%d] = %d > l_pot_max", s,
                   D->l_hartree[s]);
    FRPA_CHECK_ARG(D->n_grid[s] >= 2 && D->n_grid[s] <= D->n_hartree_grid, "sumup: n_grid[%d]", s);
  }

  // fast-path eligibility and the exact Kelvin conversion of the table
  bool fast = true;
  for (int i = 0; i < D->n_centers_hartree_potential && fast; ++i)
    if (D->centers_hartree_potential[i] != i + 1) fast = false;
  std::vector<std::vector<std::pair<int, double>>> conv(n_kelvin(L));
  for (int n = 0; n < ncc[L] && fast; ++n) {
    const int l = D->index_cc[n];
    const int i = D->index_cc[n + 2 * icc_dim0], j = D->index_cc[n + 3 * icc_dim0], k = D->index_cc[n + 4 * icc_dim0];
    const int nn = D->index_cc[n + 5 * icc_dim0];
    int lrow = 0;  // rows must be grouped by l as n_cc_lm_ijk says
    while (lrow < L && n >= ncc[lrow]) ++lrow;
    if (lrow != l || 2 * nn != l + i + j + k || nn > l) {
      fast = false;
      break;
    }
    const int s = l - nn;
    double fnn = (nn & 1) ? -1.0 : 1.0;
    for (int q = 1; q <= 2 * nn - 1; q += 2) fnn *= q;
    for (int s1 = 0; s1 <= s; ++s1)
      for (int s2 = 0; s1 + s2 <= s; ++s2) {
        const int s3 = s - s1 - s2;
        double multi = 1.0;  // s! / (s1! s2! s3!)
        for (int q = 2; q <= s; ++q) multi *= q;
        for (int q = 2; q <= s1; ++q) multi /= q;
        for (int q = 2; q <= s2; ++q) multi /= q;
        for (int q = 2; q <= s3; ++q) multi /= q;
        conv[kelvin_index(i + 2 * s1, j + 2 * s2, k + 2 * s3)].push_back({n, fnn * multi});
      }
  }
  std::vector<int> conv_ptr(n_kelvin(L) + 1, 0), conv_n;
  std::vector<double> conv_f;
  for (int q = 0; q < n_kelvin(L); ++q) {
    for (auto &e : conv[q]) {
      conv_n.push_back(e.first);
      conv_f.push_back(e.second);
    }
    conv_ptr[q + 1] = (int)conv_n.size();
  }
  // transpose (by table row) for the adjoint
  std::vector<int> convT_ptr(std::max(1, mc_dim) + 1, 0), convT_k;
  std::vector<double> convT_f;
  {
    std::vector<std::vector<std::pair<int, double>>> byrow(std::max(1, mc_dim));
    for (int q = 0; q < n_kelvin(L); ++q)
      for (auto &e : conv[q]) byrow[e.first].push_back({q, e.second});
    for (size_t n = 0; n < byrow.size(); ++n) {
      for (auto &e : byrow[n]) {
        convT_k.push_back(e.first);
        convT_f.push_back(e.second);
      }
      convT_ptr[n + 1] = (int)convT_k.size();
    }
  }
  std::vector<int> packed(std::max(1, icc_dim0), 0);
  for (int n = 0; n < ncc[L]; ++n)
    packed[n] = D->index_cc[n + 2 * icc_dim0] | (D->index_cc[n + 3 * icc_dim0] << 8) |
                (D->index_cc[n + 4 * icc_dim0] << 16) | (D->index_cc[n + 5 * icc_dim0] << 24);

  SumupPlan *P = new SumupPlan();
  FRPA_CUDA_TRY(cudaGetDevice(&P->device));
  P->T = T;
  P->L = L;
  P->L2 = (L + 1) * (L + 1);
  P->lma = lma;
  P->icc_dim0 = icc_dim0;
  P->mc_dim = mc_dim > 0 ? mc_dim : 1;
  P->hfla = D->hartree_force_l_add;
  P->n_full_points = D->n_full_points;
  P->n_valid_points = D->n_valid_points;
  P->n_centers = D->n_centers;
  P->n_chp = D->n_centers_hartree_potential;
  P->n_atoms = D->n_atoms;
  P->n_species = D->n_species;
  P->n_hartree_grid = D->n_hartree_grid;
  P->fast = fast ? 1 : 0;
  P->n_coef = n_kelvin(L);
  P->rs = rec_stride(L);
  P->n_conv = (int)conv_n.size();
  int st = FRPA_OK;
#define UP(field, src, bytes) \
  if (st == FRPA_OK) st = upload((void **)&P->field, (src), (bytes));
  UP(d_map, D->i_valid_point_2_i_full_points_map, sizeof(int) * (size_t)D->n_valid_points);
  {
    // Morton order of the valid points (21 bits per axis over their bounding box)
    const int nv = D->n_valid_points;
    std::vector<int> ord(nv);
    if (nv > 0) {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int i = 0; i < nv; ++i)
        for (int c = 0; c < 3; ++c) {
          const double x = D->coord_points[3LL * D->i_valid_point_2_i_full_points_map[i] + c];
          lo[c] = std::min(lo[c], x);
          hi[c] = std::max(hi[c], x);
        }
      auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffull;
        v = (v | v << 16) & 0x1f0000ff0000ffull;
        v = (v | v << 8) & 0x100f00f00f00f00full;
        v = (v | v << 4) & 0x10c30c30c30c30c3ull;
        v = (v | v << 2) & 0x1249249249249249ull;
        return v;
      };
      std::vector<std::pair<uint64_t, int>> key(nv);
      for (int i = 0; i < nv; ++i) {
        uint64_t k = 0;
        for (int c = 0; c < 3; ++c) {
          const double x = D->coord_points[3LL * D->i_valid_point_2_i_full_points_map[i] + c];
          const double w = hi[c] > lo[c] ? (x - lo[c]) / (hi[c] - lo[c]) : 0.0;
          const uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, w * 2097151.0));
          k |= spread(q) << c;
        }
        key[i] = {k, i};
      }
      std::sort(key.begin(), key.end());
      for (int i = 0; i < nv; ++i) ord[i] = key[i].second;
    }
    UP(d_order, ord.data(), sizeof(int) * (size_t)nv);
  }
  UP(d_coord, D->coord_points, sizeof(double) * 3 * (size_t)D->n_full_points);
  UP(d_species, D->species, sizeof(int) * D->n_atoms);
  UP(d_species_center, D->species_center, sizeof(int) * D->n_centers);
  UP(d_l_hartree, D->l_hartree, sizeof(int) * D->n_species);
  UP(d_n_grid, D->n_grid, sizeof(int) * D->n_species);
  UP(d_c2a, D->center_to_atom, sizeof(int) * D->n_centers);
  UP(d_chp, D->centers_hartree_potential, sizeof(int) * (size_t)P->n_chp);
  UP(d_icc, D->index_cc, sizeof(int) * 6 * (size_t)icc_dim0);
  UP(d_ncc, D->n_cc_lm_ijk, sizeof(int) * (lma + 1));
  UP(d_ijkmax, D->index_ijk_max_cc, sizeof(int) * 3 * (lma + 1));
  UP(d_icc_packed, packed.data(), sizeof(int) * packed.size());
  UP(d_cc, D->cc, sizeof(double) * icc_dim0);
  UP(d_cc_xyz, D->coords_center, sizeof(double) * 3 * (size_t)D->n_centers);
  UP(d_rgm, D->r_grid_min, sizeof(double) * D->n_species);
  UP(d_linc, D->log_r_grid_inc, sizeof(double) * D->n_species);
  UP(d_conv_ptr, conv_ptr.data(), sizeof(int) * conv_ptr.size());
  UP(d_conv_n, conv_n.data(), sizeof(int) * conv_n.size());
  UP(d_conv_f, conv_f.data(), sizeof(double) * conv_f.size());
  UP(d_convT_ptr, convT_ptr.data(), sizeof(int) * convT_ptr.size());
  UP(d_convT_k, convT_k.data(), sizeof(int) * convT_k.size());
  UP(d_convT_f, convT_f.data(), sizeof(double) * convT_f.size());
#undef UP
  if (st == FRPA_OK &&
      cudaMalloc((void **)&P->d_dcoef, sizeof(double) * (size_t)n_kelvin(L) * std::max(1, P->n_chp) * T) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  if (st == FRPA_OK &&
      cudaMalloc((void **)&P->d_dmc, sizeof(double) * (size_t)P->mc_dim * P->n_atoms * T) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  // adjoint: at most 64 point blocks per (slot, t), partials reduced in order
  P->adj_pts = std::max(4096, (P->n_valid_points + 63) / 64);
  P->adj_nz = std::max(1, (P->n_valid_points + P->adj_pts - 1) / P->adj_pts);
  if (st == FRPA_OK && cudaMalloc((void **)&P->d_dcoef_part, sizeof(double) * (size_t)n_kelvin(L) *
                                                                 std::max(1, P->n_chp) * T * P->adj_nz) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  {
    std::vector<int> cnt(P->n_atoms + 1, 0), slots(std::max(1, P->n_chp));
    std::vector<int> atom_of(std::max(1, P->n_chp));
    for (int q = 0; q < P->n_chp; ++q) {
      atom_of[q] = D->center_to_atom[D->centers_hartree_potential[q] - 1] - 1;
      ++cnt[atom_of[q] + 1];
    }
    for (int a = 0; a < P->n_atoms; ++a) cnt[a + 1] += cnt[a];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int q = 0; q < P->n_chp; ++q) slots[fill[atom_of[q]]++] = q;  // ascending within each atom
    if (st == FRPA_OK && (cudaMalloc((void **)&P->d_atom_slot_ptr, sizeof(int) * cnt.size()) != cudaSuccess ||
                          cudaMalloc((void **)&P->d_atom_slots, sizeof(int) * slots.size()) != cudaSuccess))
      st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
    if (st == FRPA_OK &&
        (cudaMemcpy(P->d_atom_slot_ptr, cnt.data(), sizeof(int) * cnt.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(P->d_atom_slots, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice) != cudaSuccess))
      st = fail(FRPA_ERR_CUDA, "sumup: upload failed");
  }
  if (st == FRPA_OK && cudaMalloc((void **)&P->d_mc, sizeof(double) * (size_t)P->mc_dim * P->n_atoms * T) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  if (st == FRPA_OK &&
      cudaMalloc((void **)&P->d_recs, sizeof(double) * (size_t)P->rs * std::max(1, P->n_chp) * T) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  if (st == FRPA_OK && cudaMalloc((void **)&P->d_err, sizeof(int)) != cudaSuccess)
    st = fail(FRPA_ERR_OOM, "sumup: workspace allocation failed");
  if (st == FRPA_OK) st = cudaMemset(P->d_err, 0, sizeof(int)) == cudaSuccess ? FRPA_OK : fail(FRPA_ERR_CUDA, "memset");
  if (st == FRPA_OK) st = sumup_upload_constants(P->device);
  if (st != FRPA_OK) {
    sumup_plan_free(P);
    return st;
  }
  *out = P;
  return FRPA_OK;
}

int sumup_plan_is_fast(const SumupPlan *P) { return P->fast; }

int sumup_execute(const SumupPlan *P, int n_active, int force_generic, const int *lhmfd, const double *mrs,
                  const double *opr, const double *Q, const double *spline, double *dv, unsigned char *codes,
                  cudaStream_t stream) {
  FRPA_CHECK_ARG(n_active >= 0 && n_active <= P->T, "sumup: %d active perturbations > tile %d", n_active, P->T);
  if (n_active == 0 || P->n_valid_points == 0 || P->n_chp == 0) return FRPA_OK;
  sumup_multipole_c_kernel<<<dim3(P->n_atoms, n_active), 128, 0, stream>>>(
      P->n_atoms, P->L, P->L2, P->mc_dim, P->icc_dim0, P->lma, P->d_icc, P->d_ncc, P->d_cc, lhmfd, Q, P->d_mc,
      P->d_err);
  FRPA_LAUNCH_CHECK();
  if (P->fast && !force_generic) {
    sumup_records_kernel<<<dim3(P->n_chp, n_active), 128, 0, stream>>>(
        P->L, P->n_atoms, P->n_chp, P->mc_dim, P->n_coef, P->rs, P->d_chp, P->d_c2a, P->d_species,
        P->d_species_center, P->d_l_hartree, P->d_n_grid, P->d_rgm, P->d_linc, P->d_cc_xyz, mrs, opr, P->d_mc,
        P->d_conv_ptr, P->d_conv_n, P->d_conv_f, P->d_recs);
    FRPA_LAUNCH_CHECK();
    return launch_fast(*P, n_active, spline, dv, codes, stream);
  }
  const int grid = (P->n_valid_points + SU_THREADS - 1) / SU_THREADS;
  sumup_generic_kernel<<<grid, SU_THREADS, 0, stream>>>(
      P->n_valid_points, P->n_full_points, P->d_map, P->d_coord, n_active, P->n_chp, P->n_atoms, P->L, P->L2,
      P->n_hartree_grid, P->hfla, P->d_chp, P->d_c2a, P->d_species, P->d_species_center, P->d_l_hartree,
      P->d_n_grid, P->d_rgm, P->d_linc, P->d_cc_xyz, mrs, opr, P->d_ncc, P->d_icc_packed, P->d_ijkmax, P->mc_dim,
      P->d_mc, spline, dv, codes);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

int sumup_read_error_flags(const SumupPlan *P, int *flags) {
  FRPA_CUDA_TRY(cudaMemcpy(flags, P->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  FRPA_CUDA_TRY(cudaMemset(P->d_err, 0, sizeof(int)));
  return FRPA_OK;
}

int sumup_adjoint_q(const SumupPlan *P, int n_active, const int *lhmfd, const double *mrs, const double *opr,
                    const double *Q, const double *g, double *dQ, cudaStream_t stream) {
  if (!P->fast)
    return fail(FRPA_ERR_UNSUPPORTED,
                "sumup adjoint: dQ is implemented for the fast path only (identity centers_hartree_potential and a "
                "homogeneous multipole table); this plan uses the generic far-field kernel");
  FRPA_CHECK_ARG(n_active >= 0 && n_active <= P->T, "sumup adjoint: n_active %d", n_active);
  FRPA_CUDA_TRY(cudaMemsetAsync(dQ, 0, sizeof(double) * (size_t)P->L2 * P->n_atoms * P->T, stream));
  if (n_active == 0 || P->n_chp == 0 || P->n_valid_points == 0) return FRPA_OK;
  sumup_multipole_c_kernel<<<dim3(P->n_atoms, n_active), 128, 0, stream>>>(
      P->n_atoms, P->L, P->L2, P->mc_dim, P->icc_dim0, P->lma, P->d_icc, P->d_ncc, P->d_cc, lhmfd, Q, P->d_mc,
      P->d_err);
  FRPA_LAUNCH_CHECK();
  sumup_records_kernel<<<dim3(P->n_chp, n_active), 128, 0, stream>>>(
      P->L, P->n_atoms, P->n_chp, P->mc_dim, P->n_coef, P->rs, P->d_chp, P->d_c2a, P->d_species,
      P->d_species_center, P->d_l_hartree, P->d_n_grid, P->d_rgm, P->d_linc, P->d_cc_xyz, mrs, opr, P->d_mc,
      P->d_conv_ptr, P->d_conv_n, P->d_conv_f, P->d_recs);
  FRPA_LAUNCH_CHECK();
  int st = FRPA_OK;
  st = launch_dcoef(*P, n_active, g, stream);
  if (st != FRPA_OK) return st;
  sumup_dmc_kernel<<<dim3(P->n_atoms, n_active), 128, 0, stream>>>(
      P->n_chp, P->n_atoms, P->mc_dim, P->n_coef, P->d_atom_slot_ptr, P->d_atom_slots, P->d_convT_ptr, P->d_convT_k,
      P->d_convT_f, P->d_dcoef, P->d_dmc);
  FRPA_LAUNCH_CHECK();
  sumup_dq_kernel<<<dim3(P->n_atoms, n_active), 64, 0, stream>>>(P->n_atoms, P->L, P->L2, P->mc_dim, P->icc_dim0,
                                                                  P->d_icc, P->d_ncc, P->d_cc, lhmfd, Q, P->d_dmc, dQ);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

}  // namespace frpa

// ------------------------------------------------ allocation-free variant
//
// frpa_sumup_execute_noalloc: the sum-up for callers that cannot let a
// library call cudaMalloc / cudaFree, such as a host code that hands the GPU
// a fixed memory budget managed by its own pool, or one that keeps several
// streams busy and cannot afford cudaFree's implicit device-wide
// synchronisation.  The caller passes every input and the output as device
// pointers; the only scratch this path needs (the packed multipole table and
// the per-atom multipole coefficients) lives in the file-scope array below,
// which every GPU that loads the library holds until the process exits.
// It runs the reference-mirroring (generic) kernel.

namespace frpa {

constexpr size_t NOALLOC_SCRATCH_BYTES = 8u << 20;  // 8 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

__global__ void noalloc_pack_table_kernel(int n_rows, int icc_dim0, const int *__restrict__ icc,
                                          int *__restrict__ packed) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_rows; n += gridDim.x * blockDim.x)
    packed[n] = icc[n + 2 * icc_dim0] | (icc[n + 3 * icc_dim0] << 8) | (icc[n + 4 * icc_dim0] << 16) |
                (icc[n + 5 * icc_dim0] << 24);
}

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64] = {nullptr};

// Device address of the scratch array for the current device, looked up once
// per device (host code may not use the array's name as an address).
int noalloc_scratch_address(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= 64) return fail(FRPA_ERR_UNSUPPORTED, "noalloc sum-up: device %d", device);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(FRPA_ERR_CUDA, "noalloc sum-up: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    FRPA_TRY(sumup_upload_constants(device));
    // the input-flag word at the start of the array collects the flags of
    // every call on this device until frpa_sumup_noalloc_flags reads it
    e = cudaMemset(p, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
      return fail(FRPA_ERR_CUDA, "noalloc sum-up: clearing the flag word failed: %s", cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_noalloc_addr[device]);
  return FRPA_OK;
}

}  // namespace
}  // namespace frpa

extern "C" int frpa_sumup_execute_noalloc(
    int atom_tile_size, int j_atom_begin, int j_atom_end, int n_full_points, int l_max_analytic_multipole,
    int index_cc_dim_0, int n_valid_points, int l_pot_max, int n_hartree_grid, int n_centers,
    int n_centers_hartree_potential, int n_atoms, int hartree_force_l_add, int n_species, const int *species,
    const int *species_center, const int *l_hartree_max_far_distance, const int *i_valid_point_2_i_full_points_map,
    const double *coord_points, const double *multipole_radius_sq, const double *outer_potential_radius,
    const double *multipole_moments, const double *spline, const int *l_hartree, const int *n_grid,
    const int *n_cc_lm_ijk, const int *centers_hartree_potential, const int *center_to_atom, const int *index_cc,
    const int *index_ijk_max_cc, const double *cc, const double *coords_center, const double *r_grid_min,
    const double *log_r_grid_inc, double *delta_v_hartree, void *stream_) {
  using namespace frpa;
  clear_error();
  const int T = atom_tile_size, L = l_pot_max, n_active = j_atom_end - j_atom_begin + 1;
  FRPA_CHECK_ARG(T >= 1 && T <= FRPA_MAX_ATOM_TILE, "noalloc sum-up: atom tile size %d out of range", T);
  FRPA_CHECK_ARG(L >= 0 && L <= SU_LMAX, "noalloc sum-up: l_pot_max %d unsupported (0..%d)", L, SU_LMAX);
  FRPA_CHECK_ARG(l_max_analytic_multipole >= L && index_cc_dim_0 > 0, "noalloc sum-up: bad multipole table sizes");
  FRPA_CHECK_ARG(hartree_force_l_add >= 0 && L + hartree_force_l_add <= 2 * SU_LMAX + 3,
                 "noalloc sum-up: hartree_force_l_add %d out of range", hartree_force_l_add);
  FRPA_CHECK_ARG(n_active <= T, "noalloc sum-up: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d", n_active, T);
  FRPA_CHECK_ARG(n_full_points >= 0 && n_valid_points >= 0 && n_valid_points <= n_full_points && n_atoms > 0 &&
                     n_centers > 0 && n_centers_hartree_potential >= 0 &&
                     n_centers_hartree_potential <= n_centers && n_species > 0 && n_hartree_grid >= 2,
                 "noalloc sum-up: bad sizes");
  FRPA_CHECK_ARG(species && species_center && l_hartree_max_far_distance && i_valid_point_2_i_full_points_map &&
                     coord_points && multipole_radius_sq && outer_potential_radius && multipole_moments && spline &&
                     l_hartree && n_grid && n_cc_lm_ijk && centers_hartree_potential && center_to_atom && index_cc &&
                     index_ijk_max_cc && cc && coords_center && r_grid_min && log_r_grid_inc && delta_v_hartree,
                 "noalloc sum-up: null device pointer");
  // scratch layout: [error flag | packed table rows | multipole coefficients
  // (index_cc_dim_0, n_atoms, T)]; the coefficient block is sized by
  // index_cc_dim_0, an upper bound of n_cc_lm_ijk[l_pot_max] known on the host.
  const size_t flag_bytes = 256;
  const size_t table_bytes = ((size_t)index_cc_dim_0 * sizeof(int) + 255) / 256 * 256;
  const size_t mc_bytes = sizeof(double) * (size_t)index_cc_dim_0 * n_atoms * T;
  const size_t need = flag_bytes + table_bytes + mc_bytes;
  FRPA_CHECK_ARG(need <= NOALLOC_SCRATCH_BYTES,
                 "noalloc sum-up: needs %zu bytes of scratch (index_cc_dim_0 %d x n_atoms %d x tile %d), more than "
                 "the %zu bytes this entry point has; use frpa_sumup_plan_create / frpa_sumup_execute",
                 need, index_cc_dim_0, n_atoms, T, (size_t)NOALLOC_SCRATCH_BYTES);
  int device = 0;
  FRPA_CUDA_TRY(cudaGetDevice(&device));
  unsigned char *base = nullptr;
  FRPA_TRY(noalloc_scratch_address(device, &base));
  if (n_active <= 0 || n_valid_points == 0 || n_centers_hartree_potential == 0) return FRPA_OK;
  cudaStream_t stream = (cudaStream_t)stream_;
  int *err = reinterpret_cast<int *>(base);
  int *packed = reinterpret_cast<int *>(base + flag_bytes);
  double *mc = reinterpret_cast<double *>(base + flag_bytes + table_bytes);
  const int L2 = (L + 1) * (L + 1);
  // every scratch word read below is written first in this call, so nothing
  // left by an earlier call is used; the flag word (bit 0: an
  // l_hartree_max_far_distance entry outside 0..l_pot_max, clamped) keeps
  // collecting until frpa_sumup_noalloc_flags reads and clears it
  noalloc_pack_table_kernel<<<(index_cc_dim_0 + 255) / 256, 256, 0, stream>>>(index_cc_dim_0, index_cc_dim_0,
                                                                               index_cc, packed);
  FRPA_LAUNCH_CHECK();
  sumup_multipole_c_kernel<<<dim3(n_atoms, n_active), 128, 0, stream>>>(
      n_atoms, L, L2, index_cc_dim_0, index_cc_dim_0, l_max_analytic_multipole, index_cc, n_cc_lm_ijk, cc,
      l_hartree_max_far_distance, multipole_moments, mc, err);
  FRPA_LAUNCH_CHECK();
  const int grid = (n_valid_points + SU_THREADS - 1) / SU_THREADS;
  sumup_generic_kernel<<<grid, SU_THREADS, 0, stream>>>(
      n_valid_points, n_full_points, i_valid_point_2_i_full_points_map, coord_points, n_active,
      n_centers_hartree_potential, n_atoms, L, L2, n_hartree_grid, hartree_force_l_add, centers_hartree_potential,
      center_to_atom, species, species_center, l_hartree, n_grid, r_grid_min, log_r_grid_inc, coords_center,
      multipole_radius_sq, outer_potential_radius, n_cc_lm_ijk, packed, index_ijk_max_cc, index_cc_dim_0, mc, spline,
      delta_v_hartree, nullptr);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

extern "C" int frpa_sumup_noalloc_flags(int *flags, void *stream_) {
  using namespace frpa;
  clear_error();
  FRPA_CHECK_ARG(flags != nullptr, "noalloc sum-up flags: null output");
  int device = 0;
  FRPA_CUDA_TRY(cudaGetDevice(&device));
  unsigned char *base = nullptr;
  FRPA_TRY(noalloc_scratch_address(device, &base));
  cudaStream_t stream = (cudaStream_t)stream_;
  int v = 0;
  FRPA_CUDA_TRY(cudaMemcpyAsync(&v, base, sizeof(int), cudaMemcpyDeviceToHost, stream));
  FRPA_CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(int), stream));
  FRPA_CUDA_TRY(cudaStreamSynchronize(stream));
  *flags = v;
  return FRPA_OK;
}
