/*
 * CPU parity oracle (TEST INFRASTRUCTURE; see frpa_oracle.h).
 *
 * Plain-C restatements of the reference's CPU algorithms, written for
 * readability and bit-level fidelity of every branch decision, not for speed.
 * Citations are file:line in the reference project, "B/" =
 * fast_rap_src_dfpt_gpu_eval/.  Compiled with -ffp-contract=off so products
 * and sums are rounded one at a time, as in the reference's x86-64 build.
 */
#include "frpa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_LMAX 8

/* ------------------------------------------------------------------------ */
/* rho1: B/evaluate_first_order_rho.cpp:12-210                              */
/* ------------------------------------------------------------------------ */

/* One grid batch: gather P1c (:149-159), work1 = P1c * phi (:161-175), the
 * per-point dot products (:177-200) and the scatter (:202-207). */
static void rho1_one_batch(int T, int b, int n_active, int n_full_points, int n_basis, int n_centers_basis_I,
                           int n_max_batch_size, int n_batches, const int *n_point_batches,
                           const int *n_point_batches_prefix_sum, const int *map, const int *n_compute_c_batches,
                           const int *i_basis_batches, const int *i_batch_2_wave_offset, const double *wave,
                           const double *gradient_wave, const double *P1, double *rho, const double *bias,
                           double *grad, const double *gbias, double *scratch) {
  const int np = n_point_batches[b];
  const int nc = n_compute_c_batches[b];
  if (nc <= 0) return;
  const int ncp = ((nc + 3) / 4) * 4; /* :122 */
  const int *ib = i_basis_batches + (long)n_centers_basis_I * b;
  const double *phi = wave + i_batch_2_wave_offset[b];
  const double *gphi = gradient_wave + 3L * i_batch_2_wave_offset[b];
  const int *bmap = map + n_point_batches_prefix_sum[b];
  double *P1c = scratch;                   /* nc x nc, column-major */
  double *work1 = scratch + (long)nc * nc; /* nc x np, column-major */
  const long nb2 = (long)n_basis * n_basis;
  for (int t = 0; t < T; ++t) {
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) P1c[i + (long)nc * j] = P1[(ib[i] - 1) + (long)n_basis * (ib[j] - 1) + nb2 * t];
    for (int p = 0; p < np; ++p)
      for (int i = 0; i < nc; ++i) {
        double s = 0.0;
        for (int k = 0; k < nc; ++k) s += P1c[i + (long)nc * k] * phi[k + (long)ncp * p];
        work1[i + (long)nc * p] = s;
      }
    for (int p = 0; p < np; ++p) {
      double acc = 0.0, ag0 = 0.0, ag1 = 0.0, ag2 = 0.0;
      for (int i = 0; i < nc; ++i) {
        const double w1 = work1[i + (long)nc * p];
        acc += phi[i + (long)ncp * p] * w1;
        ag0 += gphi[i + (long)ncp * (0 + 3L * p)] * w1;
        ag1 += gphi[i + (long)ncp * (1 + 3L * p)] * w1;
        ag2 += gphi[i + (long)ncp * (2 + 3L * p)] * w1;
      }
      const long gidx = 3L * (p + (long)n_max_batch_size * (b + (long)n_batches * t));
      grad[gidx + 0] = ag0 * 2 - gbias[gidx + 0];
      grad[gidx + 1] = ag1 * 2 - gbias[gidx + 1];
      grad[gidx + 2] = ag2 * 2 - gbias[gidx + 2];
      if (t < n_active)
        rho[bmap[p] + (long)n_full_points * t] =
            acc + bias[p + (long)n_max_batch_size * (b + (long)n_batches * t)];
    }
  }
}

void oracle_rho1(int T, int n_my_batches_work, int j_atom_begin, int j_atom_end, int n_full_points, int n_basis,
                 int n_atoms, int n_max_compute_ham, int n_centers_basis_I, int n_max_batch_size,
                 const int *batch_sizes, const int *n_point_batches, const int *n_point_batches_prefix_sum,
                 const int *i_valid_point_2_i_full_points_map, const int *n_compute_c_batches,
                 const int *i_basis_batches, const int *i_batch_2_wave_offset, const double *wave,
                 const double *gradient_wave, const double *first_order_density_matrix, double *first_order_rho,
                 const double *first_order_rho_bias_part2, double *first_order_gradient_rho,
                 const double *first_order_gradient_rho_bias, int n_threads) {
  (void)batch_sizes;
  (void)n_atoms;
  int n_active = j_atom_end - j_atom_begin + 1; /* scatter loop :202 */
  if (n_active > T) n_active = T;
  /* :113-114 zero both outputs */
  memset(first_order_rho, 0, sizeof(double) * (size_t)n_full_points * T);
  memset(first_order_gradient_rho, 0, sizeof(double) * 3 * (size_t)n_max_batch_size * n_my_batches_work * T);
  int ncmax = 0, npmax = 0;
  for (int b = 0; b < n_my_batches_work; ++b) {
    if (n_compute_c_batches[b] > ncmax) ncmax = n_compute_c_batches[b];
    if (n_point_batches[b] > npmax) npmax = n_point_batches[b];
  }
  (void)n_max_compute_ham;
  const size_t scratch_len = (size_t)ncmax * ncmax + (size_t)ncmax * npmax + 1;
#ifdef _OPENMP
  if (n_threads < 1) n_threads = 1;
#pragma omp parallel num_threads(n_threads)
#endif
  {
    double *scratch = (double *)malloc(sizeof(double) * scratch_len);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
    for (int b = 0; b < n_my_batches_work; ++b)
      rho1_one_batch(T, b, n_active, n_full_points, n_basis, n_centers_basis_I, n_max_batch_size,
                     n_my_batches_work, n_point_batches, n_point_batches_prefix_sum,
                     i_valid_point_2_i_full_points_map, n_compute_c_batches, i_basis_batches,
                     i_batch_2_wave_offset, wave, gradient_wave, first_order_density_matrix, first_order_rho,
                     first_order_rho_bias_part2, first_order_gradient_rho, first_order_gradient_rho_bias, scratch);
    free(scratch);
  }
}

/* ------------------------------------------------------------------------ */
/* Real spherical harmonics, reference convention (B/sheval.hpp:6-343)      */
/* ------------------------------------------------------------------------ */

/* Y_{l,m} = K_l^|m| Q_l^|m|(z) * { (-1)^m C_m (m > 0); 1 (m = 0); S_|m| (m < 0) }
 * with C_m + i S_m = (x + i y)^m, Q_l^m the Legendre recursion without the
 * Condon-Shortley phase divided by sin^m, K_l^m = sqrt(2 (2l+1)/(4 pi)
 * (l-m)!/(l+m)!) for m > 0 (no sqrt 2 for m = 0).  Index l*l + l + m. */
void oracle_ylm(int l_max, double x, double y, double z, double *ylm) {
  double C[ORACLE_LMAX + 1], S[ORACLE_LMAX + 1];
  double Q[ORACLE_LMAX + 1][ORACLE_LMAX + 1];
  C[0] = 1.0;
  S[0] = 0.0;
  for (int m = 1; m <= l_max; ++m) {
    C[m] = x * C[m - 1] - y * S[m - 1];
    S[m] = x * S[m - 1] + y * C[m - 1];
  }
  for (int m = 0; m <= l_max; ++m) {
    double dfact = 1.0;
    for (int k = 1; k <= 2 * m - 1; k += 2) dfact *= k;
    Q[m][m] = dfact;
    if (m + 1 <= l_max) Q[m + 1][m] = (2 * m + 1) * z * Q[m][m];
    for (int l = m + 2; l <= l_max; ++l)
      Q[l][m] = ((2 * l - 1) * z * Q[l - 1][m] - (l + m - 1) * Q[l - 2][m]) / (l - m);
  }
  const double four_pi = 12.566370614359172953850573533118;
  for (int l = 0; l <= l_max; ++l) {
    for (int m = 0; m <= l; ++m) {
      double ratio = 1.0; /* (l-m)!/(l+m)! */
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= k;
      double K = sqrt((2 * l + 1) / four_pi * ratio);
      if (m == 0) {
        ylm[l * l + l] = K * Q[l][0];
      } else {
        K *= sqrt(2.0);
        const double sgn = (m & 1) ? -1.0 : 1.0;
        ylm[l * l + l + m] = sgn * K * Q[l][m] * C[m];
        ylm[l * l + l - m] = K * Q[l][m] * S[m];
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Sum-up: B/sum_up_whole_potential.cpp:91-187 (far), :195-503 (driver)     */
/* ------------------------------------------------------------------------ */

/* Far field for one (point, centre slot), B/sum_up_whole_potential.cpp:91-187.
 * Like the reference, the centre used for the monomials and the multipole
 * coefficients is the loop slot i_slot itself (its :161-162, :183), while
 * dist comes from the caller's centre. */
static double far_field_pair(int lam, int i_slot, double dist, int hartree_force_l_add, int n_centers,
                             int index_cc_dim_0, int mc_dim, const double *point, const int *n_cc_lm_ijk,
                             const int *center_to_atom, const int *index_cc, const int *index_ijk_max_cc,
                             const double *coords_center, const double *mc_t) {
  (void)n_centers;
  double Fp[2 * ORACLE_LMAX + 4];
  const double dsq = dist * dist;
  int k = 1;
  Fp[0] = 1.0 / dist;
  for (int l = 1; l <= lam + hartree_force_l_add; ++l) {
    k -= 2;
    Fp[l] = Fp[l - 1] * k / dsq;
  }
  double d[3];
  for (int c = 0; c < 3; ++c) d[c] = point[c] - coords_center[c + 3L * i_slot];
  int maxpow = -1;
  for (int c = 0; c < 3; ++c)
    if (index_ijk_max_cc[c + 3 * lam] > maxpow) maxpow = index_ijk_max_cc[c + 3 * lam];
  double pw[3][2 * ORACLE_LMAX + 2];
  for (int c = 0; c < 3; ++c) {
    pw[c][0] = 1.0;
    for (int i = 1; i <= maxpow; ++i) pw[c][i] = d[c] * pw[c][i - 1];
  }
  const double *mc = mc_t + (long)mc_dim * (center_to_atom[i_slot] - 1);
  double dpot = 0.0;
  const int n_end = n_cc_lm_ijk[lam];
  for (int n = 0; n < n_end; ++n) {
    const int ii = index_cc[n + 2L * index_cc_dim_0];
    const int jj = index_cc[n + 3L * index_cc_dim_0];
    const int kk = index_cc[n + 4L * index_cc_dim_0];
    const int nn = index_cc[n + 5L * index_cc_dim_0];
    dpot += pw[0][ii] * pw[1][jj] * pw[2][kk] * Fp[nn] * mc[n];
  }
  return dpot;
}

void oracle_sumup(int T, int j_atom_begin, int j_atom_end, int n_full_points, int l_max_analytic_multipole,
                  int index_cc_dim_0, int n_valid_points, int l_pot_max, int n_hartree_grid, int n_centers,
                  int n_centers_hartree_potential, int n_atoms, int hartree_force_l_add, int n_species,
                  const int *species, const int *species_center, const int *l_hartree_max_far_distance,
                  const int *i_valid_point_2_i_full_points_map, const double *coord_points,
                  const double *multipole_radius_sq, const double *outer_potential_radius,
                  const double *multipole_moments, const double *spline_tile, const int *l_hartree,
                  const int *n_grid, const int *n_cc_lm_ijk, const int *centers_hartree_potential,
                  const int *center_to_atom, const int *index_cc, const int *index_ijk_max_cc, const double *cc,
                  const double *coords_center, const double *r_grid_min, const double *log_r_grid_inc,
                  double *delta_v_hartree, unsigned char *branch_codes, int n_threads) {
  (void)l_max_analytic_multipole;
  (void)n_species;
  int n_active = j_atom_end - j_atom_begin + 1;
  if (n_active > T) n_active = T;
  const int L2 = (l_pot_max + 1) * (l_pot_max + 1);
  const int mc_dim = n_cc_lm_ijk[l_pot_max];

  /* multipole_c = cc * Q with the l cap and the 1e-10 threshold, :357-378.
   * Entries past n_cc_lm_ijk(l_hartree_max_far_distance) are left
   * uninitialised by the reference; they are zero here. */
  double *mc = (double *)calloc((size_t)mc_dim * n_atoms * T + 1, sizeof(double));
  for (int t = 0; t < n_active; ++t)
    for (int a = 0; a < n_atoms; ++a) {
      const int lh = l_hartree_max_far_distance[a + (long)n_atoms * t];
      for (int n = 0; n < n_cc_lm_ijk[lh]; ++n) {
        const int l = index_cc[n];
        const int m = index_cc[n + index_cc_dim_0];
        const double q = multipole_moments[(l * l + l + m) + (long)L2 * (a + (long)n_atoms * t)];
        mc[n + (long)mc_dim * (a + (long)n_atoms * t)] = (l <= lh && fabs(q) > 1e-10) ? cc[n] * q : 0.0;
      }
    }

#ifdef _OPENMP
  if (n_threads < 1) n_threads = 1;
#pragma omp parallel for schedule(static) num_threads(n_threads)
#endif
  for (int iv = 0; iv < n_valid_points; ++iv) {
    const int full = i_valid_point_2_i_full_points_map[iv];
    const double *pt = coord_points + 3L * full;
    double ylm[(ORACLE_LMAX + 1) * (ORACLE_LMAX + 1)];
    for (int t = 0; t < n_active; ++t) {
      double *dv = delta_v_hartree + full + (long)n_full_points * t;
      for (int ic = 0; ic < n_centers_hartree_potential; ++ic) {
        const int cur = centers_hartree_potential[ic] - 1;
        const int atom = center_to_atom[cur] - 1;
        /* :395-402 */
        double dir[3];
        dir[0] = pt[0] - coords_center[0 + 3L * cur];
        dir[1] = pt[1] - coords_center[1 + 3L * cur];
        dir[2] = pt[2] - coords_center[2 + 3L * cur];
        double d2 = 0.0;
        d2 += dir[0] * dir[0];
        d2 += dir[1] * dir[1];
        d2 += dir[2] * dir[2];
        /* :404-407 */
        int lam = l_hartree[species[atom] - 1];
        const double *opr = outer_potential_radius + (long)(l_pot_max + 1) * (atom + (long)n_atoms * t);
        while (opr[lam] < d2 && lam > 0) lam--;
        unsigned char code = 0;
        if (d2 < multipole_radius_sq[atom + (long)n_atoms * t]) {
          /* near field, :411-477 */
          const double dist = sqrt(d2);
          double din[3] = {dir[0] / dist, dir[1] / dist, dir[2] / dist};
          const int sp = species_center[cur];
          const double r_log = 1.0 + log(dist / r_grid_min[sp - 1]) / log_r_grid_inc[sp - 1];
          double st, ct, sph, cph; /* :427-450 */
          double ab;
          const double abmax = fmax(fabs(din[0]), fabs(din[1]));
          if (abmax > 1.0e-36) {
            ab = sqrt(din[0] * din[0] + din[1] * din[1]);
            cph = din[0] / ab;
            sph = din[1] / ab;
          } else {
            cph = 1.0;
            sph = 0.0;
            ab = 0.0;
          }
          const double abcmax = fmax(abmax, fabs(din[2]));
          if (abcmax > 1.0e-36) {
            const double abc = sqrt(ab * ab + din[2] * din[2]);
            ct = din[2] / abc;
            st = ab / abc;
          } else {
            ct = 0.0;
            st = 1.0;
          }
          oracle_ylm(lam, st * cph, st * sph, ct, ylm);
          /* Hermite spline fused with the Y_lm dot, :12-52 */
          const int npts = n_grid[sp - 1];
          int i_spl = (int)r_log;
          if (i_spl < 1) i_spl = 1;
          if (i_spl > npts - 1) i_spl = npts - 1;
          const double u = r_log - i_spl;
          const double ta = (u - 1) * (u - 1) * (1 + 2 * u);
          const double tb = (u - 1) * (u - 1) * u;
          const double tc = u * u * (3 - 2 * u);
          const double td = u * u * (u - 1);
          const double *spl = spline_tile + (long)L2 * 2 * n_hartree_grid * (atom + (long)n_atoms * t);
          const double *g0 = spl + (long)L2 * 2 * (i_spl - 1);
          const double *g1 = spl + (long)L2 * 2 * i_spl;
          double acc = 0.0;
          const int nv = (lam + 1) * (lam + 1);
          for (int i = 0; i < nv; ++i)
            acc += (g0[i] * ta + g0[i + L2] * tb + g1[i] * tc + g1[i + L2] * td) * ylm[i];
          *dv += acc;
          code = (unsigned char)(1 + lam);
        } else if (d2 < 1e8) {
          /* far field, :478-499 */
          const double dist = sqrt(d2);
          *dv += far_field_pair(lam, ic, dist, hartree_force_l_add, n_centers, index_cc_dim_0, mc_dim, pt,
                                n_cc_lm_ijk, center_to_atom, index_cc, index_ijk_max_cc, coords_center,
                                mc + (long)mc_dim * n_atoms * t);
          code = (unsigned char)(16 + lam);
        }
        if (branch_codes)
          branch_codes[iv + (long)n_valid_points * (ic + (long)n_centers_hartree_potential * t)] = code;
      }
    }
  }
  free(mc);
}

/* ------------------------------------------------------------------------ */
/* First-order H with zero XC terms: B/evaluate_first_order_H.cpp:13-222    */
/* ------------------------------------------------------------------------ */

/* First-order H with every term (evaluate_first_order_H.cpp:77-215).  Per
 * batch and atom j of the tile (t = j - j_atom_begin), per point p:
 *   lfos = 2 sum_k fogr(k, p) grad_rho(k, f)                       (:146-152)
 *   pf2_k = 2 w(f) grad_rho(k, f) (v2rhosigma rho1 + v2sigma2 lfos)
 *           + 2 w(f) vsigma fogr(k, p)                             (:153-160)
 *   pf3 = w(f) (v_hartree_gradient + v2rho2 rho1 + v2rhosigma lfos) (:161-164)
 *   pf5_k = 2 vsigma w(f) grad_rho(k, f)                           (:165-168)
 *   cs1(i, p) = 0.5 (H_prefactor1 + pf3) phi_i + sum_k pf2_k dphi_i/dk (:170-178)
 *              - sum_k pf5_k hess_i(k, j_coord) for i in atom j's range (:180-189)
 * then H(ib_i, ib_j) += sum_p cs1(i, p) phi_j(p) + phi_i(p) cs1(j, p), the
 * rank-2k update (:192-205) and its symmetric scatter (:207-215).  The XC
 * arrays are indexed by their first component only, as the reference does
 * (vsigma(0, p), v2rho2(0, p), v2rhosigma(0, p), v2sigma2(0, p)); vrho and
 * H_times_psi are accepted and unused there as well. */
void oracle_first_order_h(int T, int n_my_batches_work, int j_atom_begin, int j_atom_end, int n_full_points,
                          int j_coord, int n_basis, int n_max_batch_size, int n_centers_basis_I,
                          const int *n_point_batches, const int *n_compute_c_batches, const int *i_basis_batches,
                          const int *atom_valid, int n_atoms, const int *n_point_batches_prefix_sum,
                          const int *i_valid_point_2_i_full_points_map, const double *vsigma_batches,
                          const double *gradient_rho, const int *i_batch_2_wave_offset, const double *wave,
                          const double *gradient_wave, const double *hessian_wave, const double *H_prefactor1,
                          const double *first_order_gradient_rho, const double *v_hartree_gradient,
                          const double *first_order_rho, const double *v2rho2_batches,
                          const double *v2rhosigma_batches, const double *v2sigma2_batches,
                          const double *partition_tab, double *first_order_H) {
  static const int ih[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  const long nb2 = (long)n_basis * n_basis;
  const long nmb = n_max_batch_size, nbt = n_my_batches_work;
  double *cs = NULL;
  long cs_len = 0;
  for (int b = 0; b < n_my_batches_work; ++b) {
    const int nc = n_compute_c_batches[b];
    const int np = n_point_batches[b];
    if (nc <= 0) continue;
    const int ncp = ((nc + 3) / 4) * 4;
    const int *ib = i_basis_batches + (long)n_centers_basis_I * b;
    const long off = i_batch_2_wave_offset[b];
    const double *phi = wave + off;
    const double *gph = gradient_wave + 3 * off;
    const double *hph = hessian_wave + 6 * off;
    const int *bmap = i_valid_point_2_i_full_points_map + n_point_batches_prefix_sum[b];
    if ((long)nc * np > cs_len) {
      free(cs);
      cs_len = (long)nc * np;
      cs = (double *)malloc(sizeof(double) * cs_len);
    }
    for (int ja = j_atom_begin; ja <= j_atom_end; ++ja) {
      const int t = ja - j_atom_begin;
      if (t >= T) break;
      const int vs = atom_valid[(ja - 1) + (long)(n_atoms + 1) * b];
      const int ve = atom_valid[ja + (long)(n_atoms + 1) * b];
      for (int p = 0; p < np; ++p) {
        const long f = bmap[p];
        const long bp = p + nmb * (b + nbt * t);
        const double pf1 = H_prefactor1[bp];
        const double *fog = first_order_gradient_rho + 3 * bp;
        const double *gr = gradient_rho + 3 * f;
        const double vsig = vsigma_batches[3 * nmb * b + 3 * p];
        const double v2r2 = v2rho2_batches[3 * nmb * b + 3 * p];
        const double v2rs = v2rhosigma_batches[6 * nmb * b + 6 * p];
        const double v2s2 = v2sigma2_batches[6 * nmb * b + 6 * p];
        const double w = partition_tab[f];
        const double r1 = first_order_rho[f + (long)n_full_points * t];
        double lfos = 0.0;
        for (int k = 0; k < 3; ++k) lfos += fog[k] * gr[k];
        lfos *= 2.0;
        double pf2[3], pf5[3];
        for (int k = 0; k < 3; ++k) {
          pf2[k] = 2.0 * w * gr[k] * (v2rs * r1 + v2s2 * lfos) + 2.0 * w * vsig * fog[k];
          pf5[k] = 2.0 * vsig * w * gr[k];
        }
        const double pf3 = w * (v_hartree_gradient[f + (long)n_full_points * t] + v2r2 * r1 + v2rs * lfos);
        for (int i = 0; i < nc; ++i) {
          const double c1 = (pf1 + pf3) * phi[i + (long)ncp * p];
          double c2 = 0.0;
          for (int k = 0; k < 3; ++k) c2 += pf2[k] * gph[i + (long)ncp * (k + 3L * p)];
          cs[i + (long)nc * p] = 0.5 * c1 + c2;
        }
        for (int i = vs; i < ve; ++i) {
          double c5 = 0.0;
          for (int k = 0; k < 3; ++k) c5 += pf5[k] * -hph[i + (long)ncp * (ih[k][j_coord - 1] + 6L * p)];
          cs[i + (long)nc * p] += c5;
        }
      }
      for (int i = 0; i < nc; ++i)
        for (int j = i; j < nc; ++j) {
          double s = 0.0;
          for (int p = 0; p < np; ++p)
            s += cs[j + (long)nc * p] * phi[i + (long)ncp * p] + phi[j + (long)ncp * p] * cs[i + (long)nc * p];
          const long ai = ib[i] - 1, aj = ib[j] - 1;
          double *Ht = first_order_H + nb2 * t;
          if (i == j) {
            Ht[ai + n_basis * ai] += s;
          } else {
            Ht[ai + n_basis * aj] += s;
            Ht[aj + n_basis * ai] += s;
          }
        }
    }
  }
  free(cs);
}

/* ------------------------------------------------------------------------ */
/* Spherical-form far field (long double), for table validation             */
/* ------------------------------------------------------------------------ */

static void ylm_ld(int l_max, long double x, long double y, long double z, long double *ylm) {
  long double C[ORACLE_LMAX + 1], S[ORACLE_LMAX + 1], Q[ORACLE_LMAX + 1][ORACLE_LMAX + 1];
  C[0] = 1.0L;
  S[0] = 0.0L;
  for (int m = 1; m <= l_max; ++m) {
    C[m] = x * C[m - 1] - y * S[m - 1];
    S[m] = x * S[m - 1] + y * C[m - 1];
  }
  for (int m = 0; m <= l_max; ++m) {
    long double dfact = 1.0L;
    for (int k = 1; k <= 2 * m - 1; k += 2) dfact *= k;
    Q[m][m] = dfact;
    if (m + 1 <= l_max) Q[m + 1][m] = (2 * m + 1) * z * Q[m][m];
    for (int l = m + 2; l <= l_max; ++l)
      Q[l][m] = ((2 * l - 1) * z * Q[l - 1][m] - (l + m - 1) * Q[l - 2][m]) / (l - m);
  }
  const long double four_pi = 12.566370614359172953850573533118L;
  for (int l = 0; l <= l_max; ++l)
    for (int m = 0; m <= l; ++m) {
      long double ratio = 1.0L;
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= k;
      long double K = sqrtl((2 * l + 1) / four_pi * ratio);
      if (m == 0) {
        ylm[l * l + l] = K * Q[l][0];
      } else {
        K *= sqrtl(2.0L);
        ylm[l * l + l + m] = ((m & 1) ? -1.0L : 1.0L) * K * Q[l][m] * C[m];
        ylm[l * l + l - m] = K * Q[l][m] * S[m];
      }
    }
}

void oracle_far_field_spherical(int l_max, int n_points, const double *points, int n_atoms, const double *atoms,
                                const double *Q, double *out) {
  const int nlm = (l_max + 1) * (l_max + 1);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int p = 0; p < n_points; ++p) {
    long double ylm[(ORACLE_LMAX + 1) * (ORACLE_LMAX + 1)];
    long double acc = 0.0L;
    for (int a = 0; a < n_atoms; ++a) {
      long double d[3];
      for (int c = 0; c < 3; ++c) d[c] = (long double)points[c + 3L * p] - (long double)atoms[c + 3L * a];
      const long double r = sqrtl(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      ylm_ld(l_max, d[0] / r, d[1] / r, d[2] / r, ylm);
      long double rl = 1.0L / r;
      for (int l = 0; l <= l_max; ++l) {
        long double s = 0.0L;
        for (int m = -l; m <= l; ++m) s += (long double)Q[(l * l + l + m) + (long)nlm * a] * ylm[l * l + l + m];
        acc += s * rl;
        rl /= r;
      }
    }
    out[p] += (double)acc;
  }
}

/* ------------------------------------------------------------------------ */
/* Bias producer: B/generate_first_order_rho_bias_part2.cpp:9-167           */
/* ------------------------------------------------------------------------ */

void oracle_rho_bias_part2(int T, int n_my_batches_work, int j_atom_begin, int j_atom_end, int j_coord,
                           int n_basis, int n_atoms, int n_centers_basis_I, int n_max_batch_size,
                           const int *n_point_batches, const int *n_compute_c_batches, const int *i_basis_batches,
                           const int *atom_valid_n_compute_c_batches, const int *i_batch_2_wave_offset,
                           const double *wave, const double *gradient_wave, const double *density_matrix,
                           double *first_order_rho_bias_part2) {
  for (int b = 0; b < n_my_batches_work; ++b) {
    const int np = n_point_batches[b];
    const int nc = n_compute_c_batches[b];
    if (nc <= 0) continue;
    const int ncp = ((nc + 3) / 4) * 4;
    const int *ib = i_basis_batches + (long)n_centers_basis_I * b;
    const double *phi = wave + i_batch_2_wave_offset[b];
    const double *gphi = gradient_wave + 3L * i_batch_2_wave_offset[b];
    double *D = (double *)malloc(sizeof(double) * (size_t)nc * nc);
    double *work = (double *)malloc(sizeof(double) * (size_t)nc * (np > 0 ? np : 1));
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nc; ++i) D[i + (long)nc * j] = density_matrix[(ib[i] - 1) + (long)n_basis * (ib[j] - 1)];
    for (int ja = j_atom_begin; ja <= j_atom_end; ++ja) {
      const int t = ja - j_atom_begin;
      if (t >= T) break;
      const int vs = atom_valid_n_compute_c_batches[(ja - 1) + (long)(n_atoms + 1) * b];
      const int ve = atom_valid_n_compute_c_batches[ja + (long)(n_atoms + 1) * b];
      double *out = first_order_rho_bias_part2 + (long)n_max_batch_size * (b + (long)n_my_batches_work * t);
      if (ve - vs <= 0) {
        for (int p = 0; p < np; ++p) out[p] = 0.0;
        continue;
      }
      /* first term: phi . (D(:, vs:ve) . fw(vs:ve, :)), fw = -d phi / d x_jcoord */
      for (int p = 0; p < np; ++p)
        for (int i = 0; i < nc; ++i) {
          double s = 0.0;
          for (int k = vs; k < ve; ++k)
            s += D[i + (long)nc * k] * (-gphi[k + (long)ncp * ((j_coord - 1) + 3L * p)]);
          work[i + (long)nc * p] = s;
        }
      for (int p = 0; p < np; ++p) {
        double acc = 0.0;
        for (int i = 0; i < nc; ++i) acc += phi[i + (long)ncp * p] * work[i + (long)nc * p];
        out[p] = acc;
      }
      /* second term: fw(vs:ve, :) . (D(vs:ve, :) . phi) */
      for (int p = 0; p < np; ++p) {
        double acc = 0.0;
        for (int i = vs; i < ve; ++i) {
          double s = 0.0;
          for (int k = 0; k < nc; ++k) s += D[i + (long)nc * k] * phi[k + (long)ncp * p];
          acc += (-gphi[i + (long)ncp * ((j_coord - 1) + 3L * p)]) * s;
        }
        out[p] += acc;
      }
    }
    free(D);
    free(work);
  }
}
