/*
 * CPU parity oracle for the two DFPT grid hot paths (TEST INFRASTRUCTURE).
 *
 * A plain-C restatement of the reference algorithms, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * Nothing in the product library links or calls it.  Every routine cites the
 * reference file:line it restates (paths relative to the reference project;
 * "B/" = fast_rap_src_dfpt_gpu_eval/).
 *
 * Conventions follow the reference: Fortran column-major arrays, 1-based
 * basis / species / centre / atom indices where the reference has them,
 * 0-based full-point indices in i_valid_point_2_i_full_points_map.  The
 * perturbation tile size T (the reference's compile-time ATOM_TILE_SIZE) is a
 * runtime argument here.
 */
#ifndef FRPA_ORACLE_H
#define FRPA_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* rho1 and grad-rho1; B/evaluate_first_order_rho.cpp:12-210. Outputs are
 * zeroed then written, as in the reference. n_threads > 1 splits batches over
 * OpenMP threads (outputs are disjoint per batch). */
void oracle_rho1(int T, int n_my_batches_work, int j_atom_begin, int j_atom_end, int n_full_points, int n_basis,
                 int n_atoms, int n_max_compute_ham, int n_centers_basis_I, int n_max_batch_size,
                 const int *batch_sizes, const int *n_point_batches, const int *n_point_batches_prefix_sum,
                 const int *i_valid_point_2_i_full_points_map, const int *n_compute_c_batches,
                 const int *i_basis_batches, const int *i_batch_2_wave_offset, const double *wave,
                 const double *gradient_wave, const double *first_order_density_matrix, double *first_order_rho,
                 const double *first_order_rho_bias_part2, double *first_order_gradient_rho,
                 const double *first_order_gradient_rho_bias, int n_threads);

/* Hartree potential sum-up; B/sum_up_whole_potential.cpp:195-503.  Adds into
 * delta_v_hartree (n_full_points, T).  Supports l_pot_max <= 8 (the
 * reference's SHEval stops at 6).  If branch_codes is non-NULL it receives,
 * per (valid point, centre slot, tile), 0 = skipped, 1 + l_atom_max for the
 * near branch, 16 + l_atom_max for the far branch; layout
 * (n_valid_points, n_centers_hartree_potential, T) column-major. */
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
                  double *delta_v_hartree, unsigned char *branch_codes, int n_threads);

/* Real spherical harmonics in the reference's convention (index l*l+l+m),
 * evaluated from (x, y, z) = (sin t cos p, sin t sin p, cos t) by the
 * associated-Legendre recursion; l <= 8. Matches B/sheval.hpp:6-343. */
void oracle_ylm(int l_max, double x, double y, double z, double *ylm);

/* First-order H integration with every term (B/evaluate_first_order_H.cpp:13-222),
 * argument order as the reference's (arrays in its layouts, atom_valid
 * (n_atoms + 1, n_batches)); accumulates into first_order_H (n_basis, n_basis, T).
 * With every XC array zero it is H(ib_i, ib_j, t) += sum_p w v phi_i phi_j,
 * which equals dL/dP1 for L = sum_p w v rho1. */
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
                          const double *partition_tab, double *first_order_H);

/* Spherical-form far field, in long double, for validating multipole tables:
 * out[p] += sum_atoms sum_{l<=l_max, m} Q(l*l+l+m, atom) r^-(l+1) Y_lm(r_hat),
 * r = point - atom, Q (n_lm, n_atoms) column-major, n_lm = (l_max+1)^2. */
void oracle_far_field_spherical(int l_max, int n_points, const double *points, int n_atoms, const double *atoms,
                                const double *Q, double *out);

/* Ground-state bias term; B/generate_first_order_rho_bias_part2.cpp:9-167.
 * Writes bias(p, b, t) for t in [0, j_atom_end - j_atom_begin]. */
void oracle_rho_bias_part2(int T, int n_my_batches_work, int j_atom_begin, int j_atom_end, int j_coord,
                           int n_basis, int n_atoms, int n_centers_basis_I, int n_max_batch_size,
                           const int *n_point_batches, const int *n_compute_c_batches, const int *i_basis_batches,
                           const int *atom_valid_n_compute_c_batches, const int *i_batch_2_wave_offset,
                           const double *wave, const double *gradient_wave, const double *density_matrix,
                           double *first_order_rho_bias_part2);

#ifdef __cplusplus
}
#endif
#endif
