// Writes small capture files with the reference's OWN header-only writers
// (write_first_order_rho_meta_data in
// fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho_direct_test.hpp:27-70,
// write_hartree_potential_data in .../sum_up_direct_test.hpp), so that this
// project's reader for the same byte layout is pinned against them.
// Usage: capture_writer <rho.bin> <sumup.bin>.  Values are a fixed recipe of
// small integers and doubles.  Test infrastructure.
#include <cstdio>
#include <string>
#include <type_traits>

#include "evaluate_first_order_rho_direct_test.hpp"
#include "sum_up_direct_test.hpp"

static std::vector<int> iota_vec(int n, int start, int step) {
  std::vector<int> v(n);
  for (int i = 0; i < n; ++i) v[i] = start + i * step;
  return v;
}
static std::vector<double> dvec(int n, double start, double step) {
  std::vector<double> v(n);
  for (int i = 0; i < n; ++i) v[i] = start + i * step;
  return v;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  FirstOrderRhoMetaData r;
  r.n_my_batches_work = 3;
  r.n_full_points = 11;
  r.n_basis = 7;
  r.n_atoms = 2;
  r.n_max_compute_ham = 5;
  r.n_centers_basis_I = 7;
  r.n_max_batch_size = 4;
  r.basis_atom = {1, 1, 1, 1, 2, 2, 2};
  r.batch_sizes = {4, 3, 4};
  r.n_point_batches = {4, 3, 4};
  r.n_point_batches_prefix_sum = {0, 4, 7, 11};
  r.i_valid_point_2_i_full_points_map = iota_vec(11, 10, -1);
  r.n_compute_c_batches = {5, 0, 3};
  r.i_basis_batches = iota_vec(21, 1, 1);
  r.atom_valid_n_compute_c_batches = iota_vec(9, 0, 2);
  r.i_batch_2_wave_offset = {0, 32, 32, 48};
  write_first_order_rho_meta_data(argv[1], r);

  HartreePotentialData s;
  s.j_atom_begin = 1;
  s.j_atom_end = 2;
  s.n_full_points = 6;
  s.l_max_analytic_multipole = 2;
  s.index_cc_dim_0 = 12;
  s.n_valid_points = 5;
  s.l_pot_max = 1;
  s.n_max_radial = 9;
  s.n_hartree_grid = 10;
  s.n_centers = 3;
  s.n_centers_hartree_potential = 3;
  s.n_atoms = 3;
  s.hartree_force_l_add = 1;
  s.n_species = 2;
  s.n_radial = {9, 8};
  s.species = {1, 2, 1};
  s.species_center = {1, 2, 1};
  s.l_hartree_max_far_distance = {1, 1, 0, 1, 1, 0};
  s.i_valid_point_2_i_full_points_map = {5, 4, 3, 1, 0};
  s.coord_points = dvec(18, -1.5, 0.25);
  s.multipole_radius_sq = dvec(6, 4.0, 0.5);
  s.outer_potential_radius = dvec(12, 100.0, -3.0);
  s.multipole_moments = dvec(24, 0.125, 0.0625);
  s.l_hartree = {1, 0};
  s.n_grid = {10, 10};
  s.n_cc_lm_ijk = {1, 4, 12};
  s.centers_hartree_potential = {1, 2, 3};
  s.center_to_atom = {1, 2, 3};
  s.index_cc = iota_vec(72, 0, 1);
  s.index_ijk_max_cc = iota_vec(9, 0, 1);
  s.cc = dvec(12, 0.5, 0.5);
  s.coords_center = dvec(9, 0.0, 1.0);
  s.r_grid_min = {1e-4, 2e-4};
  s.log_r_grid_inc = {0.0125, 0.015};
  s.scale_radial = {1.0, 1.5};
  s.partition_tab = dvec(6, 0.1, 0.1);
  write_hartree_potential_data(argv[2], s);
  return 0;
}
