// Test infrastructure (never part of the product): compiled against the
// reference's OWN headers next to include/frpa.h, so that the compiler checks
// that every entry point the two declare is declared alike, and linked against
// libfrpa.so, so that the reference's C++ callers' way of binding each symbol
// (C++ linkage where the reference declares it so) is exercised by a test.
//
//   evaluate_first_order_rho.h     extern "C" rho1 entry points (:3-69)
//   sum_up_whole_potential.h       extern "C" sum-up (:3-48), C++-linkage cu_host_ twin (:50-95)
//   evaluate_first_order_H.h       extern "C" first-order H (:3-43)
//   device_data.hpp / device.hpp   C++-linkage session functions (device_data.hpp:159-227, device.hpp:191-192)
//
// A C-linkage function declared differently by the two headers is a compile
// error by itself; for the C++-linkage ones a different parameter list would
// silently add an overload, so each of them is also bound to a single
// function pointer below, which fails to compile if it is overloaded.
#include "evaluate_first_order_rho.h"
#include "sum_up_whole_potential.h"
#include "evaluate_first_order_H.h"
#include "device_data.hpp"

#include "frpa.h"

namespace {
template <class F>
constexpr bool declared_once(F *) {
  return true;
}
static_assert(declared_once(&init_dfpt_device_info), "init_dfpt_device_info declared alike");
static_assert(declared_once(&free_dfpt_device_info), "free_dfpt_device_info declared alike");
static_assert(declared_once(&init_dfpt_device_data), "init_dfpt_device_data declared alike");
static_assert(declared_once(&free_dfpt_device_data), "free_dfpt_device_data declared alike");
static_assert(declared_once(&sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_),
              "sum-up cu_host_ declared alike");
static_assert(declared_once(&evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_), "rho1 declared alike");
static_assert(declared_once(&evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_),
              "rho1 cu_host_ declared alike");
static_assert(declared_once(&sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_), "sum-up declared alike");
}  // namespace

// Thin C wrappers for the test harness (ctypes cannot name C++ symbols): each
// calls the C++-linkage entry point exactly as a reference C++ caller would.
extern "C" {

void hdrchk_init_dfpt_device_info(void) { init_dfpt_device_info(); }
void hdrchk_free_dfpt_device_info(void) { free_dfpt_device_info(); }
void hdrchk_free_dfpt_device_data(void) { free_dfpt_device_data(); }

void hdrchk_init_dfpt_device_data(
    int *n_my_batches_work, int *n_full_points, int *n_valid_points, int *n_basis, int *n_atoms,
    int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *l_pot_max, int *n_max_radial,
    int *n_hartree_grid, int *n_centers, int *n_centers_hartree_potential, int *hartree_force_l_add, int *n_species,
    int *l_max_analytic_multipole, int *index_cc_dim_0, int *basis_atom, int *batch_sizes, int *n_point_batches,
    int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map, int *n_compute_c_batches,
    int *i_basis_batches, int *atom_valid_n_compute_c_batches, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *density_matrix, int *n_radial,
    int *species, int *species_center, double *coord_points, int *l_hartree, int *n_grid, int *n_cc_lm_ijk,
    int *centers_hartree_potential, int *center_to_atom, int *index_cc, int *index_ijk_max_cc, double *cc,
    double *coords_center, double *r_grid_min, double *log_r_grid_inc, double *scale_radial, double *partition_tab,
    double *first_order_density_matrix, double *first_order_rho, double *first_order_rho_bias_part2,
    double *first_order_gradient_rho, double *first_order_gradient_rho_bias_batches_atoms,
    int *l_hartree_max_far_distance, double *multipole_radius_sq, double *outer_potential_radius,
    double *multipole_moments, double *current_delta_v_hart_part_spl_tile, double *delta_v_hartree) {
  init_dfpt_device_data(
      n_my_batches_work, n_full_points, n_valid_points, n_basis, n_atoms, n_max_compute_ham, n_centers_basis_I,
      n_max_batch_size, l_pot_max, n_max_radial, n_hartree_grid, n_centers, n_centers_hartree_potential,
      hartree_force_l_add, n_species, l_max_analytic_multipole, index_cc_dim_0, basis_atom, batch_sizes,
      n_point_batches, n_point_batches_prefix_sum, i_valid_point_2_i_full_points_map, n_compute_c_batches,
      i_basis_batches, atom_valid_n_compute_c_batches, i_batch_2_wave_offset, wave_batches_compress,
      gradient_wave_batches_compress, density_matrix, n_radial, species, species_center, coord_points, l_hartree,
      n_grid, n_cc_lm_ijk, centers_hartree_potential, center_to_atom, index_cc, index_ijk_max_cc, cc, coords_center,
      r_grid_min, log_r_grid_inc, scale_radial, partition_tab, first_order_density_matrix, first_order_rho,
      first_order_rho_bias_part2, first_order_gradient_rho, first_order_gradient_rho_bias_batches_atoms,
      l_hartree_max_far_distance, multipole_radius_sq, outer_potential_radius, multipole_moments,
      current_delta_v_hart_part_spl_tile, delta_v_hartree);
}

void hdrchk_sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_(
    int j_atom_begin, int j_atom_end, int n_full_points, int l_max_analytic_multipole, int index_cc_dim_0,
    int n_valid_points, int l_pot_max, int n_max_radial, int n_hartree_grid, int n_centers,
    int n_centers_hartree_potential, int n_atoms, int hartree_force_l_add, int n_species, const int *n_radial,
    const int *species, const int *species_center, const int *l_hartree_max_far_distance,
    const int *i_valid_point_2_i_full_points_map, const double *coord_points, const double *multipole_radius_sq,
    const double *outer_potential_radius, const double *multipole_moments,
    const double *current_delta_v_hart_part_spl_tile, const int *l_hartree, const int *n_grid,
    const int *n_cc_lm_ijk, const int *centers_hartree_potential, const int *center_to_atom, const int *index_cc,
    const int *index_ijk_max_cc, const double *cc, const double *coords_center, const double *r_grid_min,
    const double *log_r_grid_inc, const double *scale_radial, const double *partition_tab,
    double *delta_v_hartree) {
  sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_(
      j_atom_begin, j_atom_end, n_full_points, l_max_analytic_multipole, index_cc_dim_0, n_valid_points, l_pot_max,
      n_max_radial, n_hartree_grid, n_centers, n_centers_hartree_potential, n_atoms, hartree_force_l_add, n_species,
      n_radial, species, species_center, l_hartree_max_far_distance, i_valid_point_2_i_full_points_map, coord_points,
      multipole_radius_sq, outer_potential_radius, multipole_moments, current_delta_v_hart_part_spl_tile, l_hartree,
      n_grid, n_cc_lm_ijk, centers_hartree_potential, center_to_atom, index_cc, index_ijk_max_cc, cc, coords_center,
      r_grid_min, log_r_grid_inc, scale_radial, partition_tab, delta_v_hartree);
}

}  // extern "C"
