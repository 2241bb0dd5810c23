/*
 * frpa: B200-native (sm_100a) DFPT grid hot paths behind a C ABI.
 *
 *  1. The first-order density rho1 and its gradient
 *     (evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_).
 *  2. The Hartree potential sum-up from atomic multipoles
 *     (sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_).
 *
 * Three layers:
 *  - Reference drop-ins: the reference's own entry-point names, argument lists
 *    and array layouts (Fortran column-major, 1-based basis / species / centre
 *    indices, 0-based full-point indices).  They take HOST pointers.  The void
 *    ones report failures through frpa_last_error() instead of exit(1).
 *    Citations are to the reference project kzwrime/fast_rpa_eval,
 *    directory fast_rap_src_dfpt_gpu_eval/.
 *  - The reference's device session (init_dfpt_device_info / _data and the
 *    *_cu_host_ twins), which keeps the constant arrays resident on the GPU.
 *  - Plans: an explicit, re-entrant, stream-ordered API on DEVICE pointers
 *    (what the Python bindings, the benchmarks and CUDA-graph capture use).
 *
 * The reference fixes the perturbation tile size ATOM_TILE_SIZE at compile
 * time (setting.h:19-21); here it is a runtime setting (default 1).
 * Everything is FP64 except the optional split-BF16 rho1 contraction.
 */
#ifndef FRPA_H
#define FRPA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ limits */
#define FRPA_MAX_N_COMPUTE 2048 /* n_compute_c per batch */
#define FRPA_MAX_ATOM_TILE 64   /* ATOM_TILE_SIZE */
#define FRPA_SUMUP_MAX_L 8      /* l_pot_max */

/* ---------------------------------------------------------------- status */
enum {
  FRPA_OK = 0,
  FRPA_ERR_INVALID = 1,     /* bad argument or inconsistent input arrays */
  FRPA_ERR_CUDA = 2,        /* CUDA runtime error (message has the details) */
  FRPA_ERR_NO_SESSION = 3,  /* *_cu_host_ called before init_dfpt_device_data */
  FRPA_ERR_OOM = 4,         /* device allocation failed */
  FRPA_ERR_UNSUPPORTED = 5, /* valid input outside what this build implements */
  FRPA_ERR_DEVICE_INPUT = 6 /* a device-side input check failed (see message) */
};

/* Status of the last failing call on this thread (FRPA_OK if none since the
 * last frpa_clear_error), and its message. */
int frpa_last_error(void);
const char *frpa_last_error_message(void);
void frpa_clear_error(void);
int frpa_version(void);

/* The GPU that plans and the session created afterwards on this thread use:
 * cudaSetDevice in the library's own CUDA runtime (it is linked statically, so
 * a caller's cudaSetDevice through another runtime need not reach it).  The
 * session (init_dfpt_device_info) takes $FRPA_DEVICE if set, else this device,
 * which is device 0 unless set -- the reference's fixed choice
 * (device.cu:7-9).  No counterpart in the reference. */
int frpa_set_device(int device);
int frpa_get_device(int *device);

/* ATOM_TILE_SIZE for the reference drop-ins (setting.h:19-21), 1..64. */
int frpa_set_atom_tile_size(int T);
int frpa_get_atom_tile_size(void);

/* rho1 contraction mode used by the reference drop-ins:
 *   FRPA_RHO1_FP64        FP64 tensor-core tiles (DMMA), the reference's arithmetic;
 *   FRPA_RHO1_SPLIT_BF16  five BF16 slices per operand on tcgen05 kind::f16, FP32 level sums;
 *   FRPA_RHO1_SPLIT_I8    five signed 8-bit digits per operand on tcgen05 kind::i8, exact
 *                         int32 level sums, operands packed by separate kernels. */
enum { FRPA_RHO1_FP64 = 0, FRPA_RHO1_SPLIT_BF16 = 1, FRPA_RHO1_SPLIT_I8 = 2 };
int frpa_set_rho1_mode(int mode);
int frpa_get_rho1_mode(void);

/* =========================================================================
 * Reference drop-ins (host pointers)
 * ======================================================================= */

/* Replaces evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_
 * (evaluate_first_order_rho.h:3-35, CPU implementation evaluate_first_order_rho.cpp:12-210).
 * Same arguments and layouts; computes on the GPU (uploads everything, runs,
 * downloads first_order_rho and first_order_gradient_rho, which are zeroed and
 * then written as in the reference).  basis_atom, partition_tab and
 * density_matrix are accepted and unused, as in the reference. */
void evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map,
    int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *first_order_density_matrix,
    double *first_order_rho, double *first_order_rho_bias_part2, double *first_order_gradient_rho,
    double *first_order_gradient_rho_bias_batches_atoms, int *basis_atom, double *partition_tab,
    double *density_matrix);

/* Replaces evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_
 * (evaluate_first_order_rho.h:37-69, evaluate_first_order_rho.cu:188-371).
 * Uses the arrays made resident by init_dfpt_device_data; per call it uploads
 * the changeable inputs first_order_density_matrix, first_order_rho_bias_part2
 * and first_order_gradient_rho_bias_batches_atoms from the host pointers,
 * computes, and downloads first_order_rho and first_order_gradient_rho (the
 * reference's host-copy mode, evaluate_first_order_rho.cu:259-263,363-367).
 * The outputs also stay resident (frpa_session_rho1_device_outputs). */
void evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map,
    int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *first_order_density_matrix,
    double *first_order_rho, double *first_order_rho_bias_part2, double *first_order_gradient_rho,
    double *first_order_gradient_rho_bias_batches_atoms, int *basis_atom, double *partition_tab,
    double *density_matrix);

/* Replaces sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_
 * (sum_up_whole_potential.h:3-48, sum_up_whole_potential.cpp:195-529).
 * Accumulates into delta_v_hartree (n_full_points, ATOM_TILE_SIZE).
 * l_pot_max <= 8 (the reference's own near field stops at 6). */
void sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_(
    const int *j_atom_begin, const int *j_atom_end, const int *n_full_points, const int *l_max_analytic_multipole,
    const int *index_cc_dim_0, const int *n_valid_points, const int *l_pot_max, const int *n_max_radial,
    const int *n_hartree_grid, const int *n_centers, const int *n_centers_hartree_potential, const int *n_atoms,
    const int *hartree_force_l_add, const int *n_species, const int *n_radial, const int *species,
    const int *species_center, const int *l_hartree_max_far_distance, const int *i_valid_point_2_i_full_points_map,
    const double *coord_points, const double *multipole_radius_sq, const double *outer_potential_radius,
    const double *multipole_moments, const double *current_delta_v_hart_part_spl_tile, const int *l_hartree,
    const int *n_grid, const int *n_cc_lm_ijk, const int *centers_hartree_potential, const int *center_to_atom,
    const int *index_cc, const int *index_ijk_max_cc, const double *cc, const double *coords_center,
    const double *r_grid_min, const double *log_r_grid_inc, const double *scale_radial, const double *partition_tab,
    double *delta_v_hartree);

/* Replaces sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_
 * (sum_up_whole_potential.h:50-95, sum_up_whole_potential.cu:548-769).
 * Scalars by value.  Constant arrays come from the session; the changeable
 * ones (l_hartree_max_far_distance, multipole_radius_sq, outer_potential_radius,
 * multipole_moments, the spline table and delta_v_hartree) are uploaded from
 * the host pointers, and delta_v_hartree is downloaded again
 * (sum_up_whole_potential.cu:641-647,768-769).
 * The reference gives this entry point C++ linkage.  The library exports it
 * twice: C++ code that includes this header (or the reference's own
 * sum_up_whole_potential.h) binds the C++-linkage symbol, as the reference's
 * C++ callers do, unmodified; C and Fortran callers bind the same function
 * under C linkage. */
#ifdef __cplusplus
} /* extern "C" */
void sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_(
    const int j_atom_begin, const int j_atom_end, const int n_full_points, const int l_max_analytic_multipole,
    const int index_cc_dim_0, const int n_valid_points, const int l_pot_max, const int n_max_radial,
    const int n_hartree_grid, const int n_centers, const int n_centers_hartree_potential, const int n_atoms,
    const int hartree_force_l_add, const int n_species, const int *n_radial, const int *species,
    const int *species_center, const int *l_hartree_max_far_distance, const int *i_valid_point_2_i_full_points_map,
    const double *coord_points, const double *multipole_radius_sq, const double *outer_potential_radius,
    const double *multipole_moments, const double *current_delta_v_hart_part_spl_tile, const int *l_hartree,
    const int *n_grid, const int *n_cc_lm_ijk, const int *centers_hartree_potential, const int *center_to_atom,
    const int *index_cc, const int *index_ijk_max_cc, const double *cc, const double *coords_center,
    const double *r_grid_min, const double *log_r_grid_inc, const double *scale_radial, const double *partition_tab,
    double *delta_v_hartree);
extern "C" {
#else
void sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_(
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
    double *delta_v_hartree);
#endif

/* Replaces generate_first_order_rho_bias_part2_
 * (generate_first_order_rho_bias_part2.cpp:11-168): the density-matrix part
 * of the rho1 bias for atoms j_atom_begin..j_atom_end along j_coord, written
 * to first_order_rho_bias_part2 (n_max_batch_size, n_batches, 4) -- the
 * reference fixes this array's atom tile at 4 (:4).  Batches without compute
 * functions are left as they were; n_full_points, n_max_compute_ham,
 * batch_sizes and partition_tab are accepted and unused, as in the reference.
 * At most 64 compute functions of one atom per batch. */
void generate_first_order_rho_bias_part2_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches,
    int *i_batch_2_wave_offset, double *wave_batches_compress, double *gradient_wave_batches_compress,
    double *first_order_rho_bias_part2, double *partition_tab, double *density_matrix);

/* Replaces evaluate_first_order_h_reduce_memory_c_v2_
 * (evaluate_first_order_H.h:3-43, CPU implementation evaluate_first_order_H.cpp:13-222):
 * the first-order H integration with every term -- H_prefactor1,
 * v_hartree_gradient, vsigma / gradient_rho / first_order_gradient_rho,
 * v2rho2, v2rhosigma, v2sigma2 (their first components, as the reference reads
 * them) and the Hessian term over each atom's compute functions -- for atoms
 * j_atom_begin..j_atom_end (at most ATOM_TILE_SIZE), ACCUMULATED into
 * first_order_H_tile (n_basis, n_basis, ATOM_TILE_SIZE) as in the reference.
 * Host arrays, same layouts; vrho_batches, H_times_psi_batches_compress,
 * n_max_compute_ham and not_use are accepted and unused, as in the reference.
 * The result does not depend on the order in which batches meet in the
 * output (bit-identical from run to run). */
void evaluate_first_order_h_reduce_memory_c_v2_(
    int *j_atom_begin, int *j_atom_end, int *n_full_points, int *j_coord, int *n_basis, int *n_atoms,
    int *n_max_compute_ham, int *n_max_batch_size, int *n_my_batches_work, int *n_centers_basis_I,
    int *n_point_batches, int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches,
    int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map, double *vrho_batches,
    double *vsigma_batches, double *gradient_rho, double *H_times_psi_batches_compress, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *hessian_wave_batches_compress,
    double *first_order_H_tile, double *H_prefactor1_batches_tile, double *first_order_gradient_rho_batches_tile,
    double *v_hartree_gradient, double *first_order_rho, double *v2rho2_batches, double *v2rhosigma_batches,
    double *v2sigma2_batches, double *partition_tab, int *not_use);

/* The reference's device session.  The reference declares these four with
 * C++ linkage (device.hpp:191-192, device_data.hpp:159-227); as for the sum-up
 * cu_host_ entry point above, C++ code including this header binds the
 * C++-linkage symbols, C and Fortran code the C-linkage ones (both exported).
 *
 * init_dfpt_device_info replaces device.cu:7-33: selects device 0 (or
 * $FRPA_DEVICE) and creates the session stream.  free_dfpt_device_info
 * replaces device.cu:35-38.
 *
 * init_dfpt_device_data replaces device_data.cu:10-361: validates and uploads
 * the constant arrays once, builds the rho1 work list (the reference's
 * valid-batch list and per-tile GEMM metadata, device_data.cu:242-300) and the
 * sum-up plan.  Wave arrays that are already device memory of the session's
 * GPU are used in place (not copied); the caller keeps them alive until
 * free_dfpt_device_data (device_data.cu:363-431). */
#ifdef __cplusplus
} /* extern "C" */
#endif
void init_dfpt_device_info(void);
void free_dfpt_device_info(void);
void init_dfpt_device_data(
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
    double *multipole_moments, double *current_delta_v_hart_part_spl_tile, double *delta_v_hartree);
void free_dfpt_device_data(void);
#ifdef __cplusplus
extern "C" {
#endif

/* Device addresses of the session's resident rho1 outputs (after a
 * *_cu_host_ call), for callers that keep working on the GPU. */
int frpa_session_rho1_device_outputs(double **first_order_rho, double **first_order_gradient_rho);

/* =========================================================================
 * Plans: device pointers, explicit stream (cudaStream_t passed as void *)
 * ======================================================================= */

typedef struct frpa_rho1_plan frpa_rho1_plan;

/* Batch metadata for rho1 (host arrays, reference layouts).  The plan builds
 * the device work list: valid batches (n_compute_c > 0) split into point tiles
 * and ordered by cost for the persistent grouped kernels. */
typedef struct {
  int atom_tile_size; /* T */
  int n_my_batches_work;
  int n_full_points;
  int n_basis;
  int n_centers_basis_I;
  int n_max_batch_size;
  const int *n_point_batches;                   /* (n_batches) */
  const int *n_point_batches_prefix_sum;        /* (n_batches + 1) */
  const int *i_valid_point_2_i_full_points_map; /* (>= prefix[n_batches]) 0-based */
  const int *n_compute_c_batches;               /* (n_batches) */
  const int *i_basis_batches;                   /* (n_centers_basis_I, n_batches) 1-based */
  const int *i_batch_2_wave_offset;             /* (n_batches + 1) */
  long long wave_alloc_len;                     /* elements available in the wave array
                                                   (0: trust i_batch_2_wave_offset) */
} frpa_rho1_desc;

int frpa_rho1_plan_create(frpa_rho1_plan **plan, const frpa_rho1_desc *desc);
int frpa_rho1_plan_destroy(frpa_rho1_plan *plan);
/* Work-list statistics: [n_items, n_valid_batches, n_valid_points]. */
int frpa_rho1_plan_info(const frpa_rho1_plan *plan, long long *info3);
/* Split-int8 mode: [groups, work items, packed P1c tiles, largest A + B scratch
 * of a group in bytes] (no counterpart in the reference).  Each group is three
 * kernel launches (pack phi, pack P1c, contraction). */
int frpa_rho1_plan_i8_info(const frpa_rho1_plan *plan, long long *info4);

/* rho1 and grad rho1 for perturbations t < T; rho1 is written for
 * t < n_active = j_atom_end - j_atom_begin + 1 (evaluate_first_order_rho.cpp:202-207).
 * wave (n elements), gradient_wave (3n), P1 (n_basis, n_basis, T),
 * bias (n_max_batch_size, n_batches, T), gbias (3, n_max_batch_size, n_batches, T);
 * outputs rho (n_full_points, T) and grad (3, n_max_batch_size, n_batches, T). */
int frpa_rho1_execute(const frpa_rho1_plan *plan, int mode, int n_active, const double *wave,
                      const double *gradient_wave, const double *P1, const double *bias, const double *gbias,
                      double *rho, double *grad, void *stream);

/* rho1 and grad rho1 as frpa_rho1_execute in the FP64 mode, with the
 * ground-state density-matrix part of the rho1 bias computed in the same
 * launch (the reference's fused form, task1_atom_tiling/version3_rho_with_bias/
 * evaluate_first_order_rho.cu.hpp:93-254, instead of a separate
 * generate_first_order_rho_bias_part2 pass): for perturbation t (atom
 * j_atom_begin + t, compute range from atom_valid (n_atoms + 1, n_batches))
 *   rho1 += sum_i phi_i sum_{k in range} (D(ib_i, ib_k) + D(ib_k, ib_i)) (-d phi_k / d x_jcoord),
 * added to rho1 only (grad rho1 as frpa_rho1_execute); the bias array is still
 * added as in frpa_rho1_execute.  density_matrix (n_basis, n_basis) and
 * atom_valid are device arrays.  No counterpart name in the reference. */
int frpa_rho1_execute_fused_bias(const frpa_rho1_plan *plan, int n_active, int n_atoms, int j_atom_begin,
                                 int j_coord, const int *atom_valid, const double *density_matrix, const double *wave,
                                 const double *gradient_wave, const double *P1, const double *bias,
                                 const double *gbias, double *rho, double *grad, void *stream);

/* The same bias on the device with a plan's work list: atom_valid
 * ((n_atoms + 1, n_batches), 0-based ranges as in the reference), wave,
 * gradient_wave, density_matrix (n_basis, n_basis) and the output
 * (n_max_batch_size, n_batches, T) are device pointers; atoms
 * j_atom_begin..j_atom_end (at most T of them, 1-based).  Ranges that leave a
 * batch's compute functions (or exceed 64 per atom) are skipped and set bit 3
 * of frpa_rho1_device_flags. */
int frpa_rho1_bias_part2(const frpa_rho1_plan *plan, int T, int n_atoms, int j_atom_begin, int j_atom_end,
                         int j_coord, const int *atom_valid, const double *wave, const double *gradient_wave,
                         const double *density_matrix, double *first_order_rho_bias_part2, void *stream);

/* Tunings of a plan's rho1 launches (no counterpart in the reference, whose
 * MAGMA batching has fixed shapes).  Keys and values:
 *   FRPA_TUNE_FP64_TILE_POINTS  64 (256 threads, up to 2 CTAs per SM) or 128
 *                               (512 threads, 1 CTA per SM: each gathered P1c
 *                               tile serves twice the points);
 *   FRPA_TUNE_FP64_CTAS_PER_SM  0 (as many as fit), 1, 2 or 3;
 *   FRPA_TUNE_SPLIT_TILE_POINTS 16..128 points per split-BF16 work item;
 *   FRPA_TUNE_ORDER             0 largest items first, 1 batch order, 2 (the
 *                               default) batches grouped by a MinHash of their
 *                               basis lists, so batches sharing functions run
 *                               together and their P1 blocks stay in L2;
 *   FRPA_TUNE_SPLIT_I8_SCRATCH_MB  MiB of packed-operand scratch per group of
 *                               batches in the split-int8 mode (default 4096;
 *                               the batches are packed and contracted group by
 *                               group, a batch larger than this is a group of
 *                               its own).
 * Results are unchanged by every setting.  Setting rebuilds and re-uploads the
 * work lists (synchronous: call it outside any stream capture). */
enum {
  FRPA_TUNE_FP64_TILE_POINTS = 1,
  FRPA_TUNE_FP64_CTAS_PER_SM = 2,
  FRPA_TUNE_SPLIT_TILE_POINTS = 3,
  FRPA_TUNE_ORDER = 4,
  FRPA_TUNE_SPLIT_I8_SCRATCH_MB = 5
};
int frpa_rho1_plan_set_tuning(frpa_rho1_plan *plan, int key, int value);
int frpa_rho1_plan_get_tuning(const frpa_rho1_plan *plan, int key, int *value);

/* The first-order H on the device with a plan's work list (the drop-in
 * evaluate_first_order_h_reduce_memory_c_v2_ runs this): perturbation t is
 * atom j_atom_begin + t (1-based), t < n_active <= T.  Device arrays in the
 * reference layouts: atom_valid (n_atoms + 1, n_batches), hessian_wave
 * (6 x the wave length), vsigma (3, nmb, nb), gradient_rho (3, n_full),
 * H_prefactor1 (nmb, nb, T), first_order_gradient_rho (3, nmb, nb, T),
 * v_hartree_gradient and first_order_rho (n_full, T), v2rho2 (3, nmb, nb),
 * v2rhosigma and v2sigma2 (6, nmb, nb), partition_tab (n_full).
 * first_order_H (n_basis, n_basis, T) is accumulated into.  The per-batch
 * contributions are added as 128-bit fixed-point integers, so the result is
 * the same bits on every run whatever the order of the additions.  The
 * accumulator ((n_basis, n_basis, T) x 16 bytes, shared with the adjoint) is
 * allocated by the plan's first such call: make it before any stream capture.
 * Device flags (frpa_rho1_device_flags): bit 3 an atom's compute range
 * leaves its batch (clipped), bit 4 a non-finite input (result incomplete). */
int frpa_rho1_first_order_h(const frpa_rho1_plan *plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                            const int *atom_valid, const double *wave, const double *gradient_wave,
                            const double *hessian_wave, const double *vsigma, const double *gradient_rho,
                            const double *H_prefactor1, const double *first_order_gradient_rho,
                            const double *v_hartree_gradient, const double *first_order_rho, const double *v2rho2,
                            const double *v2rhosigma, const double *v2sigma2, const double *partition_tab,
                            double *first_order_H, void *stream);

/* Adjoint: dP1 (n_basis, n_basis, T) += d(sum g_rho . rho1 + sum g_grad . grad)/dP1.
 * g_rho (n_full_points, T) or NULL, g_grad like grad or NULL.  dP1 is NOT zeroed.
 * Same engine and accumulation as frpa_rho1_first_order_h: deterministic
 * (bit-identical from run to run); the first call allocates the accumulator. */
int frpa_rho1_adjoint_p1(const frpa_rho1_plan *plan, int n_active, const double *wave, const double *gradient_wave,
                         const double *g_rho, const double *g_grad, double *dP1, void *stream);

/* Reads and clears the device-side status of the plan's kernels: bit 1 = a
 * pipeline wait of a tensor-core kernel timed out (the kernel gave up and left
 * its outputs incomplete), bit 2 = its final drain timed out, bit 3 = an
 * atom's compute range (atom_valid) left its batch and was clipped (bias and
 * first-order H), bit 4 = a non-finite input reached the first-order H or
 * adjoint accumulation.  0 after a good run. */
int frpa_rho1_device_flags(const frpa_rho1_plan *plan, int *flags);

typedef struct frpa_sumup_plan frpa_sumup_plan;

/* Constant sum-up inputs (host arrays, reference layouts and meanings). */
typedef struct {
  int atom_tile_size;
  int n_full_points, l_max_analytic_multipole, index_cc_dim_0, n_valid_points;
  int l_pot_max, n_hartree_grid, n_centers, n_centers_hartree_potential, n_atoms, hartree_force_l_add, n_species;
  const int *species, *species_center, *i_valid_point_2_i_full_points_map;
  const double *coord_points;
  const int *l_hartree, *n_grid, *n_cc_lm_ijk, *centers_hartree_potential, *center_to_atom, *index_cc,
      *index_ijk_max_cc;
  const double *cc, *coords_center, *r_grid_min, *log_r_grid_inc;
} frpa_sumup_desc;

int frpa_sumup_plan_create(frpa_sumup_plan **plan, const frpa_sumup_desc *desc);
int frpa_sumup_plan_destroy(frpa_sumup_plan *plan);
/* 1 if the Kelvin-polynomial far-field path applies (identity
 * centers_hartree_potential and a homogeneous multipole table). */
int frpa_sumup_plan_fast(const frpa_sumup_plan *plan);

/* Accumulates into delta_v (n_full_points, T) for t < n_active.  Per-call
 * inputs: l_hartree_max_far_distance (n_atoms, T), multipole_radius_sq
 * (n_atoms, T), outer_potential_radius (l_pot_max+1, n_atoms, T),
 * multipole_moments ((l_pot_max+1)^2, n_atoms, T), spline
 * ((l_pot_max+1)^2, 2, n_hartree_grid, n_atoms, T).  branch_codes (optional,
 * (n_valid, n_centers_hartree_potential, T) bytes): 0 skipped, 1 + l_atom_max
 * near field, 16 + l_atom_max far field.  flags: bit 0 forces the generic
 * (reference table loop) kernel. */
int frpa_sumup_execute(const frpa_sumup_plan *plan, int n_active, int flags, const int *l_hartree_max_far_distance,
                       const double *multipole_radius_sq, const double *outer_potential_radius,
                       const double *multipole_moments, const double *spline, double *delta_v,
                       unsigned char *branch_codes, void *stream);

/* Adjoint of the sum-up with respect to the multipole moments:
 * dQ ((l_pot_max+1)^2, n_atoms, T) = d(sum_p g(p, t) delta_v(p, t))/dQ, zeroed
 * first.  Implemented for the fast path (frpa_sumup_plan_fast); a plan on the
 * generic kernel returns FRPA_ERR_UNSUPPORTED.  Partial sums are reduced in a
 * fixed order: the same bits on every run. */
int frpa_sumup_adjoint_q(const frpa_sumup_plan *plan, int n_active, const int *l_hartree_max_far_distance,
                         const double *multipole_radius_sq, const double *outer_potential_radius,
                         const double *multipole_moments, const double *g, double *dQ, void *stream);

/* The sum-up without any device allocation, for callers that cannot let a
 * library call cudaMalloc or cudaFree: host codes that give the GPU a fixed
 * memory budget run by their own pool, or that keep several streams busy and
 * cannot take cudaFree's device-wide synchronisation.  No counterpart in the
 * reference.  Arguments as sum_up_..._cu_host_ with ALL arrays as device
 * pointers, the tile size explicit and a stream; accumulates into
 * delta_v_hartree with the reference-mirroring kernel.  Its scratch is one
 * 8 MiB array inside the library per GPU, held until the process exits, which
 * limits 256 + 4 index_cc_dim_0 (rounded to 256) + 8 index_cc_dim_0 n_atoms T
 * bytes to 8 MiB; larger inputs are rejected with FRPA_ERR_INVALID.  Calls
 * share that array, so calls that overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller.  The first call on a
 * device looks the array up (and loads the library's constants); make it
 * before any stream capture.  Device arrays are not range-checked: pass data
 * that frpa_sumup_plan_create would accept. */
int frpa_sumup_execute_noalloc(
    int atom_tile_size, int j_atom_begin, int j_atom_end, int n_full_points, int l_max_analytic_multipole,
    int index_cc_dim_0, int n_valid_points, int l_pot_max, int n_hartree_grid, int n_centers,
    int n_centers_hartree_potential, int n_atoms, int hartree_force_l_add, int n_species, const int *species,
    const int *species_center, const int *l_hartree_max_far_distance, const int *i_valid_point_2_i_full_points_map,
    const double *coord_points, const double *multipole_radius_sq, const double *outer_potential_radius,
    const double *multipole_moments, const double *spline, const int *l_hartree, const int *n_grid,
    const int *n_cc_lm_ijk, const int *centers_hartree_potential, const int *center_to_atom, const int *index_cc,
    const int *index_ijk_max_cc, const double *cc, const double *coords_center, const double *r_grid_min,
    const double *log_r_grid_inc, double *delta_v_hartree, void *stream);

/* Reads and clears the device-side input flags of the last executions
 * (bit 0: an l_hartree_max_far_distance entry outside 0..l_pot_max, clamped). */
int frpa_sumup_device_flags(const frpa_sumup_plan *plan, int *flags);

/* The same input flags for frpa_sumup_execute_noalloc on the current device:
 * every call of that entry point ORs into one flag word inside the library
 * (bit 0: an l_hartree_max_far_distance entry outside 0..l_pot_max was
 * clamped); this reads it after the work queued on `stream`, clears it and
 * waits for the stream.  Allocates nothing.  No counterpart in the reference. */
int frpa_sumup_noalloc_flags(int *flags, void *stream);

/* =========================================================================
 * Synthetic workload generator (benchmarks and tests)
 * ======================================================================= */

/* Fills wave / gradient_wave (device) with Gaussian basis functions
 * phi = R_lm(r - R_A) exp(-alpha |r - R_A|^2) at the batches' points.
 * points: device (3, n_valid) in valid-point order; basis_atom (0-based),
 * basis_l, basis_m, basis_alpha: host (n_basis); atoms: host (3, n_atoms).
 * Rows n_compute..n_compute_padding-1 are set to pad_value. */
int frpa_synth_basis_values(const frpa_rho1_desc *desc, const double *points, int n_atoms, const double *atoms,
                            const int *basis_atom, const int *basis_l, const int *basis_m, const double *basis_alpha,
                            double pad_value, double *wave, double *gradient_wave, void *stream);

/* Synthetic workloads: a window of a symmetric first-order density matrix
 * out (n, n, T) (device) whose entry (i, j, t) is scale x a standard-normal
 * draw keyed by (seed, t, the pair of global basis indices global_index[i],
 * global_index[j]) -- the same global P1 whichever window it is evaluated in,
 * for sweeps whose full P1 would not fit (global_index: device, n entries). */
int frpa_synth_p1_window(const int *global_index, int n, int T, double scale, unsigned long long seed, double *out,
                         void *stream);

/* Measured FP64 tensor-pipe throughput of the current device (independent
 * m8n8k4 f64 MMAs on every SM), the ceiling the plain FP64 rho1 contraction
 * is compared against.  Takes a few tens of milliseconds. */
int frpa_probe_fp64_mma_tflops(double *tflops, void *stream);
/* Same for the FP64 FMA pipe (independent DFMA chains), the ceiling of the
 * sum-up kernels. */
int frpa_probe_fp64_fma_tflops(double *tflops, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FRPA_H */
