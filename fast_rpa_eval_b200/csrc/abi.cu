// The C ABI: error state, settings, rho1 / sum-up plans, the reference
// drop-in entry points and the reference's device session.
//
// Everything a kernel indexes is validated here on the host first (batch
// sizes, basis indices, point maps, wave offsets, table ranges), so that
// device accesses stay in bounds for any input that passes; failures come
// back as status codes and messages instead of the reference's exit(1)
// (fast_rap_src_dfpt_gpu_eval/device.hpp:21-29).
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <numeric>
#include <vector>

#include "frpa_internal.cuh"

namespace frpa {

// ----------------------------------------------------------------- errors

namespace {
thread_local int t_status = FRPA_OK;
thread_local char t_msg[1024] = "";
std::atomic<int> g_tile{1};
std::atomic<int> g_rho1_mode{FRPA_RHO1_FP64};
}  // namespace

int fail(int status, const char *fmt, ...) {
  t_status = status;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
  va_end(ap);
  if (getenv("FRPA_VERBOSE")) fprintf(stderr, "[frpa] error %d: %s\n", status, t_msg);
  return status;
}

void clear_error() {
  t_status = FRPA_OK;
  t_msg[0] = 0;
}

// Declarations of the launchers implemented in the other translation units.
struct SumupPlan;
int sumup_plan_create(SumupPlan **out, const frpa_sumup_desc *D);
void sumup_plan_free(SumupPlan *P);
int sumup_plan_is_fast(const SumupPlan *P);
int sumup_execute(const SumupPlan *P, int n_active, int force_generic, const int *lhmfd, const double *mrs,
                  const double *opr, const double *Q, const double *spline, double *dv, unsigned char *codes,
                  cudaStream_t stream);
int sumup_adjoint_q(const SumupPlan *P, int n_active, const int *lhmfd, const double *mrs, const double *opr,
                    const double *Q, const double *g, double *dQ, cudaStream_t stream);
int sumup_read_error_flags(const SumupPlan *P, int *flags);
int synth_basis_values(const frpa_rho1_desc *D, const double *points, int n_atoms, const double *atoms,
                       const int *basis_atom, const int *basis_l, const int *basis_m, const double *basis_alpha,
                       double pad, double *wave, double *gwave, cudaStream_t stream);

// ------------------------------------------------------------- rho1 plan

static void rho1_plan_free(Rho1Plan *P) {
  if (!P) return;
  cudaFree(P->d_items);
  cudaFree(P->d_ib);
  cudaFree(P->d_map);
  cudaFree(P->d_counter);
  cudaFree(P->d_adj_items);
  cudaFree(P->d_h1_items_sym);
  cudaFree(P->d_h1_acc);
  cudaFree(P->d_items_split);
  cudaFree(P->d_rowmax);
  cudaFree(P->d_err);
  rho1_i8_free(P);
  delete P;
}

static int rho1_plan_build(Rho1Plan **out, const frpa_rho1_desc *D) {
  *out = nullptr;
  FRPA_CHECK_ARG(D != nullptr, "rho1: null descriptor");
  const int T = D->atom_tile_size, nb = D->n_my_batches_work;
  FRPA_CHECK_ARG(T >= 1 && T <= FRPA_MAX_ATOM_TILE, "rho1: atom tile size %d out of range 1..%d", T,
                 FRPA_MAX_ATOM_TILE);
  FRPA_CHECK_ARG(nb >= 0 && D->n_full_points >= 0 && D->n_basis >= 1 && D->n_centers_basis_I >= 0 &&
                     D->n_max_batch_size >= 0,
                 "rho1: negative size (n_batches %d, n_full_points %d, n_basis %d)", nb, D->n_full_points,
                 D->n_basis);
  FRPA_CHECK_ARG(nb == 0 || (D->n_point_batches && D->n_point_batches_prefix_sum && D->n_compute_c_batches &&
                             D->i_basis_batches && D->i_batch_2_wave_offset),
                 "rho1: null array argument");
  const long long wave_len = D->wave_alloc_len > 0 ? D->wave_alloc_len : (nb > 0 ? D->i_batch_2_wave_offset[nb] : 0);
  std::vector<Rho1WorkItem> items, batches;
  std::vector<int> ibc;
  std::vector<int> ib_off(nb, 0);
  long long map_len = 0, n_valid_pts = 0;
  int n_valid_b = 0, nc_max = 0, aligned = 1;
  for (int b = 0; b < nb; ++b) {
    const int np = D->n_point_batches[b], nc = D->n_compute_c_batches[b];
    const int pre = D->n_point_batches_prefix_sum[b];
    FRPA_CHECK_ARG(np >= 0 && np <= D->n_max_batch_size, "rho1: batch %d has %d points (n_max_batch_size %d)", b,
                   np, D->n_max_batch_size);
    FRPA_CHECK_ARG(pre >= 0 && (long long)pre + np <= D->n_full_points,
                   "rho1: batch %d point range [%d, %d) outside the %d-entry point map", b, pre, pre + np,
                   D->n_full_points);
    if (nc <= 0) continue;  // the reference skips these (evaluate_first_order_rho.cpp:126)
    FRPA_CHECK_ARG(nc <= D->n_centers_basis_I, "rho1: batch %d n_compute_c %d > n_centers_basis_I %d", b, nc,
                   D->n_centers_basis_I);
    FRPA_CHECK_ARG(nc <= FRPA_MAX_N_COMPUTE, "rho1: batch %d n_compute_c %d > supported %d", b, nc,
                   FRPA_MAX_N_COMPUTE);
    const long long off = D->i_batch_2_wave_offset[b];
    const long long ncp = (nc + 3) / 4 * 4;
    FRPA_CHECK_ARG(off >= 0 && off + ncp * np <= wave_len, "rho1: batch %d wave block [%lld, %lld) outside %lld", b,
                   off, off + ncp * np, wave_len);
    if (off & 1) aligned = 0;
    const int *col = D->i_basis_batches + (long long)D->n_centers_basis_I * b;
    ib_off[b] = (int)ibc.size();
    for (int i = 0; i < nc; ++i) {
      FRPA_CHECK_ARG(col[i] >= 1 && col[i] <= D->n_basis, "rho1: batch %d basis index %d = %d outside 1..%d", b, i,
                     col[i], D->n_basis);
      ibc.push_back(col[i]);
    }
    map_len = std::max(map_len, (long long)pre + np);
    nc_max = std::max(nc_max, nc);
    ++n_valid_b;
    n_valid_pts += np;
    batches.push_back(Rho1WorkItem{b, nc, np, 0, np, ib_off[b], pre, rho1_locality_key(col, nc), off});
  }
  for (long long i = 0; i < map_len; ++i)
    FRPA_CHECK_ARG(D->i_valid_point_2_i_full_points_map[i] >= 0 &&
                       D->i_valid_point_2_i_full_points_map[i] < D->n_full_points,
                   "rho1: i_valid_point_2_i_full_points_map[%lld] = %d outside 0..%d", i,
                   D->i_valid_point_2_i_full_points_map[i], D->n_full_points - 1);
  // locality order (batches sharing basis functions together, largest first
  // within a key): the persistent kernel takes items in this order
  std::vector<int> chunk_items, chunk_batches;
  rho1_fp64_build_items(batches, 64, 2, nb, &items, &chunk_items, &chunk_batches);

  Rho1Plan *P = new Rho1Plan();
  FRPA_CUDA_TRY(cudaGetDevice(&P->device));
  P->T = T;
  P->n_batches = nb;
  P->n_full_points = D->n_full_points;
  P->n_basis = D->n_basis;
  P->n_max_batch_size = D->n_max_batch_size;
  P->n_max_compute = nc_max;
  P->wave_len = wave_len;
  P->n_items = (int)items.size();
  P->n_valid_batches = n_valid_b;
  P->n_valid_points = n_valid_pts;
  P->wave_aligned16 = aligned;
  P->fp64_chunk_items = chunk_items;
  P->fp64_chunk_batches = chunk_batches;
  int st = FRPA_OK;
  auto up = [&](void **dst, const void *src, size_t bytes) {
    if (st != FRPA_OK) return;
    if (cudaMalloc(dst, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      st = fail(FRPA_ERR_OOM, "rho1: plan allocation of %zu bytes failed", bytes);
      return;
    }
    if (bytes && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      st = fail(FRPA_ERR_CUDA, "rho1: plan upload failed");
  };
  up((void **)&P->d_items, items.data(), sizeof(Rho1WorkItem) * items.size());
  P->h_batches = batches;
  P->h_ib = ibc;
  {
    std::vector<Rho1WorkItem> split;
    rho1_split_build_items(batches, P->split_tile_points, P->order, &split);
    P->n_items_split = (int)split.size();
    up((void **)&P->d_items_split, split.data(), sizeof(Rho1WorkItem) * split.size());
    std::vector<double> zeros((size_t)D->n_basis * T, 0.0);
    up((void **)&P->d_rowmax, zeros.data(), sizeof(double) * zeros.size());
    const int z = 0;
    up((void **)&P->d_err, &z, sizeof(int));
  }
  if (st == FRPA_OK) st = rho1_i8_build(P);
  up((void **)&P->d_ib, ibc.data(), sizeof(int) * ibc.size());
  up((void **)&P->d_map, D->i_valid_point_2_i_full_points_map, sizeof(int) * (size_t)map_len);
  const int zero = 0;
  up((void **)&P->d_counter, &zero, sizeof(int));
  {
    std::vector<int> ncb(nb), npb(nb), preb(nb);
    std::vector<long long> offb(nb);
    for (int b = 0; b < nb; ++b) {
      ncb[b] = D->n_compute_c_batches[b];
      npb[b] = D->n_point_batches[b];
      preb[b] = D->n_point_batches_prefix_sum[b];
      offb[b] = D->i_batch_2_wave_offset[b];
    }
    std::vector<unsigned char> adj, sym;
    rho1_h1_build_items(ncb.data(), npb.data(), ib_off.data(), preb.data(), offb.data(), nb, T, false, &adj);
    P->n_adj_items = (int)(adj.size() / rho1_h1_item_size());
    up(&P->d_adj_items, adj.data(), adj.size());
    rho1_h1_build_items(ncb.data(), npb.data(), ib_off.data(), preb.data(), offb.data(), nb, T, true, &sym);
    P->n_h1_items_sym = (int)(sym.size() / rho1_h1_item_size());
    up(&P->d_h1_items_sym, sym.data(), sym.size());
  }
  if (st == FRPA_OK) {
    P->grid_fp64 = rho1_fp64_grid(P->device);
    if (P->grid_fp64 <= 0) st = fail(FRPA_ERR_CUDA, "rho1: kernel attribute / occupancy query failed");
  }
  if (st != FRPA_OK) {
    rho1_plan_free(P);
    return st;
  }
  *out = P;
  return FRPA_OK;
}

static int rho1_run(Rho1Plan &P, int mode, int n_active, const double *wave, const double *gwave,
                    const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                    cudaStream_t stream) {
  FRPA_CHECK_ARG(P1 && bias && gbias && rho && grad, "rho1: null device pointer");
  FRPA_CHECK_ARG(P.n_items == 0 || (wave && gwave), "rho1: null wave pointer");
  if (n_active > P.T) return fail(FRPA_ERR_INVALID, "rho1: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d",
                                  n_active, P.T);
  if (mode == FRPA_RHO1_FP64) return rho1_fp64_launch(P, n_active, wave, gwave, P1, bias, gbias, rho, grad, stream);
  if (mode == FRPA_RHO1_SPLIT_BF16) return rho1_split_launch(P, n_active, wave, gwave, P1, bias, gbias, rho, grad, stream);
  if (mode == FRPA_RHO1_SPLIT_I8) return rho1_i8_launch(P, n_active, wave, gwave, P1, bias, gbias, rho, grad, stream);
  return fail(FRPA_ERR_INVALID, "rho1: unknown mode %d", mode);
}

// --------------------------------------------------- device buffer cache

namespace {
// Grow-only device buffers for the stateless drop-ins (one set per slot).
struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  int dev = -1;
};
std::mutex g_buf_mu;
DevBuf g_bufs[48];

int ensure(int slot, size_t bytes, void **out) {
  int dev = 0;
  FRPA_CUDA_TRY(cudaGetDevice(&dev));
  DevBuf &b = g_bufs[slot];
  if (b.p && (b.n < bytes || b.dev != dev)) {
    int cur = dev;
    cudaSetDevice(b.dev);
    cudaFree(b.p);
    cudaSetDevice(cur);
    b.p = nullptr;
    b.n = 0;
  }
  if (!b.p) {
    if (cudaMalloc(&b.p, std::max<size_t>(bytes, 256)) != cudaSuccess)
      return fail(FRPA_ERR_OOM, "device allocation of %zu bytes failed", bytes);
    b.n = std::max<size_t>(bytes, 256);
    b.dev = dev;
  }
  *out = b.p;
  return FRPA_OK;
}

template <class T>
int h2d(int slot, const T *src, size_t count, T **dst, cudaStream_t s) {
  void *p = nullptr;
  FRPA_TRY(ensure(slot, sizeof(T) * count, &p));
  if (count) FRPA_CUDA_TRY(cudaMemcpyAsync(p, src, sizeof(T) * count, cudaMemcpyHostToDevice, s));
  *dst = static_cast<T *>(p);
  return FRPA_OK;
}

// ----------------------------------------------------------- the session

struct Session {
  bool info = false;
  bool data = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  // the FP64 host-buffer entry copies the biases in and grad rho1 out chunk by
  // chunk on these streams while the kernel works on the other chunks
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_p1 = nullptr, ev_in[FP64_CHUNKS] = {}, ev_done[FP64_CHUNKS] = {};
  int T = 1;
  // rho1
  Rho1Plan *rho = nullptr;
  int n_batches = 0, n_full_points = 0, n_basis = 0, n_max_batch_size = 0;
  double *wave = nullptr, *gwave = nullptr;
  bool borrowed_wave = false;  // wave arrays were already device memory
  double *P1 = nullptr, *bias = nullptr, *gbias = nullptr, *out_rho = nullptr, *out_grad = nullptr;
  // sum-up
  SumupPlan *sumup = nullptr;
  int su_n_atoms = 0, su_L = 0, su_grid = 0, su_full = 0;
  int *lhmfd = nullptr;
  double *mrs = nullptr, *opr = nullptr, *Q = nullptr, *spline = nullptr, *dv = nullptr;
};
std::mutex g_session_mu;
Session g_session;

void session_free_data(Session &S) {
  if (S.rho) rho1_plan_free(S.rho);
  if (S.sumup) sumup_plan_free(S.sumup);
  if (S.borrowed_wave) S.wave = S.gwave = nullptr;
  S.borrowed_wave = false;
  void *ptrs[] = {S.wave, S.gwave, S.P1, S.bias, S.gbias, S.out_rho, S.out_grad, S.lhmfd, S.mrs, S.opr, S.Q, S.spline, S.dv};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  S.rho = nullptr;
  S.sumup = nullptr;
  S.wave = S.gwave = S.P1 = S.bias = S.gbias = S.out_rho = S.out_grad = nullptr;
  S.lhmfd = nullptr;
  S.mrs = S.opr = S.Q = S.spline = S.dv = nullptr;
  S.data = false;
}

void session_free_streams(Session &S) {
  for (cudaStream_t *st : {&S.stream, &S.copy_in, &S.copy_out}) {
    if (*st) cudaStreamDestroy(*st);
    *st = nullptr;
  }
  if (S.ev_p1) cudaEventDestroy(S.ev_p1);
  S.ev_p1 = nullptr;
  for (int c = 0; c < FP64_CHUNKS; ++c) {
    if (S.ev_in[c]) cudaEventDestroy(S.ev_in[c]);
    if (S.ev_done[c]) cudaEventDestroy(S.ev_done[c]);
    S.ev_in[c] = S.ev_done[c] = nullptr;
  }
}

frpa_rho1_desc rho_desc_from_ref(int T, int *n_my_batches_work, int *n_full_points, int *n_basis,
                                 int *n_centers_basis_I, int *n_max_batch_size, int *n_point_batches,
                                 int *n_point_batches_prefix_sum, int *map, int *n_compute_c_batches,
                                 int *i_basis_batches, int *i_batch_2_wave_offset) {
  frpa_rho1_desc d;
  d.atom_tile_size = T;
  d.n_my_batches_work = *n_my_batches_work;
  d.n_full_points = *n_full_points;
  d.n_basis = *n_basis;
  d.n_centers_basis_I = *n_centers_basis_I;
  d.n_max_batch_size = *n_max_batch_size;
  d.n_point_batches = n_point_batches;
  d.n_point_batches_prefix_sum = n_point_batches_prefix_sum;
  d.i_valid_point_2_i_full_points_map = map;
  d.n_compute_c_batches = n_compute_c_batches;
  d.i_basis_batches = i_basis_batches;
  d.i_batch_2_wave_offset = i_batch_2_wave_offset;
  d.wave_alloc_len = 0;
  return d;
}

frpa_sumup_desc sumup_desc_from_ref(int T, int n_full_points, int l_max_analytic_multipole, int index_cc_dim_0,
                                    int n_valid_points, int l_pot_max, int n_hartree_grid, int n_centers,
                                    int n_centers_hartree_potential, int n_atoms, int hartree_force_l_add,
                                    int n_species, const int *species, const int *species_center, const int *map,
                                    const double *coord_points, const int *l_hartree, const int *n_grid,
                                    const int *n_cc_lm_ijk, const int *chp, const int *c2a, const int *index_cc,
                                    const int *ijkmax, const double *cc, const double *coords_center,
                                    const double *rgm, const double *linc) {
  frpa_sumup_desc d;
  d.atom_tile_size = T;
  d.n_full_points = n_full_points;
  d.l_max_analytic_multipole = l_max_analytic_multipole;
  d.index_cc_dim_0 = index_cc_dim_0;
  d.n_valid_points = n_valid_points;
  d.l_pot_max = l_pot_max;
  d.n_hartree_grid = n_hartree_grid;
  d.n_centers = n_centers;
  d.n_centers_hartree_potential = n_centers_hartree_potential;
  d.n_atoms = n_atoms;
  d.hartree_force_l_add = hartree_force_l_add;
  d.n_species = n_species;
  d.species = species;
  d.species_center = species_center;
  d.i_valid_point_2_i_full_points_map = map;
  d.coord_points = coord_points;
  d.l_hartree = l_hartree;
  d.n_grid = n_grid;
  d.n_cc_lm_ijk = n_cc_lm_ijk;
  d.centers_hartree_potential = chp;
  d.center_to_atom = c2a;
  d.index_cc = index_cc;
  d.index_ijk_max_cc = ijkmax;
  d.cc = cc;
  d.coords_center = coords_center;
  d.r_grid_min = rgm;
  d.log_r_grid_inc = linc;
  return d;
}

// Host-side range check of l_hartree_max_far_distance (the per-call array
// whose values index the multipole table).
int check_lhmfd(const int *lhmfd, int n_atoms, int T, int L) {
  for (long long i = 0; i < (long long)n_atoms * T; ++i)
    FRPA_CHECK_ARG(lhmfd[i] >= 0 && lhmfd[i] <= L, "sumup: l_hartree_max_far_distance[%lld] = %d outside 0..%d", i,
                   lhmfd[i], L);
  return FRPA_OK;
}

}  // namespace
}  // namespace frpa

// ---------------------------------------------------- public C functions

using namespace frpa;

extern "C" {

int frpa_last_error(void) { return t_status; }
const char *frpa_last_error_message(void) { return t_msg; }
void frpa_clear_error(void) { clear_error(); }
int frpa_version(void) { return 10000; }

int frpa_set_device(int device) {
  int count = 0;
  FRPA_CUDA_TRY(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(FRPA_ERR_INVALID, "device %d outside 0..%d", device, count - 1);
  FRPA_CUDA_TRY(cudaSetDevice(device));
  return FRPA_OK;
}
int frpa_get_device(int *device) {
  if (!device) return fail(FRPA_ERR_INVALID, "frpa_get_device: null argument");
  FRPA_CUDA_TRY(cudaGetDevice(device));
  return FRPA_OK;
}
int frpa_set_atom_tile_size(int T) {
  if (T < 1 || T > FRPA_MAX_ATOM_TILE) return fail(FRPA_ERR_INVALID, "atom tile size %d out of range", T);
  g_tile = T;
  return FRPA_OK;
}
int frpa_get_atom_tile_size(void) { return g_tile; }
int frpa_set_rho1_mode(int mode) {
  if (mode != FRPA_RHO1_FP64 && mode != FRPA_RHO1_SPLIT_BF16 && mode != FRPA_RHO1_SPLIT_I8)
    return fail(FRPA_ERR_INVALID, "rho1 mode %d", mode);
  g_rho1_mode = mode;
  return FRPA_OK;
}
int frpa_get_rho1_mode(void) { return g_rho1_mode; }

struct frpa_rho1_plan {
  Rho1Plan *p;
};
struct frpa_sumup_plan {
  SumupPlan *p;
};

int frpa_rho1_plan_create(frpa_rho1_plan **plan, const frpa_rho1_desc *desc) {
  if (!plan) return fail(FRPA_ERR_INVALID, "rho1: null plan pointer");
  *plan = nullptr;
  Rho1Plan *p = nullptr;
  FRPA_TRY(rho1_plan_build(&p, desc));
  *plan = new frpa_rho1_plan{p};
  return FRPA_OK;
}

int frpa_rho1_plan_destroy(frpa_rho1_plan *plan) {
  if (plan) {
    rho1_plan_free(plan->p);
    delete plan;
  }
  return FRPA_OK;
}

int frpa_rho1_plan_info(const frpa_rho1_plan *plan, long long *info3) {
  if (!plan || !info3) return fail(FRPA_ERR_INVALID, "rho1: null argument");
  info3[0] = plan->p->n_items;
  info3[1] = plan->p->n_valid_batches;
  info3[2] = plan->p->n_valid_points;
  return FRPA_OK;
}

int frpa_rho1_plan_i8_info(const frpa_rho1_plan *plan, long long *info4) {
  if (!plan || !info4) return fail(FRPA_ERR_INVALID, "rho1: null argument");
  const Rho1Plan &P = *plan->p;
  long long items = 0, tiles = 0, scratch = 0;
  for (const I8Group &g : P.i8_groups) {
    items += g.item1 - g.item0;
    tiles += g.tile1 - g.tile0;
    scratch = std::max(scratch, g.a_bytes + g.b_bytes);
  }
  info4[0] = (long long)P.i8_groups.size();
  info4[1] = items;
  info4[2] = tiles;
  info4[3] = scratch;
  return FRPA_OK;
}

int frpa_rho1_execute(const frpa_rho1_plan *plan, int mode, int n_active, const double *wave,
                      const double *gradient_wave, const double *P1, const double *bias, const double *gbias,
                      double *rho, double *grad, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "rho1: null plan");
  return rho1_run(*plan->p, mode, n_active, wave, gradient_wave, P1, bias, gbias, rho, grad, (cudaStream_t)stream);
}

int frpa_rho1_execute_fused_bias(const frpa_rho1_plan *plan, int n_active, int n_atoms, int j_atom_begin,
                                 int j_coord, const int *atom_valid, const double *density_matrix, const double *wave,
                                 const double *gradient_wave, const double *P1, const double *bias,
                                 const double *gbias, double *rho, double *grad, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "rho1: null plan");
  Rho1Plan &P = *plan->p;
  FRPA_CHECK_ARG(P1 && bias && gbias && rho && grad && atom_valid && density_matrix, "rho1 fused bias: null pointer");
  FRPA_CHECK_ARG(P.n_items == 0 || (wave && gradient_wave), "rho1 fused bias: null wave pointer");
  FRPA_CHECK_ARG(n_active >= 0 && n_active <= P.T, "rho1 fused bias: n_active %d outside 0..%d", n_active, P.T);
  FRPA_CHECK_ARG(j_coord >= 1 && j_coord <= 3, "rho1 fused bias: j_coord %d outside 1..3", j_coord);
  FRPA_CHECK_ARG(n_active == 0 || (j_atom_begin >= 1 && j_atom_begin + n_active - 1 <= n_atoms),
                 "rho1 fused bias: atoms %d..%d outside 1..%d", j_atom_begin, j_atom_begin + n_active - 1, n_atoms);
  return rho1_fp64_fused_bias_launch(P, n_active, n_atoms, j_atom_begin, j_coord, atom_valid, density_matrix, wave,
                                     gradient_wave, P1, bias, gbias, rho, grad, (cudaStream_t)stream);
}

int frpa_rho1_device_flags(const frpa_rho1_plan *plan, int *flags) {
  if (!plan || !flags) return fail(FRPA_ERR_INVALID, "rho1: null argument");
  FRPA_CUDA_TRY(cudaMemcpy(flags, plan->p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  FRPA_CUDA_TRY(cudaMemset(plan->p->d_err, 0, sizeof(int)));
  return FRPA_OK;
}

// Re-uploads a work list (synchronous; not inside a stream capture).
static int replace_items(Rho1WorkItem **dst, int *count, const std::vector<Rho1WorkItem> &items) {
  Rho1WorkItem *d = nullptr;
  FRPA_CUDA_TRY(cudaMalloc(&d, sizeof(Rho1WorkItem) * std::max<size_t>(items.size(), 1)));
  if (!items.empty() &&
      cudaMemcpy(d, items.data(), sizeof(Rho1WorkItem) * items.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return fail(FRPA_ERR_CUDA, "rho1: work-list upload failed");
  }
  cudaFree(*dst);
  *dst = d;
  *count = (int)items.size();
  return FRPA_OK;
}

int frpa_rho1_plan_set_tuning(frpa_rho1_plan *plan, int key, int value) {
  if (!plan) return fail(FRPA_ERR_INVALID, "rho1: null plan");
  Rho1Plan &P = *plan->p;
  switch (key) {
    case FRPA_TUNE_FP64_TILE_POINTS:
      FRPA_CHECK_ARG(value == 64 || value == 128, "rho1 tuning: FP64 tile points %d not 64 or 128", value);
      P.fp64_tile_points = value;
      break;
    case FRPA_TUNE_FP64_CTAS_PER_SM:
      FRPA_CHECK_ARG(value >= 0 && value <= 3, "rho1 tuning: CTAs per SM %d not 0..3", value);
      P.fp64_ctas_per_sm = value;
      return FRPA_OK;
    case FRPA_TUNE_SPLIT_TILE_POINTS:
      FRPA_CHECK_ARG(value >= 16 && value <= 128, "rho1 tuning: split tile points %d not 16..128", value);
      P.split_tile_points = value;
      break;
    case FRPA_TUNE_ORDER:
      FRPA_CHECK_ARG(value >= 0 && value <= 2, "rho1 tuning: order %d not 0, 1 or 2", value);
      P.order = value;
      break;
    case FRPA_TUNE_SPLIT_I8_SCRATCH_MB:
      FRPA_CHECK_ARG(value >= 1, "rho1 tuning: split-int8 scratch %d MiB not >= 1", value);
      P.i8_budget = (long long)value << 20;
      rho1_i8_free(&P);  // groups change: new lists, scratch reallocated by the next execution
      return rho1_i8_build(&P);
    default:
      return fail(FRPA_ERR_INVALID, "rho1 tuning: unknown key %d", key);
  }
  std::vector<Rho1WorkItem> items, split;
  rho1_fp64_build_items(P.h_batches, P.fp64_tile_points, P.order, P.n_batches, &items, &P.fp64_chunk_items,
                        &P.fp64_chunk_batches);
  rho1_split_build_items(P.h_batches, P.split_tile_points, P.order, &split);
  FRPA_TRY(replace_items(&P.d_items, &P.n_items, items));
  FRPA_TRY(replace_items(&P.d_items_split, &P.n_items_split, split));
  return FRPA_OK;
}

int frpa_rho1_plan_get_tuning(const frpa_rho1_plan *plan, int key, int *value) {
  if (!plan || !value) return fail(FRPA_ERR_INVALID, "rho1: null argument");
  const Rho1Plan &P = *plan->p;
  switch (key) {
    case FRPA_TUNE_FP64_TILE_POINTS: *value = P.fp64_tile_points; return FRPA_OK;
    case FRPA_TUNE_FP64_CTAS_PER_SM: *value = P.fp64_ctas_per_sm; return FRPA_OK;
    case FRPA_TUNE_SPLIT_TILE_POINTS: *value = P.split_tile_points; return FRPA_OK;
    case FRPA_TUNE_ORDER: *value = P.order; return FRPA_OK;
    case FRPA_TUNE_SPLIT_I8_SCRATCH_MB: *value = (int)(P.i8_budget >> 20); return FRPA_OK;
    default: return fail(FRPA_ERR_INVALID, "rho1 tuning: unknown key %d", key);
  }
}

int frpa_rho1_bias_part2(const frpa_rho1_plan *plan, int T, int n_atoms, int j_atom_begin, int j_atom_end,
                         int j_coord, const int *atom_valid, const double *wave, const double *gradient_wave,
                         const double *density_matrix, double *first_order_rho_bias_part2, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "bias part 2: null plan");
  return rho1_bias_part2_launch(*plan->p, nullptr, atom_valid, n_atoms, j_atom_begin, j_atom_end, j_coord, T, wave,
                                gradient_wave, density_matrix, first_order_rho_bias_part2, (cudaStream_t)stream);
}

int frpa_rho1_first_order_h(const frpa_rho1_plan *plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                            const int *atom_valid, const double *wave, const double *gradient_wave,
                            const double *hessian_wave, const double *vsigma, const double *gradient_rho,
                            const double *H_prefactor1, const double *first_order_gradient_rho,
                            const double *v_hartree_gradient, const double *first_order_rho, const double *v2rho2,
                            const double *v2rhosigma, const double *v2sigma2, const double *partition_tab,
                            double *first_order_H, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "first-order H: null plan");
  Rho1Plan &P = *plan->p;
  FRPA_CHECK_ARG(n_active >= 0 && n_active <= P.T, "first-order H: j_atom_end - j_atom_begin + 1 = %d outside 0..%d",
                 n_active, P.T);
  FRPA_CHECK_ARG(j_coord >= 1 && j_coord <= 3, "first-order H: j_coord %d outside 1..3", j_coord);
  FRPA_CHECK_ARG(n_active == 0 || (j_atom_begin >= 1 && j_atom_begin + n_active - 1 <= n_atoms),
                 "first-order H: atoms %d..%d outside 1..%d", j_atom_begin, j_atom_begin + n_active - 1, n_atoms);
  FRPA_CHECK_ARG(first_order_H && atom_valid && vsigma && gradient_rho && H_prefactor1 && first_order_gradient_rho &&
                     v_hartree_gradient && first_order_rho && v2rho2 && v2rhosigma && v2sigma2 && partition_tab,
                 "first-order H: null device pointer");
  FRPA_CHECK_ARG(P.n_items == 0 || (wave && gradient_wave && hessian_wave), "first-order H: null wave pointer");
  if (n_active == 0) return FRPA_OK;
  return rho1_first_order_h_run(P, n_active, n_atoms, j_atom_begin, j_coord, atom_valid, wave, gradient_wave,
                                hessian_wave, vsigma, gradient_rho, H_prefactor1, first_order_gradient_rho,
                                v_hartree_gradient, first_order_rho, v2rho2, v2rhosigma, v2sigma2, partition_tab,
                                first_order_H, (cudaStream_t)stream);
}

int frpa_rho1_adjoint_p1(const frpa_rho1_plan *plan, int n_active, const double *wave, const double *gradient_wave,
                         const double *g_rho, const double *g_grad, double *dP1, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "rho1: null plan");
  FRPA_CHECK_ARG(dP1 && (g_rho || g_grad), "rho1 adjoint: null output or no upstream gradient");
  FRPA_CHECK_ARG(n_active <= plan->p->T, "rho1 adjoint: n_active %d > tile %d", n_active, plan->p->T);
  return rho1_adjoint_run(*plan->p, n_active, wave,
                                   gradient_wave, g_rho, g_grad, dP1, (cudaStream_t)stream);
}

int frpa_sumup_plan_create(frpa_sumup_plan **plan, const frpa_sumup_desc *desc) {
  if (!plan) return fail(FRPA_ERR_INVALID, "sumup: null plan pointer");
  *plan = nullptr;
  SumupPlan *p = nullptr;
  FRPA_TRY(sumup_plan_create(&p, desc));
  *plan = new frpa_sumup_plan{p};
  return FRPA_OK;
}

int frpa_sumup_plan_destroy(frpa_sumup_plan *plan) {
  if (plan) {
    sumup_plan_free(plan->p);
    delete plan;
  }
  return FRPA_OK;
}

int frpa_sumup_plan_fast(const frpa_sumup_plan *plan) { return plan ? sumup_plan_is_fast(plan->p) : 0; }

int frpa_sumup_execute(const frpa_sumup_plan *plan, int n_active, int flags, const int *lhmfd, const double *mrs,
                       const double *opr, const double *Q, const double *spline, double *delta_v,
                       unsigned char *branch_codes, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "sumup: null plan");
  FRPA_CHECK_ARG(lhmfd && mrs && opr && Q && spline && delta_v, "sumup: null device pointer");
  return sumup_execute(plan->p, n_active, flags & 1, lhmfd, mrs, opr, Q, spline, delta_v, branch_codes,
                       (cudaStream_t)stream);
}

int frpa_sumup_adjoint_q(const frpa_sumup_plan *plan, int n_active, const int *lhmfd, const double *mrs,
                         const double *opr, const double *Q, const double *g, double *dQ, void *stream) {
  if (!plan) return fail(FRPA_ERR_INVALID, "sumup: null plan");
  FRPA_CHECK_ARG(lhmfd && mrs && opr && Q && g && dQ, "sumup adjoint: null device pointer");
  return sumup_adjoint_q(plan->p, n_active, lhmfd, mrs, opr, Q, g, dQ, (cudaStream_t)stream);
}

int frpa_sumup_device_flags(const frpa_sumup_plan *plan, int *flags) {
  if (!plan || !flags) return fail(FRPA_ERR_INVALID, "sumup: null argument");
  return sumup_read_error_flags(plan->p, flags);
}

int frpa_synth_basis_values(const frpa_rho1_desc *desc, const double *points, int n_atoms, const double *atoms,
                            const int *basis_atom, const int *basis_l, const int *basis_m, const double *basis_alpha,
                            double pad_value, double *wave, double *gradient_wave, void *stream) {
  return synth_basis_values(desc, points, n_atoms, atoms, basis_atom, basis_l, basis_m, basis_alpha, pad_value, wave,
                            gradient_wave, (cudaStream_t)stream);
}

int frpa_synth_p1_window(const int *global_index, int n, int T, double scale, unsigned long long seed, double *out,
                         void *stream) {
  return synth_p1_window(global_index, n, T, scale, seed, out, (cudaStream_t)stream);
}

// ------------------------------------------------- reference drop-ins

void evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map,
    int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *first_order_density_matrix,
    double *first_order_rho, double *first_order_rho_bias_part2, double *first_order_gradient_rho,
    double *first_order_gradient_rho_bias_batches_atoms, int *basis_atom, double *partition_tab,
    double *density_matrix) {
  (void)j_coord;
  (void)n_atoms;
  (void)n_max_compute_ham;
  (void)batch_sizes;
  (void)atom_valid_n_compute_c_batches;
  (void)basis_atom;
  (void)partition_tab;
  (void)density_matrix;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  clear_error();
  const int T = g_tile;
  frpa_rho1_desc d = rho_desc_from_ref(T, n_my_batches_work, n_full_points, n_basis, n_centers_basis_I,
                                       n_max_batch_size, n_point_batches, n_point_batches_prefix_sum,
                                       i_valid_point_2_i_full_points_map, n_compute_c_batches, i_basis_batches,
                                       i_batch_2_wave_offset);
  Rho1Plan *P = nullptr;
  if (rho1_plan_build(&P, &d) != FRPA_OK) return;
  const int nb = d.n_my_batches_work;
  const size_t wl = (size_t)P->wave_len, nb2 = (size_t)d.n_basis * d.n_basis * T;
  const size_t nbias = (size_t)d.n_max_batch_size * nb * T, nrho = (size_t)d.n_full_points * T;
  double *w = nullptr, *gw = nullptr, *p1 = nullptr, *bi = nullptr, *gb = nullptr, *r = nullptr, *g = nullptr;
  cudaStream_t s = 0;
  int st = FRPA_OK;
  if (st == FRPA_OK) st = h2d(0, wave_batches_compress, wl, &w, s);
  if (st == FRPA_OK) st = h2d(1, gradient_wave_batches_compress, 3 * wl, &gw, s);
  if (st == FRPA_OK) st = h2d(2, first_order_density_matrix, nb2, &p1, s);
  if (st == FRPA_OK) st = h2d(3, first_order_rho_bias_part2, nbias, &bi, s);
  if (st == FRPA_OK) st = h2d(4, first_order_gradient_rho_bias_batches_atoms, 3 * nbias, &gb, s);
  if (st == FRPA_OK) st = ensure(5, sizeof(double) * nrho, (void **)&r);
  if (st == FRPA_OK) st = ensure(6, sizeof(double) * 3 * nbias, (void **)&g);
  if (st == FRPA_OK)
    st = rho1_run(*P, g_rho1_mode, *j_atom_end - *j_atom_begin + 1, w, gw, p1, bi, gb, r, g, s);
  if (st == FRPA_OK && cudaMemcpyAsync(first_order_rho, r, sizeof(double) * nrho, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    st = fail(FRPA_ERR_CUDA, "rho1: download failed");
  if (st == FRPA_OK &&
      cudaMemcpyAsync(first_order_gradient_rho, g, sizeof(double) * 3 * nbias, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    st = fail(FRPA_ERR_CUDA, "rho1: download failed");
  if (st == FRPA_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) fail(FRPA_ERR_CUDA, "rho1: %s", cudaGetErrorString(e));
  }
  rho1_plan_free(P);
}

void evaluate_first_order_h_reduce_memory_c_v2_(
    int *j_atom_begin, int *j_atom_end, int *n_full_points, int *j_coord, int *n_basis, int *n_atoms,
    int *n_max_compute_ham, int *n_max_batch_size, int *n_my_batches_work, int *n_centers_basis_I,
    int *n_point_batches, int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches,
    int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map, double *vrho_batches,
    double *vsigma_batches, double *gradient_rho, double *H_times_psi_batches_compress, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *hessian_wave_batches_compress,
    double *first_order_H_tile, double *H_prefactor1_batches_tile, double *first_order_gradient_rho_batches_tile,
    double *v_hartree_gradient, double *first_order_rho, double *v2rho2_batches, double *v2rhosigma_batches,
    double *v2sigma2_batches, double *partition_tab, int *not_use) {
  (void)n_max_compute_ham;
  (void)vrho_batches;                  // unused by the reference as well
  (void)H_times_psi_batches_compress;  // unused by the reference as well
  (void)not_use;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  clear_error();
  const int T = g_tile;
  if (!j_atom_begin || !j_atom_end || !n_my_batches_work || !n_atoms || !j_coord || !first_order_H_tile) {
    fail(FRPA_ERR_INVALID, "first-order H: null argument");
    return;
  }
  const int n_active = *j_atom_end - *j_atom_begin + 1;
  if (n_active > T) {
    fail(FRPA_ERR_INVALID, "first-order H: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d", n_active, T);
    return;
  }
  frpa_rho1_desc d = rho_desc_from_ref(T, n_my_batches_work, n_full_points, n_basis, n_centers_basis_I,
                                       n_max_batch_size, n_point_batches, n_point_batches_prefix_sum,
                                       i_valid_point_2_i_full_points_map, n_compute_c_batches, i_basis_batches,
                                       i_batch_2_wave_offset);
  Rho1Plan *P = nullptr;
  if (rho1_plan_build(&P, &d) != FRPA_OK) return;
  const int nb = d.n_my_batches_work, nmb = d.n_max_batch_size, nf = d.n_full_points;
  const size_t wl = (size_t)P->wave_len, nH = (size_t)d.n_basis * d.n_basis * T;
  const size_t nav = (size_t)(*n_atoms + 1) * nb, nbt = (size_t)nmb * nb;
  double *w = nullptr, *gw = nullptr, *hw = nullptr, *vs = nullptr, *gr = nullptr, *pf1 = nullptr, *fog = nullptr,
         *vhg = nullptr, *r1 = nullptr, *v2r2 = nullptr, *v2rs = nullptr, *v2s2 = nullptr, *pt = nullptr,
         *H = nullptr;
  int *av = nullptr;
  cudaStream_t s = 0;
  int st = FRPA_OK;
  if (st == FRPA_OK) st = h2d(24, wave_batches_compress, wl, &w, s);
  if (st == FRPA_OK) st = h2d(25, gradient_wave_batches_compress, 3 * wl, &gw, s);
  if (st == FRPA_OK) st = h2d(26, hessian_wave_batches_compress, 6 * wl, &hw, s);
  if (st == FRPA_OK) st = h2d(27, vsigma_batches, 3 * nbt, &vs, s);
  if (st == FRPA_OK) st = h2d(28, gradient_rho, 3 * (size_t)nf, &gr, s);
  if (st == FRPA_OK) st = h2d(29, H_prefactor1_batches_tile, nbt * T, &pf1, s);
  if (st == FRPA_OK) st = h2d(30, first_order_gradient_rho_batches_tile, 3 * nbt * T, &fog, s);
  if (st == FRPA_OK) st = h2d(31, v_hartree_gradient, (size_t)nf * T, &vhg, s);
  if (st == FRPA_OK) st = h2d(32, first_order_rho, (size_t)nf * T, &r1, s);
  if (st == FRPA_OK) st = h2d(33, v2rho2_batches, 3 * nbt, &v2r2, s);
  if (st == FRPA_OK) st = h2d(34, v2rhosigma_batches, 6 * nbt, &v2rs, s);
  if (st == FRPA_OK) st = h2d(35, v2sigma2_batches, 6 * nbt, &v2s2, s);
  if (st == FRPA_OK) st = h2d(36, partition_tab, (size_t)nf, &pt, s);
  if (st == FRPA_OK) st = h2d(37, first_order_H_tile, nH, &H, s);
  if (st == FRPA_OK) st = h2d(38, atom_valid_n_compute_c_batches, nav, &av, s);
  frpa_rho1_plan handle{P};
  if (st == FRPA_OK)
    st = frpa_rho1_first_order_h(&handle, std::max(0, n_active), *n_atoms, *j_atom_begin, *j_coord, av, w, gw, hw, vs,
                                 gr, pf1, fog, vhg, r1, v2r2, v2rs, v2s2, pt, H, s);
  if (st == FRPA_OK &&
      cudaMemcpyAsync(first_order_H_tile, H, sizeof(double) * nH, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    st = fail(FRPA_ERR_CUDA, "first-order H: download failed");
  if (st == FRPA_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = fail(FRPA_ERR_CUDA, "first-order H: %s", cudaGetErrorString(e));
  }
  if (st == FRPA_OK) {
    int flags = 0;
    if (cudaMemcpy(&flags, P->d_err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && flags)
      fail(FRPA_ERR_DEVICE_INPUT,
           "first-order H: device input flags 0x%x (8: an atom's compute range leaves its batch, clipped; 16: a "
           "non-finite input, result incomplete)",
           flags);
  }
  rho1_plan_free(P);
}

void generate_first_order_rho_bias_part2_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches,
    int *i_batch_2_wave_offset, double *wave_batches_compress, double *gradient_wave_batches_compress,
    double *first_order_rho_bias_part2, double *partition_tab, double *density_matrix) {
  (void)n_full_points;
  (void)n_max_compute_ham;
  (void)batch_sizes;
  (void)partition_tab;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  clear_error();
  constexpr int T = 4;  // generate_first_order_rho_bias_part2.cpp:4
  if (!n_my_batches_work || !n_point_batches || !atom_valid_n_compute_c_batches || !density_matrix ||
      !first_order_rho_bias_part2) {
    fail(FRPA_ERR_INVALID, "bias part 2: null argument");
    return;
  }
  const int nb = *n_my_batches_work;
  // the reference does not use the point map here: a contiguous numbering
  std::vector<int> pre(nb + 1, 0);
  for (int b = 0; b < nb; ++b) pre[b + 1] = pre[b] + std::max(0, n_point_batches[b]);
  std::vector<int> ident(std::max(1, pre[nb]));
  for (size_t i = 0; i < ident.size(); ++i) ident[i] = (int)i;
  int n_full = std::max(1, pre[nb]);
  frpa_rho1_desc d = rho_desc_from_ref(T, n_my_batches_work, &n_full, n_basis, n_centers_basis_I, n_max_batch_size,
                                       n_point_batches, pre.data(), ident.data(), n_compute_c_batches,
                                       i_basis_batches, i_batch_2_wave_offset);
  Rho1Plan *P = nullptr;
  if (rho1_plan_build(&P, &d) != FRPA_OK) return;
  const size_t wl = (size_t)P->wave_len, nbias = (size_t)d.n_max_batch_size * nb * T;
  const size_t nav = (size_t)(*n_atoms + 1) * nb, ndm = (size_t)d.n_basis * d.n_basis;
  double *w = nullptr, *gw = nullptr, *dm = nullptr, *bi = nullptr;
  int *av = nullptr;
  cudaStream_t s = 0;
  int st = FRPA_OK;
  if (st == FRPA_OK) st = h2d(16, wave_batches_compress, wl, &w, s);
  if (st == FRPA_OK) st = h2d(17, gradient_wave_batches_compress, 3 * wl, &gw, s);
  if (st == FRPA_OK) st = h2d(18, density_matrix, ndm, &dm, s);
  if (st == FRPA_OK) st = h2d(19, first_order_rho_bias_part2, nbias, &bi, s);
  if (st == FRPA_OK) st = h2d(20, atom_valid_n_compute_c_batches, nav, &av, s);
  if (st == FRPA_OK)
    st = rho1_bias_part2_launch(*P, atom_valid_n_compute_c_batches, av, *n_atoms, *j_atom_begin, *j_atom_end,
                                *j_coord, T, w, gw, dm, bi, s);
  if (st == FRPA_OK &&
      cudaMemcpyAsync(first_order_rho_bias_part2, bi, sizeof(double) * nbias, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess)
    st = fail(FRPA_ERR_CUDA, "bias part 2: download failed");
  if (st == FRPA_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) fail(FRPA_ERR_CUDA, "bias part 2: %s", cudaGetErrorString(e));
  }
  rho1_plan_free(P);
}

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
    double *delta_v_hartree) {
  (void)n_max_radial;
  (void)n_radial;
  (void)scale_radial;
  (void)partition_tab;
  std::lock_guard<std::mutex> lk(g_buf_mu);
  clear_error();
  const int T = g_tile;
  frpa_sumup_desc d = sumup_desc_from_ref(
      T, *n_full_points, *l_max_analytic_multipole, *index_cc_dim_0, *n_valid_points, *l_pot_max, *n_hartree_grid,
      *n_centers, *n_centers_hartree_potential, *n_atoms, *hartree_force_l_add, *n_species, species, species_center,
      i_valid_point_2_i_full_points_map, coord_points, l_hartree, n_grid, n_cc_lm_ijk, centers_hartree_potential,
      center_to_atom, index_cc, index_ijk_max_cc, cc, coords_center, r_grid_min, log_r_grid_inc);
  const int n_active = *j_atom_end - *j_atom_begin + 1;
  if (n_active > T) {
    fail(FRPA_ERR_INVALID, "sumup: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d", n_active, T);
    return;
  }
  if (check_lhmfd(l_hartree_max_far_distance, *n_atoms, T, *l_pot_max) != FRPA_OK) return;
  SumupPlan *P = nullptr;
  if (sumup_plan_create(&P, &d) != FRPA_OK) return;
  const int L2 = (*l_pot_max + 1) * (*l_pot_max + 1);
  const size_t na = (size_t)*n_atoms * T;
  cudaStream_t s = 0;
  int *lh = nullptr;
  double *mr = nullptr, *op = nullptr, *q = nullptr, *sp = nullptr, *dv = nullptr;
  int st = FRPA_OK;
  if (st == FRPA_OK) st = h2d(10, l_hartree_max_far_distance, na, &lh, s);
  if (st == FRPA_OK) st = h2d(11, multipole_radius_sq, na, &mr, s);
  if (st == FRPA_OK) st = h2d(12, outer_potential_radius, (size_t)(*l_pot_max + 1) * na, &op, s);
  if (st == FRPA_OK) st = h2d(13, multipole_moments, (size_t)L2 * na, &q, s);
  if (st == FRPA_OK) st = h2d(14, current_delta_v_hart_part_spl_tile, (size_t)L2 * 2 * (*n_hartree_grid) * na, &sp, s);
  if (st == FRPA_OK) st = h2d(15, delta_v_hartree, (size_t)*n_full_points * T, &dv, s);
  if (st == FRPA_OK) st = sumup_execute(P, std::max(0, n_active), 0, lh, mr, op, q, sp, dv, nullptr, s);
  if (st == FRPA_OK &&
      cudaMemcpyAsync(delta_v_hartree, dv, sizeof(double) * (size_t)*n_full_points * T, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess)
    st = fail(FRPA_ERR_CUDA, "sumup: download failed");
  if (st == FRPA_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) fail(FRPA_ERR_CUDA, "sumup: %s", cudaGetErrorString(e));
  }
  sumup_plan_free(P);
}

}  // extern "C"

// ------------------------------------------------ the reference session
//
// The reference declares the session functions (device.hpp:191-192,
// device_data.hpp:159-227) and the sum-up's cu_host_ twin
// (sum_up_whole_potential.h:50-95) with C++ linkage; frpa.h does the same for
// C++ callers.  Each is defined here with C linkage, inside a namespace so that
// it can sit beside the header's C++ declaration (for C and Fortran callers and
// ctypes), and exported a second time with C++ linkage at the end of the file,
// forwarding to the first, so that the reference's C++ callers link unmodified.

namespace frpa {
namespace c_exports {
extern "C" {


void init_dfpt_device_info(void) {
  std::lock_guard<std::mutex> lk(g_session_mu);
  clear_error();
  Session &S = g_session;
  if (S.info) return;
  // $FRPA_DEVICE, else the library's current device (frpa_set_device; 0 unless set)
  int dev = 0;
  if (const char *e = getenv("FRPA_DEVICE"))
    dev = atoi(e);
  else if (cudaGetDevice(&dev) != cudaSuccess)
    dev = 0;
  int count = 0;
  cudaError_t err = cudaGetDeviceCount(&count);
  if (err != cudaSuccess || dev < 0 || dev >= count) {
    fail(FRPA_ERR_CUDA, "init_dfpt_device_info: device %d unavailable (%d devices, %s)", dev, count,
         cudaGetErrorString(err));
    return;
  }
  bool ok = cudaSetDevice(dev) == cudaSuccess &&
            cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&S.copy_in, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&S.copy_out, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&S.ev_p1, cudaEventDisableTiming) == cudaSuccess;
  for (int c = 0; ok && c < FP64_CHUNKS; ++c)
    ok = cudaEventCreateWithFlags(&S.ev_in[c], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&S.ev_done[c], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    session_free_streams(S);
    fail(FRPA_ERR_CUDA, "init_dfpt_device_info: stream creation failed");
    return;
  }
  S.device = dev;
  S.info = true;
}

void free_dfpt_device_info(void) {
  std::lock_guard<std::mutex> lk(g_session_mu);
  Session &S = g_session;
  if (S.data) session_free_data(S);
  session_free_streams(S);
  S.info = false;
}

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
    double *multipole_moments, double *current_delta_v_hart_part_spl_tile, double *delta_v_hartree) {
  (void)n_max_compute_ham;
  (void)n_max_radial;
  (void)basis_atom;
  (void)batch_sizes;
  (void)atom_valid_n_compute_c_batches;
  (void)density_matrix;
  (void)n_radial;
  (void)scale_radial;
  (void)partition_tab;
  (void)first_order_density_matrix;
  (void)first_order_rho;
  (void)first_order_rho_bias_part2;
  (void)first_order_gradient_rho;
  (void)first_order_gradient_rho_bias_batches_atoms;
  (void)l_hartree_max_far_distance;
  (void)multipole_radius_sq;
  (void)outer_potential_radius;
  (void)multipole_moments;
  (void)current_delta_v_hart_part_spl_tile;
  (void)delta_v_hartree;
  std::lock_guard<std::mutex> lk(g_session_mu);
  clear_error();
  Session &S = g_session;
  if (!S.info) {
    fail(FRPA_ERR_NO_SESSION, "init_dfpt_device_data: call init_dfpt_device_info first");
    return;
  }
  if (S.data) session_free_data(S);
  cudaSetDevice(S.device);
  S.T = g_tile;
  const int T = S.T;
  frpa_rho1_desc d = rho_desc_from_ref(T, n_my_batches_work, n_full_points, n_basis, n_centers_basis_I,
                                       n_max_batch_size, n_point_batches, n_point_batches_prefix_sum,
                                       i_valid_point_2_i_full_points_map, n_compute_c_batches, i_basis_batches,
                                       i_batch_2_wave_offset);
  if (rho1_plan_build(&S.rho, &d) != FRPA_OK) return;
  S.n_batches = *n_my_batches_work;
  S.n_full_points = *n_full_points;
  S.n_basis = *n_basis;
  S.n_max_batch_size = *n_max_batch_size;
  const size_t wl = (size_t)S.rho->wave_len;
  const size_t nbias = (size_t)S.n_max_batch_size * S.n_batches * T;
  auto alloc = [&](void **p, size_t bytes) {
    if (t_status != FRPA_OK) return;
    if (cudaMalloc(p, std::max<size_t>(bytes, 256)) != cudaSuccess)
      fail(FRPA_ERR_OOM, "init_dfpt_device_data: allocation of %zu bytes failed", bytes);
  };
  // Wave arrays that are already device memory of this GPU (e.g. computed
  // there by the caller) are used in place instead of copied; the caller
  // keeps them alive until free_dfpt_device_data.
  cudaPointerAttributes wa{}, ga{};
  const bool dev_wave = cudaPointerGetAttributes(&wa, wave_batches_compress) == cudaSuccess &&
                        cudaPointerGetAttributes(&ga, gradient_wave_batches_compress) == cudaSuccess &&
                        wa.type == cudaMemoryTypeDevice && ga.type == cudaMemoryTypeDevice &&
                        wa.device == S.device && ga.device == S.device;
  cudaGetLastError();
  if (dev_wave) {
    S.wave = wave_batches_compress;
    S.gwave = gradient_wave_batches_compress;
    S.borrowed_wave = true;
  } else {
    alloc((void **)&S.wave, sizeof(double) * wl);
    alloc((void **)&S.gwave, sizeof(double) * 3 * wl);
  }
  alloc((void **)&S.P1, sizeof(double) * (size_t)S.n_basis * S.n_basis * T);
  alloc((void **)&S.bias, sizeof(double) * nbias);
  alloc((void **)&S.gbias, sizeof(double) * 3 * nbias);
  alloc((void **)&S.out_rho, sizeof(double) * (size_t)S.n_full_points * T);
  alloc((void **)&S.out_grad, sizeof(double) * 3 * nbias);
  if (t_status == FRPA_OK && !dev_wave &&
      (cudaMemcpy(S.wave, wave_batches_compress, sizeof(double) * wl, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(S.gwave, gradient_wave_batches_compress, sizeof(double) * 3 * wl, cudaMemcpyHostToDevice) !=
           cudaSuccess))
    fail(FRPA_ERR_CUDA, "init_dfpt_device_data: wave upload failed");
  // sum-up constants (skipped when the caller has no sum-up data)
  if (t_status == FRPA_OK && n_valid_points && *n_valid_points > 0 && l_pot_max && index_cc) {
    frpa_sumup_desc sd = sumup_desc_from_ref(
        T, *n_full_points, *l_max_analytic_multipole, *index_cc_dim_0, *n_valid_points, *l_pot_max, *n_hartree_grid,
        *n_centers, *n_centers_hartree_potential, *n_atoms, *hartree_force_l_add, *n_species, species,
        species_center, i_valid_point_2_i_full_points_map, coord_points, l_hartree, n_grid, n_cc_lm_ijk,
        centers_hartree_potential, center_to_atom, index_cc, index_ijk_max_cc, cc, coords_center, r_grid_min,
        log_r_grid_inc);
    if (sumup_plan_create(&S.sumup, &sd) == FRPA_OK) {
      S.su_n_atoms = *n_atoms;
      S.su_L = *l_pot_max;
      S.su_grid = *n_hartree_grid;
      S.su_full = *n_full_points;
      const int L2 = (S.su_L + 1) * (S.su_L + 1);
      const size_t na = (size_t)S.su_n_atoms * T;
      alloc((void **)&S.lhmfd, sizeof(int) * na);
      alloc((void **)&S.mrs, sizeof(double) * na);
      alloc((void **)&S.opr, sizeof(double) * (S.su_L + 1) * na);
      alloc((void **)&S.Q, sizeof(double) * L2 * na);
      alloc((void **)&S.spline, sizeof(double) * (size_t)L2 * 2 * S.su_grid * na);
      alloc((void **)&S.dv, sizeof(double) * (size_t)S.su_full * T);
    }
  }
  if (t_status != FRPA_OK) {
    session_free_data(S);
    return;
  }
  S.data = true;
}

void free_dfpt_device_data(void) {
  std::lock_guard<std::mutex> lk(g_session_mu);
  if (g_session.data) session_free_data(g_session);
}

int frpa_session_rho1_device_outputs(double **rho, double **grad) {
  std::lock_guard<std::mutex> lk(g_session_mu);
  if (!g_session.data) return fail(FRPA_ERR_NO_SESSION, "no device session");
  if (rho) *rho = g_session.out_rho;
  if (grad) *grad = g_session.out_grad;
  return FRPA_OK;
}

// The session's FP64 step with host buffers, chunk by chunk: P1 goes in first,
// the biases follow chunk by chunk on copy_in, the kernel runs one chunk of
// batches after another on the session stream, and each finished chunk's
// grad rho1 goes out on copy_out while the next chunk computes; rho1 (scattered
// over all points) goes out last. Results are identical to one launch (every
// work item computes the same way). All three streams are idle on return.
static int rho1_session_chunked(Session &S, int n_active, const double *hP1, const double *hbias,
                                const double *hgbias, double *hrho, double *hgrad) {
  Rho1Plan &P = *S.rho;
  if (n_active > P.T)
    return fail(FRPA_ERR_INVALID, "rho1: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d", n_active, P.T);
  const int T = S.T, nb = S.n_batches;
  const size_t nmb = (size_t)S.n_max_batch_size, nbias = nmb * nb * T, nrho = (size_t)S.n_full_points * T;
  cudaStream_t s = S.stream, ci = S.copy_in, co = S.copy_out;
  int st = FRPA_OK;
  auto run = [&]() -> int {
    FRPA_CUDA_TRY(cudaMemcpyAsync(S.P1, hP1, sizeof(double) * (size_t)S.n_basis * S.n_basis * T,
                                  cudaMemcpyHostToDevice, s));
    FRPA_CUDA_TRY(cudaEventRecord(S.ev_p1, s));
    FRPA_CUDA_TRY(cudaStreamWaitEvent(ci, S.ev_p1, 0));  // the biases queue behind P1 on the link
    for (int c = 0; c < FP64_CHUNKS; ++c) {
      const size_t b0 = P.fp64_chunk_batches[c], b1 = P.fp64_chunk_batches[c + 1];
      for (int t = 0; t < T && b1 > b0; ++t) {
        const size_t off = nmb * (b0 + (size_t)nb * t), len = nmb * (b1 - b0);
        FRPA_CUDA_TRY(cudaMemcpyAsync(S.bias + off, hbias + off, sizeof(double) * len, cudaMemcpyHostToDevice, ci));
        FRPA_CUDA_TRY(cudaMemcpyAsync(S.gbias + 3 * off, hgbias + 3 * off, sizeof(double) * 3 * len,
                                      cudaMemcpyHostToDevice, ci));
      }
      FRPA_CUDA_TRY(cudaEventRecord(S.ev_in[c], ci));
    }
    // evaluate_first_order_rho.cpp:113-114 zeroes both outputs first
    FRPA_CUDA_TRY(cudaMemsetAsync(S.out_rho, 0, sizeof(double) * nrho, s));
    FRPA_CUDA_TRY(cudaMemsetAsync(S.out_grad, 0, sizeof(double) * 3 * nbias, s));
    for (int c = 0; c < FP64_CHUNKS; ++c) {
      FRPA_CUDA_TRY(cudaStreamWaitEvent(s, S.ev_in[c], 0));
      FRPA_TRY(rho1_fp64_launch_chunk(P, c, n_active, S.wave, S.gwave, S.P1, S.bias, S.gbias, S.out_rho, S.out_grad,
                                      s));
      FRPA_CUDA_TRY(cudaEventRecord(S.ev_done[c], s));
      FRPA_CUDA_TRY(cudaStreamWaitEvent(co, S.ev_done[c], 0));
      const size_t b0 = P.fp64_chunk_batches[c], b1 = P.fp64_chunk_batches[c + 1];
      for (int t = 0; t < T && b1 > b0; ++t) {
        const size_t off = 3 * nmb * (b0 + (size_t)nb * t), len = 3 * nmb * (b1 - b0);
        FRPA_CUDA_TRY(cudaMemcpyAsync(hgrad + off, S.out_grad + off, sizeof(double) * len, cudaMemcpyDeviceToHost, co));
      }
    }
    FRPA_CUDA_TRY(cudaMemcpyAsync(hrho, S.out_rho, sizeof(double) * nrho, cudaMemcpyDeviceToHost, s));
    return FRPA_OK;
  };
  st = run();
  // leave no copy of the caller's buffers in flight, whatever happened
  for (cudaStream_t x : {s, ci, co}) {
    const cudaError_t e = cudaStreamSynchronize(x);
    if (e != cudaSuccess && st == FRPA_OK) st = fail(FRPA_ERR_CUDA, "rho1 cu_host: %s", cudaGetErrorString(e));
  }
  return st;
}

void evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_(
    int *n_my_batches_work, int *j_atom_begin, int *j_atom_end, int *j_coord, int *n_full_points, int *n_basis,
    int *n_atoms, int *n_max_compute_ham, int *n_centers_basis_I, int *n_max_batch_size, int *batch_sizes,
    int *n_point_batches, int *n_point_batches_prefix_sum, int *i_valid_point_2_i_full_points_map,
    int *n_compute_c_batches, int *i_basis_batches, int *atom_valid_n_compute_c_batches, int *i_batch_2_wave_offset,
    double *wave_batches_compress, double *gradient_wave_batches_compress, double *first_order_density_matrix,
    double *first_order_rho, double *first_order_rho_bias_part2, double *first_order_gradient_rho,
    double *first_order_gradient_rho_bias_batches_atoms, int *basis_atom, double *partition_tab,
    double *density_matrix) {
  (void)j_coord;
  (void)n_atoms;
  (void)n_max_compute_ham;
  (void)n_centers_basis_I;
  (void)batch_sizes;
  (void)n_point_batches;
  (void)n_point_batches_prefix_sum;
  (void)i_valid_point_2_i_full_points_map;
  (void)n_compute_c_batches;
  (void)i_basis_batches;
  (void)atom_valid_n_compute_c_batches;
  (void)i_batch_2_wave_offset;
  (void)wave_batches_compress;
  (void)gradient_wave_batches_compress;
  (void)basis_atom;
  (void)partition_tab;
  (void)density_matrix;
  std::lock_guard<std::mutex> lk(g_session_mu);
  clear_error();
  Session &S = g_session;
  if (!S.data || !S.rho) {
    fail(FRPA_ERR_NO_SESSION, "rho1 cu_host: call init_dfpt_device_info and init_dfpt_device_data first");
    return;
  }
  if (*n_my_batches_work != S.n_batches || *n_full_points != S.n_full_points || *n_basis != S.n_basis ||
      *n_max_batch_size != S.n_max_batch_size) {
    fail(FRPA_ERR_INVALID, "rho1 cu_host: sizes differ from init_dfpt_device_data");
    return;
  }
  cudaSetDevice(S.device);
  const int T = S.T;
  const size_t nbias = (size_t)S.n_max_batch_size * S.n_batches * T, nrho = (size_t)S.n_full_points * T;
  cudaStream_t s = S.stream;
  if (g_rho1_mode == FRPA_RHO1_FP64 && (int)S.rho->fp64_chunk_items.size() == FP64_CHUNKS + 1) {
    rho1_session_chunked(S, *j_atom_end - *j_atom_begin + 1, first_order_density_matrix, first_order_rho_bias_part2,
                         first_order_gradient_rho_bias_batches_atoms, first_order_rho, first_order_gradient_rho);
    return;
  }
  if (cudaMemcpyAsync(S.P1, first_order_density_matrix, sizeof(double) * (size_t)S.n_basis * S.n_basis * T,
                      cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S.bias, first_order_rho_bias_part2, sizeof(double) * nbias, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(S.gbias, first_order_gradient_rho_bias_batches_atoms, sizeof(double) * 3 * nbias,
                      cudaMemcpyHostToDevice, s) != cudaSuccess) {
    fail(FRPA_ERR_CUDA, "rho1 cu_host: upload failed");
    return;
  }
  if (rho1_run(*S.rho, g_rho1_mode, *j_atom_end - *j_atom_begin + 1, S.wave, S.gwave, S.P1, S.bias, S.gbias,
               S.out_rho, S.out_grad, s) != FRPA_OK)
    return;
  if (cudaMemcpyAsync(first_order_rho, S.out_rho, sizeof(double) * nrho, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(first_order_gradient_rho, S.out_grad, sizeof(double) * 3 * nbias, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess) {
    fail(FRPA_ERR_CUDA, "rho1 cu_host: download failed");
    return;
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) fail(FRPA_ERR_CUDA, "rho1 cu_host: %s", cudaGetErrorString(e));
}

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
    double *delta_v_hartree) {
  (void)l_max_analytic_multipole;
  (void)index_cc_dim_0;
  (void)n_valid_points;
  (void)n_max_radial;
  (void)n_centers;
  (void)n_centers_hartree_potential;
  (void)hartree_force_l_add;
  (void)n_species;
  (void)n_radial;
  (void)species;
  (void)species_center;
  (void)i_valid_point_2_i_full_points_map;
  (void)coord_points;
  (void)l_hartree;
  (void)n_grid;
  (void)n_cc_lm_ijk;
  (void)centers_hartree_potential;
  (void)center_to_atom;
  (void)index_cc;
  (void)index_ijk_max_cc;
  (void)cc;
  (void)coords_center;
  (void)r_grid_min;
  (void)log_r_grid_inc;
  (void)scale_radial;
  (void)partition_tab;
  std::lock_guard<std::mutex> lk(g_session_mu);
  clear_error();
  Session &S = g_session;
  if (!S.data || !S.sumup) {
    fail(FRPA_ERR_NO_SESSION, "sumup cu_host: call init_dfpt_device_info and init_dfpt_device_data first");
    return;
  }
  if (n_atoms != S.su_n_atoms || l_pot_max != S.su_L || n_hartree_grid != S.su_grid || n_full_points != S.su_full) {
    fail(FRPA_ERR_INVALID, "sumup cu_host: sizes differ from init_dfpt_device_data");
    return;
  }
  const int T = S.T, n_active = j_atom_end - j_atom_begin + 1;
  if (n_active > T) {
    fail(FRPA_ERR_INVALID, "sumup cu_host: j_atom_end - j_atom_begin + 1 = %d > ATOM_TILE_SIZE %d", n_active, T);
    return;
  }
  if (check_lhmfd(l_hartree_max_far_distance, n_atoms, T, l_pot_max) != FRPA_OK) return;
  cudaSetDevice(S.device);
  const int L2 = (l_pot_max + 1) * (l_pot_max + 1);
  const size_t na = (size_t)n_atoms * T;
  cudaStream_t s = S.stream;
  if (cudaMemcpyAsync(S.lhmfd, l_hartree_max_far_distance, sizeof(int) * na, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S.mrs, multipole_radius_sq, sizeof(double) * na, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S.opr, outer_potential_radius, sizeof(double) * (l_pot_max + 1) * na, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemcpyAsync(S.Q, multipole_moments, sizeof(double) * L2 * na, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S.spline, current_delta_v_hart_part_spl_tile, sizeof(double) * (size_t)L2 * 2 * n_hartree_grid * na,
                      cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(S.dv, delta_v_hartree, sizeof(double) * (size_t)n_full_points * T, cudaMemcpyHostToDevice, s) !=
          cudaSuccess) {
    fail(FRPA_ERR_CUDA, "sumup cu_host: upload failed");
    return;
  }
  if (sumup_execute(S.sumup, std::max(0, n_active), 0, S.lhmfd, S.mrs, S.opr, S.Q, S.spline, S.dv, nullptr, s) !=
      FRPA_OK)
    return;
  if (cudaMemcpyAsync(delta_v_hartree, S.dv, sizeof(double) * (size_t)n_full_points * T, cudaMemcpyDeviceToHost, s) !=
      cudaSuccess) {
    fail(FRPA_ERR_CUDA, "sumup cu_host: download failed");
    return;
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) fail(FRPA_ERR_CUDA, "sumup cu_host: %s", cudaGetErrorString(e));
}

}  // extern "C"
}  // namespace c_exports
}  // namespace frpa

// ------------------------------------------- C++-linkage exports (see above)

void init_dfpt_device_info() { frpa::c_exports::init_dfpt_device_info(); }

void free_dfpt_device_info() { frpa::c_exports::free_dfpt_device_info(); }

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
    double *multipole_moments, double *current_delta_v_hart_part_spl_tile, double *delta_v_hartree) {
  frpa::c_exports::init_dfpt_device_data(
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

void free_dfpt_device_data() { frpa::c_exports::free_dfpt_device_data(); }

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
    double *delta_v_hartree) {
  frpa::c_exports::sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_(
      j_atom_begin, j_atom_end, n_full_points, l_max_analytic_multipole, index_cc_dim_0, n_valid_points, l_pot_max,
      n_max_radial, n_hartree_grid, n_centers, n_centers_hartree_potential, n_atoms, hartree_force_l_add, n_species,
      n_radial, species, species_center, l_hartree_max_far_distance, i_valid_point_2_i_full_points_map, coord_points,
      multipole_radius_sq, outer_potential_radius, multipole_moments, current_delta_v_hart_part_spl_tile, l_hartree,
      n_grid, n_cc_lm_ijk, centers_hartree_potential, center_to_atom, index_cc, index_ijk_max_cc, cc, coords_center,
      r_grid_min, log_r_grid_inc, scale_radial, partition_tab, delta_v_hartree);
}
