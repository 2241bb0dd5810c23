// Internal helpers shared by the frpa CUDA sources (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "frpa.h"

namespace frpa {

// ---------------------------------------------------------------- errors --

// Records a failure for frpa_last_error()/frpa_last_error_message() and
// returns the status so callers can `return fail(...)`.
int fail(int status, const char *fmt, ...);
void clear_error();

#define FRPA_CUDA_TRY(call)                                                                      \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return ::frpa::fail(FRPA_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call,             \
                          cudaGetErrorString(e_));                                               \
  } while (0)

#define FRPA_CHECK_ARG(cond, ...)                                                                \
  do {                                                                                           \
    if (!(cond)) return ::frpa::fail(FRPA_ERR_INVALID, __VA_ARGS__);                             \
  } while (0)

#define FRPA_TRY(call)                                                                           \
  do {                                                                                           \
    int s_ = (call);                                                                             \
    if (s_ != FRPA_OK) return s_;                                                                \
  } while (0)

// Launch-time check: configuration errors surface here, execution errors at
// the next synchronising call.
#define FRPA_LAUNCH_CHECK() FRPA_CUDA_TRY(cudaGetLastError())

// One-time setup per device (kernel attributes, constant-memory uploads) that
// several host threads may reach at the same time: `fn` runs under a lock and
// is retried by the next caller until it has succeeded once for `device`.
class PerDeviceOnce {
 public:
  template <class F>
  int run(int device, F &&fn) {
    std::lock_guard<std::mutex> lk(mu_);
    if (device >= 0 && device < 64 && done_[device]) return FRPA_OK;
    const int st = fn();
    if (st == FRPA_OK && device >= 0 && device < 64) done_[device] = true;
    return st;
  }

 private:
  std::mutex mu_;
  bool done_[64] = {};
};

// ------------------------------------------------------------ device math --

// Exactly rounded product and sum (no FMA contraction), used wherever the
// reference's x86-64 arithmetic decides a branch (dist^2 vs radii).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// 64-bit FP tensor-core MMA, m8n8k4 (A row-major 8x4, B col-major 4x8).
// Fragments: a = A[lane>>2][lane&3], b = B[lane&3][lane>>2],
// c/d = C[lane>>2][2*(lane&3) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// cp.async with zero fill: copies `src_bytes` (0 or the full size) and
// zero-fills the rest of the destination.
__device__ __forceinline__ void cp_async_8(void *smem_dst, const void *gmem_src, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem_src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_16(void *smem_dst, const void *gmem_src, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem_src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

// ------------------------------------------------------------ rho1 plan --

// One unit of rho1 work: a point tile of one non-empty grid batch
// (the reference's valid-batch list, device_data.cu:242-260, refined into
// point tiles and ordered by decreasing cost for the persistent scheduler).
struct Rho1WorkItem {
  int batch;         // index into the caller's batch arrays
  int nc;            // n_compute_c of the batch
  int np;            // points in the batch
  int p0;            // first point of this tile
  int pn;            // points in this tile
  int ib_off;        // offset of the batch's basis list in the compact list
  int prefix;        // n_point_batches_prefix_sum[batch]
  int key;           // locality key: MinHash of the batch's basis functions
  long long wave_off;  // i_batch_2_wave_offset[batch]
};
static_assert(sizeof(Rho1WorkItem) == 40, "work item layout");

// Split-int8 rho1 (rho1_split_i8.cu).  A work item is a point tile of one
// batch; its phi digits live in the A scratch, the batch's P1c digits (per
// perturbation) in the B scratch.  Offsets are relative to the scratch of
// the item's group: groups of consecutive batches are packed and contracted
// in turn, so the scratch holds one group at a time.
struct I8Item {
  int batch, nc, p0, pn;
  int prefix, rows8, n_nt, n_kc;  // rows8 = pn rounded up to 8; N tiles of 32 rows; K chunks of 32
  long long wave_off;
  long long a_off;       // bytes of the item's first A chunk
  long long b_off;       // bytes of the batch's first B chunk (t = 0)
  long long b_tstride;   // B bytes per perturbation
  int sa_off;            // first per-point scale of the item
  int sb_off;            // first per-row scale of the batch (t = 0)
  int sb_tstride;        // per-row scales per perturbation (n_nt * 32)
  int pad_;
};
static_assert(sizeof(I8Item) == 80, "I8Item layout");

// One N tile of one batch and perturbation, packed by one CTA.
struct I8BTile {
  int ib_off, nc, jn, t;
  int n_rows, n_kc, sb_off, pad_;  // rows of this tile (32; rows past n_compute are zero)
  long long b_off;                 // bytes of the tile's first chunk
};
static_assert(sizeof(I8BTile) == 40, "I8BTile layout");

struct I8Group {
  int item0, item1;   // items [item0, item1)
  int tile0, tile1;   // B tiles [tile0, tile1)
  long long a_bytes, b_bytes;
  int sa_len, sb_len;
};

struct Rho1Plan {
  int device = 0;
  int T = 1;
  int n_batches = 0;
  int n_full_points = 0;
  int n_basis = 0;
  int n_max_batch_size = 0;
  int n_max_compute = 0;
  long long wave_len = 0;
  int n_items = 0;
  int n_valid_batches = 0;
  long long n_valid_points = 0;  // points in batches with n_compute > 0
  int wave_aligned16 = 0;        // every batch offset even -> 16-byte loads
  // device copies
  Rho1WorkItem *d_items = nullptr;
  int *d_ib = nullptr;        // compact 1-based basis lists
  int *d_map = nullptr;       // i_valid_point_2_i_full_points_map
  int *d_counter = nullptr;   // persistent scheduler cursor
  int grid_fp64 = 0;
  // adjoint work list (batch, i tile, j tile, t), built with the plan, and
  // the first-order H's list of the tiles with j >= i; their 128-bit
  // fixed-point accumulator (allocated by the first call)
  void *d_adj_items = nullptr;
  int n_adj_items = 0;
  void *d_h1_items_sym = nullptr;
  int n_h1_items_sym = 0;
  unsigned long long *d_h1_acc = nullptr;
  // split-BF16 path: <= 128-point tiles, per-row P1 scales, device error flags
  Rho1WorkItem *d_items_split = nullptr;
  int n_items_split = 0;
  double *d_rowmax = nullptr;
  int *d_err = nullptr;
  // tunings (frpa_rho1_plan_set_tuning) and the host copy of the valid
  // batches the work lists are rebuilt from (one item per batch, p0 = 0)
  int fp64_tile_points = 64;   // 64 or 128 points per FP64 work item
  int fp64_ctas_per_sm = 0;    // 0: as many as fit
  int split_tile_points = 128; // <= 128 points per split-BF16 work item
  int order = 2;               // 0: largest items first, 1: batch order, 2: locality key
  // the FP64 work list in FP64_CHUNKS pieces of consecutive batches (6%, 44%,
  // 44%, 6% of the cost): chunk c holds items [fp64_chunk_items[c], fp64_chunk_items[c + 1])
  // of batches [fp64_chunk_batches[c], fp64_chunk_batches[c + 1]), so the
  // host-buffer entry point can overlap copies with compute chunk by chunk
  std::vector<int> fp64_chunk_items, fp64_chunk_batches;
  std::vector<Rho1WorkItem> h_batches;
  std::vector<int> h_ib;  // host copy of the compact basis lists
  // split-int8 path: work lists (built with the plan) and the scratch
  // (allocated by the first split-int8 execution, reused afterwards)
  I8Item *d_i8_items = nullptr;
  I8BTile *d_i8_tiles = nullptr;
  std::vector<I8Group> i8_groups;
  long long i8_budget = 4LL << 30;  // bytes of A + B scratch per group
  int i8_wave4 = 0;                  // every batch's phi offset a multiple of 4 doubles
  // two scratch sets: group g is packed into set g % 2 on a side stream while
  // group g - 1 is contracted on the caller's stream
  unsigned char *d_i8_a[2] = {nullptr, nullptr}, *d_i8_b[2] = {nullptr, nullptr};
  double *d_i8_sa[2] = {nullptr, nullptr}, *d_i8_sb[2] = {nullptr, nullptr};
  cudaStream_t i8_side = nullptr;
  cudaEvent_t i8_ev_start = nullptr, i8_ev_packed[2] = {nullptr, nullptr}, i8_ev_done[2] = {nullptr, nullptr};
};

// Work lists of a plan's valid batches (one entry per batch in `batches`).
// work-list order (0 largest first, 1 batch order, 2 locality key) and the key
void rho1_order_items(std::vector<Rho1WorkItem> *items, int order);
int rho1_locality_key(const int *ib, int nc);
constexpr int FP64_CHUNKS = 4;
// FP64 work items, chunk by chunk (FP64_CHUNKS ranges of consecutive batches
// holding 6%, 44%, 44% and 6% of the cost, n_batches = the caller's batch
// count), each chunk in the given order; the chunk boundaries go to
// chunk_items / chunk_batches
void rho1_fp64_build_items(const std::vector<Rho1WorkItem> &batches, int tile_points, int order, int n_batches,
                           std::vector<Rho1WorkItem> *out, std::vector<int> *chunk_items,
                           std::vector<int> *chunk_batches);

int rho1_fp64_launch(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave,
                     const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                     cudaStream_t stream);
// The FP64 kernel over the items of one chunk only, without zeroing the
// outputs (the caller zeroes them once before the first chunk).
int rho1_fp64_launch_chunk(const Rho1Plan &plan, int chunk, int n_active, const double *wave, const double *gwave,
                           const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                           cudaStream_t stream);
int rho1_fp64_grid(int device);
int rho1_fp64_fused_bias_launch(const Rho1Plan &plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                                const int *atom_valid, const double *density_matrix, const double *wave,
                                const double *gwave, const double *P1, const double *bias, const double *gbias,
                                double *rho, double *grad, cudaStream_t stream);
int rho1_split_launch(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave,
                      const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                      cudaStream_t stream);
void rho1_split_build_items(const std::vector<Rho1WorkItem> &batches, int tile_points, int order,
                            std::vector<Rho1WorkItem> *out);

int p1_rowmax_launch(const Rho1Plan &plan, const double *P1, cudaStream_t stream);
int rho1_i8_build(Rho1Plan *plan);  // work lists and groups from plan->h_batches
void rho1_i8_free(Rho1Plan *plan);
int rho1_i8_launch(Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *P1,
                   const double *bias, const double *gbias, double *rho, double *grad, cudaStream_t stream);

int synth_p1_window(const int *gidx, int n, int T, double scale, unsigned long long seed, double *out,
                    cudaStream_t stream);
int rho1_bias_part2_launch(const Rho1Plan &plan, const int *h_atom_valid, const int *d_atom_valid, int n_atoms,
                           int j_atom_begin, int j_atom_end, int j_coord, int T, const double *wave,
                           const double *gwave, const double *dm, double *bias, cudaStream_t stream);
// First-order H and the rho1 adjoint (first_order_h.cu): deterministic
// fixed-point accumulation into an (n_basis, n_basis, T) output.
size_t rho1_h1_item_size();
void rho1_h1_build_items(const int *nc_b, const int *np_b, const int *ib_off, const int *prefix,
                         const long long *wave_off, int n_batches, int T, bool sym, std::vector<unsigned char> *host);
int rho1_adjoint_run(Rho1Plan &plan, int n_active, const double *wave, const double *gwave, const double *g_rho,
                     const double *g_grad, double *dP1, cudaStream_t stream);
int rho1_first_order_h_run(Rho1Plan &plan, int n_active, int n_atoms, int j_atom_begin, int j_coord,
                           const int *atom_valid, const double *wave, const double *gwave, const double *hwave,
                           const double *vsigma, const double *gradient_rho, const double *H_prefactor1,
                           const double *fogr, const double *vhg, const double *rho1, const double *v2rho2,
                           const double *v2rhosigma, const double *v2sigma2, const double *partition_tab,
                           double *first_order_H, cudaStream_t stream);

// ----------------------------------------------------------- sum-up plan --

struct SumupPlan;  // defined in sumup.cu

}  // namespace frpa
