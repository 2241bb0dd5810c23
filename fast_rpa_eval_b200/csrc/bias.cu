// First-order density bias, part 2: the density-matrix term of rho1 for the
// displacement of atom j along j_coord, the input `first_order_rho_bias_part2`
// of the rho1 step.  Per grid batch and atom j of the tile, with
// fw = -d phi / d x_{j_coord} and A_j the batch's compute functions of atom j
// (the range atom_valid_n_compute_c_batches(j-1 .. j, batch)):
//   bias(p, j) = sum_i phi_i(p) sum_{k in A_j} DM(ib_i, ib_k) fw_k(p)
//              + sum_{i in A_j} fw_i(p) sum_k DM(ib_i, ib_k) phi_k(p)
// Reference: fast_rap_src_dfpt_gpu_eval/generate_first_order_rho_bias_part2.cpp:11-168
// (two DGEMMs and two per-point dot products per (batch, atom), through the
// host).  Here the two terms are one contraction with the symmetrised slab
//   S(i, k) = DM(ib_i, ib_k) + DM(ib_k, ib_i),  k in A_j,
// bias(p, j) = sum_i phi_i(p) sum_k S(i, k) fw_k(p): one CTA per work item of
// the rho1 plan (a batch's point tile), one thread per point, S staged in
// shared memory in 32-row chunks, FP64 throughout.  Atoms with no compute
// function in a batch get bias 0, as in the reference (:152-156); batches
// without compute functions are left untouched.
#include <algorithm>

#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int BZ_THREADS = 128;  // >= points per work item (64 or 128)
constexpr int BZ_IC = 32;        // rows i per staged chunk of S
constexpr int BZ_MAXA = 64;      // compute functions of one atom in one batch

struct BiasSmem {
  double S[BZ_IC][BZ_MAXA];
  double g[BZ_MAXA][BZ_THREADS];  // fw_k(p) of the tile's points
  int ib[FRPA_MAX_N_COMPUTE];
};

__global__ void __launch_bounds__(BZ_THREADS) bias_part2_kernel(
    const Rho1WorkItem *__restrict__ items, const int *__restrict__ ib_all, const int *__restrict__ atom_valid,
    int n_atoms, int j_atom_begin, int n_active, int j_coord, int n_basis, int n_max_batch_size, int n_batches,
    const double *__restrict__ wave, const double *__restrict__ gwave, const double *__restrict__ dm,
    double *__restrict__ bias, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BiasSmem &S = *reinterpret_cast<BiasSmem *>(smem_raw);
  const Rho1WorkItem W = items[blockIdx.x];
  const int p = threadIdx.x, nc = W.nc, ncp = (nc + 3) & ~3;
  const bool live = p < W.pn;
  for (int i = p; i < nc; i += BZ_THREADS) S.ib[i] = ib_all[W.ib_off + i] - 1;
  const double *phi = wave + W.wave_off + (long long)(W.p0 + (live ? p : 0)) * ncp;
  const double *fwp = gwave + 3 * W.wave_off + 3LL * (W.p0 + (live ? p : 0)) * ncp + (long long)(j_coord - 1) * ncp;
  const int *av = atom_valid + (long long)(n_atoms + 1) * W.batch;
  for (int t = 0; t < n_active; ++t) {
    const int j_atom = j_atom_begin + t;
    const int vs = av[j_atom - 1], cnt = av[j_atom] - vs;
    double *out = bias + (W.p0 + p) + (long long)n_max_batch_size * (W.batch + (long long)n_batches * t);
    __syncthreads();  // ib staged; the previous atom's S and g consumed
    if (cnt <= 0) {
      if (live) *out = 0.0;
      continue;
    }
    if (vs < 0 || cnt > BZ_MAXA || vs + cnt > nc) {  // outside the batch: flag, write nothing
      if (p == 0) atomicOr(err, 8);
      continue;
    }
    for (int k = 0; k < cnt; ++k) S.g[k][p] = live ? -__ldg(fwp + vs + k) : 0.0;
    double acc = 0.0;
    for (int i0 = 0; i0 < nc; i0 += BZ_IC) {
      __syncthreads();
      for (int e = p; e < BZ_IC * cnt; e += BZ_THREADS) {
        const int ii = e / cnt, k = e - ii * cnt, i = i0 + ii;
        double v = 0.0;
        if (i < nc) {
          const long long bi = S.ib[i], bk = S.ib[vs + k];
          v = __ldg(dm + bi + bk * n_basis) + __ldg(dm + bk + bi * n_basis);
        }
        S.S[ii][k] = v;
      }
      __syncthreads();
      if (live) {
        const int iend = min(BZ_IC, nc - i0);
        for (int ii = 0; ii < iend; ++ii) {
          double s = 0.0;
          for (int k = 0; k < cnt; ++k) s = fma(S.S[ii][k], S.g[k][p], s);
          acc = fma(__ldg(phi + i0 + ii), s, acc);
        }
      }
    }
    if (live) *out = acc;
  }
}

}  // namespace

// Host checks of the atom ranges, then one launch over the plan's work items.
int rho1_bias_part2_launch(const Rho1Plan &plan, const int *h_atom_valid, const int *d_atom_valid, int n_atoms,
                           int j_atom_begin, int j_atom_end, int j_coord, int T, const double *wave,
                           const double *gwave, const double *dm, double *bias, cudaStream_t stream) {
  const int n_active = j_atom_end - j_atom_begin + 1;
  FRPA_CHECK_ARG(j_coord >= 1 && j_coord <= 3, "bias part 2: j_coord %d not 1..3", j_coord);
  FRPA_CHECK_ARG(n_active >= 1 && n_active <= T, "bias part 2: atoms %d..%d do not fit the tile of %d", j_atom_begin,
                 j_atom_end, T);
  FRPA_CHECK_ARG(j_atom_begin >= 1 && j_atom_end <= n_atoms, "bias part 2: atoms %d..%d outside 1..%d", j_atom_begin,
                 j_atom_end, n_atoms);
  FRPA_CHECK_ARG(wave && gwave && dm && bias && d_atom_valid, "bias part 2: null device pointer");
  if (h_atom_valid) {
    for (const Rho1WorkItem &b : plan.h_batches)
      for (int j = j_atom_begin; j <= j_atom_end; ++j) {
        const int *av = h_atom_valid + (long long)(n_atoms + 1) * b.batch;
        const int vs = av[j - 1], ve = av[j];
        FRPA_CHECK_ARG(vs >= 0 && ve >= vs && ve <= b.nc && ve - vs <= BZ_MAXA,
                       "bias part 2: batch %d atom %d compute range [%d, %d) invalid (n_compute %d, at most %d per "
                       "atom)",
                       b.batch, j, vs, ve, b.nc, BZ_MAXA);
      }
  }
  if (plan.n_items == 0) return FRPA_OK;
  static PerDeviceOnce configured;
  FRPA_TRY(configured.run(plan.device, []() -> int {
    FRPA_CUDA_TRY(
        cudaFuncSetAttribute(bias_part2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BiasSmem)));
    return FRPA_OK;
  }));
  bias_part2_kernel<<<plan.n_items, BZ_THREADS, sizeof(BiasSmem), stream>>>(
      plan.d_items, plan.d_ib, d_atom_valid, n_atoms, j_atom_begin, n_active, j_coord, plan.n_basis,
      plan.n_max_batch_size, plan.n_batches, wave, gwave, dm, bias, plan.d_err);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

}  // namespace frpa
