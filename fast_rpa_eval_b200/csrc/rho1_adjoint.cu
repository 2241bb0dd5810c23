// Adjoint of rho1 with respect to the first-order density matrix P1.
//
// Forward (fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho.cpp:149-207):
//   rho1(map p, t)  = sum_ij P1(ib_i, ib_j, t) phi_i(p) phi_j(p) + bias
//   grad(d, p, b, t) = 2 sum_ij grad_d phi_i(p) P1(ib_i, ib_j, t) phi_j(p) - gbias
// so for upstream gradients g_rho (n_full_points, T) and g_grad
// (3, n_max_batch_size, n_batches, T):
//   dP1(ib_i, ib_j, t) += sum_p A(i, p) phi_j(p),
//   A(i, p) = g_rho(map p, t) phi_i(p) + 2 sum_d g_grad(d, p, b, t) grad_d phi_i(p)
// (the g_rho term only for t < n_active, the perturbations rho1 is written
// for).  With g_rho = w v and no g_grad this is the first-order-H integration
// sum_p w v phi_i phi_j of fast_rap_src_dfpt_gpu_eval/evaluate_first_order_H.cpp:145-215
// with its XC terms zero.
//
// One CTA computes a 64 x 64 (i, j) tile of one batch's contribution on the
// FP64 MMA, building A in shared memory from phi, grad phi and the upstream
// gradients as it streams the point dimension; nothing is saved from the
// forward pass.  Tiles are scatter-added into dP1 with double atomics (batches
// overlap in P1), so the summation order across batches is not fixed.
#include <cstring>
#include <vector>

#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int BM = 64, BN = 64, KC = 16, THREADS = 256;
constexpr int LDA = BM + 4;  // As[k = point][m = i]
constexpr int LDB = KC + 4;  // Bs[n = j][k = point]

struct AdjItem {
  int batch, nc, np, ib_off, prefix, m0, n0, t;
  long long wave_off;
};

__global__ void __launch_bounds__(THREADS)
    rho1_adjoint_kernel(const AdjItem *__restrict__ items, int n_items, const int *__restrict__ ib_all,
                        const int *__restrict__ map, int n_active, int n_basis, int n_full_points,
                        int n_max_batch_size, int n_batches, const double *__restrict__ wave,
                        const double *__restrict__ gwave, const double *__restrict__ g_rho,
                        const double *__restrict__ g_grad, double *__restrict__ dP1) {
  __shared__ __align__(16) double As[KC * LDA];
  __shared__ __align__(16) double Bs[BN * LDB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3, g = lane >> 2, q = lane & 3;
  const long long nb2 = (long long)n_basis * n_basis;

  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const AdjItem W = items[it];
    const int nc = W.nc, np = W.np, t = W.t;
    const int ncp = (nc + 3) & ~3;
    const double *phi = wave + W.wave_off;
    const double *gph = gwave + 3 * W.wave_off;
    const bool use_rho = (g_rho != nullptr) && t < n_active;
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    for (int k0 = 0; k0 < np; k0 += KC) {
      // A tile: (KC points) x (BM rows i)
#pragma unroll
      for (int j = 0; j < (BM * KC) / THREADS; ++j) {
        const int e = tid + THREADS * j;
        const int m = e & (BM - 1), k = e / BM;
        const int i = W.m0 + m, p = k0 + k;
        double v = 0.0;
        if (i < nc && p < np) {
          const long long pc = (long long)p * ncp;
          if (use_rho) v = g_rho[map[W.prefix + p] + (long long)n_full_points * t] * phi[i + pc];
          if (g_grad) {
            const long long gi = 3 * (p + (long long)n_max_batch_size * (W.batch + (long long)n_batches * t));
            const double *gp = gph + i + 3 * pc;
            v += 2.0 * (g_grad[gi] * gp[0] + g_grad[gi + 1] * gp[ncp] + g_grad[gi + 2] * gp[2 * ncp]);
          }
        }
        As[k * LDA + m] = v;
      }
      // B tile: Bs[j][p] = phi(j, p)
#pragma unroll
      for (int j = 0; j < (BN * KC) / THREADS; ++j) {
        const int e = tid + THREADS * j;
        const int n = e & (BN - 1), k = e / BN;
        const int jj = W.n0 + n, p = k0 + k;
        Bs[n * LDB + k] = (jj < nc && p < np) ? phi[jj + (long long)p * ncp] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int ks = 0; ks < KC / 4; ++ks) {
        double a[4], b[2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = As[(ks * 4 + q) * LDA + wm * 32 + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) b[ni] = Bs[(wn * 16 + ni * 8 + g) * LDB + ks * 4 + q];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int ni = 0; ni < 2; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
      }
      __syncthreads();
    }
    // scatter-add the tile
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int i = W.m0 + wm * 32 + mi * 8 + g;
      if (i >= nc) continue;
      const long long row = ib_all[W.ib_off + i] - 1;
#pragma unroll
      for (int ni = 0; ni < 2; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int jj = W.n0 + wn * 16 + ni * 8 + 2 * q + h;
          if (jj < nc) {
            const long long col = ib_all[W.ib_off + jj] - 1;
            atomicAdd(dP1 + row + col * n_basis + t * nb2, acc[mi][ni][h]);
          }
        }
    }
  }
}

}  // namespace

int rho1_adjoint_launch_items(const Rho1Plan &plan, const void *d_items, int n_items, int n_active,
                              const double *wave, const double *gwave, const double *g_rho, const double *g_grad,
                              double *dP1, cudaStream_t stream) {
  if (n_items == 0) return FRPA_OK;
  int n_sm = 148;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, plan.device);
  int grid = n_sm * 4;
  if (grid > n_items) grid = n_items;
  rho1_adjoint_kernel<<<grid, THREADS, 0, stream>>>(static_cast<const AdjItem *>(d_items), n_items, plan.d_ib,
                                                    plan.d_map, n_active, plan.n_basis, plan.n_full_points,
                                                    plan.n_max_batch_size, plan.n_batches, wave, gwave, g_rho,
                                                    g_grad, dP1);
  FRPA_LAUNCH_CHECK();
  return FRPA_OK;
}

size_t rho1_adjoint_item_size() { return sizeof(AdjItem); }

// Packs (batch, i tile, j tile, t) items; `host` receives raw AdjItem bytes.
void rho1_adjoint_build_items(const int *nc_b, const int *np_b, const int *ib_off, const int *prefix,
                              const long long *wave_off, int n_batches, int T, std::vector<unsigned char> *host) {
  std::vector<AdjItem> v;
  for (int b = 0; b < n_batches; ++b) {
    if (nc_b[b] <= 0 || np_b[b] <= 0) continue;
    for (int t = 0; t < T; ++t)
      for (int m0 = 0; m0 < nc_b[b]; m0 += BM)
        for (int n0 = 0; n0 < nc_b[b]; n0 += BN)
          v.push_back(AdjItem{b, nc_b[b], np_b[b], ib_off[b], prefix[b], m0, n0, t, wave_off[b]});
  }
  host->resize(v.size() * sizeof(AdjItem));
  if (!v.empty()) memcpy(host->data(), v.data(), host->size());
}

}  // namespace frpa
