// Synthetic workload generator: analytic Gaussian basis functions and their
// gradients at the grid batches' points, written straight into the reference's
// compressed wave layouts (wave (ncp, np) and gradient_wave (ncp, 3, np) per
// batch at i_batch_2_wave_offset).  Used by the benchmarks to build large
// workloads on the device; not part of the rho1 / sum-up path.
//   phi(r) = R_lm(r - R_A) exp(-alpha |r - R_A|^2),  R_lm = r^l Y_lm
// with Y_lm in the reference's real convention (index l*l + l + m).
#include <cmath>
#include <map>
#include <tuple>
#include <vector>

#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int SY_LMAX = 4;
constexpr int SY_NLM = (SY_LMAX + 1) * (SY_LMAX + 1);
constexpr int SY_MAXT = 16;

struct Mono {
  double c;
  int a, b, k;
};
__constant__ Mono c_mono[SY_NLM][SY_MAXT];
__constant__ int c_nmono[SY_NLM];

using Poly = std::map<std::tuple<int, int, int>, double>;

Poly pmul(const Poly &p, const Poly &q) {
  Poly r;
  for (auto &x : p)
    for (auto &y : q) {
      auto key = std::make_tuple(std::get<0>(x.first) + std::get<0>(y.first), std::get<1>(x.first) + std::get<1>(y.first),
                                 std::get<2>(x.first) + std::get<2>(y.first));
      r[key] += x.second * y.second;
    }
  return r;
}
Poly padd(const Poly &p, const Poly &q, double s) {
  Poly r = p;
  for (auto &y : q) r[y.first] += s * y.second;
  return r;
}

// Regular solid harmonics r^l Y_lm as monomial lists (same recursion as the
// oracle's Y_lm, written homogeneously in x, y, z).
int build_monomials(std::vector<Mono> *out, std::vector<int> *count) {
  const Poly X{{{1, 0, 0}, 1.0}}, Y{{{0, 1, 0}, 1.0}}, Z{{{0, 0, 1}, 1.0}}, ONE{{{0, 0, 0}, 1.0}};
  const Poly R2{{{2, 0, 0}, 1.0}, {{0, 2, 0}, 1.0}, {{0, 0, 2}, 1.0}};
  const double four_pi = 12.566370614359172953850573533118;
  out->assign(SY_NLM * SY_MAXT, Mono{0, 0, 0, 0});
  count->assign(SY_NLM, 0);
  std::vector<Poly> C(SY_LMAX + 1), S(SY_LMAX + 1);
  C[0] = ONE;
  for (int m = 1; m <= SY_LMAX; ++m) {
    C[m] = padd(pmul(X, C[m - 1]), pmul(Y, S[m - 1]), -1.0);
    S[m] = padd(pmul(X, S[m - 1]), pmul(Y, C[m - 1]), 1.0);
  }
  for (int m = 0; m <= SY_LMAX; ++m) {
    std::vector<Poly> Q(SY_LMAX + 1);
    double df = 1.0;
    for (int k = 1; k <= 2 * m - 1; k += 2) df *= k;
    Q[m] = Poly{{{0, 0, 0}, df}};
    for (int l = m + 1; l <= SY_LMAX; ++l) {
      Poly a = pmul(Z, Q[l - 1]);
      for (auto &e : a) e.second *= (double)(2 * l - 1) / (l - m);
      if (l >= m + 2) {
        Poly b = pmul(R2, Q[l - 2]);
        a = padd(a, b, -(double)(l + m - 1) / (l - m));
      }
      Q[l] = a;
    }
    for (int l = m; l <= SY_LMAX; ++l) {
      double ratio = 1.0;
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= k;
      double K = std::sqrt((2 * l + 1) / four_pi * ratio);
      if (m > 0) K *= std::sqrt(2.0);
      for (int sgn = (m == 0 ? 0 : -1); sgn <= (m == 0 ? 0 : 1); sgn += 2) {
        if (m > 0 && sgn == 0) continue;
        Poly p = m == 0 ? Q[l] : pmul(Q[l], sgn > 0 ? C[m] : S[m]);
        const double f = (m > 0 && sgn > 0 && (m & 1)) ? -K : K;
        const int lm = l * l + l + (m == 0 ? 0 : sgn * m);
        int n = 0;
        for (auto &e : p) {
          if (e.second == 0.0) continue;
          if (n >= SY_MAXT) return fail(FRPA_ERR_UNSUPPORTED, "synth: monomial table too small");
          (*out)[lm * SY_MAXT + n] = Mono{f * e.second, std::get<0>(e.first), std::get<1>(e.first), std::get<2>(e.first)};
          ++n;
        }
        (*count)[lm] = n;
        if (m == 0) break;
      }
    }
  }
  return FRPA_OK;
}

struct SynBatch {
  int nc, np, prefix, ib_off;
  long long wave_off;
};

__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}

__global__ void synth_kernel(int n_batches, const SynBatch *__restrict__ batches, const int *__restrict__ ib,
                             const double *__restrict__ points, const double *__restrict__ atoms,
                             const int *__restrict__ b_atom, const int *__restrict__ b_lm,
                             const double *__restrict__ b_alpha, double pad, double *__restrict__ wave,
                             double *__restrict__ gwave) {
  for (int b = blockIdx.x; b < n_batches; b += gridDim.x) {
    const SynBatch B = batches[b];
    const int ncp = (B.nc + 3) & ~3;
    const long long n_el = (long long)ncp * B.np;
    for (long long e = threadIdx.x; e < n_el; e += blockDim.x) {
      const int i = (int)(e % ncp);
      const int p = (int)(e / ncp);
      double v = pad, gx = pad, gy = pad, gz = pad;
      if (i < B.nc) {
        const int f = ib[B.ib_off + i] - 1;
        const int a = b_atom[f];
        const double *pt = points + 3LL * (B.prefix + p);
        const double x = pt[0] - atoms[3 * a], y = pt[1] - atoms[3 * a + 1], z = pt[2] - atoms[3 * a + 2];
        const double al = b_alpha[f];
        const double gau = exp(-al * (x * x + y * y + z * z));
        const int lm = b_lm[f];
        double R = 0.0, Rx = 0.0, Ry = 0.0, Rz = 0.0;
        for (int t = 0; t < c_nmono[lm]; ++t) {
          const Mono M = c_mono[lm][t];
          const double xa = ipow(x, M.a), yb = ipow(y, M.b), zk = ipow(z, M.k);
          R += M.c * xa * yb * zk;
          if (M.a) Rx += M.c * M.a * ipow(x, M.a - 1) * yb * zk;
          if (M.b) Ry += M.c * M.b * xa * ipow(y, M.b - 1) * zk;
          if (M.k) Rz += M.c * M.k * xa * yb * ipow(z, M.k - 1);
        }
        v = R * gau;
        gx = (Rx - 2 * al * x * R) * gau;
        gy = (Ry - 2 * al * y * R) * gau;
        gz = (Rz - 2 * al * z * R) * gau;
      }
      wave[B.wave_off + e] = v;
      double *g = gwave + 3 * B.wave_off + i + 3LL * ncp * p;
      g[0] = gx;
      g[ncp] = gy;
      g[2 * ncp] = gz;
    }
  }
}

}  // namespace

int synth_basis_values(const frpa_rho1_desc *D, const double *points, int n_atoms, const double *atoms,
                       const int *basis_atom, const int *basis_l, const int *basis_m, const double *basis_alpha,
                       double pad, double *wave, double *gwave, cudaStream_t stream) {
  FRPA_CHECK_ARG(D && points && atoms && basis_atom && basis_l && basis_m && basis_alpha && wave && gwave,
                 "synth: null argument");
  const int nb = D->n_my_batches_work, n_basis = D->n_basis;
  for (int f = 0; f < n_basis; ++f) {
    FRPA_CHECK_ARG(basis_l[f] >= 0 && basis_l[f] <= SY_LMAX && basis_m[f] >= -basis_l[f] && basis_m[f] <= basis_l[f],
                   "synth: basis function %d has unsupported (l, m)", f);
    FRPA_CHECK_ARG(basis_atom[f] >= 0 && basis_atom[f] < n_atoms, "synth: basis_atom[%d]", f);
  }
  std::vector<Mono> mono;
  std::vector<int> cnt;
  FRPA_TRY(build_monomials(&mono, &cnt));
  FRPA_CUDA_TRY(cudaMemcpyToSymbolAsync(c_mono, mono.data(), sizeof(Mono) * mono.size(), 0, cudaMemcpyHostToDevice, stream));
  FRPA_CUDA_TRY(cudaMemcpyToSymbolAsync(c_nmono, cnt.data(), sizeof(int) * cnt.size(), 0, cudaMemcpyHostToDevice, stream));
  std::vector<SynBatch> bt;
  std::vector<int> ibc;
  for (int b = 0; b < nb; ++b) {
    const int nc = D->n_compute_c_batches[b];
    if (nc <= 0) continue;
    FRPA_CHECK_ARG(nc <= D->n_centers_basis_I, "synth: n_compute_c exceeds n_centers_basis_I");
    bt.push_back(SynBatch{nc, D->n_point_batches[b], D->n_point_batches_prefix_sum[b], (int)ibc.size(),
                          (long long)D->i_batch_2_wave_offset[b]});
    const int *col = D->i_basis_batches + (long long)D->n_centers_basis_I * b;
    for (int i = 0; i < nc; ++i) {
      FRPA_CHECK_ARG(col[i] >= 1 && col[i] <= n_basis, "synth: i_basis_batches entry out of range");
      ibc.push_back(col[i]);
    }
  }
  if (bt.empty()) return FRPA_OK;
  std::vector<int> lm(n_basis);
  for (int f = 0; f < n_basis; ++f) lm[f] = basis_l[f] * basis_l[f] + basis_l[f] + basis_m[f];
  SynBatch *d_bt = nullptr;
  int *d_ib = nullptr, *d_atom = nullptr, *d_lm = nullptr;
  double *d_alpha = nullptr, *d_atoms = nullptr;
  int st = FRPA_OK;
  auto up = [&](void **dst, const void *src, size_t bytes) {
    if (st != FRPA_OK) return;
    if (cudaMalloc(dst, bytes) != cudaSuccess || cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      st = fail(FRPA_ERR_CUDA, "synth: upload failed");
  };
  up((void **)&d_bt, bt.data(), sizeof(SynBatch) * bt.size());
  up((void **)&d_ib, ibc.data(), sizeof(int) * ibc.size());
  up((void **)&d_atom, basis_atom, sizeof(int) * n_basis);
  up((void **)&d_lm, lm.data(), sizeof(int) * n_basis);
  up((void **)&d_alpha, basis_alpha, sizeof(double) * n_basis);
  up((void **)&d_atoms, atoms, sizeof(double) * 3 * n_atoms);
  if (st == FRPA_OK) {
    synth_kernel<<<std::min<int>((int)bt.size(), 148 * 8), 256, 0, stream>>>(
        (int)bt.size(), d_bt, d_ib, points, d_atoms, d_atom, d_lm, d_alpha, pad, wave, gwave);
    if (cudaGetLastError() != cudaSuccess) st = fail(FRPA_ERR_CUDA, "synth: launch failed");
    if (st == FRPA_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = fail(FRPA_ERR_CUDA, "synth: kernel failed");
  }
  cudaFree(d_bt);
  cudaFree(d_ib);
  cudaFree(d_atom);
  cudaFree(d_lm);
  cudaFree(d_alpha);
  cudaFree(d_atoms);
  return st;
}

namespace {

// splitmix64 finaliser: a counter-based hash of the entry's coordinates.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// out(i, j, t) = scale N(0,1)-like draw keyed by (seed, t, min(g_i, g_j),
// max(g_i, g_j)) with g the window's global basis indices: a symmetric P1
// whose entries do not depend on the window they are evaluated in
// (Box-Muller on two 53-bit uniforms from the hash).
__global__ void synth_p1_window_kernel(const int *__restrict__ gidx, int n, int T, double scale,
                                       unsigned long long seed, double *__restrict__ out) {
  const long long nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn * T;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / nn, r = e - t * nn;
    const int i = (int)(r % n), j = (int)(r / n);
    const unsigned long long a = (unsigned long long)min(gidx[i], gidx[j]);
    const unsigned long long b = (unsigned long long)max(gidx[i], gidx[j]);
    const unsigned long long h1 = mix64(seed ^ mix64(a * 0x100000001B3ull + b) ^ mix64((unsigned long long)t + 7));
    const unsigned long long h2 = mix64(h1 ^ 0xD1B54A32D192ED03ull);
    const double u1 = ((h1 >> 11) + 1) * 0x1.0p-53;  // (0, 1]
    const double u2 = (h2 >> 11) * 0x1.0p-53;
    out[e] = scale * sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}

}  // namespace

int synth_p1_window(const int *gidx, int n, int T, double scale, unsigned long long seed, double *out,
                    cudaStream_t stream) {
  FRPA_CHECK_ARG(gidx && out && n >= 0 && T >= 1, "synth P1 window: bad argument");
  if (n == 0) return FRPA_OK;
  const long long total = (long long)n * n * T;
  const int grid = (int)std::min<long long>((total + 255) / 256, 148 * 32);
  synth_p1_window_kernel<<<grid, 256, 0, stream>>>(gidx, n, T, scale, seed, out);
  if (cudaGetLastError() != cudaSuccess) return fail(FRPA_ERR_CUDA, "synth P1 window: launch failed");
  return FRPA_OK;
}

}  // namespace frpa
