// Measured FP64 tensor-pipe ceiling for the roofline of the plain FP64 rho1
// path: a kernel that does nothing but independent m8n8k4 f64 MMAs on every
// SM, timed with CUDA events.  Measurement only; not on any compute path.
#include "frpa_internal.cuh"

namespace frpa {
namespace {

constexpr int PROBE_THREADS = 256;
constexpr int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(PROBE_THREADS) dmma_peak_kernel(int iters, double *out) {
  const double a = 1.0 + threadIdx.x * 1e-12, b = 1.0 - threadIdx.x * 1e-12;
  double c[PROBE_CHAINS][2];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) c[k][0] = c[k][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k) dmma_8x8x4(c[k][0], c[k][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += c[k][0] + c[k][1];
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(PROBE_THREADS) dfma_peak_kernel(int iters, double *out) {
  const double a = 1.0 + threadIdx.x * 1e-12, b = 1.0 - threadIdx.x * 1e-12;
  double c[PROBE_CHAINS];
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) c[k] = k * 1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; ++k) c[k] = fma(c[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PROBE_CHAINS; ++k) s += c[k];
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

}  // namespace
}  // namespace frpa

using namespace frpa;

static int probe(bool mma, double *tflops, void *stream_) {
  if (!tflops) return fail(FRPA_ERR_INVALID, "probe: null output");
  cudaStream_t stream = (cudaStream_t)stream_;
  int dev = 0, n_sm = 0;
  FRPA_CUDA_TRY(cudaGetDevice(&dev));
  FRPA_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  const int grid = n_sm * 8, iters = 4096;
  double *out = nullptr;
  FRPA_CUDA_TRY(cudaMalloc(&out, sizeof(double) * grid));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0, stream);
    if (mma)
      dmma_peak_kernel<<<grid, PROBE_THREADS, 0, stream>>>(iters, out);
    else
      dfma_peak_kernel<<<grid, PROBE_THREADS, 0, stream>>>(iters * 16, out);
    cudaEventRecord(e1, stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // first launch is a warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  FRPA_CUDA_TRY(cudaGetLastError());
  const double flops = mma ? (double)grid * (PROBE_THREADS / 32) * iters * PROBE_CHAINS * 512.0
                           : (double)grid * PROBE_THREADS * iters * 16.0 * PROBE_CHAINS * 2.0;
  *tflops = flops / (best * 1e-3) / 1e12;
  return FRPA_OK;
}

extern "C" int frpa_probe_fp64_mma_tflops(double *tflops, void *stream) { return probe(true, tflops, stream); }
extern "C" int frpa_probe_fp64_fma_tflops(double *tflops, void *stream) { return probe(false, tflops, stream); }
