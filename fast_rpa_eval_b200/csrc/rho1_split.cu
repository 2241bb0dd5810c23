// Split-precision rho1 contraction (placeholder until the tcgen05 kernel lands).
#include "frpa_internal.cuh"

namespace frpa {

int rho1_split_launch(const Rho1Plan &plan, int n_active, const double *wave, const double *gwave,
                      const double *P1, const double *bias, const double *gbias, double *rho, double *grad,
                      cudaStream_t stream) {
  (void)plan; (void)n_active; (void)wave; (void)gwave; (void)P1; (void)bias; (void)gbias; (void)rho; (void)grad;
  (void)stream;
  return fail(FRPA_ERR_UNSUPPORTED, "rho1: split-BF16 mode not built yet");
}

}  // namespace frpa
