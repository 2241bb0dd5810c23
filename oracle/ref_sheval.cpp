// Exports the reference's own real spherical harmonics (SHEval_s in
// fast_rap_src_dfpt_gpu_eval/sheval.hpp:331-343, internal linkage there)
// under a C name, so the oracle's Y_lm restatement can be pinned against it.
// Compiled into oracle/_ref/ only.  Test infrastructure.
#include "sheval.hpp"
extern "C" void ref_sheval(int lmax, double sintheta, double costheta, double sinphi, double cosphi, double *out) {
  SHEval_s(lmax, sintheta, costheta, sinphi, cosphi, out);
}
