// Stand-in for MAGMA's header, for compiling the reference's CPU sources
// only.  device.hpp (pulled in through sheval.hpp) includes magma_v2.h and
// names a few MAGMA types; no MAGMA routine is called on the CPU path.
// sheval.hpp also names CUDA's double2 in a function that the CPU path never
// calls, so a plain struct of the same shape is declared here.
#pragma once
typedef long long magma_int_t;
typedef void *magma_queue_t;
static inline const char *magma_strerror(magma_int_t) { return "magma stub"; }
struct double2 {
  double x, y;
};
