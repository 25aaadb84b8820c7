/*
 * broccoli_oracle.c -- CPU oracle of BROCCOLI's registration and filtering
 * path (TEST INFRASTRUCTURE ONLY; never linked into the product).
 * The algorithm body lives in orc_impl.h and is instantiated here for float
 * (the FP32 parity target) and double (the FP64 accuracy oracle).
 */
#include "broccoli_oracle.h"

#include <math.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define REAL float
#define REAL_IS_FLOAT 1
#define SFX _f32
#include "orc_impl.h"
#undef REAL
#undef REAL_IS_FLOAT
#undef SFX

#define REAL double
#define REAL_IS_FLOAT 0
#define SFX _f64
#include "orc_impl.h"
#undef REAL
#undef REAL_IS_FLOAT
#undef SFX

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Threads of the following OpenMP regions (the process's OpenMP runtime is
 * shared with the reference-kernel build, so this also sets its count). */
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
