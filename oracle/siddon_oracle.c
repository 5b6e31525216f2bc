/*
 * siddon_oracle.c — CPU oracle for the Siddon projector.
 *
 * TEST INFRASTRUCTURE ONLY (see siddon_oracle_impl.h for what each routine
 * restates and which reference file:line it follows).  Built by
 * oracle/Makefile into oracle/_build/libsiddon_oracle.so with
 * -ffp-contract=off so that no multiply-add is fused unless the source asks
 * for it with FMA_.  Exported names carry _f32 (IEEE single, the reference's
 * arithmetic) or _f64 (the FP64 oracle) suffixes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* single precision */
#define REAL float
#define SUFFIX _f32
#define FMA_ fmaf
#define SQRT_ sqrtf
#define FABS_ fabsf
#define FMIN_ fminf
#define FMAX_ fmaxf
#define FLOOR_ floorf
#define CEIL_ ceilf
#define ROUND_ roundf
#define HYPOT_ hypotf
#define NEARBYINT_ nearbyintf
#define ISINF_(x) (isinf(x) != 0)
#include "siddon_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef FMA_
#undef SQRT_
#undef FABS_
#undef FMIN_
#undef FMAX_
#undef FLOOR_
#undef CEIL_
#undef ROUND_
#undef HYPOT_
#undef NEARBYINT_
#undef ISINF_

/* double precision (FP64 oracle) */
#define REAL double
#define SUFFIX _f64
#define FMA_ fma
#define SQRT_ sqrt
#define FABS_ fabs
#define FMIN_ fmin
#define FMAX_ fmax
#define FLOOR_ floor
#define CEIL_ ceil
#define ROUND_ round
#define HYPOT_ hypot
#define NEARBYINT_ nearbyint
#define ISINF_(x) (isinf(x) != 0)
#include "siddon_oracle_impl.h"

/* Threads the OpenMP runtime will use (1 when built without OpenMP). */
int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
