/*
 * hv_oracle.c -- CPU restatement of the hyper-vlasov hot path.
 * TEST INFRASTRUCTURE ONLY (see hv_oracle.h): the checker, never the product.
 * Build: oracle/Makefile (gcc -std=c11 -O2 -ffp-contract=off -fopenmp).
 */
#define _POSIX_C_SOURCE 199309L
#include "hv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* wall clock in seconds */
static double orc_wtime(void) {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
#endif
}

/* std::numbers::pi_v<T> (used via pi<T>, include/sim_structs.hpp:37) */
#define ORC_PI 3.141592653589793238462643383279502884

#define R double
#define S d
#define EXPR(v) exp(v)
#define POWR(a, b) pow(a, b)
#define SQRTR(v) sqrt(v)
#define FABSR(v) fabs(v)
#include "hv_oracle_impl.h"
#undef R
#undef S
#undef EXPR
#undef POWR
#undef SQRTR
#undef FABSR

#define R float
#define S f
#define EXPR(v) expf(v)
#define POWR(a, b) powf(a, b)
#define SQRTR(v) sqrtf(v)
#define FABSR(v) fabsf(v)
#include "hv_oracle_impl.h"
#undef R
#undef S
#undef EXPR
#undef POWR
#undef SQRTR
#undef FABSR

#ifdef _OPENMP
#include <omp.h>
#endif
/* OpenMP thread count of the restatement (no effect without OpenMP). */
void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
