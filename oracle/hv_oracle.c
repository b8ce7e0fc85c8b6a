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

/* ---- seeded synthetic nucleus -------------------------------------------
 * The inputs of every workload: positions uniform in the open ball of
 * `radius`, wavenumbers uniform in the open ball of `k_fermi`, protons first,
 * all positions drawn before all wavenumbers.  Each uniform is the top 53 bits
 * of one MT19937-64 output times 2^-53, and a coordinate is r (2 u - 1), with
 * rejection of triples outside the ball.  This restates the generator the
 * CUDA library's host side uses (its hv_generate_nucleus_*), so that the CPU
 * baseline and the checks get their inputs without loading the product.
 *
 * MT19937-64 is Matsumoto and Nishimura's 64-bit Mersenne Twister (Nishimura,
 * ACM TOMACS 10 (2000) 348-357), the engine std::mt19937_64 of the C++
 * standard library: degree 312, middle word 156, 31 lower bits in the split
 * word, and its published twist and tempering constants. */
#include <stdint.h>

typedef struct orc_mt64 {
    uint64_t mt[312];
    int i;
} orc_mt64;

static void orc_mt64_seed(orc_mt64 *s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; i++)
        s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    s->i = 312;
}

static uint64_t orc_mt64_next(orc_mt64 *s) {
    if (s->i >= 312) {
        for (int k = 0; k < 312; k++) {
            const uint64_t y = (s->mt[k] & 0xFFFFFFFF80000000ULL) | (s->mt[(k + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t v = s->mt[(k + 156) % 312] ^ (y >> 1);
            if (y & 1u) v ^= 0xB5026F5AA96619E9ULL;
            s->mt[k] = v;
        }
        s->i = 0;
    }
    uint64_t x = s->mt[s->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

uint64_t orc_mt64_nth(uint64_t seed, long long n) {
    orc_mt64 s;
    orc_mt64_seed(&s, seed);
    uint64_t v = 0;
    for (long long i = 0; i < n; i++) v = orc_mt64_next(&s);
    return v;
}

static double orc_sym(orc_mt64 *s, double r) {
    const double u = (double)(orc_mt64_next(s) >> 11) * 0x1.0p-53;
    return r * (2.0 * u - 1.0);
}

/* fills xyz[0..2][0..total) with draws in the ball of radius r */
static void orc_ball(orc_mt64 *s, long total, double r, double *a, double *b, double *c) {
    const double r2 = r * r;
    for (long i = 0; i < total; i++) {
        double u, v, w;
        do {
            u = orc_sym(s, r);
            v = orc_sym(s, r);
            w = orc_sym(s, r);
        } while (u * u + v * v + w * w >= r2);
        a[i] = u;
        b[i] = v;
        c[i] = w;
    }
}

int orc_generate_nucleus_d(uint64_t seed, int protons, int neutrons, double radius, double k_fermi, double *x,
                           double *y, double *z, double *kx, double *ky, double *kz) {
    if (protons < 0 || neutrons < 0 || !(radius > 0.0) || !(k_fermi > 0.0)) return 1;
    const long total = (long)protons + neutrons;
    orc_mt64 *s = (orc_mt64 *)malloc(sizeof(orc_mt64));
    if (!s) return 1;
    orc_mt64_seed(s, seed);
    orc_ball(s, total, radius, x, y, z);
    orc_ball(s, total, k_fermi, kx, ky, kz);
    free(s);
    return 0;
}

int orc_generate_nucleus_f(uint64_t seed, int protons, int neutrons, double radius, double k_fermi, float *x,
                           float *y, float *z, float *kx, float *ky, float *kz) {
    if (protons < 0 || neutrons < 0) return 1;
    const long total = (long)protons + neutrons;
    double *tmp = (double *)malloc(sizeof(double) * 6 * (size_t)(total > 0 ? total : 1));
    if (!tmp) return 1;
    const int st = orc_generate_nucleus_d(seed, protons, neutrons, radius, k_fermi, tmp, tmp + total,
                                          tmp + 2 * total, tmp + 3 * total, tmp + 4 * total, tmp + 5 * total);
    float *out[6] = {x, y, z, kx, ky, kz};
    for (int a = 0; st == 0 && a < 6; a++)
        for (long i = 0; i < total; i++) out[a][i] = (float)tmp[a * total + i];
    free(tmp);
    return st;
}
