// Seeded synthetic nucleus and parameter helpers (host code).
//
// The reference initialises particles with a Woods-Saxon self-consistency loop
// driven by rand() and a GSL fit (include/physics.hpp:34-97,
// include/tools.hpp:234-254).  That loop is not part of the step; the
// synthetic generator below stands in for it so that the GPU path and the
// oracle start from identical, reproducible inputs.
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "hv_b200.h"

namespace {

constexpr double kRho0 = 0.16;  // rho_0 (include/sim_structs.hpp:34)

struct Uniform {
    std::mt19937_64 eng;
    explicit Uniform(uint64_t seed) : eng(seed) {}
    // 53 random bits -> [0, 1)
    double next() { return static_cast<double>(eng() >> 11) * 0x1.0p-53; }
    // uniform in [-r, r)
    double sym(double r) { return r * (2.0 * next() - 1.0); }
};

template <typename T>
hv_status generate(uint64_t seed, int protons, int neutrons, double radius, double k_fermi,
                   T *x, T *y, T *z, T *kx, T *ky, T *kz) {
    if (protons < 0 || neutrons < 0 || !(radius > 0.0) || !(k_fermi > 0.0))
        return HV_ERR_BAD_ARG;
    const long total = static_cast<long>(protons) + neutrons;
    if (total > 0 && (!x || !y || !z || !kx || !ky || !kz)) return HV_ERR_BAD_ARG;
    Uniform u(seed);
    const double r2 = radius * radius;
    for (long i = 0; i < total; ++i) {
        double a, b, c;
        do {
            a = u.sym(radius);
            b = u.sym(radius);
            c = u.sym(radius);
        } while (a * a + b * b + c * c >= r2);
        x[i] = static_cast<T>(a);
        y[i] = static_cast<T>(b);
        z[i] = static_cast<T>(c);
    }
    const double k2 = k_fermi * k_fermi;
    for (long i = 0; i < total; ++i) {
        double a, b, c;
        do {
            a = u.sym(k_fermi);
            b = u.sym(k_fermi);
            c = u.sym(k_fermi);
        } while (a * a + b * b + c * c >= k2);
        kx[i] = static_cast<T>(a);
        ky[i] = static_cast<T>(b);
        kz[i] = static_cast<T>(c);
    }
    return HV_OK;
}

}  // namespace

extern "C" {

void hv_sor_reference_defaults(hv_sor_params *p) {
    if (!p) return;
    p->omega = 1.5;
    p->tol = 1e-4;
    p->criterion = HV_SOR_MAX_UPDATE;
    p->max_iter = 512;
}

void hv_skyrme_from_t0t3(double t0, double t3, double sigma, double a_sym, hv_skyrme *out) {
    if (!out) return;
    out->A = 0.75 * t0 * kRho0;
    out->B = (sigma + 2.0) / 16.0 * t3 * std::pow(kRho0, sigma + 1.0);
    out->gamma = sigma + 1.0;
    out->C = a_sym;
}

hv_status hv_generate_nucleus_f64(uint64_t seed, int protons, int neutrons, double radius,
                                  double k_fermi, double *x, double *y, double *z, double *kx,
                                  double *ky, double *kz) {
    return generate<double>(seed, protons, neutrons, radius, k_fermi, x, y, z, kx, ky, kz);
}

hv_status hv_generate_nucleus_f32(uint64_t seed, int protons, int neutrons, double radius,
                                  double k_fermi, float *x, float *y, float *z, float *kx,
                                  float *ky, float *kz) {
    return generate<float>(seed, protons, neutrons, radius, k_fermi, x, y, z, kx, ky, kz);
}

}  // extern "C"
