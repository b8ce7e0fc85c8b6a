// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own step routines, compiled unmodified from the
// reference tree's include/ directory, behind extern "C" wrappers so that the
// tests can pin the C restatement (hv_oracle.c) against them and so that the
// CPU baseline can time them.  Nothing here is part of the product library.
//
// Build: oracle/Makefile target `ref` (needs the reference tree; writes only
// into oracle/_ref/).  FIT_ALGORITHM_H is predefined so that physics.hpp skips
// include/fit_algorithm.hpp (GSL, absent here); its only user,
// initialize_particles (include/physics.hpp:34-97), is a template that is
// never instantiated below.
#define FIT_ALGORITHM_H
#include "init.hpp"
#include "physics.hpp"
#include "sim_structs.hpp"
#include "tools.hpp"

#include <cstring>
#include <omp.h>

namespace {

template <typename T>
World<T> mk_world(const int *n, const double *d_max) {
    World<T> w;
    for (int a = 0; a < 3; a++) {
        w.n[a] = n[a];
        w.d_max[a] = T(d_max[a]);
    }
    return w;
}

template <typename T>
TestParticles<T> mk_part(int protons, int neutrons, T *x, T *y, T *z, T *kx, T *ky, T *kz, T *fx,
                         T *fy, T *fz) {
    TestParticles<T> p;
    std::memset(&p, 0, sizeof(p));
    p.protons = protons;
    p.neutrons = neutrons;
    p.x = x; p.y = y; p.z = z;
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.fx = fx; p.fy = fy; p.fz = fz;
    return p;
}

template <typename T>
Parameters<T> mk_param(double sigma_r, int ppn, int z, int n, double eta) {
    Parameters<T> p;
    std::memset(&p, 0, sizeof(p));
    p.sigma_r = T(sigma_r);
    p.part_per_nucleon = ppn;
    p.z = z;
    p.n = n;
    p.eta_exc = T(eta);
    return p;
}

}  // namespace

#define REF_API(T, S)                                                                              \
    extern "C" void ref_deposit_##S(const int *n, const double *dm, int protons, int neutrons,     \
                                    T *x, T *y, T *z, T *rho) {                                    \
        World<T> w = mk_world<T>(n, dm);                                                           \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, 0, 0, 0, 0, 0, 0);             \
        ScalarField<T> f{rho};                                                                     \
        distribute_volumetric_particles_cic(&f, &p, w);                                            \
    }                                                                                              \
    extern "C" void ref_smooth_##S(const int *n, const double *dm, double sigma_r, int ppn,        \
                                   T *rho, T *tmp) {                                               \
        World<T> w = mk_world<T>(n, dm);                                                           \
        Parameters<T> pr = mk_param<T>(sigma_r, ppn, 0, 0, 0.0);                                   \
        ScalarField<T> d{rho}, t{tmp};                                                             \
        compute_volumetric_densities(&d, &t, pr, w);                                               \
    }                                                                                              \
    extern "C" void ref_skyrme_##S(const int *n, const double *dm, double A, double B, double C,   \
                                   double gamma, T *rho, T *U) {                                   \
        World<T> w = mk_world<T>(n, dm);                                                           \
        Skyrme<T> s{T(A), T(B), T(C), T(gamma)};                                                   \
        ScalarField<T> d{rho}, u{U};                                                               \
        compute_volumetric_skyrme_potentials(&u, d, s, w);                                         \
    }                                                                                              \
    extern "C" void ref_boundary_##S(const int *n, const double *dm, int z, T *phi) {              \
        World<T> w = mk_world<T>(n, dm);                                                           \
        ScalarField<T> c{phi};                                                                     \
        set_initial_coulomb_boundaries(&c, w, z);                                                  \
    }                                                                                              \
    extern "C" void ref_sor_##S(const int *n, const double *dm, T *phi, T *rho) {                  \
        World<T> w = mk_world<T>(n, dm);                                                           \
        ScalarField<T> c{phi}, d{rho};                                                             \
        compute_volumetric_coulomb_potentials_sor(&c, d, w);                                       \
    }                                                                                              \
    extern "C" void ref_merge_##S(const int *n, const double *dm, T *U, T *phi) {                  \
        World<T> w = mk_world<T>(n, dm);                                                           \
        ScalarField<T> u{U}, c{phi};                                                               \
        merge_volumetric_potentials(&u, c, w);                                                     \
    }                                                                                              \
    extern "C" void ref_fdm_##S(const int *n, const double *dm, T *U, T *Fx, T *Fy, T *Fz) {       \
        World<T> w = mk_world<T>(n, dm);                                                           \
        ScalarField<T> u{U};                                                                       \
        VectorField<T> f{Fx, Fy, Fz};                                                              \
        compute_volumetric_forces_fdm(&f, u, w);                                                   \
    }                                                                                              \
    extern "C" void ref_gather_##S(const int *n, const double *dm, int protons, int neutrons,      \
                                   T *x, T *y, T *z, T *Fx, T *Fy, T *Fz, T *fx, T *fy, T *fz) {   \
        World<T> w = mk_world<T>(n, dm);                                                           \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, 0, 0, 0, fx, fy, fz);          \
        VectorField<T> f{Fx, Fy, Fz};                                                              \
        distribute_forces_to_particles_cic(&p, f, w);                                              \
    }                                                                                              \
    extern "C" void ref_kick_half_##S(int protons, int neutrons, T *kx, T *ky, T *kz, T *fx,       \
                                      T *fy, T *fz, double dt) {                                   \
        TestParticles<T> p = mk_part<T>(protons, neutrons, 0, 0, 0, kx, ky, kz, fx, fy, fz);       \
        update_momenta_half(&p, T(dt));                                                            \
    }                                                                                              \
    extern "C" void ref_drift_##S(int protons, int neutrons, T *x, T *y, T *z, T *kx, T *ky,       \
                                  T *kz, double dt) {                                              \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, kx, ky, kz, 0, 0, 0);          \
        update_positions_full(&p, T(dt));                                                          \
    }                                                                                              \
    extern "C" void ref_excite_##S(int protons, int neutrons, T *kz, int Z, int N, double eta) {   \
        TestParticles<T> p = mk_part<T>(protons, neutrons, 0, 0, 0, 0, 0, kz, 0, 0, 0);            \
        Parameters<T> pr = mk_param<T>(0.0, 1, Z, N, eta);                                         \
        nuclear_excitation(&p, pr);                                                                \
    }                                                                                              \
    extern "C" double ref_center_of_mass_##S(int protons, int neutrons, T *z, int species) {       \
        TestParticles<T> p = mk_part<T>(protons, neutrons, 0, 0, z, 0, 0, 0, 0, 0, 0);             \
        return (double)center_of_mass(p, species);                                                 \
    }                                                                                              \
    extern "C" double ref_mean_squared_radius_##S(const int *n, const double *dm, int protons,     \
                                                  int neutrons, T *x, T *y, T *z, int species) {   \
        World<T> w = mk_world<T>(n, dm);                                                           \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, 0, 0, 0, 0, 0, 0);             \
        return (double)mean_squared_radius(p, w, species);                                         \
    }

REF_API(double, d)
REF_API(float, f)

// compute_particle_densities (include/tools.hpp:170-203) into dp, dn.
#define REF_PDENS(T, S)                                                                            \
    extern "C" void ref_particle_densities_##S(int protons, int neutrons, T *x, T *y, T *z,        \
                                               double sigma_r, int ppn, T *dp, T *dn) {            \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, 0, 0, 0, 0, 0, 0);             \
        p.density_p = dp;                                                                          \
        p.density_n = dn;                                                                          \
        Parameters<T> pr = mk_param<T>(sigma_r, ppn, 0, 0, 0.0);                                   \
        compute_particle_densities(&p, pr);                                                        \
    }
REF_PDENS(double, d)
REF_PDENS(float, f)

// OpenMP thread count of the reference routines (1 gives the reproducible
// particle-order summation of the deposit's array reduction, tools.hpp:45).
extern "C" void ref_set_threads(int n) { omp_set_num_threads(n); }
extern "C" int ref_get_threads(void) { return omp_get_max_threads(); }

// The reference's VTK frame writer (include/init.hpp:159-254) in the order of
// src/hyper_vlasov.cpp:79-82: header, forces, density, potentials.
#define REF_VTK(T, S)                                                                                \
    extern "C" int ref_write_vtk_##S(const char *path, const int *n, const double *dm, T *Fx, T *Fy, \
                                     T *Fz, T *rho, T *U) {                                          \
        World<T> w = mk_world<T>(n, dm);                                                             \
        FILE *out = std::fopen(path, "wb");                                                          \
        if (!out) return 1;                                                                          \
        VectorField<T> f{Fx, Fy, Fz};                                                                \
        ScalarField<T> d{rho}, u{U};                                                                 \
        output_vtk_header_start(out, w);                                                             \
        output_vector_field(out, f, w, "forces");                                                    \
        output_scalar_field(out, d, w, "density");                                                   \
        output_scalar_field(out, u, w, "potentials");                                                \
        std::fclose(out);                                                                            \
        return 0;                                                                                    \
    }
REF_VTK(double, d)
REF_VTK(float, f)
