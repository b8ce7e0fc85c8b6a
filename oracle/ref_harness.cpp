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
// initialize_particles (include/physics.hpp:34-97), is instantiated below with
// the oracle's restatement of the fit in GSL's place (ref_initialize_particles).
#define FIT_ALGORITHM_H
#include "init.hpp"
#include "physics.hpp"
#include "sim_structs.hpp"
#include "tools.hpp"

#include <cstdlib>
#include <cstring>
#include <omp.h>

#include "hv_oracle.h"

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

// compute_particle_energies (include/tools.hpp:226-232) into energy; ws = {V0,
// R12, a} of protons then neutrons.
#define REF_ENERGY(T, S)                                                                           \
    extern "C" void ref_particle_energies_##S(int protons, int neutrons, T *x, T *y, T *z, T *kx,  \
                                              T *ky, T *kz, const double *ws, double sigma_k,      \
                                              int zc, T *energy) {                                 \
        TestParticles<T> p = mk_part<T>(protons, neutrons, x, y, z, kx, ky, kz, 0, 0, 0);          \
        p.energy = energy;                                                                         \
        Parameters<T> pr = mk_param<T>(0.0, 1, zc, 0, 0.0);                                        \
        pr.sigma_k = T(sigma_k);                                                                   \
        WoodsSaxon<T> w[2];                                                                        \
        for (int s = 0; s < 2; s++) set_woods_saxon(&w[s], T(ws[3 * s]), T(ws[3 * s + 1]),         \
                                                    T(ws[3 * s + 2]));                             \
        compute_particle_energies(&p, w, pr);                                                      \
    }
REF_ENERGY(double, d)
REF_ENERGY(float, f)

// initialize_particles (include/physics.hpp:34-97), the reference's own loop,
// with its Woods-Saxon fit.  The reference's fit (minim_woods_saxon,
// include/fit_algorithm.hpp:95-137) calls GSL, which is absent; the overload
// below, found by argument-dependent lookup when initialize_particles is
// instantiated, runs the oracle's Levenberg-Marquardt restatement
// (orc_fit_woods_saxon) on the same residuals instead.  Everything else -- the
// rand() sampling, the energies, the Fermi-level update, the densities and the
// relaxation -- is the reference's code.
namespace {
int g_fit_calls = 0;
int g_fit_iters[2] = {0, 0}, g_fit_status[2] = {0, 0};
}  // namespace

inline int orc_fit(int n, const double *x, const double *y, const double *z, const double *dp, const double *dn,
                   int type, const orc_skyrme *s, double *ws, int *it) {
    return orc_fit_woods_saxon_d(n, x, y, z, dp, dn, type, s, ws, 100, 1e-4, 1e-4, it);
}
inline int orc_fit(int n, const float *x, const float *y, const float *z, const float *dp, const float *dn,
                   int type, const orc_skyrme *s, double *ws, int *it) {
    return orc_fit_woods_saxon_f(n, x, y, z, dp, dn, type, s, ws, 100, 1e-4, 1e-4, it);
}

template <typename T>
void minim_woods_saxon(TestParticles<T> *part, WoodsSaxon<T> *ws, Skyrme<T> skm) {
    g_fit_calls++;
    const orc_skyrme s = {double(skm.A), double(skm.B), double(skm.C), double(skm.gamma)};
    for (int type = 0; type <= 1; type++) {
        const int start = type == 0 ? 0 : part->protons;
        const int total = type == 0 ? part->protons : part->neutrons;
        double w[3] = {double(ws[type].V0), double(ws[type].R12), double(ws[type].a)};
        g_fit_status[type] = orc_fit(total, part->x + start, part->y + start, part->z + start,
                                     part->density_p + start, part->density_n + start, type, &s, w,
                                     &g_fit_iters[type]);
        ws[type].V0 = T(w[0]);
        ws[type].R12 = T(w[1]);
        ws[type].a = T(w[2]);
    }
}

// srand(seed), then initialize_particles with the parameters that
// read_input_file and set_parameters derive (include/init.hpp:44-58,326-336):
// r_max = 1.5 A^(1/3), max_test_part = max_particles(r_max, k_max, ppn).
// io: ws[6] = {V0, R12, a} x 2 (in: the start, R12 is taken as given), fermi[2];
// out: particles (protons * ppn ... as the reference orders them), their
// densities and energies, info[0] = loop passes, info[1..2] = iterations of
// the last fits, info[3..4] their status.
#define REF_INIT(T, S)                                                                             \
    extern "C" void ref_initialize_particles_##S(int z, int n, int ppn, double sigma_k,            \
                                                 double sigma_r, const double *skm, double *ws,    \
                                                 double *fermi, unsigned seed, T *x, T *y, T *zz,  \
                                                 T *kx, T *ky, T *kz, T *dp, T *dn, T *energy,     \
                                                 int *info) {                                      \
        Parameters<T> pr;                                                                          \
        std::memset(&pr, 0, sizeof(pr));                                                           \
        set_parameters(&pr, z, n, ppn, 1, 1, false, T(sigma_k), T(sigma_r), T(1), T(0), T(0));     \
        Skyrme<T> sk;                                                                              \
        set_skyrme(&sk, T(skm[0]), T(skm[1]), T(skm[2]), T(skm[3]));                               \
        WoodsSaxon<T> w[2];                                                                        \
        for (int s = 0; s < 2; s++) set_woods_saxon(&w[s], T(ws[3 * s]), T(ws[3 * s + 1]),         \
                                                    T(ws[3 * s + 2]));                             \
        Fermi<T> fl;                                                                               \
        set_fermi_levels(&fl, T(fermi[0]), T(fermi[1]));                                           \
        TestParticles<T> part;                                                                     \
        g_fit_calls = 0;                                                                           \
        std::srand(seed);                                                                          \
        initialize_particles(&part, w, sk, &fl, pr);                                               \
        const int total = part.protons + part.neutrons;                                            \
        std::memcpy(x, part.x, sizeof(T) * total);                                                 \
        std::memcpy(y, part.y, sizeof(T) * total);                                                 \
        std::memcpy(zz, part.z, sizeof(T) * total);                                                \
        std::memcpy(kx, part.kx, sizeof(T) * total);                                               \
        std::memcpy(ky, part.ky, sizeof(T) * total);                                               \
        std::memcpy(kz, part.kz, sizeof(T) * total);                                               \
        std::memcpy(dp, part.density_p, sizeof(T) * total);                                        \
        std::memcpy(dn, part.density_n, sizeof(T) * total);                                        \
        std::memcpy(energy, part.energy, sizeof(T) * total);                                       \
        for (int s = 0; s < 2; s++) {                                                              \
            ws[3 * s] = double(w[s].V0);                                                           \
            ws[3 * s + 1] = double(w[s].R12);                                                      \
            ws[3 * s + 2] = double(w[s].a);                                                        \
        }                                                                                          \
        fermi[0] = double(fl.epsilon_p);                                                           \
        fermi[1] = double(fl.epsilon_n);                                                           \
        info[0] = g_fit_calls;                                                                     \
        info[1] = g_fit_iters[0]; info[2] = g_fit_iters[1];                                        \
        info[3] = g_fit_status[0]; info[4] = g_fit_status[1];                                      \
        free_particles(&part);                                                                     \
    }
REF_INIT(double, d)
REF_INIT(float, f)

// max_test_part and r_max as set_parameters derives them (init.hpp:55-57).
extern "C" void ref_init_sizes(int z, int n, int ppn, double *r_max, int *max_test_part) {
    Parameters<double> pr;
    std::memset(&pr, 0, sizeof(pr));
    set_parameters(&pr, z, n, ppn, 1, 1, false, 0.1, 0.6, 1.0, 0.0, 0.0);
    *r_max = pr.r_max;
    *max_test_part = pr.max_test_part;
}

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
