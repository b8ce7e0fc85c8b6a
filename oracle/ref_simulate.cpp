// ref_simulate.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The cpu_simulate loop (src/hyper_vlasov.cpp:32-104) driven by the
// reference's own routines, without the VTK and stats.txt I/O, for golden
// vectors and for the timed CPU baseline.  The smoothing call can be the
// reference's O(G^2) compute_volumetric_densities (include/physics.hpp:202-234)
// or the offset-table restatement from hv_oracle.c (identical pair set; the
// O(G^2) form is infeasible beyond ~48^3).
#define FIT_ALGORITHM_H
#include "physics.hpp"
#include "sim_structs.hpp"
#include "tools.hpp"

#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <vector>

#include "hv_oracle.h"

namespace {

template <typename T> struct OrcSmooth;
template <> struct OrcSmooth<double> {
    static void run(const orc_world *w, double s, int ppn, double *r, double *t) { orc_smooth_d(w, s, ppn, r, t); }
};
template <> struct OrcSmooth<float> {
    static void run(const orc_world *w, double s, int ppn, float *r, float *t) { orc_smooth_f(w, s, ppn, r, t); }
};

// One row per step: t, rms_p, rms_n, zcm_p, zcm_n (src/hyper_vlasov.cpp:66-70).
// step_seconds (may be null): [0] the initial field solve, [1 + s] step s.
template <typename T>
double simulate(const int *n, const double *dm, int protons, int neutrons, T *x, T *y, T *z, T *kx,
                T *ky, T *kz, double sigma_r, int ppn, int Z, int N, double A, double B, double C,
                double gamma, double dt_d, double t_exc, double eta, int steps, int smooth_mode,
                double *rows, T *fields_out, double *step_seconds) {
    World<T> world;
    orc_world ow;
    for (int a = 0; a < 3; a++) {
        world.n[a] = n[a];
        world.d_max[a] = T(dm[a]);
        ow.n[a] = n[a];
        ow.d_max[a] = dm[a];
    }
    const long G = (long)n[0] * n[1] * n[2];
    const int total = protons + neutrons;
    std::vector<T> fx(total > 0 ? total : 1), fy(total > 0 ? total : 1), fz(total > 0 ? total : 1);
    TestParticles<T> part;
    std::memset(&part, 0, sizeof(part));
    part.protons = protons;
    part.neutrons = neutrons;
    part.x = x; part.y = y; part.z = z;
    part.kx = kx; part.ky = ky; part.kz = kz;
    part.fx = fx.data(); part.fy = fy.data(); part.fz = fz.data();
    Parameters<T> param;
    std::memset(&param, 0, sizeof(param));
    param.sigma_r = T(sigma_r);
    param.part_per_nucleon = ppn;
    param.z = Z;
    param.n = N;
    param.eta_exc = T(eta);
    param.t_exc = T(t_exc);
    param.steps = steps;
    Skyrme<T> skm{T(A), T(B), T(C), T(gamma)};
    const T dt = T(dt_d);
    bool excited_nucleus = false;

    std::vector<T> fxg(2 * G, T(0)), fyg(2 * G, T(0)), fzg(2 * G, T(0)), coul(G, T(0)), dens(2 * G, T(0)),
        pot(2 * G, T(0)), tmpd(2 * G, T(0));
    VectorField<T> forces{fxg.data(), fyg.data(), fzg.data()};
    ScalarField<T> potentials{pot.data()}, coulomb{coul.data()}, temp_density{tmpd.data()}, density{dens.data()};

    auto smooth = [&]() {
        if (smooth_mode == 0)
            compute_volumetric_densities(&density, &temp_density, param, world);
        else
            OrcSmooth<T>::run(&ow, sigma_r, ppn, density.v, temp_density.v);
    };

    double t0 = omp_get_wtime();
    distribute_volumetric_particles_cic(&density, &part, world);
    smooth();
    set_initial_coulomb_boundaries(&coulomb, world, Z);
    compute_volumetric_skyrme_potentials(&potentials, density, skm, world);
    compute_volumetric_coulomb_potentials_sor(&coulomb, density, world);
    merge_volumetric_potentials(&potentials, coulomb, world);
    compute_volumetric_forces_fdm(&forces, potentials, world);
    distribute_forces_to_particles_cic(&part, forces, world);
    double t_init = omp_get_wtime() - t0;
    if (step_seconds) step_seconds[0] = t_init;
    for (int step = 0; step < steps; step++) {
        double ts = omp_get_wtime();
        if (rows) {
            T x_p = center_of_mass(part, PROTONS);
            T x_n = center_of_mass(part, NEUTRONS);
            T msr_p = mean_squared_radius(part, world, PROTONS);
            T msr_n = mean_squared_radius(part, world, NEUTRONS);
            rows[5 * step + 0] = (double)(step * dt);
            rows[5 * step + 1] = (double)std::sqrt(msr_p);
            rows[5 * step + 2] = (double)std::sqrt(msr_n);
            rows[5 * step + 3] = (double)x_p;
            rows[5 * step + 4] = (double)x_n;
        }
        if (step * dt >= param.t_exc && !excited_nucleus) {
            excited_nucleus = true;
            nuclear_excitation(&part, param);
        }
        update_momenta_half(&part, dt);
        update_positions_full(&part, dt);
        distribute_volumetric_particles_cic(&density, &part, world);
        smooth();
        compute_volumetric_skyrme_potentials(&potentials, density, skm, world);
        compute_volumetric_coulomb_potentials_sor(&coulomb, density, world);
        merge_volumetric_potentials(&potentials, coulomb, world);
        compute_volumetric_forces_fdm(&forces, potentials, world);
        distribute_forces_to_particles_cic(&part, forces, world);
        update_momenta_half(&part, dt);
        if (step_seconds) step_seconds[1 + step] = omp_get_wtime() - ts;
    }
    double elapsed = omp_get_wtime() - t0;
    if (fields_out) {  // rho(2G) U(2G) phi(G) Fx(2G) Fy(2G) Fz(2G)
        std::memcpy(fields_out, dens.data(), sizeof(T) * 2 * G);
        std::memcpy(fields_out + 2 * G, pot.data(), sizeof(T) * 2 * G);
        std::memcpy(fields_out + 4 * G, coul.data(), sizeof(T) * G);
        std::memcpy(fields_out + 5 * G, fxg.data(), sizeof(T) * 2 * G);
        std::memcpy(fields_out + 7 * G, fyg.data(), sizeof(T) * 2 * G);
        std::memcpy(fields_out + 9 * G, fzg.data(), sizeof(T) * 2 * G);
    }
    return elapsed;
}

}  // namespace

#define REF_SIM(T, S)                                                                               \
    extern "C" double ref_simulate_##S(const int *n, const double *dm, int protons, int neutrons,   \
                                       T *x, T *y, T *z, T *kx, T *ky, T *kz, double sigma_r,       \
                                       int ppn, int Z, int N, double A, double B, double C,         \
                                       double gamma, double dt, double t_exc, double eta,           \
                                       int steps, int smooth_mode, double *rows, T *fields_out,     \
                                       double *step_seconds) {                                      \
        return simulate<T>(n, dm, protons, neutrons, x, y, z, kx, ky, kz, sigma_r, ppn, Z, N, A, B, \
                           C, gamma, dt, t_exc, eta, steps, smooth_mode, rows, fields_out,          \
                           step_seconds);                                                           \
    }

REF_SIM(double, d)
REF_SIM(float, f)
