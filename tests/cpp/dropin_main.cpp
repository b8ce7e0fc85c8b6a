// Drives the reference's cpu_simulate step order (src/hyper_vlasov.cpp:53-103)
// through hv_b200.hpp -- the same calls the reference makes, in the same
// order, on the same struct layouts -- and then the gpu_simulate slot.
//
//   dropin_main <steps> <output_dir>
//
// Prints one line per step "t zcm_p zcm_n rms_p rms_n" (observed where the
// reference records them), then "final <sum of x> <sum of kz>", then the
// path of the stats.txt written by gpu_simulate.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hv_b200.hpp"

using namespace hvb200;

int main(int argc, char **argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 5;
    const char *outdir = argc > 2 ? argv[2] : ".";
    // 40Ca, 100 test particles per nucleon, 32^3 grid with h = 1 fm
    const int Z = 20, N = 20, ppn = 100, P = Z * ppn, Nn = N * ppn, total = P + Nn;
    std::vector<double> x(total), y(total), z(total), kx(total), ky(total), kz(total), fx(total), fy(total),
        fz(total), energy(total), dp(total), dn(total);
    const double radius = 1.2 * std::cbrt(40.0), kf = std::cbrt(3.0 * M_PI * M_PI * 0.08 / 2.0);
    if (hv_generate_nucleus_f64(0, P, Nn, radius, kf, x.data(), y.data(), z.data(), kx.data(), ky.data(),
                                kz.data()) != HV_OK)
        return 2;
    TestParticles<double> part{P, Nn, x.data(), y.data(), z.data(), kx.data(), ky.data(), kz.data(),
                               energy.data(), dp.data(), dn.data(), fx.data(), fy.data(), fz.data()};
    World<double> world{{32, 32, 32}, {16.0, 16.0, 16.0}};
    Parameters<double> param{};
    param.sigma_r = 1.444 / (2.0 * std::sqrt(2.0 * std::log(2.0)));
    param.part_per_nucleon = ppn;
    param.z = Z;
    param.n = N;
    param.eta_exc = 30.0 / 197.33;
    param.t_exc = 0.0;
    param.steps = steps;
    param.substeps = 1;
    param.t_f = 0.5 * steps;
    hv_skyrme hk;
    hv_skyrme_from_t0t3(-2645.0, 15595.0, 1.0 / 6.0, 32.0, &hk);
    Skyrme<double> skm{hk.A, hk.B, hk.C, hk.gamma};
    const double dt = param.t_f / param.steps;
    const size_t G = 32 * 32 * 32;
    std::vector<double> fxg(2 * G), fyg(2 * G), fzg(2 * G), coul(G, 0.0), dens(2 * G), pot(2 * G), tmp(2 * G);
    VectorField<double> forces{fxg.data(), fyg.data(), fzg.data()};
    ScalarField<double> potentials{pot.data()}, coulomb{coul.data()}, temp_density{tmp.data()}, density{dens.data()};

    // initial solve (src/hyper_vlasov.cpp:53-62)
    distribute_volumetric_particles_cic(&density, &part, world);
    compute_volumetric_densities(&density, &temp_density, param, world);
    set_initial_coulomb_boundaries(&coulomb, world, param.z);
    compute_volumetric_skyrme_potentials(&potentials, density, skm, world);
    compute_volumetric_coulomb_potentials_sor(&coulomb, density, world);
    merge_volumetric_potentials(&potentials, coulomb, world);
    compute_volumetric_forces_fdm(&forces, potentials, world);
    distribute_forces_to_particles_cic(&part, forces, world);
    bool excited = false;
    for (int step = 0; step < steps; step++) {  // src/hyper_vlasov.cpp:63-104
        double xp = center_of_mass(part, PROTONS), xn = center_of_mass(part, NEUTRONS);
        double mp = mean_squared_radius(part, world, PROTONS), mn = mean_squared_radius(part, world, NEUTRONS);
        std::printf("%.17g %.17g %.17g %.17g %.17g\n", step * dt, xp, xn, std::sqrt(mp), std::sqrt(mn));
        if (step * dt >= param.t_exc && !excited) {
            excited = true;
            nuclear_excitation(&part, param);
        }
        update_momenta_half(&part, dt);
        update_positions_full(&part, dt);
        distribute_volumetric_particles_cic(&density, &part, world);
        compute_volumetric_densities(&density, &temp_density, param, world);
        compute_volumetric_skyrme_potentials(&potentials, density, skm, world);
        compute_volumetric_coulomb_potentials_sor(&coulomb, density, world);
        merge_volumetric_potentials(&potentials, coulomb, world);
        compute_volumetric_forces_fdm(&forces, potentials, world);
        distribute_forces_to_particles_cic(&part, forces, world);
        update_momenta_half(&part, dt);
    }
    double sx = 0.0, skz = 0.0;
    for (int i = 0; i < total; i++) {
        sx += x[i];
        skz += kz[i];
    }
    std::printf("final %.17g %.17g\n", sx, skz);

    // the gpu_simulate slot on a fresh copy of the initial nucleus
    hv_generate_nucleus_f64(0, P, Nn, radius, kf, x.data(), y.data(), z.data(), kx.data(), ky.data(), kz.data());
    gpu_simulate(outdir, &part, skm, param, world);
    std::printf("stats %s/stats.txt\n", outdir);
    release_contexts();
    return 0;
}
