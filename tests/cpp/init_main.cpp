// The reference's initialisation call shape (src/hyper_vlasov.cpp:125-141)
// written against include/hv_b200.hpp: srand(seed), initialize_particles,
// then the final Woods-Saxon parameters, Fermi levels and particle arrays to
// a binary file.
//
//   init_main <out.bin> Z N ppn sigma_k sigma_r r_max max_test_part seed
//             A B C gamma V0p R12p ap V0n R12n an eps_p eps_n
#include <cstdio>
#include <cstdlib>

#include "hv_b200.hpp"

int main(int argc, char **argv) {
    if (argc != 22) {
        std::fprintf(stderr, "BAD ARGUMENTS!\n");
        return 1;
    }
    hvb200::Parameters<double> param{};
    param.z = std::atoi(argv[2]);
    param.n = std::atoi(argv[3]);
    param.part_per_nucleon = std::atoi(argv[4]);
    param.sigma_k = std::atof(argv[5]);
    param.sigma_r = std::atof(argv[6]);
    param.r_max = std::atof(argv[7]);
    param.max_test_part = std::atoi(argv[8]);
    const unsigned seed = (unsigned)std::atoi(argv[9]);
    hvb200::Skyrme<double> skm{std::atof(argv[10]), std::atof(argv[11]), std::atof(argv[12]), std::atof(argv[13])};
    hvb200::WoodsSaxon<double> ws[2] = {{std::atof(argv[14]), std::atof(argv[15]), std::atof(argv[16])},
                                        {std::atof(argv[17]), std::atof(argv[18]), std::atof(argv[19])}};
    hvb200::Fermi<double> fermi{std::atof(argv[20]), std::atof(argv[21])};
    hvb200::TestParticles<double> part{};
    std::srand(seed);
    hvb200::initialize_particles(&part, ws, skm, &fermi, param);
    FILE *out = std::fopen(argv[1], "wb");
    if (!out) return 1;
    const double head[8] = {ws[0].V0, ws[0].R12, ws[0].a, ws[1].V0, ws[1].R12, ws[1].a, fermi.epsilon_p,
                            fermi.epsilon_n};
    std::fwrite(head, sizeof(double), 8, out);
    const int total = part.protons + part.neutrons;
    double *arrays[9] = {part.x, part.y, part.z, part.kx, part.ky, part.kz, part.density_p, part.density_n,
                         part.energy};
    for (double *a : arrays) std::fwrite(a, sizeof(double), total, out);
    std::fclose(out);
    double *all[12] = {part.x, part.y, part.z, part.kx, part.ky, part.kz,
                       part.fx, part.fy, part.fz, part.energy, part.density_p, part.density_n};
    for (double *a : all) std::free(a);
    hvb200::release_contexts();
    return 0;
}
