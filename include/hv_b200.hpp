// hv_b200.hpp -- C++ drop-in for the reference's step routines.
//
// The reference (BanuDarius/hyper-vlasov) exposes its step as function
// templates over the POD structs of include/sim_structs.hpp, operating on
// host memory, called in a fixed order by cpu_simulate
// (src/hyper_vlasov.cpp:32-118).  This header provides the same templates,
// with the same names, argument roles and struct layouts, in namespace
// hvb200; each call runs the routine on the GPU through the C ABI of
// hv_b200.h (host -> device copy, kernel, device -> host copy).  It also fills
// the reference's empty gpu_simulate slot (src/hyper_vlasov.cpp:120-123) with
// a device-resident run that writes the reference's stats.txt.
//
// Errors follow the reference: a failure prints a message to stderr and
// calls exit(1) (as include/init.hpp:94-96 does); define
// HVB200_THROW_ON_ERROR before including this header to get hvb200::error
// exceptions instead.  A non-converged SOR prints the reference's warning
// "SOR COULOMB DID NOT CONVERGE!" (include/physics.hpp:155-156) and carries on.
//
// Device contexts are cached per thread and per (world, particle counts,
// precision); they are released by hvb200::release_contexts() or at thread
// exit.
#ifndef HV_B200_HPP
#define HV_B200_HPP

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "hv_b200.h"

namespace hvb200 {

// ---- the reference's structs (include/sim_structs.hpp:48-91), same layout ----
template <typename T>
struct Parameters {
    bool use_gpu;
    T sigma_k, sigma_r, r_max, t_f, t_exc, eta_exc, d_max_scale;
    int part_per_nucleon, max_test_part, substeps, steps, z, n;
};

template <typename T>
struct TestParticles {
    int protons, neutrons;
    T *x, *y, *z, *kx, *ky, *kz;
    T *energy, *density_p, *density_n, *fx, *fy, *fz;
};

template <typename T>
struct ScalarField {
    T *v;
};

template <typename T>
struct VectorField {
    T *x, *y, *z;
};

template <typename T>
struct World {
    int n[3];
    T d_max[3];
};

template <typename T>
struct Skyrme {
    T A, B, C, gamma;
};

template <typename T>
struct WoodsSaxon {
    T V0, R12, a;
};

template <typename T>
struct Fermi {
    T epsilon_p, epsilon_n;
};

constexpr int PROTONS = 0;   // include/sim_structs.hpp:28
constexpr int NEUTRONS = 1;  // include/sim_structs.hpp:29

struct error : std::runtime_error {
    hv_status status;
    error(hv_status s, const std::string &where)
        : std::runtime_error(where + ": " + hv_status_string(s) + " " + hv_last_error()), status(s) {}
};

namespace detail {

inline void fail(hv_status s, const char *where) {
#ifdef HVB200_THROW_ON_ERROR
    throw error(s, where);
#else
    std::fprintf(stderr, "%s: %s %s\n", where, hv_status_string(s), hv_last_error());
    std::exit(1);
#endif
}

inline void check(hv_status s, const char *where) {
    if (s != HV_OK) fail(s, where);
}

template <typename T>
constexpr hv_precision prec() {
    static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value, "T must be float or double");
    return std::is_same<T, double>::value ? HV_F64 : HV_F32;
}

template <typename T>
hv_world to_world(const World<T> &w) {
    hv_world o;
    for (int a = 0; a < 3; a++) {
        o.n[a] = w.n[a];
        o.d_max[a] = (double)w.d_max[a];
    }
    return o;
}

// Run parameters that the routines do not take from their arguments.
inline hv_run_params base_params() {
    hv_run_params p;
    std::memset(&p, 0, sizeof(p));
    p.z = 1;
    p.n = 0;
    p.part_per_nucleon = 1;
    p.sigma_r = 1.0;
    p.dt = 0.0;
    hv_sor_reference_defaults(&p.sor);
    p.deposit_mode = HV_DEPOSIT_SORTED;  // reproduces a single-threaded reference run
    return p;
}

struct CtxDeleter {
    void operator()(hv_ctx *c) const { hv_ctx_destroy(c); }
};

using Key = std::tuple<int, int, int, double, double, double, int, int, int>;

inline std::map<Key, std::unique_ptr<hv_ctx, CtxDeleter>> &cache() {
    static thread_local std::map<Key, std::unique_ptr<hv_ctx, CtxDeleter>> m;
    return m;
}

// Context for (world, counts, precision), with its run parameters updated.
template <typename T>
hv_ctx *context(const World<T> &w, int protons, int neutrons, const hv_run_params &p) {
    const hv_world hw = to_world(w);
    Key k{hw.n[0], hw.n[1], hw.n[2], hw.d_max[0], hw.d_max[1], hw.d_max[2], protons, neutrons, (int)prec<T>()};
    auto &m = cache();
    auto it = m.find(k);
    if (it == m.end()) {
        hv_ctx *c = nullptr;
        check(hv_ctx_create(&hw, protons, neutrons, prec<T>(), &p, -1, &c), "hv_ctx_create");
        it = m.emplace(k, std::unique_ptr<hv_ctx, CtxDeleter>(c)).first;
        return c;
    }
    hv_run_params cur;
    hv_ctx_get_params(it->second.get(), &cur);
    if (std::memcmp(&cur, &p, sizeof(p)) != 0) check(hv_ctx_set_params(it->second.get(), &p), "hv_ctx_set_params");
    return it->second.get();
}

template <typename T>
size_t nodes(const World<T> &w) {
    return (size_t)w.n[0] * w.n[1] * w.n[2];
}

}  // namespace detail

// Releases every cached device context of this thread.
inline void release_contexts() { detail::cache().clear(); }

// ---- one routine each, reference names and argument roles ------------------

// include/tools.hpp:35-96
template <typename T>
void distribute_volumetric_particles_cic(ScalarField<T> *density, TestParticles<T> *part, const World<T> &world) {
    hv_ctx *c = detail::context(world, part->protons, part->neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, nullptr, nullptr, nullptr), "upload");
    detail::check(hv_deposit_cic(c), "hv_deposit_cic");
    detail::check(hv_download_field(c, HV_FIELD_DENSITY_RAW, density->v), "download");
}

// include/physics.hpp:202-234 (temp_density receives the input counts, as in
// the reference)
template <typename T>
void compute_volumetric_densities(ScalarField<T> *density, ScalarField<T> *temp_density, const Parameters<T> &param,
                                  const World<T> &world) {
    hv_run_params p = detail::base_params();
    p.sigma_r = (double)param.sigma_r;
    p.part_per_nucleon = param.part_per_nucleon;
    hv_ctx *c = detail::context(world, 0, 0, p);
    std::memcpy(temp_density->v, density->v, sizeof(T) * 2 * detail::nodes(world));
    detail::check(hv_upload_field(c, HV_FIELD_DENSITY_RAW, density->v), "upload");
    detail::check(hv_smooth_density(c), "hv_smooth_density");
    detail::check(hv_download_field(c, HV_FIELD_DENSITY, density->v), "download");
}

// include/physics.hpp:272-281
template <typename T>
void compute_volumetric_skyrme_potentials(ScalarField<T> *potentials, const ScalarField<T> &density,
                                          const Skyrme<T> &skm, const World<T> &world) {
    hv_run_params p = detail::base_params();
    p.skyrme = {(double)skm.A, (double)skm.B, (double)skm.C, (double)skm.gamma};
    hv_ctx *c = detail::context(world, 0, 0, p);
    detail::check(hv_upload_field(c, HV_FIELD_DENSITY, density.v), "upload");
    detail::check(hv_skyrme_potential(c), "hv_skyrme_potential");
    detail::check(hv_download_field(c, HV_FIELD_POTENTIAL, potentials->v), "download");
}

// include/tools.hpp:283-300 (writes the six faces only)
template <typename T>
void set_initial_coulomb_boundaries(ScalarField<T> *coulomb, const World<T> &world, int z) {
    hv_run_params p = detail::base_params();
    p.z = z;
    hv_ctx *c = detail::context(world, 0, 0, p);
    const size_t G = detail::nodes(world);
    std::vector<T> tmp(G);
    detail::check(hv_coulomb_boundary(c), "hv_coulomb_boundary");
    detail::check(hv_download_field(c, HV_FIELD_COULOMB, tmp.data()), "download");
    const int nx = world.n[0], ny = world.n[1], nz = world.n[2];
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++)
                if (i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1) {
                    size_t id = ((size_t)i * ny + j) * nz + k;
                    coulomb->v[id] = tmp[id];
                }
}

// include/physics.hpp:99-157 (omega 1.5, |dphi| < 1e-4, 512 iterations)
template <typename T>
void compute_volumetric_coulomb_potentials_sor(ScalarField<T> *coulomb, const ScalarField<T> &density,
                                               const World<T> &world) {
    hv_ctx *c = detail::context(world, 0, 0, detail::base_params());
    detail::check(hv_upload_field(c, HV_FIELD_COULOMB, coulomb->v), "upload");
    detail::check(hv_upload_field(c, HV_FIELD_DENSITY, density.v), "upload");
    hv_status s = hv_coulomb_sor(c, nullptr, nullptr);
    if (s == HV_ERR_NOT_CONVERGED) std::fprintf(stderr, "SOR COULOMB DID NOT CONVERGE!\n");
    else detail::check(s, "hv_coulomb_sor");
    detail::check(hv_download_field(c, HV_FIELD_COULOMB, coulomb->v), "download");
}

// include/tools.hpp:377-384 (first G nodes)
template <typename T>
void merge_volumetric_potentials(ScalarField<T> *potential_a, const ScalarField<T> &potential_b,
                                 const World<T> &world) {
    hv_ctx *c = detail::context(world, 0, 0, detail::base_params());
    detail::check(hv_upload_field(c, HV_FIELD_POTENTIAL, potential_a->v), "upload");
    detail::check(hv_upload_field(c, HV_FIELD_COULOMB, potential_b.v), "upload");
    detail::check(hv_merge_potentials(c), "hv_merge_potentials");
    detail::check(hv_download_field(c, HV_FIELD_POTENTIAL, potential_a->v), "download");
}

// include/physics.hpp:159-200
template <typename T>
void compute_volumetric_forces_fdm(VectorField<T> *forces, ScalarField<T> potentials, const World<T> &world) {
    hv_ctx *c = detail::context(world, 0, 0, detail::base_params());
    detail::check(hv_upload_field(c, HV_FIELD_POTENTIAL, potentials.v), "upload");
    detail::check(hv_forces_fdm(c), "hv_forces_fdm");
    detail::check(hv_download_field(c, HV_FIELD_FORCE_X, forces->x), "download");
    detail::check(hv_download_field(c, HV_FIELD_FORCE_Y, forces->y), "download");
    detail::check(hv_download_field(c, HV_FIELD_FORCE_Z, forces->z), "download");
}

// include/tools.hpp:98-168
template <typename T>
void distribute_forces_to_particles_cic(TestParticles<T> *part, const VectorField<T> &forces,
                                        const World<T> &world) {
    hv_ctx *c = detail::context(world, part->protons, part->neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, nullptr, nullptr, nullptr), "upload");
    detail::check(hv_upload_field(c, HV_FIELD_FORCE_X, forces.x), "upload");
    detail::check(hv_upload_field(c, HV_FIELD_FORCE_Y, forces.y), "upload");
    detail::check(hv_upload_field(c, HV_FIELD_FORCE_Z, forces.z), "upload");
    detail::check(hv_gather_cic(c), "hv_gather_cic");
    detail::check(hv_download_particle_array(c, HV_PART_FX, part->fx), "download");
    detail::check(hv_download_particle_array(c, HV_PART_FY, part->fy), "download");
    detail::check(hv_download_particle_array(c, HV_PART_FZ, part->fz), "download");
}

// include/physics.hpp:248-258
template <typename T>
void update_momenta_half(TestParticles<T> *part, T dt) {
    World<T> w{{3, 3, 3}, {T(1), T(1), T(1)}};
    hv_ctx *c = detail::context(w, part->protons, part->neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, nullptr, nullptr, nullptr, part->kx, part->ky, part->kz), "upload");
    detail::check(hv_upload_particle_array(c, HV_PART_FX, part->fx), "upload");
    detail::check(hv_upload_particle_array(c, HV_PART_FY, part->fy), "upload");
    detail::check(hv_upload_particle_array(c, HV_PART_FZ, part->fz), "upload");
    detail::check(hv_kick_half(c, (double)dt), "hv_kick_half");
    detail::check(hv_download_particles(c, nullptr, nullptr, nullptr, part->kx, part->ky, part->kz), "download");
}

// include/physics.hpp:260-270
template <typename T>
void update_positions_full(TestParticles<T> *part, T dt) {
    World<T> w{{3, 3, 3}, {T(1), T(1), T(1)}};
    hv_ctx *c = detail::context(w, part->protons, part->neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, part->kx, part->ky, part->kz), "upload");
    detail::check(hv_drift(c, (double)dt), "hv_drift");
    detail::check(hv_download_particles(c, part->x, part->y, part->z, nullptr, nullptr, nullptr), "download");
}

// include/physics.hpp:236-246
template <typename T>
void nuclear_excitation(TestParticles<T> *part, const Parameters<T> &param) {
    World<T> w{{3, 3, 3}, {T(1), T(1), T(1)}};
    hv_run_params p = detail::base_params();
    p.z = param.z;
    p.n = param.n;
    hv_ctx *c = detail::context(w, part->protons, part->neutrons, p);
    detail::check(hv_upload_particle_array(c, HV_PART_KZ, part->kz), "upload");
    detail::check(hv_excite(c, (double)param.eta_exc), "hv_excite");
    detail::check(hv_download_particle_array(c, HV_PART_KZ, part->kz), "download");
}

// include/tools.hpp:327-338 (summed in double on the device)
template <typename T>
T center_of_mass(const TestParticles<T> &part, int type) {
    World<T> w{{3, 3, 3}, {T(1), T(1), T(1)}};
    hv_ctx *c = detail::context(w, part.protons, part.neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, part.x, part.y, part.z, nullptr, nullptr, nullptr), "upload");
    hv_observables o;
    detail::check(hv_observe(c, &o), "hv_observe");
    return (T)(type == PROTONS ? o.zcm_p : o.zcm_n);
}

// include/tools.hpp:302-325
template <typename T>
T mean_squared_radius(const TestParticles<T> &part, const World<T> &world, int type) {
    hv_ctx *c = detail::context(world, part.protons, part.neutrons, detail::base_params());
    detail::check(hv_upload_particles(c, part.x, part.y, part.z, nullptr, nullptr, nullptr), "upload");
    hv_observables o;
    detail::check(hv_observe(c, &o), "hv_observe");
    const double r = type == PROTONS ? o.rms_p : o.rms_n;
    return (T)(r * r);
}

// ---- the gpu_simulate slot (src/hyper_vlasov.cpp:120-123) -----------------
//
// Runs cpu_simulate's loop (src/hyper_vlasov.cpp:32-104) on the device: the
// initial field solve, param.steps steps of dt = t_f / steps with the
// excitation at t_exc, particles advanced in place.  Writes
// output_directory/stats.txt with the reference's rows "t rms_p rms_n zcm_p
// zcm_n" every param.substeps steps (src/hyper_vlasov.cpp:64-70).  float runs
// take the fused path, double runs the plain (reference-order) path.  The SOR
// settings are the reference's (omega 1.5, |dphi| < 1e-4, 512 iterations)
// unless `sor` is given.
template <typename T>
void gpu_simulate(const char *output_directory, TestParticles<T> *part, const Skyrme<T> &skm,
                  const Parameters<T> &param, const World<T> &world, const hv_sor_params *sor = nullptr) {
    hv_run_params p = detail::base_params();
    p.z = param.z;
    p.n = param.n;
    p.part_per_nucleon = param.part_per_nucleon;
    p.sigma_r = (double)param.sigma_r;
    p.dt = (double)(param.t_f / param.steps);  // src/hyper_vlasov.cpp:35
    p.t_exc = (double)param.t_exc;
    p.eta_exc = (double)param.eta_exc;
    p.skyrme = {(double)skm.A, (double)skm.B, (double)skm.C, (double)skm.gamma};
    if (sor) p.sor = *sor;
    p.deposit_mode = std::is_same<T, float>::value ? HV_DEPOSIT_ATOMIC : HV_DEPOSIT_SORTED;
    const int path = std::is_same<T, float>::value ? HV_PATH_FUSED : HV_PATH_PLAIN;
    std::vector<hv_observables> rows(param.steps > 0 ? param.steps : 1);
    const hv_world hw = detail::to_world(world);
    detail::check(hv_simulate(&hw, part->protons, part->neutrons, detail::prec<T>(), &p, path, param.steps, part->x,
                              part->y, part->z, part->kx, part->ky, part->kz, rows.data()),
                  "hv_simulate");
    std::string name = std::string(output_directory) + "/stats.txt";
    FILE *stats = std::fopen(name.c_str(), "w");
    if (!stats) {
        std::fprintf(stderr, "CANNOT OPEN STATS FILE!\n");
        std::exit(1);
    }
    const int sub = param.substeps > 0 ? param.substeps : 1;
    for (int s = 0; s < param.steps; s++)
        if (s % sub == 0)
            std::fprintf(stats, "%e %e %e %e %e\n", (double)(T(s) * T(p.dt)), rows[s].rms_p, rows[s].rms_n,
                         rows[s].zcm_p, rows[s].zcm_n);
    std::fclose(stats);
}

// ---- the initialisation -------------------------------------------------

namespace detail {

// A context holding only particles (the routines below use no grid).
template <typename T>
hv_ctx *particle_context(int protons, int neutrons, const hv_run_params &p) {
    World<T> w;
    for (int a = 0; a < 3; a++) {
        w.n[a] = 8;
        w.d_max[a] = T(1);
    }
    return context(w, protons, neutrons, p);
}

template <typename T>
hv_run_params init_params(const Parameters<T> &param, const Skyrme<T> *skm) {
    hv_run_params p = base_params();
    p.z = param.z;
    p.n = param.n;
    p.part_per_nucleon = param.part_per_nucleon;
    p.sigma_r = (double)param.sigma_r;
    if (skm) p.skyrme = {(double)skm->A, (double)skm->B, (double)skm->C, (double)skm->gamma};
    return p;
}

template <typename T>
void to_ws(const WoodsSaxon<T> *ws, hv_woods_saxon *o) {
    for (int q = 0; q < 2; q++) o[q] = {(double)ws[q].V0, (double)ws[q].R12, (double)ws[q].a};
}

template <typename T>
void from_ws(const hv_woods_saxon *o, WoodsSaxon<T> *ws) {
    for (int q = 0; q < 2; q++) {
        ws[q].V0 = T(o[q].V0);
        ws[q].R12 = T(o[q].R12);
        ws[q].a = T(o[q].a);
    }
}

}  // namespace detail

// include/tools.hpp:170-203: part->density_p / density_n from the positions
template <typename T>
void compute_particle_densities(TestParticles<T> *part, const Parameters<T> &param) {
    hv_ctx *c = detail::particle_context<T>(part->protons, part->neutrons, detail::init_params<T>(param, nullptr));
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, nullptr, nullptr, nullptr), "upload");
    detail::check(hv_particle_densities(c, part->density_p, part->density_n), "hv_particle_densities");
}

// include/tools.hpp:226-232: part->energy
template <typename T>
void compute_particle_energies(TestParticles<T> *part, const WoodsSaxon<T> *ws, const Parameters<T> &param) {
    hv_ctx *c = detail::particle_context<T>(part->protons, part->neutrons, detail::init_params<T>(param, nullptr));
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, part->kx, part->ky, part->kz), "upload");
    hv_woods_saxon h[2];
    detail::to_ws(ws, h);
    detail::check(hv_particle_energies(c, h, (double)param.sigma_k, part->energy), "hv_particle_energies");
}

// include/fit_algorithm.hpp:95-137: the Woods-Saxon fit of each species, from
// ws (in/out).  The densities are recomputed from the positions, as the
// loop's preceding compute_particle_densities gives them; the fit restates
// GSL's driver as Levenberg-Marquardt (hv_fit_woods_saxon).  param supplies
// Z, N, part_per_nucleon and sigma_r (the reference's signature has none:
// its densities come with the particles).
template <typename T>
void minim_woods_saxon(TestParticles<T> *part, WoodsSaxon<T> *ws, Skyrme<T> skm, const Parameters<T> &param) {
    hv_ctx *c = detail::particle_context<T>(part->protons, part->neutrons, detail::init_params<T>(param, &skm));
    detail::check(hv_upload_particles(c, part->x, part->y, part->z, nullptr, nullptr, nullptr), "upload");
    hv_woods_saxon h[2];
    detail::to_ws(ws, h);
    detail::check(hv_fit_woods_saxon(c, nullptr, h, nullptr, nullptr), "hv_fit_woods_saxon");
    detail::from_ws(h, ws);
}

// include/physics.hpp:34-97: allocates part (as create_particles,
// include/init.hpp:133-157: free with the reference's free_particles) and
// fills it with the loop's final particles, their densities and energies;
// ws and fermi_levels receive the final parameters.  The candidates are drawn
// from rand() in the reference's order, so after the same srand() the run is
// the reference's (with the fit restated, GSL being absent).  Prints the
// reference's per-pass lines and its warning when the loop does not converge.
template <typename T>
void initialize_particles(TestParticles<T> *part, WoodsSaxon<T> *ws, const Skyrme<T> &skm, Fermi<T> *fermi_levels,
                          const Parameters<T> &param) {
    const int total_p = param.z * param.part_per_nucleon, total_n = param.n * param.part_per_nucleon;
    const int total = total_p + total_n;
    hv_ctx *c = detail::particle_context<T>(total_p, total_n, detail::init_params<T>(param, &skm));
    hv_woods_saxon h[2];
    detail::to_ws(ws, h);
    hv_fermi f = {(double)fermi_levels->epsilon_p, (double)fermi_levels->epsilon_n};
    hv_init_params ip;
    hv_init_params_default(&ip);
    ip.sigma_k = (double)param.sigma_k;
    ip.r_max = (double)param.r_max;
    ip.max_test_part = param.max_test_part;
    ip.rng = HV_RNG_LIBC;
    hv_init_report rep;
    std::vector<hv_init_row> rows(32);
    detail::check(hv_initialize_particles(c, nullptr, h, &f, &ip, &rep, rows.data()), "hv_initialize_particles");
    for (int it = 0; it < rep.iterations; it++) {  // include/physics.hpp:84-90
        const hv_init_row &r = rows[it];
        std::printf("---------------------------\n");
        std::printf("EQUAL P %i EQUAL N %i\n", r.equal_p, r.equal_n);
        for (int q = 0; q < 2; q++) std::printf("V0 %0.2lf R12 %0.2lf a %0.2lf\n", r.ws[q].V0, r.ws[q].R12, r.ws[q].a);
        std::printf("FERMI P %0.2lf FERMI N %0.2lf\n", r.epsilon_p, r.epsilon_n);
        std::printf("DELTA EPSILON %0.2lf\nITERATION %i\n", r.delta_epsilon, it + 1);
    }
    if (!rep.converged) std::fprintf(stderr, "INITIALIZATION DID NOT CONVERGE!\n");
    part->protons = total_p;
    part->neutrons = total_n;
    T **arrays[12] = {&part->x, &part->y, &part->z, &part->kx, &part->ky, &part->kz,
                      &part->fx, &part->fy, &part->fz, &part->energy, &part->density_p, &part->density_n};
    for (T **a : arrays) {
        *a = (T *)std::malloc((size_t)(total > 0 ? total : 1) * sizeof(T));
        if (!*a) {
            std::fprintf(stderr, "ERROR ALLOCATING MEMORY!\n");
            std::exit(1);
        }
    }
    detail::check(hv_download_particles(c, part->x, part->y, part->z, part->kx, part->ky, part->kz), "download");
    detail::check(hv_particle_densities(c, part->density_p, part->density_n), "hv_particle_densities");
    detail::check(hv_particle_energies(c, h, (double)param.sigma_k, part->energy), "hv_particle_energies");
    std::memset(part->fx, 0, sizeof(T) * total);
    std::memset(part->fy, 0, sizeof(T) * total);
    std::memset(part->fz, 0, sizeof(T) * total);
    detail::from_ws(h, ws);
    fermi_levels->epsilon_p = T(f.epsilon_p);
    fermi_levels->epsilon_n = T(f.epsilon_n);
}

}  // namespace hvb200

#endif  // HV_B200_HPP
