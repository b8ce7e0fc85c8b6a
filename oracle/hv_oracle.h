/*
 * hv_oracle.h -- CPU restatement of the hyper-vlasov per-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA library, not
 * part of it: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product library never links or calls it.
 *
 * Each function restates one routine of BanuDarius/hyper-vlasov (file:line
 * cited at the definition in hv_oracle_impl.h) in plain C, for double (_d)
 * and float (_f), with the reference's operation order and no FMA
 * contraction (built with -ffp-contract=off, as the reference's ISO C++20
 * build is).  Parity of this restatement is pinned against the reference's
 * own routines compiled from source (oracle/ref_harness.cpp) and against the
 * golden vectors in tests/golden/.
 *
 * Differences from the reference, all deliberate:
 *  - orc_smooth_* visits the same node pairs as compute_volumetric_densities
 *    (include/physics.hpp:202-234) in the same order, but through a table of
 *    offsets built once, instead of testing all G^2 pairs.  Weights come from
 *    the node coordinates of the grid centre and its offset partners; they
 *    are bit-identical to the reference when node coordinates are exact
 *    binary fractions (all grids with power-of-two n and d_max) and within
 *    one rounding otherwise.
 *  - orc_sor_* takes omega, the stopping rule, tolerance and iteration cap as
 *    arguments; (1.5, max-update, 1e-4, 512) reproduces the reference.
 *  - observables are also returned as double sums.
 */
#ifndef HV_ORACLE_H
#define HV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_world {
    int n[3];
    double d_max[3];
} orc_world;

typedef struct orc_skyrme {
    double A, B, C, gamma;
} orc_skyrme;

typedef struct orc_run {
    int z, n, part_per_nucleon;
    double sigma_r, dt, t_exc, eta_exc;
    orc_skyrme skyrme;
    double sor_omega, sor_tol;
    int sor_criterion; /* 0 = max update (reference), 1 = relative residual */
    int sor_max_iter;
} orc_run;

typedef struct orc_obs {
    double t, rms_p, rms_n, zcm_p, zcm_n, dipole;
    int sor_iterations, flags;
} orc_obs;

#define ORC_DECLARE(R, S)                                                                     \
    void orc_deposit_cic_##S(const orc_world *w, int protons, int neutrons, const R *x,       \
                             const R *y, const R *z, R *rho);                                 \
    int orc_smooth_table_size_##S(const orc_world *w, double sigma_r);                        \
    void orc_smooth_##S(const orc_world *w, double sigma_r, int ppn, R *rho, R *tmp);         \
    void orc_skyrme_##S(const orc_world *w, const orc_skyrme *s, const R *rho, R *U);         \
    void orc_coulomb_boundary_##S(const orc_world *w, int z, R *phi);                         \
    int orc_sor_##S(const orc_world *w, R *phi, const R *rho, double omega, int criterion,    \
                    double tol, int max_iter, double *metric);                                \
    double orc_rel_residual_##S(const orc_world *w, const R *phi, const R *rho);              \
    void orc_merge_##S(const orc_world *w, R *U, const R *phi);                               \
    void orc_fdm_##S(const orc_world *w, const R *U, R *fx, R *fy, R *fz);                    \
    void orc_gather_cic_##S(const orc_world *w, int protons, int neutrons, const R *x,        \
                            const R *y, const R *z, const R *Fx, const R *Fy, const R *Fz,    \
                            R *fx, R *fy, R *fz);                                             \
    void orc_kick_half_##S(int total, R *kx, R *ky, R *kz, const R *fx, const R *fy,          \
                           const R *fz, R dt);                                                \
    void orc_drift_##S(int total, R *x, R *y, R *z, const R *kx, const R *ky, const R *kz,    \
                       R dt);                                                                 \
    void orc_excite_##S(int protons, int neutrons, R *kz, int Z, int N, R eta);               \
    void orc_observe_##S(const orc_world *w, int protons, int neutrons, const R *x,           \
                         const R *y, const R *z, orc_obs *out);                               \
    void orc_particle_densities_##S(int protons, int neutrons, const R *x, const R *y,         \
                                    const R *z, double sigma_r, int ppn, R *dp, R *dn);        \
    void orc_particle_energies_##S(int protons, int neutrons, const R *x, const R *y,          \
                                   const R *z, const R *kx, const R *ky, const R *kz,         \
                                   const double *ws, double sigma_k, int zc, R *energy);      \
    int orc_fit_woods_saxon_##S(int n, const R *x, const R *y, const R *z, const R *dp,       \
                                const R *dn, int type, const orc_skyrme *skm, double *ws,     \
                                int max_iter, double xtol, double gtol, int *iters);          \
    int orc_simulate_##S(const orc_world *w, const orc_run *run, int protons, int neutrons,    \
                         R *x, R *y, R *z, R *kx, R *ky, R *kz, int steps, orc_obs *obs,      \
                         R *fields_out, double *step_seconds);

ORC_DECLARE(double, d)
ORC_DECLARE(float, f)

#undef ORC_DECLARE

/* OpenMP thread count of the restatement. */
void orc_set_threads(int n);

/* Seeded synthetic nucleus (MT19937-64), the inputs of every workload: see
 * hv_oracle.c.  Returns 0, or 1 for a bad argument. */
#include <stdint.h>
int orc_generate_nucleus_d(uint64_t seed, int protons, int neutrons, double radius, double k_fermi, double *x,
                           double *y, double *z, double *kx, double *ky, double *kz);
int orc_generate_nucleus_f(uint64_t seed, int protons, int neutrons, double radius, double k_fermi, float *x,
                           float *y, float *z, float *kx, float *ky, float *kz);
/* the n-th output (n >= 1) of MT19937-64 seeded with `seed` */
uint64_t orc_mt64_nth(uint64_t seed, long long n);

#ifdef __cplusplus
}
#endif

#endif
