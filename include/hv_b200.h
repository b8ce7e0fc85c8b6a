/*
 * hv_b200.h -- C ABI of the B200 (sm_100a) implementation of the hyper-vlasov
 * per-step hot path.
 *
 * The reference (BanuDarius/hyper-vlasov) has no FFI: its surface is a set of
 * C++ function templates over the POD structs of include/sim_structs.hpp,
 * called in a fixed order by cpu_simulate (src/hyper_vlasov.cpp:32-118), with
 * an empty GPU slot gpu_simulate (src/hyper_vlasov.cpp:120-123).  Every entry
 * point below replaces one of those routines (cited per function) and keeps
 * its argument roles.  The C++ header hv_b200.hpp wraps these entry points
 * with the reference's own call shapes (TestParticles<T>*, ScalarField<T>*,
 * const World<T>& ...).
 *
 * Conventions
 *  - Plain C types only.  Device buffers are owned by an hv_ctx; host buffers
 *    are owned by the caller and are never retained after a call returns.
 *  - Every function returns hv_status and never exits the process (the
 *    reference prints and calls exit(1); include/init.hpp:94-96).
 *  - All work of one context is ordered on the context's own CUDA stream.  A
 *    context is not thread-safe; distinct contexts are independent.
 *  - Particle arrays are structure-of-arrays with protons first, exactly as
 *    TestParticles<T> (include/sim_structs.hpp:55-60).  Species grids are
 *    stacked: protons at [0,G), neutrons at [G,2G), G = n[0]*n[1]*n[2], index
 *    IDX(i,j,k) = (i*n[1] + j)*n[2] + k (include/sim_structs.hpp:38).
 */
#ifndef HV_B200_H
#define HV_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HV_API __attribute__((visibility("default")))
#else
#define HV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hv_status {
    HV_OK = 0,
    HV_ERR_BAD_ARG = 1,        /* invalid size, pointer or parameter            */
    HV_ERR_CUDA = 2,           /* a CUDA runtime call failed                    */
    HV_ERR_NOT_CONVERGED = 3,  /* SOR reached max_iter; fields are still written */
    HV_ERR_NO_DEVICE = 4,      /* no usable sm_100 device                       */
    HV_ERR_OOM = 5,            /* device allocation failed                      */
    HV_ERR_TIMEOUT = 6,        /* a bounded device-side wait gave up            */
    HV_ERR_UNSUPPORTED = 7,    /* combination of options not provided           */
    HV_ERR_NONFINITE = 8       /* NaN/Inf detected in a checked quantity        */
} hv_status;

/* Arithmetic type of a context.  HV_F64 is the plain drop-in (the reference's
 * default double instantiation); HV_F32 keeps particles, grids and stencils in
 * float and uses double only for the SOR residual norm / convergence test, the
 * Coulomb boundary monopole and the observable sums. */
typedef enum hv_precision { HV_F64 = 0, HV_F32 = 1 } hv_precision;

/* How the CIC deposit reduces contributions into the density grid. */
typedef enum hv_deposit_mode {
    HV_DEPOSIT_ATOMIC = 0,  /* warp-aggregated atomics; order not reproducible   */
    HV_DEPOSIT_SORTED = 1   /* sort by cell, then per-node sum in particle-index
                               order: deterministic and, in HV_F64, bit-identical
                               to a single-threaded run of the reference         */
} hv_deposit_mode;

/* SOR stopping rule. */
typedef enum hv_sor_criterion {
    HV_SOR_MAX_UPDATE = 0,   /* stop when max|phi_new - phi_old| < tol over one
                                red+black iteration (physics.hpp:152)            */
    HV_SOR_REL_RESIDUAL = 1  /* stop when ||b + lap_h phi||_2 / ||b||_2 <= tol,
                                b = 4*pi*1.44*rho_p on interior nodes (FP64)     */
} hv_sor_criterion;

/* How hv_run advances the state. */
typedef enum hv_step_path {
    HV_PATH_PLAIN = 0,  /* one kernel per reference routine, in cpu_simulate order,
                           SOR convergence tested on the host each iteration     */
    HV_PATH_FUSED = 1   /* fused particle kernel, fused field kernels, device-side
                           SOR loop, whole step replayed from a CUDA graph       */
} hv_step_path;

/* World<T> (include/sim_structs.hpp:72-75).  Node i on axis a sits at
 * d_max[a] * (2 i / n[a] - 1) (include/tools.hpp:394-401). */
typedef struct hv_world {
    int n[3];
    double d_max[3];
} hv_world;

/* Skyrme<T> (include/sim_structs.hpp:82-84):
 * U_q = A t + B t^gamma + 2 tau C (rho_n - rho_p)/rho0, t = rho/rho0,
 * tau = -1 protons, +1 neutrons (include/physics_formulas.hpp:70-77). */
typedef struct hv_skyrme {
    double A, B, C, gamma;
} hv_skyrme;

/* Coulomb SOR controls.  The reference hard-codes omega = 1.5, tol = 1e-4,
 * max_iter = 512 with HV_SOR_MAX_UPDATE (include/physics.hpp:103-104,152). */
typedef struct hv_sor_params {
    double omega;
    double tol;
    int criterion;   /* hv_sor_criterion */
    int max_iter;
} hv_sor_params;

/* Parameters<T> fields that the step uses (include/sim_structs.hpp:49-53). */
typedef struct hv_run_params {
    int z, n;                 /* proton and neutron numbers of the nucleus     */
    int part_per_nucleon;     /* test particles per nucleon                    */
    double sigma_r;           /* Gaussian smoothing width (fm)                 */
    double dt;                /* time step (fm/c); the reference uses t_f/steps */
    double t_exc;             /* time of the one-shot dipole excitation (fm/c) */
    double eta_exc;           /* excitation strength (fm^-1)                   */
    hv_skyrme skyrme;
    hv_sor_params sor;
    int deposit_mode;         /* hv_deposit_mode                               */
} hv_run_params;

/* Fields held by a context.  Sizes: COULOMB has G nodes, all others 2G. */
typedef enum hv_field {
    HV_FIELD_DENSITY_RAW = 0,  /* CIC counts after the deposit                   */
    HV_FIELD_DENSITY = 1,      /* smoothed density (fm^-3)                       */
    HV_FIELD_POTENTIAL = 2,    /* mean-field potential U (MeV), Coulomb merged   */
    HV_FIELD_COULOMB = 3,      /* Coulomb potential phi (MeV)                    */
    HV_FIELD_FORCE_X = 4,      /* -dU/dx (MeV/fm)                                */
    HV_FIELD_FORCE_Y = 5,
    HV_FIELD_FORCE_Z = 6
} hv_field;

/* Particle arrays of TestParticles<T> that the step reads or writes. */
typedef enum hv_particle_array {
    HV_PART_X = 0, HV_PART_Y = 1, HV_PART_Z = 2,
    HV_PART_KX = 3, HV_PART_KY = 4, HV_PART_KZ = 5,
    HV_PART_FX = 6, HV_PART_FY = 7, HV_PART_FZ = 8
} hv_particle_array;

/* Per-step observables, one row per recorded step (src/hyper_vlasov.cpp:64-70
 * writes t, rms_p, rms_n, zcm_p, zcm_n).  Sums are accumulated in double. */
typedef struct hv_observables {
    double t;
    double rms_p, rms_n;   /* sqrt of mean_squared_radius (tools.hpp:302-325) */
    double zcm_p, zcm_n;   /* center_of_mass (tools.hpp:327-338)              */
    double dipole;         /* D = N Z / A (zcm_p - zcm_n) (scripts/programs.py:99) */
    int sor_iterations;    /* SOR iterations spent in this step               */
    int flags;             /* HV_OBS_* bits                                   */
} hv_observables;

/* hv_observables.flags: the step's SOR reached max_iter (the reference prints
 * "SOR COULOMB DID NOT CONVERGE!" and carries on, include/physics.hpp:155-156). */
#define HV_OBS_SOR_NOT_CONVERGED 1

typedef struct hv_ctx hv_ctx;

/* ---- library / device ------------------------------------------------- */

/* Version string of the library. */
HV_API const char *hv_version(void);
/* Human-readable name of a status code. */
HV_API const char *hv_status_string(hv_status s);
/* Last CUDA error text recorded by this thread (empty if none). */
HV_API const char *hv_last_error(void);
/* Number of visible sm_100 devices (0 when none).  Never fails. */
HV_API int hv_device_count(void);

/* ---- defaults and parameter helpers ----------------------------------- */

/* Fills *p with the reference's SOR controls (omega 1.5, |dphi| < 1e-4,
 * 512 iterations; include/physics.hpp:103-104,152, sim_structs.hpp:36,45). */
HV_API void hv_sor_reference_defaults(hv_sor_params *p);

/* Skyrme coefficients from (t0, t3, sigma, a_sym):
 * A = 3/4 t0 rho0, B = (sigma+2)/16 t3 rho0^(sigma+1), gamma = sigma+1,
 * C = a_sym, with rho0 = 0.16 fm^-3 (include/sim_structs.hpp:34). */
HV_API void hv_skyrme_from_t0t3(double t0, double t3, double sigma, double a_sym, hv_skyrme *out);

/* Seeded synthetic nucleus (replaces initialize_particles,
 * include/physics.hpp:34-97, which needs GSL).  std::mt19937_64(seed); each
 * uniform is (draw >> 11) * 2^-53; coordinates are radius*(2u-1) with
 * rejection to the open ball.  All positions are drawn first (protons first),
 * then all wavenumbers, in the ball of radius k_fermi (fm^-1).  The _f32
 * variant rounds the same double draws to float. */
HV_API hv_status hv_generate_nucleus_f64(uint64_t seed, int protons, int neutrons,
                                  double radius, double k_fermi,
                                  double *x, double *y, double *z,
                                  double *kx, double *ky, double *kz);
HV_API hv_status hv_generate_nucleus_f32(uint64_t seed, int protons, int neutrons,
                                  double radius, double k_fermi,
                                  float *x, float *y, float *z,
                                  float *kx, float *ky, float *kz);

/* ---- context lifetime ------------------------------------------------- */

/* Allocates the device state of one run: particles (TestParticles<T>,
 * include/init.hpp:133-157) and the fields of cpu_simulate
 * (src/hyper_vlasov.cpp:44-51).  Requires n[a] >= 3, d_max[a] > 0,
 * protons, neutrons >= 0.  device < 0 selects the current device. */
HV_API hv_status hv_ctx_create(const hv_world *world, int protons, int neutrons,
                        hv_precision prec, const hv_run_params *params,
                        int device, hv_ctx **out);
HV_API hv_status hv_ctx_destroy(hv_ctx *ctx);
/* Replaces the run parameters (sizes are fixed at creation). */
HV_API hv_status hv_ctx_set_params(hv_ctx *ctx, const hv_run_params *params);
HV_API hv_status hv_ctx_get_params(const hv_ctx *ctx, hv_run_params *out);
/* The context's CUDA stream (a cudaStream_t). */
HV_API void *hv_ctx_stream(hv_ctx *ctx);
/* Blocks until all work queued on the context has finished. */
HV_API hv_status hv_ctx_synchronize(hv_ctx *ctx);

/* ---- host <-> device transfers (caller-owned host memory) ------------- */
/* Element type of every host pointer is the context precision (double for
 * HV_F64, float for HV_F32).  Particle counts are those given at creation. */

/* Uploads x,y,z,kx,ky,kz (any may be NULL to keep the device copy). */
HV_API hv_status hv_upload_particles(hv_ctx *ctx, const void *x, const void *y, const void *z,
                              const void *kx, const void *ky, const void *kz);
/* Downloads the particle arrays in the caller's original particle order. */
HV_API hv_status hv_download_particles(hv_ctx *ctx, void *x, void *y, void *z,
                                void *kx, void *ky, void *kz);
HV_API hv_status hv_upload_particle_array(hv_ctx *ctx, int which, const void *host);
HV_API hv_status hv_download_particle_array(hv_ctx *ctx, int which, void *host);
HV_API hv_status hv_upload_field(hv_ctx *ctx, int field, const void *host);
HV_API hv_status hv_download_field(hv_ctx *ctx, int field, void *host);
/* Device address of a field (valid until hv_ctx_destroy). */
HV_API hv_status hv_field_device_ptr(hv_ctx *ctx, int field, void **dev_ptr);

/* ---- one entry per reference routine (device-resident state) ---------- */

/* distribute_volumetric_particles_cic (include/tools.hpp:35-96):
 * particles -> DENSITY_RAW, using params.deposit_mode. */
HV_API hv_status hv_deposit_cic(hv_ctx *ctx);
/* compute_volumetric_densities (include/physics.hpp:202-234):
 * DENSITY_RAW -> DENSITY.  Same node-pair set (|r_i - r_j|^2 <= 16 sigma_r^2,
 * zero padding) and normalisation 1/(ppn (2 pi sigma_r^2)^1.5). */
HV_API hv_status hv_smooth_density(hv_ctx *ctx);
/* compute_volumetric_skyrme_potentials (include/physics.hpp:272-281):
 * DENSITY -> POTENTIAL. */
HV_API hv_status hv_skyrme_potential(hv_ctx *ctx);
/* set_initial_coulomb_boundaries (include/tools.hpp:283-300): writes
 * phi = 1.44 Z / |r| on the six faces of COULOMB (evaluated in double). */
HV_API hv_status hv_coulomb_boundary(hv_ctx *ctx);
/* compute_volumetric_coulomb_potentials_sor (include/physics.hpp:99-157):
 * red-black SOR on the interior of COULOMB, warm-started from its contents,
 * source = proton DENSITY.  *iterations (may be NULL) receives the number of
 * red+black iterations; *metric (may be NULL) the final value of the stopping
 * quantity.  Returns HV_ERR_NOT_CONVERGED when max_iter was reached. */
HV_API hv_status hv_coulomb_sor(hv_ctx *ctx, int *iterations, double *metric);
/* merge_volumetric_potentials (include/tools.hpp:377-384): U_p += phi. */
HV_API hv_status hv_merge_potentials(hv_ctx *ctx);
/* compute_volumetric_forces_fdm (include/physics.hpp:159-200):
 * POTENTIAL -> FORCE_{X,Y,Z}. */
HV_API hv_status hv_forces_fdm(hv_ctx *ctx);
/* distribute_forces_to_particles_cic (include/tools.hpp:98-168):
 * FORCE_{X,Y,Z} -> particle fx,fy,fz (zero outside the grid). */
HV_API hv_status hv_gather_cic(hv_ctx *ctx);
/* update_momenta_half (include/physics.hpp:248-258): k += dt/(2 hbar c) f. */
HV_API hv_status hv_kick_half(hv_ctx *ctx, double dt);
/* update_positions_full (include/physics.hpp:260-270): x += dt hbar c/mc2 k. */
HV_API hv_status hv_drift(hv_ctx *ctx, double dt);
/* nuclear_excitation (include/physics.hpp:236-246): kz += eta N/A (protons),
 * kz -= eta Z/A (neutrons), Z = params.z, N = params.n. */
HV_API hv_status hv_excite(hv_ctx *ctx, double eta);
/* center_of_mass (include/tools.hpp:327-338) and mean_squared_radius
 * (include/tools.hpp:302-325) of both species, summed in double. */
HV_API hv_status hv_observe(hv_ctx *ctx, hv_observables *out);

/* Observables (as hv_observe) of particle arrays held in the caller's device
 * memory, computed without allocating any device memory.  No counterpart in
 * the reference: it is for callers that cannot call cudaMalloc, such as a
 * host framework that has reserved the GPU's memory for its own allocator, or
 * code running where allocation is not permitted.  The caller passes the
 * inputs (x, y, z: protons + neutrons values of the precision's type, protons
 * first) and receives *out on the host; D uses nucleus_z and nucleus_n.
 * Scratch is a fixed 256 KiB array inside the library, held by every GPU that
 * loads it until the process exits; one call handles at most
 * HV_NOALLOC_MAX_PARTICLES particles and rejects more with HV_ERR_BAD_ARG.
 * Each call looks up the array's address on the current device (a lookup
 * that allocates nothing).  All calls share the array: calls whose work
 * overlaps on the GPU race.  Work is queued on `stream` (a cudaStream_t,
 * NULL for the default stream) and the call returns after it completes. */
#define HV_NOALLOC_MAX_PARTICLES (4096 * 1024)
HV_API hv_status hv_observe_noalloc(const hv_world *world, int protons, int neutrons, int nucleus_z,
                                    int nucleus_n, hv_precision prec, const void *x, const void *y,
                                    const void *z, void *stream, hv_observables *out);

/* ---- fused-path options ------------------------------------------------ */

 /* SOR starting guess of each step's solve in the fused path (the plain path
 * always starts from the previous step's phi, as the reference does). */
typedef enum hv_warm_start {
    HV_WARM_PREVIOUS = 0,    /* the previous step's phi, as the reference does  */
    HV_WARM_EXTRAPOLATE = 1, /* 2 phi(t) - phi(t - dt): the same stopping rule
                                from a closer guess, about half the iterations */
    HV_WARM_QUADRATIC = 2    /* 3 phi(t) - 3 phi(t - dt) + phi(t - 2 dt) (the
                                default): a quarter of the linear guess's
                                iterations on 208Pb / 2.08 M; the converged phi
                                differs from the previous-guess solve within
                                the tolerance (D(t) by ~6e-9 relative)         */
} hv_warm_start;

/* How the blocks of the fused SOR exchange boundary corrections. */
typedef enum hv_sor_exchange {
    HV_SOR_EXCHANGE_AUTO = 0,   /* tagged mirror words where supported (float,
                                   z extent a multiple of 8), else counters    */
    HV_SOR_EXCHANGE_FLAGS = 1   /* per-block phase counters after each sweep   */
} hv_sor_exchange;

/* Controls of HV_PATH_FUSED that have no counterpart in the reference. */
typedef struct hv_fast_options {
    int sor_warm_start;   /* hv_warm_start                                      */
    int sor_inner_min;    /* red+black iterations between two FP64 residual     */
    int sor_inner_max;    /*   checks: the first cycle of a solve runs 7/8 of the
                             previous solve's iterations (at most max), the
                             later ones follow the observed rate, clamped to
                             [min, max]                                        */
    int sort_every;       /* hv_run on HV_PATH_FUSED re-sorts the particle slots
                             by cell (protons before neutrons) every n steps, at
                             most once per graph launch (0 = off); downloads
                             stay in the caller's order.  Batched runs keep
                             their slot order                                  */
    int graph_steps;      /* steps captured per CUDA graph launch (0 = no graph) */
    int sor_exchange;     /* hv_sor_exchange                                    */
    int smooth_fft;       /* Gaussian smoothing as an FFT convolution where it is
                             exact (power-of-two axes up to 128, no density
                             within the stencil of a face; elsewhere the direct
                             form runs): 2 always, 1 for stencils of half-width
                             6 nodes or more (the default; 89 against 321 us at
                             128^3, half-width 9), 0 never                      */
    double sor_omega;     /* relaxation of the fused solver's sweeps on the
                             correction in plain cycles (no coarse-grid
                             correction: sor_coarse 0, or where it does not
                             run); 0 (the default): the run's
                             hv_sor_params.omega.  The stopping rule stays the
                             FP64 residual test; on 208Pb 128^3 (rule 1e-6)
                             1.8 / 1.85 / 1.9 / 1.93 took 169 / 144 / 120 / 105
                             iterations per step with D(t) equal to 1e-8      */
    int sor_wait_limit;   /* polls a device-side wait of the fused solver (grid
                             barrier, neighbour row) makes before it gives up
                             and the run returns HV_ERR_TIMEOUT; 0 (the
                             default): 2^24 for barriers, 2^22 per row entry
                             (about a second).  The context stays usable after
                             a timeout                                         */
    int sor_coarse;       /* 1 (the default): each cycle of the fused float
                             solve starts its correction from the correction
                             equation solved exactly on a coarse grid (every
                             F-th node, F the smallest power of two leaving at
                             most 15 interior coarse nodes per axis; grids of
                             fewer than 48^3 nodes or whose axes F does not
                             divide, double solves, the max-update rule and
                             batched waves of generic sweeps go without), and
                             runs sor_coarse_sweeps red+black iterations after
                             it; 0: plain SOR cycles.  The stopping rule is
                             unchanged, so only the iterations per solve
                             change                                            */
    int sor_coarse_sweeps;/* red+black iterations after each coarse correction
                             (default 12)                                      */
    int deposit_aggregate;/* 1 (the default): the float atomic deposit of the
                             fused particle step sums the CIC weights of
                             neighbouring lanes with the same base node (the
                             slots are re-sorted by cell) and adds each run
                             once; 0: one set of atomics per particle          */
    double sor_coarse_omega;/* relaxation of the sweeps after each coarse
                             correction (they smooth what the coarse grid
                             leaves); 0 (the default): 1.7.  With 12 sweeps
                             the solves of 208Pb end in two cycles, 24
                             iterations, on 48^3 to 128^3 grids, where the
                             run's omega 1.8 with 16 sweeps takes 32 (128^3)
                             or 48; the stopping rule is unchanged            */
} hv_fast_options;

/* Defaults: HV_WARM_QUADRATIC, inner 8..256, sort every 16 steps, 8-step graphs,
 * HV_SOR_EXCHANGE_AUTO, smooth_fft 1, sor_omega 0 (the run's omega),
 * sor_wait_limit 0, sor_coarse 1 with 12 sweeps per cycle at sor_coarse_omega 0
 * (1.7), deposit_aggregate 1. */
HV_API void hv_fast_options_default(hv_fast_options *o);
HV_API hv_status hv_ctx_set_fast_options(hv_ctx *ctx, const hv_fast_options *o);
HV_API hv_status hv_ctx_get_fast_options(const hv_ctx *ctx, hv_fast_options *o);

/* What hv_ctx_autotune chose. */
typedef struct hv_autotune_report {
    int particle_block;    /* threads per block of the particle step          */
    int particle_grid;     /* its blocks (a multiple of the SM count)         */
    int sor_planes;        /* the SOR tile: planes x rows owned by one block  */
    int sor_rows;
    int sor_blocks;        /* blocks of the solve                             */
    int sor_tile_rank;     /* rank of the tile in the plan's own order (0: the
                              plan's heuristic choice)                        */
    int candidates;        /* configurations timed                            */
    double particle_ms;    /* device ms per launch of the chosen particle step */
    double sor_ms;         /* device ms per launch of the solve with the chosen
                              tile                                             */
} hv_autotune_report;

/* Chooses the fused path's launch configuration for this context by timing
 * candidates over trial_steps steps each (CUDA events around each launch):
 * first the particle step's block size (128, 256, 512 threads) and grid (2, 4,
 * 8 blocks per SM) with the planned SOR tile, then the SOR tile among the
 * plan's four best-ranked P x R partitions (the ranking hv_run's plan uses:
 * fewest quads per thread, then least exchanged face, then fewest blocks).
 * The trial steps advance the run like hv_run (solving the initial fields
 * first if needed); the choice holds for later hv_run calls on the context.
 * No counterpart in the reference. */
HV_API hv_status hv_ctx_autotune(hv_ctx *ctx, int trial_steps, hv_autotune_report *report);

/* Kernels of one fused step, for hv_ctx_kernel_times. */
typedef enum hv_kernel_id {
    HV_K_PARTICLE = 0,  /* gather + kicks + drift + deposit + observables      */
    HV_K_SMOOTH = 1,    /* Gaussian smoothing                                  */
    HV_K_SKYRME = 2,    /* Skyrme + symmetry potential                         */
    HV_K_SOR = 3,       /* persistent Coulomb SOR                              */
    HV_K_FORCES = 4,    /* -grad(U + phi) into the interleaved force field     */
    HV_K_COUNT = 5
} hv_kernel_id;

/* Per-kernel CUDA-event timing of fused steps.  While enabled, steps are
 * launched directly (not from a graph) with an event pair around each kernel
 * on the context stream; hv_ctx_kernel_times returns the accumulated device
 * milliseconds and launch counts per hv_kernel_id since the last enable. */
HV_API hv_status hv_ctx_set_profiling(hv_ctx *ctx, int enable);
HV_API hv_status hv_ctx_kernel_times(hv_ctx *ctx, double *total_ms, int *launches, int n);

/* ---- output ------------------------------------------------------------ */

/* Writes the context's forces, density and potential as one VTK frame in the
 * reference's format (output_vtk_header_start, output_vector_field,
 * output_scalar_field: include/init.hpp:159-254; the frame of
 * src/hyper_vlasov.cpp:72-84): ASCII STRUCTURED_POINTS header, big-endian
 * float32 blocks with x varying fastest. */
HV_API hv_status hv_write_vtk(hv_ctx *ctx, const char *path);

/* ---- whole-step drivers ----------------------------------------------- */

/* The initial field solve of cpu_simulate (src/hyper_vlasov.cpp:53-62):
 * deposit, smooth, Coulomb boundary, Skyrme, SOR, merge, FDM, gather. */
HV_API hv_status hv_initial_solve(hv_ctx *ctx, int *sor_iterations);

/* Advances n_steps time steps of the cpu_simulate loop
 * (src/hyper_vlasov.cpp:63-104): [excite at t >= t_exc, once] -> kick/2 ->
 * drift -> deposit -> smooth -> Skyrme -> SOR -> merge -> FDM -> gather ->
 * kick/2.  obs (may be NULL) receives n_steps rows, observed at the start of
 * each step as the reference records them.  path selects hv_step_path. */
HV_API hv_status hv_run(hv_ctx *ctx, int n_steps, int path, hv_observables *obs);

/* The whole gpu_simulate slot (src/hyper_vlasov.cpp:120-123) with host
 * buffers: uploads the particles, runs the initial solve and n_steps steps,
 * downloads the final particles (in place) and n_steps observable rows.
 * Element type of the particle pointers follows prec.  Runs on the current
 * device.  The device context of a call is kept afterwards and reused by the
 * next call with the same device, world, particle counts and precision (any
 * run parameters), reset to the state a new context starts from, so that a
 * caller stepping many nuclei of one shape pays for allocation and planning
 * once; at most four idle contexts are kept, and a call that fails destroys
 * its context.  Concurrent calls never share a context. */
HV_API hv_status hv_simulate(const hv_world *world, int protons, int neutrons,
                      hv_precision prec, const hv_run_params *params, int path,
                      int n_steps, void *x, void *y, void *z,
                      void *kx, void *ky, void *kz, hv_observables *obs);
/* Destroys the contexts hv_simulate keeps between calls (device memory is
 * returned); the next call creates a new one. */
HV_API hv_status hv_simulate_release(void);

/* compute_particle_densities (include/tools.hpp:170-203), part of the
 * reference's initialisation (initialize_particles, include/physics.hpp:34-97):
 * for every particle of the context, the Gaussian-weighted (sigma_r of the
 * run parameters) sum over all particles within 4 sigma_r, by species, times
 * 1 / (part_per_nucleon (2 pi sigma_r^2)^1.5) -- the reference's
 * TestParticles<T>::density_p / density_n.  The reference loops over all pairs
 * (O(N^2)); here cell lists of edge 4 sigma_r find the partners.  Host arrays
 * of the context's precision, in the caller's particle order. */
HV_API hv_status hv_particle_densities(hv_ctx *ctx, void *density_p, void *density_n);

/* ---- initialisation: the Woods-Saxon self-consistency loop ---------------
 * initialize_particles (include/physics.hpp:34-97) on the device: Fermi levels
 * from 2M temporary particles, the run's particles as (r, k) / (-r, -k) pairs
 * below the levels, their densities, a Woods-Saxon fit per species, relaxation
 * by 0.6, repeated until |d eps_p| + |d eps_n| <= 0.1 or max_iterations. */

/* WoodsSaxon<T> (include/sim_structs.hpp:78-81): V(r) = V0 / (1 + exp((r - R12) / a)). */
typedef struct hv_woods_saxon {
    double V0, R12, a;
} hv_woods_saxon;

/* Fermi<T> (include/sim_structs.hpp:88-90). */
typedef struct hv_fermi {
    double epsilon_p, epsilon_n;
} hv_fermi;

/* Source of the uniform numbers of the rejection sampling. */
typedef enum hv_rng {
    /* the C library's rand(), drawn on the host in the reference's order
     * (rand_val, include/math_functions.hpp:29-33): after srand(seed) the run
     * is the reference's, and rand() continues afterwards exactly as after the
     * reference's loop.  Host-bound (6 rand() calls per candidate pair). */
    HV_RNG_LIBC = 0,
    /* Philox4x32-10 on the device, keyed by hv_init_params.seed */
    HV_RNG_PHILOX = 1
} hv_rng;

typedef struct hv_init_params {
    double sigma_k;      /* Parameters::sigma_k = calc_sigma(k_fwhm) (init.hpp:322) */
    double r_max;        /* 0: nuclear_radius(Z + N) = 1.5 A^(1/3) (init.hpp:55)    */
    int max_test_part;   /* temporaries per species; 0: max_particles(r_max, k_max, ppn) (init.hpp:57) */
    int max_iterations;  /* 0: MAX_INIT_ITERATIONS = 32 (sim_structs.hpp:28)        */
    int rng;             /* hv_rng                                                 */
    unsigned long long seed;  /* HV_RNG_PHILOX key                                 */
} hv_init_params;

/* One pass of the loop: what the reference prints (physics.hpp:85-90). */
typedef struct hv_init_row {
    int equal_p, equal_n;          /* 2 x temporaries below each Fermi level     */
    double epsilon_p, epsilon_n;   /* Fermi levels after the update              */
    double delta_epsilon;          /* |d eps_n| + |d eps_p|                      */
    hv_woods_saxon ws[2];          /* after the fit and the relaxation           */
    int fit_iterations[2];         /* iterations of the fit, protons / neutrons  */
    int fit_status[2];             /* as hv_fit_woods_saxon's status             */
} hv_init_row;

typedef struct hv_init_report {
    int iterations;                /* passes of the loop                         */
    int converged;                 /* the last |d eps| sum was <= 0.1 (else the  */
                                   /* reference prints "INITIALIZATION DID NOT CONVERGE!") */
    double delta_epsilon;
    double chi_squared_p, chi_squared_n;  /* chi_squared (tools.hpp:340-366)   */
    long long candidates;          /* candidates drawn (3 or 6 numbers each)     */
    int max_test_part;             /* temporaries per species used               */
    double r_max;                  /* sampling radius used                       */
} hv_init_report;

/* Defaults: sigma_k = calc_sigma(0.346) (auto_compute.py:54), r_max and
 * max_test_part derived, 32 passes, HV_RNG_PHILOX, seed 128. */
HV_API void hv_init_params_default(hv_init_params *p);

/* initialize_particles (include/physics.hpp:34-97): replaces the context's
 * particles (which must number Z ppn protons and N ppn neutrons, an even total,
 * from the run parameters) by the loop's final ones, in the reference's order.
 * ws[2] (protons, neutrons) and fermi are the starting values and receive the
 * final ones, as the reference's pointers do; skm NULL takes the run
 * parameters' Skyrme.  rows (NULL or max_iterations entries) receives one row
 * per pass.  The Woods-Saxon fit restates GSL's driver (absent here) as
 * Levenberg-Marquardt; HV_ERR_NOT_CONVERGED when no candidate can be kept
 * (the reference would loop for ever). */
HV_API hv_status hv_initialize_particles(hv_ctx *ctx, const hv_skyrme *skm, hv_woods_saxon ws[2],
                                         hv_fermi *fermi, const hv_init_params *params,
                                         hv_init_report *report, hv_init_row *rows);

/* minim_woods_saxon (include/fit_algorithm.hpp:95-137) on the context's
 * particles and their compute_particle_densities: per species, the least-squares
 * fit of V0 / (1 + exp((r - R12) / a)) to skyrme_potential of the particle's
 * densities, from ws (in/out).  Levenberg-Marquardt with More's scaling, step
 * and gradient tests xtol = gtol = 1e-4, at most 100 iterations (the
 * reference's GSL call arguments; its ftol is not tested).  status: 1 xtol,
 * 2 gtol, 0 iterations exhausted, -1 no acceptable step, -2 fewer than 3
 * particles (ws unchanged). */
HV_API hv_status hv_fit_woods_saxon(hv_ctx *ctx, const hv_skyrme *skm, hv_woods_saxon ws[2],
                                    int iterations[2], int status[2]);

/* compute_particle_energies (include/tools.hpp:226-232) of the context's
 * particles: host array of the context's precision, caller's order. */
HV_API hv_status hv_particle_energies(hv_ctx *ctx, const hv_woods_saxon ws[2], double sigma_k,
                                      void *energy);

/* ---- adjoint: gradients of a D(t) objective ----------------------------
 * No counterpart in the reference, which has no derivative code: the
 * hand-written adjoint of the plain FP64 step (cpu_simulate's order,
 * src/hyper_vlasov.cpp:63-104), for the gradient of an objective J(D_0 ..
 * D_{n-1}) with respect to the Skyrme parameters theta = (t0, t3, sigma,
 * a_sym) that hv_skyrme_from_t0t3 maps to the context's hv_skyrme.  HV_F64
 * contexts only (HV_ERR_UNSUPPORTED otherwise).
 *
 * hv_adjoint_forward runs n_steps plain steps from the context's current
 * state (solving its fields first if nothing has), writing one observable row
 * per step as hv_run does, and keeps the particle state and phi every
 * checkpoint_every steps (device memory: (n / K + 1) (9 N + G) doubles for the
 * checkpoints, K (3 N + 8 G) for a recomputed segment).
 * hv_adjoint_backward takes dJ/dD_n for those rows and returns dJ/dtheta at
 * theta (which must be the parameters the forward ran with), and, when
 * grad_skyrme is not NULL, dJ/d(A, B, C, gamma).  It recomputes each segment
 * from its checkpoint and runs the reversed steps through it: the transposed
 * gather is a deposit, the transposed deposit a gather of weight gradients,
 * the transposed Poisson solve a second SOR solve with the context's SOR
 * settings (warm-started from the previous one).  The context is left in the
 * state the forward run ended in, with its fields marked stale.  A later
 * hv_adjoint_forward replaces the checkpoints. */
HV_API hv_status hv_adjoint_forward(hv_ctx *ctx, int n_steps, int checkpoint_every, hv_observables *obs);
HV_API hv_status hv_adjoint_backward(hv_ctx *ctx, const double *dJ_dD, const double theta[4],
                                     double grad_theta[4], double grad_skyrme[4]);

/* hv_adjoint_forward on a chosen path (no counterpart in the reference).
 * HV_PATH_PLAIN is hv_adjoint_forward.  HV_PATH_FUSED runs the forward as
 * fused FP64 steps (hv_run(HV_PATH_FUSED) per segment; missing fields are
 * solved with the fused kernels), and the following hv_adjoint_backward
 * recomputes its segments with the same steps and runs each transposed
 * Poisson solve on the persistent SOR kernel, started from the extrapolation
 * of the previous reversed steps' solutions as the fused forward starts phi.
 * Slot re-sorting (hv_fast_options.sort_every) is paused during both passes,
 * since the adjoint state is indexed by slot.  Device memory: (n / K + 1)
 * (9 N + 13 G) doubles for the checkpoints (phi and its two earlier
 * solutions, the interleaved forces and the smoothed density besides the
 * particle state), K (3 N + 10 G) for a recomputed segment.  A bounded wait of
 * the solver that runs out returns HV_ERR_TIMEOUT with the fields marked
 * stale. */
HV_API hv_status hv_adjoint_forward_path(hv_ctx *ctx, int path, int n_steps, int checkpoint_every,
                                         hv_observables *obs);

/* After hv_adjoint_backward: the path of the forward run, the iterations of
 * all transposed Poisson solves of the backward pass, and how many of them
 * stopped at the iteration cap (no counterpart in the reference). */
HV_API hv_status hv_adjoint_stats(const hv_ctx *ctx, int *path, int *adjoint_sor_iterations,
                                  int *adjoint_sor_unconverged);

/* ---- batched runs -------------------------------------------------------
 * No counterpart in the reference, which runs one nucleus per process: many
 * independent runs (own nucleus, test particles, grid and parameters, each an
 * HV_F32 context on the same device, particles uploaded) advanced together on
 * the fused path.  Per step every instance's particle step, smoothing and
 * Skyrme potential run as parallel branches, the Coulomb solves as a few
 * cooperative launches that each solve several instances ("waves"), then the
 * forces; chunks of steps are replayed from one CUDA graph.  Each instance's
 * observables are those of hv_run(HV_PATH_FUSED) on its own, up to float
 * rounding.  The contexts stay owned by the caller and must outlive the batch;
 * while it exists they are advanced only through it.
 *
 * hv_batch_create solves each instance's initial fields if needed and plans
 * with each instance's own SOR plan.  hv_batch_plan re-plans every instance's
 * SOR with at most sor_max_blocks blocks (0: the instance's own plan; an
 * instance whose grid needs more blocks' shared memory gets twice the cap, and
 * so on) and packs the solves into waves of at most one block per SM.  hv_batch_autotune
 * times trial_steps batched steps (plus one) for each candidate cap and keeps
 * the fastest, then does the same for the particle step's block size (128,
 * 256 or 512 threads, the same for every instance); the trial steps advance
 * every run.  hv_batch_tiles reports, for the first n instances, the SOR tile
 * (planes x rows per block), the blocks of the solve and the particle step's
 * block size (any pointer may be NULL).  hv_batch_run advances all
 * instances n_steps and writes n_steps observable rows per instance,
 * instance-major (obs[i * n_steps + s]; may be NULL). */
typedef struct hv_batch hv_batch;
HV_API hv_status hv_batch_create(int n_instances, hv_ctx *const *ctxs, hv_batch **out);
HV_API hv_status hv_batch_destroy(hv_batch *batch);
HV_API hv_status hv_batch_plan(hv_batch *batch, int sor_max_blocks);
HV_API hv_status hv_batch_autotune(hv_batch *batch, int trial_steps, int *chosen_cap);
HV_API hv_status hv_batch_run(hv_batch *batch, int n_steps, hv_observables *obs);
HV_API int hv_batch_waves(const hv_batch *batch);
HV_API hv_status hv_batch_tiles(const hv_batch *batch, int *sor_planes, int *sor_rows, int *sor_blocks,
                                int *particle_block, int n);

#ifdef __cplusplus
}
#endif

#endif /* HV_B200_H */
