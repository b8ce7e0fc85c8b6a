// Internal declarations of the B200 step library: the context, device
// buffers and the kernel launchers shared by the translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "hv_b200.h"

namespace hv {

// Physical constants of the reference (include/sim_structs.hpp:32-37).
constexpr double kMc2 = 935.0;
constexpr double kHbarC = 197.33;
constexpr double kRho0 = 0.16;
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kE2 = 1.44;  // e^2 in MeV fm

// Records a CUDA error for hv_last_error() and maps it to a status.
hv_status cuda_status(cudaError_t e, const char *what);
void set_last_error(const std::string &msg);

#define HV_CUDA(call)                                                 \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return ::hv::cuda_status(e_, #call);   \
    } while (0)

#define HV_TRY(call)                      \
    do {                                  \
        hv_status s_ = (call);            \
        if (s_ != HV_OK) return s_;       \
    } while (0)

// Grid geometry used by every kernel (plain values, passed by value).
struct Geom {
    int nx, ny, nz;
    long long G;          // nodes per species
    double dmx, dmy, dmz; // d_max per axis
};

// One tap of the smoothing stencil: offset (a,b,c) packed as
// ((a + 512) << 20) | ((b + 512) << 10) | (c + 512).
struct TapTable {
    int count = 0;
    int lim[3] = {0, 0, 0};
    std::vector<int> packed;
    std::vector<double> w64;
    std::vector<float> w32;
};
TapTable build_taps(const hv_world &w, double sigma_r);

// Device buffers of one precision T.
template <typename T>
struct State {
    // particles (SoA, protons first, slot order; perm[slot] = caller index)
    T *x = nullptr, *y = nullptr, *z = nullptr;
    T *kx = nullptr, *ky = nullptr, *kz = nullptr;
    T *fx = nullptr, *fy = nullptr, *fz = nullptr;
    // fields; rho_raw holds 2G values and then 4 more, the first of which is,
    // as an int, the count of the FFT smoothing's wrap list (zeroed with the
    // raw density by each fused step)
    T *rho_raw = nullptr, *rho = nullptr, *U = nullptr, *phi = nullptr;
    T *Fx = nullptr, *Fy = nullptr, *Fz = nullptr;
    T *taps_w = nullptr;
};

struct Scratch {
    double *partials = nullptr;     // deterministic reduction partials
    size_t partials_len = 0;
    unsigned long long *maxbits = nullptr;  // SOR max|dphi| as ordered bits
    double *result = nullptr;       // small device results (reductions)
    double *h_result = nullptr;     // pinned host mirror of result
    // sorted-deposit buffers
    unsigned int *keys = nullptr, *keys_alt = nullptr;
    int *vals = nullptr, *vals_alt = nullptr;
    int *cell_start = nullptr;      // [2G + 1]
    void *cub_tmp = nullptr;
    size_t cub_tmp_bytes = 0;
    void *sort_tmp = nullptr;       // total x 8 bytes: the slot re-sort's gather buffer, and the stage of
                                    // uploads and downloads in permuted slot order
};

// Partition and device buffers of the persistent SOR solver (k_sor_fast.cu).
struct SorFast {
    bool ok = false;           // a partition that fits on chip was found
    int P = 0, R = 0;          // planes and rows owned by one block
    int bx = 0, by = 0;        // blocks along x (interior planes) and y
    int nblocks = 0;
    int threads = 0;
    size_t smem = 0;
    int nz2 = 0;               // (nz + 1) / 2: length of one colour half-line
    bool src_smem = false;     // the residual source also lives in shared memory
    bool tables = false;       // shared memory also holds the tagged sweeps' row tables
    void *delta = nullptr;     // SOR correction, colour-split layout
    void *src = nullptr;       // residual source, colour-split layout
    double *resid = nullptr;   // FP64 residual of phi per grid node, carried between checks
    double *partials = nullptr;
    unsigned *phase = nullptr; // per-block publish counters
    unsigned *bar = nullptr;   // [0] arrivals, [1] generation
    int *status = nullptr;     // [0] error, [1] iterations, [2] converged, [3] m hint
    double *metric = nullptr;  // final stopping quantity
    // coarse-grid correction: factor F (0: none for this grid), interior
    // extents of the coarse grid, restriction stage buffers
    int cf = 0, cmx = 0, cmy = 0, cmz = 0;
    float *t1 = nullptr, *t2 = nullptr;
    int tile_candidates = 0;   // ranked P x R candidates of a float solve
    int tile_rank = 0;         // the one planned
};

// Decomposed smoothing plan (k_smooth_fast.cu).
constexpr int kSmoothMaxR = 16;  // largest |a|, |b| or z half-width handled
// Capacity of the FFT smoothing's wrap list: particles that deposit within the
// stencil of a face in one step (more: the direct form recomputes the field).
constexpr int kWrapParticles = 65536;
struct SmoothFast {
    bool ok = false;           // tap table is symmetric with contiguous runs
    int A = 0, B = 0, W = 0;   // max |a|, |b|, z half-width
    float gx[kSmoothMaxR + 1] = {}, gy[kSmoothMaxR + 1] = {}, gz[kSmoothMaxR + 1] = {};
    int bm[kSmoothMaxR + 1] = {};                        // largest |b| for each |a| (-1: none)
    int wt[(kSmoothMaxR + 1) * (kSmoothMaxR + 1)] = {};  // w(|a|, |b|) (-1: none)
    size_t smem = 0;
    int per = 0;               // R = max(A, B, W): the kernel instantiation
    int xsplit = 1;            // x segments per column tile (the plan's choice)
    // FFT form (power-of-two axes up to 128): the circular convolution by the
    // stencil's spectrum, exact while no density lies within (A, B, W) of a
    // face, and made exact otherwise by subtracting the wrapped pairs
    bool fft = false;
    bool fft128 = false;       // 128^3: the register-transform kernels (khat in natural z order)
    void *fwork = nullptr;     // nx ny nz complex floats: both species' transform
    float *khat = nullptr;     // nx ny nz: the stencil's spectrum x term / (nx ny nz)
    void *tw = nullptr;        // 64 complex twiddles exp(-2 pi i m / 128)
    int *edge = nullptr;       // [nx]: nonzero densities found within the stencil of a face
    unsigned *occ = nullptr;   // [2][nx] (128^3 transforms): bit q set when raw density of the species
                               // lies in rows 4q..4q+3 of the x plane (written by the forward pass)
    void *wlist = nullptr;     // kWrapParticles float4: the particles depositing within the
                               // stencil of a face (grid coordinates, species), from the particle step
    double fft_term = 0.0;     // the term folded into khat
};

// Fast-path (fused) buffers.
struct Fused {
    bool ready = false;
    double *phi64 = nullptr;      // Coulomb potential (double for every precision)
    double *phi64_prev = nullptr; // previous step's phi (extrapolated warm start)
    double *phi64_prev2 = nullptr; // the step before's (quadratic extrapolation)
    void *F4 = nullptr;           // interleaved forces, 4 x T per node
    double *obs_partials = nullptr;  // per-step observable partials
    int obs_blocks = 0;           // blocks of the particle step (one partial row each)
    int pblock = 256;             // threads per block of the particle step
    int obs_rows = 0;             // capacity in steps
    int *sor_its = nullptr;       // per-step SOR iterations (device)
    double *obs_rows_dev = nullptr;  // reduced rows (device)
    cudaGraphExec_t graph = nullptr;
    int graph_len = 0;
    int last_sort = -(1 << 30);   // step of the last slot re-sort
    bool prev_valid = false;      // phi64_prev holds the previous step's phi
    bool f4_current = false;      // F4 holds the forces of the current positions
    int m_hint = 8;               // iterations of the previous SOR solve (seeds the first cycle)
    SorFast sor;
    SmoothFast smooth;
};

// Per-kernel CUDA-event timing of fused steps (hv_ctx_set_profiling).
struct Profile {
    bool on = false;
    std::vector<cudaEvent_t> events;  // event pairs (start, stop)
    std::vector<int> kernel;          // kernel id of each pair in use
    double ms[HV_K_COUNT] = {0, 0, 0, 0, 0};
    int launches[HV_K_COUNT] = {0, 0, 0, 0, 0};
};

}  // namespace hv

namespace hv {
struct Adjoint;  // adjoint.cu
}

struct hv_ctx {
    hv_world world{};
    hv::Geom geom{};
    int protons = 0, neutrons = 0, total = 0;
    hv_precision prec = HV_F64;
    hv_run_params params{};
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    hv::State<double> d64;
    hv::State<float> d32;
    int *perm = nullptr;
    hv::TapTable taps;
    int taps_count = 0;
    int *taps_dev = nullptr;
    hv::Scratch scratch;
    hv::Fused fused;
    hv::Profile prof;
    hv_fast_options fast{};
    bool boundary_set = false;
    bool fields_valid = false;  // forces correspond to the current positions
    bool permuted = false;   // particle slots reordered by the fused path
    bool excited = false;
    int step_index = 0;      // steps taken so far (time = step_index * dt)
    void *staging = nullptr; // pinned host staging
    size_t staging_bytes = 0;
    hv::Adjoint *adjoint = nullptr;  // checkpoints and work arrays of the adjoint
};

namespace hv {

// ---- kernel launchers (templated on the arithmetic type) ----------------
template <typename T>
hv_status launch_deposit_atomic(hv_ctx *c, const T *x, const T *y, const T *z, T *rho);
template <typename T>
hv_status launch_deposit_sorted(hv_ctx *c, const T *x, const T *y, const T *z, T *rho);
hv_status fused_sort_slots(hv_ctx *c);
template <typename T>
hv_status launch_smooth(hv_ctx *c, const T *rho_raw, T *rho);
template <typename T>
hv_status launch_skyrme(hv_ctx *c, const T *rho, T *U);
template <typename T>
hv_status launch_boundary(hv_ctx *c, T *phi);
template <typename T>
hv_status launch_sor_plain(hv_ctx *c, T *phi, const T *rho, int *iters, double *metric);
template <typename T>
hv_status launch_merge(hv_ctx *c, T *U, const T *phi);
template <typename T>
hv_status launch_fdm(hv_ctx *c, const T *U, T *Fx, T *Fy, T *Fz);
template <typename T>
hv_status launch_gather(hv_ctx *c, const T *x, const T *y, const T *z, const T *Fx,
                        const T *Fy, const T *Fz, T *fx, T *fy, T *fz);
template <typename T>
hv_status launch_kick(hv_ctx *c, T *kx, T *ky, T *kz, const T *fx, const T *fy, const T *fz,
                      double dt_half_fact);
template <typename T>
hv_status launch_drift(hv_ctx *c, T *x, T *y, T *z, const T *kx, const T *ky, const T *kz,
                       double dt);
template <typename T>
hv_status launch_excite(hv_ctx *c, T *kz, double eta);
template <typename T>
hv_status launch_observe(hv_ctx *c, const T *x, const T *y, const T *z, hv_observables *out);

// Fused fast path (k_fused.cu, k_sor_fast.cu)
hv_status fused_prepare(hv_ctx *c);
hv_status fused_release(hv_ctx *c);
hv_status fused_run(hv_ctx *c, int n_steps, hv_observables *obs);
hv_status fused_autotune(hv_ctx *c, int trial, hv_autotune_report *rep);
void fused_invalidate(hv_ctx *c);

// Several float SOR solves run by one cooperative launch (k_sor_fast.cu).
struct SorWave {
    int nblocks = 0;                 // all instances' blocks
    size_t smem = 0;                 // the largest instance's dynamic shared memory
    const void *kern = nullptr;
    void *args = nullptr;            // device: the instances' kernel arguments
    int *binst = nullptr, *bfirst = nullptr;  // device: block -> instance, instance -> first block
    std::vector<hv_ctx *> ctx;
};
hv_status sor_wave_build(SorWave &w, const std::vector<hv_ctx *> &cs, const std::vector<const float *> &rho,
                         const std::vector<int *> &ctl, const std::vector<int *> &its_ring, int ring);
hv_status sor_wave_launch(const SorWave &w, cudaStream_t st);
void sor_wave_release(SorWave &w);
// Lets a kernel launch with up to the device's opt-in shared memory per block.
// The attribute belongs to the function, which every context shares, so it is
// raised to the maximum once rather than set to one plan's need.
hv_status allow_max_dynamic_smem(const void *kern, int device);
// the context's particle and field buffers of type T (ctx.cu)
template <typename T>
State<T> &state(hv_ctx *c);
template <>
State<double> &state<double>(hv_ctx *c);
template <>
State<float> &state<float>(hv_ctx *c);
// a per-particle device array in slot order to a host array in the caller's
// particle order (element type of the context's precision; synchronous)
hv_status download_slots(hv_ctx *c, const void *dev, void *host);
// re-plans a context's fused SOR with at most max_blocks blocks (0: all SMs)
hv_status sor_fast_replan(hv_ctx *c, int max_blocks);
// re-plans it with the tile of the given rank (float solves; see plan_for)
hv_status sor_fast_replan_rank(hv_ctx *c, int rank, int *count);

// parts of fused float steps for the batched driver (k_fused.cu)
hv_status fused_batch_ready(hv_ctx *c);
hv_status fused_batch_begin(hv_ctx *c, int n_steps, int *exc);
hv_status fused_batch_phase_a(hv_ctx *c, cudaStream_t s);
hv_status fused_batch_phase_c(hv_ctx *c, cudaStream_t s);
hv_status fused_batch_rows(hv_ctx *c, cudaStream_t s, int s0, int k, hv_observables *obs);
hv_status fused_batch_end(hv_ctx *c, int n_steps, int exc);
void fused_batch_sor_inputs(hv_ctx *c, const float **rho, int **ctl, int **its_ring, int *ring);
void adjoint_release(hv_ctx *c);
// fused FP64 steps one at a time for the adjoint (k_fused.cu): the control
// words set for n_steps steps from the context's step (forces and phi packed
// from the plain buffers first when stale; synchronous), then one step per
// call (stream-ordered).  fused_ctl: the device control words, fused_ctl_words
// of them.
hv_status fused_adjoint_begin(hv_ctx *c, int n_steps);
hv_status fused_adjoint_step(hv_ctx *c);
int *fused_ctl(hv_ctx *c);
int fused_ctl_words();
// A double solve of lap mu = -4 pi e^2 src with mu's boundary nodes held (the
// adjoint's transposed Coulomb solve), on the persistent SOR kernel with the
// context's SOR settings, warm-started from mu and its history mu_prev,
// mu_prev2 as the context's warm-start rule says; ctl: its own control words
// ([1] iterations of the previous solve, [2] solutions held).  The outcome is
// left in the solver's status words (sor_fast_status_words).
hv_status sor_fast_launch_adjoint(hv_ctx *c, const double *src, double *mu, double *mu_prev, double *mu_prev2,
                                  int *ctl);
const int *sor_fast_status_words(hv_ctx *c);
// compute_particle_densities of N particles (protons first) given by device
// positions, into dp / dn at the same indices (pdens.cu; stream-ordered)
template <typename T>
hv_status particle_densities_at(hv_ctx *c, int N, int protons, const T *x, const T *y, const T *z, T *dp, T *dn);
// writes per-particle device arrays in the caller's order into the context's
// particle slots (x, y, z, kx, ky, kz; ctx.cu; stream-ordered)
template <typename T>
hv_status store_particles(hv_ctx *c, const T *const src[6]);
// one plain FP64 step / the field solve and gather of the current positions
hv_status plain_step_f64(hv_ctx *c, hv_observables *row);
hv_status plain_fields_f64(hv_ctx *c, int *sor_its);

// geometry helpers
inline Geom make_geom(const hv_world &w) {
    Geom g;
    g.nx = w.n[0];
    g.ny = w.n[1];
    g.nz = w.n[2];
    g.G = (long long)w.n[0] * w.n[1] * w.n[2];
    g.dmx = w.d_max[0];
    g.dmy = w.d_max[1];
    g.dmz = w.d_max[2];
    return g;
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace hv
