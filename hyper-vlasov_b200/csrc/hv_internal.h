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
    // fields
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
};

// Fast-path (fused) buffers.
struct Fused {
    bool ready = false;
    double *phi64 = nullptr;    // Coulomb potential, always double
    double *phi64_prev = nullptr;
    float *delta = nullptr;     // SOR correction (float)
    float *src = nullptr;       // SOR source (float residual)
    double *delta64 = nullptr;  // SOR correction when T = double
    double *src64 = nullptr;
    void *F4 = nullptr;         // interleaved forces, T4 per node
    double *obs_dev = nullptr;  // per-step observables ring
    int obs_cap = 0;
    int *sor_its_dev = nullptr;
    int *flags = nullptr;       // device status / control words
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int prev_valid = 0;
};

}  // namespace hv

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
    bool boundary_set = false;
    bool permuted = false;   // particle slots reordered by the fused path
    bool excited = false;
    int step_index = 0;      // steps taken so far (time = step_index * dt)
    void *staging = nullptr; // pinned host staging
    size_t staging_bytes = 0;
};

namespace hv {

// ---- kernel launchers (templated on the arithmetic type) ----------------
template <typename T>
hv_status launch_deposit_atomic(hv_ctx *c, const T *x, const T *y, const T *z, T *rho);
template <typename T>
hv_status launch_deposit_sorted(hv_ctx *c, const T *x, const T *y, const T *z, T *rho);
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
