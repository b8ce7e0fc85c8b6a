// Context lifetime, host<->device transfers, the per-routine C entry points
// and the plain (reference-order) step driver.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include <cub/cub.cuh>

#include "hv_internal.h"

namespace hv {

size_t sorted_deposit_tmp_bytes(int total);  // k_plain.cu

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

hv_status cuda_status(cudaError_t e, const char *what) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    cudaGetLastError();  // clear a non-sticky error
    if (e == cudaErrorMemoryAllocation) return HV_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return HV_ERR_NO_DEVICE;
    return HV_ERR_CUDA;
}

// Offsets and weights of the smoothing stencil: all (a,b,c) whose node
// distance satisfies |r_i - r_j|^2 <= 16 sigma_r^2 (include/physics.hpp:205,
// 217-219), in increasing (a,b,c) -- the order of the reference's linear j
// loop -- with weights exp(-d^2 / (2 sigma_r^2)) (physics.hpp:221).  The
// distance is taken between the grid's centre node and its partner, with
// node coordinates d_max (2 i / n - 1) (include/tools.hpp:394-401), once in
// double and once in float (the two instantiations of the reference).
template <typename T>
static void taps_for(const hv_world &w, double sigma_r_d, std::vector<int> *packed, std::vector<T> *wt,
                     int lim_out[3]) {
    const T sigma_r = T(sigma_r_d);
    const T exp_term = T(1.0) / (T(2.0) * sigma_r * sigma_r);
    const T cutoff = T(16.0) * sigma_r * sigma_r;
    int lim[3], ctr[3];
    T dm[3];
    for (int a = 0; a < 3; a++) {
        dm[a] = T(w.d_max[a]);
        double h = 2.0 * w.d_max[a] / w.n[a];
        lim[a] = (int)(4.0 * sigma_r_d / h) + 2;
        if (lim[a] > w.n[a] - 1) lim[a] = w.n[a] - 1;
        ctr[a] = w.n[a] / 2;
        lim_out[a] = 0;
    }
    auto pos = [](T d, int i, int n) { return d * (T(2.0) * (T)i / (T)n - T(1.0)); };
    for (int a = -lim[0]; a <= lim[0]; a++)
        for (int b = -lim[1]; b <= lim[1]; b++)
            for (int c = -lim[2]; c <= lim[2]; c++) {
                T d0 = pos(dm[0], ctr[0], w.n[0]) - pos(dm[0], ctr[0] + a, w.n[0]);
                T d1 = pos(dm[1], ctr[1], w.n[1]) - pos(dm[1], ctr[1] + b, w.n[1]);
                T d2 = pos(dm[2], ctr[2], w.n[2]) - pos(dm[2], ctr[2] + c, w.n[2]);
                T dist2 = d0 * d0 + d1 * d1 + d2 * d2;
                if (dist2 > cutoff) continue;
                if (packed) packed->push_back(((a + 512) << 20) | ((b + 512) << 10) | (c + 512));
                wt->push_back(std::exp(-dist2 * exp_term));
                lim_out[0] = std::max(lim_out[0], std::abs(a));
                lim_out[1] = std::max(lim_out[1], std::abs(b));
                lim_out[2] = std::max(lim_out[2], std::abs(c));
            }
}

TapTable build_taps(const hv_world &w, double sigma_r) {
    TapTable t;
    int lim64[3], lim32[3];
    taps_for<double>(w, sigma_r, &t.packed, &t.w64, lim64);
    std::vector<int> packed32;
    taps_for<float>(w, sigma_r, &packed32, &t.w32, lim32);
    // the float and double pair sets agree except for pairs within one
    // rounding of the cutoff; keep the double set and drop float weights that
    // do not line up
    if (packed32 != t.packed) {
        std::vector<float> w32(t.packed.size(), 0.0f);
        size_t j = 0;
        for (size_t i = 0; i < t.packed.size(); i++) {
            while (j < packed32.size() && packed32[j] < t.packed[i]) j++;
            if (j < packed32.size() && packed32[j] == t.packed[i]) w32[i] = t.w32[j];
        }
        t.w32.swap(w32);
    }
    t.count = (int)t.packed.size();
    for (int a = 0; a < 3; a++) t.lim[a] = lim64[a];
    return t;
}

template <typename T>
State<T> &state(hv_ctx *c);
template <>
State<double> &state<double>(hv_ctx *c) { return c->d64; }
template <>
State<float> &state<float>(hv_ctx *c) { return c->d32; }

namespace {

template <typename T>
hv_status alloc_state(hv_ctx *c) {
    State<T> &s = state<T>(c);
    const size_t n = (size_t)(c->total > 0 ? c->total : 1);
    const size_t G2 = (size_t)(2 * c->geom.G);
    T **parts[] = {&s.x, &s.y, &s.z, &s.kx, &s.ky, &s.kz, &s.fx, &s.fy, &s.fz};
    for (T **p : parts) {
        HV_CUDA(cudaMalloc((void **)p, n * sizeof(T)));
        HV_CUDA(cudaMemsetAsync(*p, 0, n * sizeof(T), c->stream));
    }
    T **grids[] = {&s.rho_raw, &s.rho, &s.U, &s.Fx, &s.Fy, &s.Fz};
    for (T **p : grids) {
        // rho_raw: 4 more values, the wrap list's count (State)
        const size_t len = G2 + (p == &s.rho_raw ? 4 : 0);
        HV_CUDA(cudaMalloc((void **)p, len * sizeof(T)));
        HV_CUDA(cudaMemsetAsync(*p, 0, len * sizeof(T), c->stream));
    }
    HV_CUDA(cudaMalloc((void **)&s.phi, (size_t)c->geom.G * sizeof(T)));
    HV_CUDA(cudaMemsetAsync(s.phi, 0, (size_t)c->geom.G * sizeof(T), c->stream));
    const size_t nt = (size_t)(c->taps_count > 0 ? c->taps_count : 1);
    HV_CUDA(cudaMalloc((void **)&s.taps_w, nt * sizeof(T)));
    const void *src = sizeof(T) == 8 ? (const void *)c->taps.w64.data() : (const void *)c->taps.w32.data();
    if (c->taps_count > 0)
        HV_CUDA(cudaMemcpyAsync(s.taps_w, src, c->taps_count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return HV_OK;
}

template <typename T>
void free_state(State<T> &s) {
    T *ptrs[] = {s.x, s.y, s.z, s.kx, s.ky, s.kz, s.fx, s.fy, s.fz, s.rho_raw, s.rho, s.U, s.phi, s.Fx, s.Fy, s.Fz, s.taps_w};
    for (T *p : ptrs)
        if (p) cudaFree(p);
    s = State<T>();
}

hv_status check_world(const hv_world *w) {
    if (!w) return HV_ERR_BAD_ARG;
    for (int a = 0; a < 3; a++) {
        if (w->n[a] < 3 || w->n[a] > 1024) return HV_ERR_BAD_ARG;
        if (!(w->d_max[a] > 0.0) || !std::isfinite(w->d_max[a])) return HV_ERR_BAD_ARG;
    }
    long long G = (long long)w->n[0] * w->n[1] * w->n[2];
    if (2 * G >= (1ll << 31)) return HV_ERR_BAD_ARG;
    return HV_OK;
}

hv_status check_params(const hv_run_params *p) {
    if (!p) return HV_ERR_BAD_ARG;
    if (p->z < 0 || p->n < 0 || p->z + p->n <= 0) return HV_ERR_BAD_ARG;
    if (p->part_per_nucleon <= 0) return HV_ERR_BAD_ARG;
    if (!(p->sigma_r > 0.0) || !std::isfinite(p->sigma_r)) return HV_ERR_BAD_ARG;
    if (!std::isfinite(p->dt) || !std::isfinite(p->t_exc) || !std::isfinite(p->eta_exc)) return HV_ERR_BAD_ARG;
    if (!(p->sor.omega > 0.0 && p->sor.omega < 2.0)) return HV_ERR_BAD_ARG;
    if (!(p->sor.tol > 0.0) || p->sor.max_iter < 1) return HV_ERR_BAD_ARG;
    if (p->sor.criterion != HV_SOR_MAX_UPDATE && p->sor.criterion != HV_SOR_REL_RESIDUAL) return HV_ERR_BAD_ARG;
    if (p->deposit_mode != HV_DEPOSIT_ATOMIC && p->deposit_mode != HV_DEPOSIT_SORTED) return HV_ERR_BAD_ARG;
    return HV_OK;
}

__global__ void k_iota(int n, int *p) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

// out[perm[s]] = in[s]: slot order -> caller order
template <typename T>
__global__ void k_unpermute(int n, const int *__restrict__ perm, const T *__restrict__ in, T *out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[perm[s]] = in[s];
}

// out[s] = in[perm[s]]: caller order -> slot order
template <typename T>
__global__ void k_permute(int n, const int *__restrict__ perm, const T *__restrict__ in, T *out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[s] = in[perm[s]];
}

// Keys of the fused path's slot re-sort: species * (G + 1) + the particle's
// CIC base cell, G for a particle outside the grid, so that the sort keeps the
// protons' slots before the neutrons'.
template <typename T>
__global__ void k_slot_keys(Geom g, int protons, int total, const T *__restrict__ x, const T *__restrict__ y,
                            const T *__restrict__ z, unsigned int *keys, int *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const T cx = (g.nx / T(2.0)) * (x[i] / T(g.dmx) + T(1.0));
    const T cy = (g.ny / T(2.0)) * (y[i] / T(g.dmy) + T(1.0));
    const T cz = (g.nz / T(2.0)) * (z[i] / T(g.dmz) + T(1.0));
    long long cell = g.G;
    if (cx >= T(0) && cy >= T(0) && cz >= T(0) && cx < g.nx && cy < g.ny && cz < g.nz)
        cell = ((long long)(int)cx * g.ny + (int)cy) * g.nz + (int)cz;
    keys[i] = (unsigned int)(cell + (i < protons ? 0 : g.G + 1));
    vals[i] = i;
}

template <typename T>
hv_status sort_slots_typed(hv_ctx *c, State<T> &s) {
    const int n = c->total;
    if (n == 0) return HV_OK;
    Scratch &sc = c->scratch;
    k_slot_keys<T><<<div_up(n, 256), 256, 0, c->stream>>>(c->geom, c->protons, n, s.x, s.y, s.z, sc.keys, sc.vals);
    HV_CUDA(cudaGetLastError());
    const unsigned long long nkeys = 2ull * ((unsigned long long)c->geom.G + 1);
    int end_bit = 1;
    while ((1ull << end_bit) < nkeys) end_bit++;
    size_t bytes = sc.cub_tmp_bytes;
    HV_CUDA(cub::DeviceRadixSort::SortPairs(sc.cub_tmp, bytes, sc.keys, sc.keys_alt, sc.vals, sc.vals_alt, n, 0,
                                            end_bit, c->stream));
    // every per-particle array and the caller permutation follow the new order
    T *tmp = reinterpret_cast<T *>(sc.sort_tmp);
    T *arrs[] = {s.x, s.y, s.z, s.kx, s.ky, s.kz, s.fx, s.fy, s.fz};
    for (T *a : arrs) {
        k_permute<T><<<div_up(n, 256), 256, 0, c->stream>>>(n, sc.vals_alt, a, tmp);
        HV_CUDA(cudaMemcpyAsync(a, tmp, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
    }
    int *ptmp = reinterpret_cast<int *>(sc.sort_tmp);
    k_permute<int><<<div_up(n, 256), 256, 0, c->stream>>>(n, sc.vals_alt, c->perm, ptmp);
    HV_CUDA(cudaMemcpyAsync(c->perm, ptmp, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
    HV_CUDA(cudaGetLastError());
    c->permuted = true;
    return HV_OK;
}

template <typename T>
T *part_ptr(State<T> &s, int which) {
    switch (which) {
        case HV_PART_X: return s.x;
        case HV_PART_Y: return s.y;
        case HV_PART_Z: return s.z;
        case HV_PART_KX: return s.kx;
        case HV_PART_KY: return s.ky;
        case HV_PART_KZ: return s.kz;
        case HV_PART_FX: return s.fx;
        case HV_PART_FY: return s.fy;
        case HV_PART_FZ: return s.fz;
        default: return nullptr;
    }
}

template <typename T>
T *field_ptr(State<T> &s, int which, long long *count, long long G) {
    *count = 2 * G;
    switch (which) {
        case HV_FIELD_DENSITY_RAW: return s.rho_raw;
        case HV_FIELD_DENSITY: return s.rho;
        case HV_FIELD_POTENTIAL: return s.U;
        case HV_FIELD_COULOMB: *count = G; return s.phi;
        case HV_FIELD_FORCE_X: return s.Fx;
        case HV_FIELD_FORCE_Y: return s.Fy;
        case HV_FIELD_FORCE_Z: return s.Fz;
        default: return nullptr;
    }
}

bool slots_permuted(hv_ctx *c);

template <typename T>
hv_status upload_part(hv_ctx *c, int which, const void *host) {
    T *d = part_ptr(state<T>(c), which);
    if (!d) return HV_ERR_BAD_ARG;
    if (c->total == 0) return HV_OK;
    if (!host) return HV_ERR_BAD_ARG;
    const size_t bytes = sizeof(T) * c->total;
    if (slots_permuted(c)) {
        // stage in caller order (the re-sort's gather buffer), then gather
        // into slot order
        T *stage = reinterpret_cast<T *>(c->scratch.sort_tmp);
        HV_CUDA(cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, c->stream));
        k_permute<T><<<div_up(c->total, 256), 256, 0, c->stream>>>(c->total, c->perm, stage, d);
        HV_CUDA(cudaGetLastError());
    } else {
        HV_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    return HV_OK;
}

template <typename T>
hv_status download_part(hv_ctx *c, int which, void *host) {
    T *d = part_ptr(state<T>(c), which);
    if (!d) return HV_ERR_BAD_ARG;
    if (c->total == 0) return HV_OK;
    if (!host) return HV_ERR_BAD_ARG;
    const size_t bytes = sizeof(T) * c->total;
    if (slots_permuted(c)) {
        T *stage = reinterpret_cast<T *>(c->scratch.sort_tmp);
        k_unpermute<T><<<div_up(c->total, 256), 256, 0, c->stream>>>(c->total, c->perm, d, stage);
        HV_CUDA(cudaGetLastError());
        HV_CUDA(cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    } else {
        HV_CUDA(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

// ---- one step of the plain path, cpu_simulate order (src/hyper_vlasov.cpp)
template <typename T>
hv_status fields_and_gather(hv_ctx *c, int *sor_its) {
    State<T> &s = state<T>(c);
    if (c->params.deposit_mode == HV_DEPOSIT_SORTED)
        HV_TRY(launch_deposit_sorted<T>(c, s.x, s.y, s.z, s.rho_raw));
    else
        HV_TRY(launch_deposit_atomic<T>(c, s.x, s.y, s.z, s.rho_raw));
    HV_TRY(launch_smooth<T>(c, s.rho_raw, s.rho));
    if (!c->boundary_set) {  // set once before the first solve (hyper_vlasov.cpp:56)
        HV_TRY(launch_boundary<T>(c, s.phi));
        c->boundary_set = true;
    }
    HV_TRY(launch_skyrme<T>(c, s.rho, s.U));
    hv_status st = launch_sor_plain<T>(c, s.phi, s.rho, sor_its, nullptr);
    if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
    HV_TRY(launch_merge<T>(c, s.U, s.phi));
    HV_TRY(launch_fdm<T>(c, s.U, s.Fx, s.Fy, s.Fz));
    HV_TRY(launch_gather<T>(c, s.x, s.y, s.z, s.Fx, s.Fy, s.Fz, s.fx, s.fy, s.fz));
    return st;
}

template <typename T>
hv_status plain_step(hv_ctx *c, hv_observables *row) {
    State<T> &s = state<T>(c);
    const double dt = c->params.dt;
    const T tnow = T(c->step_index) * T(dt);
    if (row) {
        HV_TRY(launch_observe<T>(c, s.x, s.y, s.z, row));
        row->t = (double)tnow;
    }
    if (tnow >= T(c->params.t_exc) && !c->excited) {  // hyper_vlasov.cpp:86-89
        c->excited = true;
        HV_TRY(launch_excite<T>(c, s.kz, c->params.eta_exc));
    }
    HV_TRY(launch_kick<T>(c, s.kx, s.ky, s.kz, s.fx, s.fy, s.fz, dt));
    HV_TRY(launch_drift<T>(c, s.x, s.y, s.z, s.kx, s.ky, s.kz, dt));
    int its = 0;
    hv_status st = fields_and_gather<T>(c, &its);
    if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
    HV_TRY(launch_kick<T>(c, s.kx, s.ky, s.kz, s.fx, s.fy, s.fz, dt));
    if (row) {
        row->sor_iterations = its;
        if (st == HV_ERR_NOT_CONVERGED) row->flags |= HV_OBS_SOR_NOT_CONVERGED;
    }
    c->step_index++;
    return HV_OK;
}

bool slots_permuted(hv_ctx *c) { return c->permuted; }

}  // namespace

// Re-sorts the particle slots by CIC cell within each species (a stable radix
// sort), so that the particles of a warp gather and deposit in few cells; the
// fused path calls it every hv_fast_options.sort_every steps, between graph
// launches.  Downloads and uploads follow the slot permutation.
hv_status fused_sort_slots(hv_ctx *c) {
    return c->prec == HV_F64 ? sort_slots_typed<double>(c, c->d64) : sort_slots_typed<float>(c, c->d32);
}

hv_status plain_step_f64(hv_ctx *c, hv_observables *row) { return plain_step<double>(c, row); }

namespace {
template <typename T>
hv_status download_slots_t(hv_ctx *c, const T *d, T *host) {
    const size_t bytes = sizeof(T) * c->total;
    if (slots_permuted(c)) {
        T *stage = reinterpret_cast<T *>(c->scratch.sort_tmp);
        k_unpermute<T><<<div_up(c->total, 256), 256, 0, c->stream>>>(c->total, c->perm, d, stage);
        HV_CUDA(cudaGetLastError());
        HV_CUDA(cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, c->stream));
    } else {
        HV_CUDA(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}
}  // namespace

template <typename T>
hv_status store_particles(hv_ctx *c, const T *const src[6]) {
    if (c->total == 0) return HV_OK;
    State<T> &st = state<T>(c);
    T *dst[6] = {st.x, st.y, st.z, st.kx, st.ky, st.kz};
    for (int a = 0; a < 6; a++) {
        if (slots_permuted(c)) {
            k_permute<T><<<div_up(c->total, 256), 256, 0, c->stream>>>(c->total, c->perm, src[a], dst[a]);
            HV_CUDA(cudaGetLastError());
        } else {
            HV_CUDA(cudaMemcpyAsync(dst[a], src[a], sizeof(T) * c->total, cudaMemcpyDeviceToDevice, c->stream));
        }
    }
    c->fields_valid = false;
    fused_invalidate(c);
    return HV_OK;
}
template hv_status store_particles<double>(hv_ctx *, const double *const[6]);
template hv_status store_particles<float>(hv_ctx *, const float *const[6]);

hv_status download_slots(hv_ctx *c, const void *dev, void *host) {
    if (c->total == 0) return HV_OK;
    return c->prec == HV_F64 ? download_slots_t<double>(c, (const double *)dev, (double *)host)
                             : download_slots_t<float>(c, (const float *)dev, (float *)host);
}

hv_status allow_max_dynamic_smem(const void *kern, int device) {
    cudaFuncAttributes fa;
    HV_CUDA(cudaFuncGetAttributes(&fa, kern));
    int optin = 0;
    HV_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (fa.maxDynamicSharedSizeBytes < dyn)
        HV_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return HV_OK;
}
hv_status plain_fields_f64(hv_ctx *c, int *sor_its) { return fields_and_gather<double>(c, sor_its); }

}  // namespace hv

using namespace hv;

extern "C" {

const char *hv_version(void) { return "hv_b200 0.1.0 (sm_100a)"; }

const char *hv_status_string(hv_status s) {
    switch (s) {
        case HV_OK: return "ok";
        case HV_ERR_BAD_ARG: return "bad argument";
        case HV_ERR_CUDA: return "CUDA error";
        case HV_ERR_NOT_CONVERGED: return "SOR not converged";
        case HV_ERR_NO_DEVICE: return "no sm_100 device";
        case HV_ERR_OOM: return "out of device memory";
        case HV_ERR_TIMEOUT: return "device wait timed out";
        case HV_ERR_UNSUPPORTED: return "unsupported";
        case HV_ERR_NONFINITE: return "non-finite value";
    }
    return "unknown";
}

const char *hv_last_error(void) { return g_last_error.c_str(); }

int hv_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int ok = 0;
    for (int d = 0; d < n; d++) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ok++;
    }
    return ok;
}

hv_status hv_ctx_create(const hv_world *world, int protons, int neutrons, hv_precision prec,
                        const hv_run_params *params, int device, hv_ctx **out) {
    if (!out) return HV_ERR_BAD_ARG;
    *out = nullptr;
    HV_TRY(check_world(world));
    HV_TRY(check_params(params));
    if (protons < 0 || neutrons < 0 || (long long)protons + neutrons > (1ll << 30)) return HV_ERR_BAD_ARG;
    if (prec != HV_F64 && prec != HV_F32) return HV_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return HV_ERR_NO_DEVICE;
    }
    if (device < 0) HV_CUDA(cudaGetDevice(&device));
    if (device >= ndev) return HV_ERR_BAD_ARG;
    cudaDeviceProp prop;
    HV_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_last_error("device is not sm_100 (compute capability 10.x)");
        return HV_ERR_NO_DEVICE;
    }
    HV_CUDA(cudaSetDevice(device));
    hv_ctx *c = new (std::nothrow) hv_ctx();
    if (!c) return HV_ERR_OOM;
    c->world = *world;
    c->geom = make_geom(*world);
    c->protons = protons;
    c->neutrons = neutrons;
    c->total = protons + neutrons;
    c->prec = prec;
    c->params = *params;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    hv_fast_options_default(&c->fast);
    hv_status st = HV_OK;
    auto fail = [&](hv_status s) {
        hv_ctx_destroy(c);
        return s;
    };
    if ((st = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) != HV_OK &&
        c->stream == nullptr)
        return fail(st);
    c->taps = build_taps(*world, params->sigma_r);
    c->taps_count = c->taps.count;
    for (int a = 0; a < 3; a++)
        if (c->taps.lim[a] > 500) return fail(HV_ERR_UNSUPPORTED);
    if (cudaMalloc((void **)&c->taps_dev, sizeof(int) * (c->taps_count > 0 ? c->taps_count : 1)) != cudaSuccess)
        return fail(cuda_status(cudaErrorMemoryAllocation, "taps"));
    if (c->taps_count > 0 &&
        cudaMemcpyAsync(c->taps_dev, c->taps.packed.data(), sizeof(int) * c->taps_count, cudaMemcpyHostToDevice,
                        c->stream) != cudaSuccess)
        return fail(cuda_status(cudaGetLastError(), "taps upload"));
    st = prec == HV_F64 ? alloc_state<double>(c) : alloc_state<float>(c);
    if (st != HV_OK) return fail(st);
    const int n = c->total > 0 ? c->total : 1;
    Scratch &s = c->scratch;
    s.partials_len = (size_t)8 * 4 * c->sm_count + 64;
    s.cub_tmp_bytes = sorted_deposit_tmp_bytes(n);
    if (cudaMalloc((void **)&c->perm, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc((void **)&s.partials, sizeof(double) * s.partials_len) != cudaSuccess ||
        cudaMalloc((void **)&s.maxbits, sizeof(unsigned long long) * 4) != cudaSuccess ||
        cudaMalloc((void **)&s.result, sizeof(double) * 64) != cudaSuccess ||
        cudaMallocHost((void **)&s.h_result, sizeof(double) * 64) != cudaSuccess ||
        cudaMalloc((void **)&s.keys, sizeof(unsigned int) * n) != cudaSuccess ||
        cudaMalloc((void **)&s.keys_alt, sizeof(unsigned int) * n) != cudaSuccess ||
        cudaMalloc((void **)&s.vals, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc((void **)&s.vals_alt, sizeof(int) * n) != cudaSuccess ||
        cudaMalloc((void **)&s.cell_start, sizeof(int) * (2 * c->geom.G + 1)) != cudaSuccess ||
        cudaMalloc(&s.cub_tmp, s.cub_tmp_bytes > 0 ? s.cub_tmp_bytes : 16) != cudaSuccess ||
        cudaMalloc(&s.sort_tmp, sizeof(double) * (size_t)n) != cudaSuccess)
        return fail(cuda_status(cudaErrorMemoryAllocation, "scratch"));
    k_iota<<<div_up(n, 256), 256, 0, c->stream>>>(n, c->perm);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(cuda_status(cudaGetLastError(), "create"));
    *out = c;
    return HV_OK;
}

hv_status hv_ctx_destroy(hv_ctx *c) {
    if (!c) return HV_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    fused_release(c);
    adjoint_release(c);
    for (cudaEvent_t e : c->prof.events) cudaEventDestroy(e);
    c->prof.events.clear();
    free_state(c->d64);
    free_state(c->d32);
    Scratch &s = c->scratch;
    void *ptrs[] = {c->perm, c->taps_dev, s.partials, s.maxbits, s.result, s.keys, s.keys_alt, s.vals, s.vals_alt,
                    s.cell_start, s.cub_tmp, s.sort_tmp};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (s.h_result) cudaFreeHost(s.h_result);
    if (c->staging) cudaFreeHost(c->staging);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HV_OK;
}

hv_status hv_ctx_set_params(hv_ctx *c, const hv_run_params *p) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_TRY(check_params(p));
    bool taps_change = p->sigma_r != c->params.sigma_r;
    c->params = *p;
    if (taps_change) {
        HV_CUDA(cudaSetDevice(c->device));
        TapTable t = build_taps(c->world, p->sigma_r);
        if (t.count != c->taps_count) {
            HV_CUDA(cudaStreamSynchronize(c->stream));
            cudaFree(c->taps_dev);
            c->taps_dev = nullptr;
            HV_CUDA(cudaMalloc((void **)&c->taps_dev, sizeof(int) * (t.count > 0 ? t.count : 1)));
            if (c->d64.taps_w) { cudaFree(c->d64.taps_w); HV_CUDA(cudaMalloc((void **)&c->d64.taps_w, sizeof(double) * (t.count > 0 ? t.count : 1))); }
            if (c->d32.taps_w) { cudaFree(c->d32.taps_w); HV_CUDA(cudaMalloc((void **)&c->d32.taps_w, sizeof(float) * (t.count > 0 ? t.count : 1))); }
        }
        c->taps = t;
        c->taps_count = t.count;
        if (t.count > 0) {
            HV_CUDA(cudaMemcpyAsync(c->taps_dev, t.packed.data(), sizeof(int) * t.count, cudaMemcpyHostToDevice, c->stream));
            if (c->d64.taps_w)
                HV_CUDA(cudaMemcpyAsync(c->d64.taps_w, t.w64.data(), sizeof(double) * t.count, cudaMemcpyHostToDevice, c->stream));
            if (c->d32.taps_w)
                HV_CUDA(cudaMemcpyAsync(c->d32.taps_w, t.w32.data(), sizeof(float) * t.count, cudaMemcpyHostToDevice, c->stream));
        }
        HV_CUDA(cudaStreamSynchronize(c->stream));
    }
    HV_CUDA(cudaStreamSynchronize(c->stream));
    fused_release(c);  // plans and graphs depend on the parameters
    return HV_OK;
}

hv_status hv_ctx_get_params(const hv_ctx *c, hv_run_params *out) {
    if (!c || !out) return HV_ERR_BAD_ARG;
    *out = c->params;
    return HV_OK;
}

void *hv_ctx_stream(hv_ctx *c) { return c ? (void *)c->stream : nullptr; }

hv_status hv_ctx_synchronize(hv_ctx *c) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

#define DISPATCH(c, EXPR_D, EXPR_F) ((c)->prec == HV_F64 ? (EXPR_D) : (EXPR_F))

hv_status hv_upload_particle_array(hv_ctx *c, int which, const void *host) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (which <= HV_PART_Z) c->fields_valid = false;
    fused_invalidate(c);
    HV_TRY(DISPATCH(c, upload_part<double>(c, which, host), upload_part<float>(c, which, host)));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

hv_status hv_download_particle_array(hv_ctx *c, int which, void *host) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    return DISPATCH(c, download_part<double>(c, which, host), download_part<float>(c, which, host));
}

hv_status hv_upload_particles(hv_ctx *c, const void *x, const void *y, const void *z, const void *kx,
                              const void *ky, const void *kz) {
    if (!c) return HV_ERR_BAD_ARG;
    const void *src[6] = {x, y, z, kx, ky, kz};
    HV_CUDA(cudaSetDevice(c->device));
    if (x || y || z) c->fields_valid = false;
    fused_invalidate(c);
    for (int a = 0; a < 6; a++)
        if (src[a]) HV_TRY(DISPATCH(c, upload_part<double>(c, a, src[a]), upload_part<float>(c, a, src[a])));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

hv_status hv_download_particles(hv_ctx *c, void *x, void *y, void *z, void *kx, void *ky, void *kz) {
    if (!c) return HV_ERR_BAD_ARG;
    void *dst[6] = {x, y, z, kx, ky, kz};
    HV_CUDA(cudaSetDevice(c->device));
    for (int a = 0; a < 6; a++)
        if (dst[a]) HV_TRY(DISPATCH(c, download_part<double>(c, a, dst[a]), download_part<float>(c, a, dst[a])));
    return HV_OK;
}

hv_status hv_upload_field(hv_ctx *c, int field, const void *host) {
    if (!c || !host) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    long long n = 0;
    void *d = DISPATCH(c, (void *)field_ptr(c->d64, field, &n, c->geom.G), (void *)field_ptr(c->d32, field, &n, c->geom.G));
    if (!d) return HV_ERR_BAD_ARG;
    const size_t es = c->prec == HV_F64 ? 8 : 4;
    fused_invalidate(c);
    HV_CUDA(cudaMemcpyAsync(d, host, es * n, cudaMemcpyHostToDevice, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    if (field == HV_FIELD_COULOMB) c->boundary_set = true;  // the caller owns phi now
    return HV_OK;
}

hv_status hv_download_field(hv_ctx *c, int field, void *host) {
    if (!c || !host) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    long long n = 0;
    void *d = DISPATCH(c, (void *)field_ptr(c->d64, field, &n, c->geom.G), (void *)field_ptr(c->d32, field, &n, c->geom.G));
    if (!d) return HV_ERR_BAD_ARG;
    const size_t es = c->prec == HV_F64 ? 8 : 4;
    HV_CUDA(cudaMemcpyAsync(host, d, es * n, cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

hv_status hv_field_device_ptr(hv_ctx *c, int field, void **dev_ptr) {
    if (!c || !dev_ptr) return HV_ERR_BAD_ARG;
    long long n = 0;
    void *d = DISPATCH(c, (void *)field_ptr(c->d64, field, &n, c->geom.G), (void *)field_ptr(c->d32, field, &n, c->geom.G));
    if (!d) return HV_ERR_BAD_ARG;
    *dev_ptr = d;
    return HV_OK;
}

// ---- per-routine entry points -------------------------------------------
#define STAGE_BEGIN(c)                          \
    if (!(c)) return HV_ERR_BAD_ARG;            \
    HV_CUDA(cudaSetDevice((c)->device));        \
    fused_invalidate(c);

#define SYNC_END(c)                                  \
    HV_CUDA(cudaStreamSynchronize((c)->stream));     \
    return HV_OK;

hv_status hv_deposit_cic(hv_ctx *c) {
    STAGE_BEGIN(c);
    if (c->params.deposit_mode == HV_DEPOSIT_SORTED)
        HV_TRY(DISPATCH(c, launch_deposit_sorted<double>(c, c->d64.x, c->d64.y, c->d64.z, c->d64.rho_raw),
                        launch_deposit_sorted<float>(c, c->d32.x, c->d32.y, c->d32.z, c->d32.rho_raw)));
    else
        HV_TRY(DISPATCH(c, launch_deposit_atomic<double>(c, c->d64.x, c->d64.y, c->d64.z, c->d64.rho_raw),
                        launch_deposit_atomic<float>(c, c->d32.x, c->d32.y, c->d32.z, c->d32.rho_raw)));
    SYNC_END(c);
}

hv_status hv_smooth_density(hv_ctx *c) {
    STAGE_BEGIN(c);
    HV_TRY(DISPATCH(c, launch_smooth<double>(c, c->d64.rho_raw, c->d64.rho),
                    launch_smooth<float>(c, c->d32.rho_raw, c->d32.rho)));
    SYNC_END(c);
}

hv_status hv_skyrme_potential(hv_ctx *c) {
    STAGE_BEGIN(c);
    HV_TRY(DISPATCH(c, launch_skyrme<double>(c, c->d64.rho, c->d64.U), launch_skyrme<float>(c, c->d32.rho, c->d32.U)));
    SYNC_END(c);
}

hv_status hv_coulomb_boundary(hv_ctx *c) {
    STAGE_BEGIN(c);
    HV_TRY(DISPATCH(c, launch_boundary<double>(c, c->d64.phi), launch_boundary<float>(c, c->d32.phi)));
    c->boundary_set = true;
    SYNC_END(c);
}

hv_status hv_coulomb_sor(hv_ctx *c, int *iterations, double *metric) {
    STAGE_BEGIN(c);
    hv_status st = DISPATCH(c, launch_sor_plain<double>(c, c->d64.phi, c->d64.rho, iterations, metric),
                            launch_sor_plain<float>(c, c->d32.phi, c->d32.rho, iterations, metric));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return st;
}

hv_status hv_merge_potentials(hv_ctx *c) {
    STAGE_BEGIN(c);
    HV_TRY(DISPATCH(c, launch_merge<double>(c, c->d64.U, c->d64.phi), launch_merge<float>(c, c->d32.U, c->d32.phi)));
    SYNC_END(c);
}

hv_status hv_forces_fdm(hv_ctx *c) {
    STAGE_BEGIN(c);
    HV_TRY(DISPATCH(c, launch_fdm<double>(c, c->d64.U, c->d64.Fx, c->d64.Fy, c->d64.Fz),
                    launch_fdm<float>(c, c->d32.U, c->d32.Fx, c->d32.Fy, c->d32.Fz)));
    SYNC_END(c);
}

hv_status hv_gather_cic(hv_ctx *c) {
    STAGE_BEGIN(c);
    State<double> &a = c->d64;
    State<float> &b = c->d32;
    HV_TRY(DISPATCH(c, launch_gather<double>(c, a.x, a.y, a.z, a.Fx, a.Fy, a.Fz, a.fx, a.fy, a.fz),
                    launch_gather<float>(c, b.x, b.y, b.z, b.Fx, b.Fy, b.Fz, b.fx, b.fy, b.fz)));
    SYNC_END(c);
}

hv_status hv_kick_half(hv_ctx *c, double dt) {
    STAGE_BEGIN(c);
    if (!std::isfinite(dt)) return HV_ERR_BAD_ARG;
    State<double> &a = c->d64;
    State<float> &b = c->d32;
    HV_TRY(DISPATCH(c, launch_kick<double>(c, a.kx, a.ky, a.kz, a.fx, a.fy, a.fz, dt),
                    launch_kick<float>(c, b.kx, b.ky, b.kz, b.fx, b.fy, b.fz, dt)));
    SYNC_END(c);
}

hv_status hv_drift(hv_ctx *c, double dt) {
    STAGE_BEGIN(c);
    if (!std::isfinite(dt)) return HV_ERR_BAD_ARG;
    State<double> &a = c->d64;
    State<float> &b = c->d32;
    HV_TRY(DISPATCH(c, launch_drift<double>(c, a.x, a.y, a.z, a.kx, a.ky, a.kz, dt),
                    launch_drift<float>(c, b.x, b.y, b.z, b.kx, b.ky, b.kz, dt)));
    SYNC_END(c);
}

hv_status hv_excite(hv_ctx *c, double eta) {
    STAGE_BEGIN(c);
    if (!std::isfinite(eta)) return HV_ERR_BAD_ARG;
    HV_TRY(DISPATCH(c, launch_excite<double>(c, c->d64.kz, eta), launch_excite<float>(c, c->d32.kz, eta)));
    SYNC_END(c);
}

hv_status hv_observe(hv_ctx *c, hv_observables *out) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (!out) return HV_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    HV_TRY(DISPATCH(c, launch_observe<double>(c, c->d64.x, c->d64.y, c->d64.z, out),
                    launch_observe<float>(c, c->d32.x, c->d32.y, c->d32.z, out)));
    out->t = c->step_index * c->params.dt;
    return HV_OK;
}

void hv_fast_options_default(hv_fast_options *o) {
    if (!o) return;
    o->sor_warm_start = HV_WARM_QUADRATIC;
    o->sor_inner_min = 8;
    o->sor_inner_max = 256;
    o->sort_every = 16;
    o->graph_steps = 8;
    o->sor_exchange = HV_SOR_EXCHANGE_AUTO;
    o->smooth_fft = 1;
    o->sor_omega = 0.0;
    o->sor_wait_limit = 0;
    o->sor_coarse = 1;
    o->sor_coarse_sweeps = 12;
    o->deposit_aggregate = 1;
    o->sor_coarse_omega = 0.0;
}

hv_status hv_ctx_set_fast_options(hv_ctx *c, const hv_fast_options *o) {
    if (!c || !o) return HV_ERR_BAD_ARG;
    if (o->sor_warm_start != HV_WARM_PREVIOUS && o->sor_warm_start != HV_WARM_EXTRAPOLATE &&
        o->sor_warm_start != HV_WARM_QUADRATIC)
        return HV_ERR_BAD_ARG;
    if (o->sor_inner_min < 1 || o->sor_inner_max < o->sor_inner_min || o->sor_inner_max > 4096) return HV_ERR_BAD_ARG;
    if (o->sort_every < 0 || o->graph_steps < 0 || o->graph_steps > 64) return HV_ERR_BAD_ARG;
    if (o->sor_exchange != HV_SOR_EXCHANGE_AUTO && o->sor_exchange != HV_SOR_EXCHANGE_FLAGS) return HV_ERR_BAD_ARG;
    if (o->smooth_fft < 0 || o->smooth_fft > 2) return HV_ERR_BAD_ARG;
    if (!(o->sor_omega == 0.0 || (o->sor_omega > 0.0 && o->sor_omega < 2.0))) return HV_ERR_BAD_ARG;
    if (o->sor_wait_limit < 0) return HV_ERR_BAD_ARG;
    if (o->sor_coarse < 0 || o->sor_coarse > 1 || o->sor_coarse_sweeps < 1 || o->sor_coarse_sweeps > 4096)
        return HV_ERR_BAD_ARG;
    if (o->deposit_aggregate < 0 || o->deposit_aggregate > 1) return HV_ERR_BAD_ARG;
    if (!(o->sor_coarse_omega == 0.0 || (o->sor_coarse_omega > 0.0 && o->sor_coarse_omega < 2.0)))
        return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    if (c->fused.graph) {
        cudaGraphExecDestroy(c->fused.graph);
        c->fused.graph = nullptr;
        c->fused.graph_len = 0;
    }
    c->fast = *o;
    return HV_OK;
}

hv_status hv_ctx_get_fast_options(const hv_ctx *c, hv_fast_options *o) {
    if (!c || !o) return HV_ERR_BAD_ARG;
    *o = c->fast;
    return HV_OK;
}

hv_status hv_ctx_set_profiling(hv_ctx *c, int enable) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    c->prof.on = enable != 0;
    c->prof.kernel.clear();
    for (int k = 0; k < HV_K_COUNT; k++) {
        c->prof.ms[k] = 0.0;
        c->prof.launches[k] = 0;
    }
    return HV_OK;
}

hv_status hv_ctx_autotune(hv_ctx *c, int trial_steps, hv_autotune_report *report) {
    if (!c || trial_steps < 1 || trial_steps > 1024) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (report) std::memset(report, 0, sizeof(*report));
    return fused_autotune(c, trial_steps, report);
}

hv_status hv_ctx_kernel_times(hv_ctx *c, double *total_ms, int *launches, int n) {
    if (!c || n < 0 || n > HV_K_COUNT) return HV_ERR_BAD_ARG;
    for (int k = 0; k < n; k++) {
        if (total_ms) total_ms[k] = c->prof.ms[k];
        if (launches) launches[k] = c->prof.launches[k];
    }
    return HV_OK;
}

hv_status hv_initial_solve(hv_ctx *c, int *sor_iterations) {
    STAGE_BEGIN(c);
    int its = 0;
    hv_status st = DISPATCH(c, fields_and_gather<double>(c, &its), fields_and_gather<float>(c, &its));
    if (sor_iterations) *sor_iterations = its;
    if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
    HV_CUDA(cudaStreamSynchronize(c->stream));
    c->fields_valid = true;
    return HV_OK;
}

hv_status hv_run(hv_ctx *c, int n_steps, int path, hv_observables *obs) {
    if (!c) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (n_steps < 0) return HV_ERR_BAD_ARG;
    if (path != HV_PATH_PLAIN && path != HV_PATH_FUSED) return HV_ERR_BAD_ARG;
    // a run starts from forces of the current positions: solve for them first
    // if nothing has (the fused path uses its own kernels for that solve)
    if (path == HV_PATH_FUSED) return fused_run(c, n_steps, obs);
    if (!c->fields_valid) HV_TRY(hv_initial_solve(c, nullptr));
    fused_invalidate(c);  // the plain step rewrites the fields
    for (int s = 0; s < n_steps; s++) {
        hv_observables *row = obs ? &obs[s] : nullptr;
        if (row) std::memset(row, 0, sizeof(*row));
        HV_TRY(DISPATCH(c, plain_step<double>(c, row), plain_step<float>(c, row)));
    }
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

}  // extern "C"

namespace hv {
namespace {

// Contexts kept between hv_simulate calls, keyed by what fixes their device
// buffers: device, world, particle counts and precision.  A context is taken
// out of the cache for the length of a call, so concurrent calls never share
// one; at most kSimCacheMax idle contexts are kept (the oldest is destroyed
// first).  The cache is never destroyed at exit: freeing device memory after
// the CUDA runtime has shut down is not safe, and the process's memory goes
// with it anyway.
struct SimKey {
    int device;
    hv_world world;
    int protons, neutrons;
    hv_precision prec;
};

bool same_key(const SimKey &a, const SimKey &b) {
    if (a.device != b.device || a.protons != b.protons || a.neutrons != b.neutrons || a.prec != b.prec) return false;
    for (int i = 0; i < 3; i++)
        if (a.world.n[i] != b.world.n[i] || a.world.d_max[i] != b.world.d_max[i]) return false;
    return true;
}

bool same_params(const hv_run_params &a, const hv_run_params &b) {
    return a.z == b.z && a.n == b.n && a.part_per_nucleon == b.part_per_nucleon && a.sigma_r == b.sigma_r &&
           a.dt == b.dt && a.t_exc == b.t_exc && a.eta_exc == b.eta_exc && a.skyrme.A == b.skyrme.A &&
           a.skyrme.B == b.skyrme.B && a.skyrme.C == b.skyrme.C && a.skyrme.gamma == b.skyrme.gamma &&
           a.sor.omega == b.sor.omega && a.sor.tol == b.sor.tol && a.sor.criterion == b.sor.criterion &&
           a.sor.max_iter == b.sor.max_iter && a.deposit_mode == b.deposit_mode;
}

constexpr size_t kSimCacheMax = 4;
std::mutex g_sim_mutex;
std::vector<std::pair<SimKey, hv_ctx *>> &sim_cache() {
    static auto *cache = new std::vector<std::pair<SimKey, hv_ctx *>>();
    return *cache;
}

hv_ctx *sim_take(const SimKey &k) {
    std::lock_guard<std::mutex> lock(g_sim_mutex);
    auto &cache = sim_cache();
    for (size_t i = 0; i < cache.size(); i++)
        if (same_key(cache[i].first, k)) {
            hv_ctx *c = cache[i].second;
            cache.erase(cache.begin() + (long)i);
            return c;
        }
    return nullptr;
}

void sim_put(const SimKey &k, hv_ctx *c) {
    hv_ctx *evict = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_sim_mutex);
        auto &cache = sim_cache();
        cache.emplace_back(k, c);
        if (cache.size() > kSimCacheMax) {
            evict = cache.front().second;
            cache.erase(cache.begin());
        }
    }
    if (evict) hv_ctx_destroy(evict);
}

// A cached context brought back to the state hv_ctx_create leaves: step 0,
// not excited, Coulomb boundary and fields unset, phi zero, identity slot
// order and the fused solver's first-cycle seed at its initial value, so that
// the call computes what it would on a new context.  Plans, graphs and
// buffers are kept (new parameters re-plan the fused path).
hv_status sim_reset(hv_ctx *c, const hv_run_params *params) {
    HV_CUDA(cudaSetDevice(c->device));
    if (!same_params(c->params, *params)) HV_TRY(hv_ctx_set_params(c, params));
    c->step_index = 0;
    c->excited = false;
    c->boundary_set = false;
    c->fields_valid = false;
    const size_t es = c->prec == HV_F64 ? 8 : 4;
    void *phi = c->prec == HV_F64 ? (void *)c->d64.phi : (void *)c->d32.phi;
    HV_CUDA(cudaMemsetAsync(phi, 0, es * (size_t)c->geom.G, c->stream));
    if (c->permuted && c->total > 0) {
        k_iota<<<div_up(c->total, 256), 256, 0, c->stream>>>(c->total, c->perm);
        HV_CUDA(cudaGetLastError());
    }
    c->permuted = false;
    fused_invalidate(c);
    c->fused.m_hint = Fused().m_hint;
    return HV_OK;
}

}  // namespace
}  // namespace hv

extern "C" {

hv_status hv_simulate(const hv_world *world, int protons, int neutrons, hv_precision prec,
                      const hv_run_params *params, int path, int n_steps, void *x, void *y, void *z, void *kx,
                      void *ky, void *kz, hv_observables *obs) {
    if (n_steps < 0 || !world || !params) return HV_ERR_BAD_ARG;
    if (protons + neutrons > 0 && (!x || !y || !z || !kx || !ky || !kz)) return HV_ERR_BAD_ARG;
    HV_TRY(check_world(world));
    HV_TRY(check_params(params));
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("no CUDA device");
        return HV_ERR_NO_DEVICE;
    }
    const SimKey key{device, *world, protons, neutrons, prec};
    hv_ctx *c = sim_take(key);
    hv_status st = HV_OK;
    if (c) st = sim_reset(c, params);
    else st = hv_ctx_create(world, protons, neutrons, prec, params, device, &c);
    if (st == HV_OK) st = hv_upload_particles(c, x, y, z, kx, ky, kz);
    // hv_run performs the initial field solve on the chosen path
    if (st == HV_OK) st = hv_run(c, n_steps, path, obs);
    if (st == HV_OK) st = hv_download_particles(c, x, y, z, kx, ky, kz);
    if (!c) return st;
    if (st == HV_OK) sim_put(key, c);  // kept for the next call of the same shape
    else hv_ctx_destroy(c);
    return st;
}

hv_status hv_simulate_release(void) {
    std::vector<std::pair<SimKey, hv_ctx *>> held;
    {
        std::lock_guard<std::mutex> lock(g_sim_mutex);
        held.swap(sim_cache());
    }
    for (auto &e : held) hv_ctx_destroy(e.second);
    return HV_OK;
}

}  // extern "C"
