// Adjoint of the plain FP64 step: the gradient of an objective of the dipole
// series D(t) with respect to the Skyrme parameters.
//
// The reference has no derivative code; this is the differentiated form of
// its step (cpu_simulate, src/hyper_vlasov.cpp:63-104):
//
//   [D_n = obs(x_n)]  k_h = k_n + a f_n  x_{n+1} = x_n + b k_h
//   f_{n+1} = force(x_{n+1}; theta)      k_{n+1} = k_h + a f_{n+1}
//
// with a = dt / (2 hbar c) (physics.hpp:251) and b = dt hbar c / mc^2
// (physics.hpp:263).  Reversed, step n is
//
//   lf += a lk;  lx += dforce(x_{n+1})^T lf,  g_theta += dforce/dtheta^T lf
//   lk += b lx;  lx += dD_n/dx_n lD_n;  lf = a lk
//
// and the transposed force map at x is, stage by stage:
//   gather (tools.hpp:98-168): its transpose in the force field is a deposit
//     of lf with the CIC weights; in the positions, the CIC weight gradients
//     against F . lf;
//   -grad (physics.hpp:159-200): the transposed central / one-sided stencil;
//   merge and Skyrme (physics_formulas.hpp:70-77): the pointwise Jacobian of
//     U_q = A t + B t^gamma + 2 tau_q C (rho_n - rho_p) / rho0, and its
//     derivatives in (A, B, gamma, C) summed over the grid;
//   Coulomb SOR (physics.hpp:99-157): lap phi = -c rho_p, so the transposed
//     solve is a second SOR solve, lap mu = l_phi with zero boundary, and
//     l_rho_p += -c mu;
//   smoothing (physics.hpp:202-234): symmetric, its own transpose;
//   deposit (tools.hpp:35-96): the CIC weight gradients against l_rho_raw.
//
// The forward keeps the particle state and phi every K steps; the backward
// recomputes each segment (storing x, F and the smoothed density per step)
// and runs the reversed steps through it.  All arithmetic is double.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kBlock = 256;

inline int nblocks(long long n) { return div_up(n > 0 ? n : 1, kBlock); }

__device__ __forceinline__ double cell(double pos, double dmax, int n) { return (n / 2.0) * (pos / dmax + 1.0); }

// lam_F(c) += w_c(x_p) lam_f(p): the transposed gather, a deposit of lam_f.
__global__ void k_adj_gather_field(Geom g, int protons, int total, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   const double *__restrict__ lfx, const double *__restrict__ lfy,
                                   const double *__restrict__ lfz, double *LFx, double *LFy, double *LFz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double cx = cell(x[i], g.dmx, nx), cy = cell(y[i], g.dmy, ny), cz = cell(z[i], g.dmz, nz);
    if (cx < 0.0 || cy < 0.0 || cz < 0.0 || cx >= nx || cy >= ny || cz >= nz) return;
    const int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    const double dx = cx - x0, dy = cy - y0, dz = cz - z0;
    const double wx[2] = {1.0 - dx, dx}, wy[2] = {1.0 - dy, dy}, wz[2] = {1.0 - dz, dz};
    const long long off = i < protons ? 0 : g.G, sx = (long long)ny * nz, sy = nz;
    const double fx = lfx[i], fy = lfy[i], fz = lfz[i];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                if (x0 + a >= nx || y0 + b >= ny || z0 + cc >= nz) continue;  // dropped corners
                const long long id = off + (x0 + a) * sx + (y0 + b) * sy + z0 + cc;
                const double w = wx[a] * wy[b] * wz[cc];
                atomicAdd(LFx + id, w * fx);
                atomicAdd(LFy + id, w * fy);
                atomicAdd(LFz + id, w * fz);
            }
}

// Position adjoint of the CIC weights of gather and deposit:
// lam_x(p) += sum_c grad w_c(x_p) [ F(c) . lam_f(p) + lam_raw(c) ].
// The force field is read at Fx[fs id] (fs 1: separate arrays; 4: the fused
// path's interleaved (Fx, Fy, Fz, 0) per node).
__global__ void k_adj_weights(Geom g, int protons, int total, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ z,
                              const double *__restrict__ lfx, const double *__restrict__ lfy,
                              const double *__restrict__ lfz, const double *__restrict__ Fx,
                              const double *__restrict__ Fy, const double *__restrict__ Fz, long long fs,
                              const double *__restrict__ lraw, double *lx, double *ly, double *lz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double cx = cell(x[i], g.dmx, nx), cy = cell(y[i], g.dmy, ny), cz = cell(z[i], g.dmz, nz);
    if (cx < 0.0 || cy < 0.0 || cz < 0.0 || cx >= nx || cy >= ny || cz >= nz) return;
    const int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    const double dx = cx - x0, dy = cy - y0, dz = cz - z0;
    const double hx = nx / (2.0 * g.dmx), hy = ny / (2.0 * g.dmy), hz = nz / (2.0 * g.dmz);  // dc/dpos
    const double wx[2] = {1.0 - dx, dx}, wy[2] = {1.0 - dy, dy}, wz[2] = {1.0 - dz, dz};
    const double gxw[2] = {-hx, hx}, gyw[2] = {-hy, hy}, gzw[2] = {-hz, hz};
    const long long off = i < protons ? 0 : g.G, sx = (long long)ny * nz, sy = nz;
    const double fx = lfx[i], fy = lfy[i], fz = lfz[i];
    double ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                if (x0 + a >= nx || y0 + b >= ny || z0 + cc >= nz) continue;
                const long long id = off + (x0 + a) * sx + (y0 + b) * sy + z0 + cc;
                const double v = Fx[fs * id] * fx + Fy[fs * id] * fy + Fz[fs * id] * fz + lraw[id];
                ax += gxw[a] * wy[b] * wz[cc] * v;
                ay += wx[a] * gyw[b] * wz[cc] * v;
                az += wx[a] * wy[b] * gzw[cc] * v;
            }
    lx[i] += ax;
    ly[i] += ay;
    lz[i] += az;
}

// One axis of the transposed k_fdm stencil at index m of n, values L along
// the axis with the given stride and spacing d.
__device__ __forceinline__ double fdm_t(const double *L, long long base, long long stride, int m, int n, double d) {
    double s = 0.0;
    if (m - 1 >= 1 && m - 1 <= n - 2) s += L[base + (m - 1) * stride] / (2.0 * d);
    if (m + 1 >= 1 && m + 1 <= n - 2) s -= L[base + (m + 1) * stride] / (2.0 * d);
    if (m == 1) s += L[base] / d;
    if (m == 0) s -= L[base] / d;
    if (m == n - 1) s += L[base + (n - 1) * stride] / d;
    if (m == n - 2) s -= L[base + (n - 1) * stride] / d;
    return s;
}

// lam_U = (-grad)^T lam_F over both species.
__global__ void k_adj_fdm(Geom g, double dx, double dy, double dz, const double *__restrict__ LFx,
                          const double *__restrict__ LFy, const double *__restrict__ LFz, double *LU) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * g.G) return;
    const long long off = i >= g.G ? g.G : 0, id = i - off;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const int k = (int)(id % nz), j = (int)((id / nz) % ny), ii = (int)(id / sx);
    const double s = fdm_t(LFx, off + (long long)j * sy + k, sx, ii, nx, dx) +
                     fdm_t(LFy, off + (long long)ii * sx + k, sy, j, ny, dy) +
                     fdm_t(LFz, off + (long long)ii * sx + (long long)j * sy, 1, k, nz, dz);
    LU[i] = -s;
}

// Transposed Skyrme map and its parameter derivatives: lam_rho from lam_U,
// and per-block sums of lam_U . dU/d(A, B, gamma, C).
__global__ void k_adj_skyrme(long long G, double A, double B, double C, double gamma, const double *__restrict__ rho,
                             const double *__restrict__ LU, double *Lrho, double *partials) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < G;
         i += (long long)gridDim.x * blockDim.x) {
        const double rp = rho[i], rn = rho[i + G], lp = LU[i], ln = LU[i + G];
        const double t = (rp + rn) / kRho0;
        const double tg = pow(t, gamma), tg1 = t > 0.0 ? pow(t, gamma - 1.0) : 0.0;
        const double S = (A + B * gamma * tg1) / kRho0, sum = lp + ln, dif = ln - lp;
        Lrho[i] = S * sum - (2.0 * C / kRho0) * dif;
        Lrho[i + G] = S * sum + (2.0 * C / kRho0) * dif;
        s[0] += sum * t;
        s[1] += sum * tg;
        s[2] += t > 0.0 ? sum * B * tg * log(t) : 0.0;
        s[3] += dif * 2.0 * (rn - rp) / kRho0;
    }
    __shared__ double sh[4][kBlock];
    for (int q = 0; q < 4; q++) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int q = 0; q < 4; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 4) partials[4 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// acc[0..3] += the block partials, summed in block order.
__global__ void k_adj_accumulate(const double *__restrict__ partials, int nb, double *acc) {
    if (threadIdx.x >= 4) return;
    double v = 0.0;
    for (int b = 0; b < nb; b++) v += partials[4 * b + threadIdx.x];
    acc[threadIdx.x] += v;
}

// Source of the transposed Poisson solve: the SOR kernel solves
// lap mu = -c src, so src = -lam_phi / c gives lap mu = lam_phi.
__global__ void k_adj_coulomb_src(long long G, double inv_c, const double *__restrict__ LU, double *src) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) src[i] = -LU[i] * inv_c;
}

__global__ void k_adj_coulomb_add(long long G, double c, const double *__restrict__ mu, double *Lrho) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) Lrho[i] += -c * mu[i];
}

// lam_z += dD/dz lam_D: D = N Z / A (sum z_p / Z_count - sum z_n / N_count).
__global__ void k_adj_observe(int protons, int total, double cp, double cn, double *lz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) lz[i] += i < protons ? cp : -cn;
}

__global__ void k_axpy3d(int total, double f, double *a0, double *a1, double *a2, const double *__restrict__ b0,
                         const double *__restrict__ b1, const double *__restrict__ b2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    a0[i] += f * b0[i];
    a1[i] += f * b1[i];
    a2[i] += f * b2[i];
}

__global__ void k_scale3d(int total, double f, double *a0, double *a1, double *a2, const double *__restrict__ b0,
                          const double *__restrict__ b1, const double *__restrict__ b2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    a0[i] = f * b0[i];
    a1[i] = f * b1[i];
    a2[i] = f * b2[i];
}

}  // namespace

// Device buffers and checkpoints of one adjoint run.
struct Adjoint {
    int steps = 0, every = 0, nseg = 0, cap_steps = 0, cap_every = 0;
    hv_step_path path = HV_PATH_PLAIN, cap_path = HV_PATH_PLAIN;  // the forward's path; the buffers' layout
    // checkpoints: [nseg + 1] x (9 N particle state + G phi) on the plain path;
    // the fused path adds phi's two earlier solutions (the extrapolated start),
    // the interleaved force field (8 G) and the smoothed density (2 G); the
    // last checkpoint is the final state
    double *ckpt = nullptr;
    int *ck_ctl = nullptr;   // fused path: [nseg + 1] x the fused control words
    std::vector<int> ck_step, ck_mhint;
    std::vector<char> ck_excited, ck_boundary;
    // per-step data of a recomputed segment: [every] x (3 N positions + the
    // force field (6 G separate, or 8 G interleaved on the fused path) + 2 G density)
    double *seg = nullptr;
    // adjoints of the particle state (9 N: x, k, f) and grid work arrays
    double *lam = nullptr;
    double *LF = nullptr;    // 3 x 2G
    double *LU = nullptr;    // 2G
    double *Lrho = nullptr;  // 2G
    double *Lraw = nullptr;  // 2G
    double *src = nullptr;   // G
    double *mu = nullptr;    // G, zero on the boundary
    double *mu_hist = nullptr;  // fused path: 2 G, mu's two earlier solutions
    int *actl = nullptr;     // fused path: the transposed solves' control words (8) and counts (2)
    double *partials = nullptr;
    double *acc = nullptr;   // 4: dJ/d(A, B, gamma, C)
    // the slot-to-caller permutation of the checkpointed particle state (the
    // steps of a forward run keep the slot order, so one copy serves all
    // checkpoints); restored with them, since a fused run between forward and
    // backward may re-sort the slots
    int *perm = nullptr;
    bool permuted = false;
    int nb_sky = 0;
    int adj_sor_its = 0;     // iterations of the transposed solves of the last backward pass
    int adj_sor_unconverged = 0;  // of those solves, the ones that stopped at max_iter
    bool ready = false;      // a forward run's checkpoints are held
};

void adjoint_release(hv_ctx *c) {
    Adjoint *a = c->adjoint;
    if (!a) return;
    double *bufs[] = {a->ckpt, a->seg, a->lam, a->LF, a->LU, a->Lrho, a->Lraw, a->src, a->mu, a->mu_hist,
                      a->partials, a->acc};
    for (double *p : bufs)
        if (p) cudaFree(p);
    int *ibufs[] = {a->perm, a->ck_ctl, a->actl};
    for (int *p : ibufs)
        if (p) cudaFree(p);
    delete a;
    c->adjoint = nullptr;
}

namespace {

bool fused_layout(hv_step_path p) { return p == HV_PATH_FUSED; }
size_t ck_stride(const hv_ctx *c, hv_step_path p) {
    return (size_t)9 * c->total + (size_t)(fused_layout(p) ? 13 : 1) * c->geom.G;
}
size_t seg_stride(const hv_ctx *c, hv_step_path p) {
    return (size_t)3 * c->total + (size_t)(fused_layout(p) ? 10 : 8) * c->geom.G;
}

hv_status adjoint_alloc(hv_ctx *c, int steps, int every, hv_step_path path) {
    const int nseg = (steps + every - 1) / every;
    Adjoint *a = c->adjoint;
    if (a && a->cap_path == path && a->cap_every >= every &&
        (a->cap_steps + a->cap_every - 1) / a->cap_every >= nseg)
        return HV_OK;
    adjoint_release(c);
    a = c->adjoint = new Adjoint();
    const size_t N = c->total, G = c->geom.G;
    auto alloc = [&](double **p, size_t n) -> hv_status {
        if (cudaMalloc((void **)p, sizeof(double) * (n > 0 ? n : 1)) != cudaSuccess) {
            cudaGetLastError();
            return HV_ERR_OOM;
        }
        return HV_OK;
    };
    auto alloci = [&](int **p, size_t n) -> hv_status {
        if (cudaMalloc((void **)p, sizeof(int) * (n > 0 ? n : 1)) != cudaSuccess) {
            cudaGetLastError();
            return HV_ERR_OOM;
        }
        return HV_OK;
    };
    HV_TRY(alloc(&a->ckpt, ck_stride(c, path) * (nseg + 1)));
    HV_TRY(alloc(&a->seg, seg_stride(c, path) * every));
    HV_TRY(alloc(&a->lam, 9 * N));
    HV_TRY(alloc(&a->LF, 6 * G));
    HV_TRY(alloc(&a->LU, 2 * G));
    HV_TRY(alloc(&a->Lrho, 2 * G));
    HV_TRY(alloc(&a->Lraw, 2 * G));
    HV_TRY(alloc(&a->src, G));
    HV_TRY(alloc(&a->mu, G));
    a->nb_sky = 2 * c->sm_count;
    HV_TRY(alloc(&a->partials, 4 * (size_t)a->nb_sky));
    HV_TRY(alloc(&a->acc, 4));
    HV_TRY(alloci(&a->perm, N));
    if (fused_layout(path)) {
        HV_TRY(alloc(&a->mu_hist, 2 * G));
        HV_TRY(alloci(&a->ck_ctl, (size_t)fused_ctl_words() * (nseg + 1)));
        HV_TRY(alloci(&a->actl, 10));
    }
    a->cap_steps = steps;
    a->cap_every = every;
    a->cap_path = path;
    return HV_OK;
}

// Particle state (x..kz, fx..fz) and phi to / from checkpoint slot s; on the
// fused path also phi's history, the interleaved forces, the smoothed density
// and the control words, so that a recomputed segment repeats the forward's
// steps.
hv_status save_ckpt(hv_ctx *c, int s) {
    Adjoint *a = c->adjoint;
    State<double> &st = c->d64;
    const size_t N = c->total, G = c->geom.G;
    const bool fz = fused_layout(a->path);
    double *dst = a->ckpt + ck_stride(c, a->path) * s;
    double *src[9] = {st.x, st.y, st.z, st.kx, st.ky, st.kz, st.fx, st.fy, st.fz};
    for (int k = 0; k < 9; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(dst + k * N, src[k], sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    double *g = dst + 9 * N;
    if (!fz) {
        HV_CUDA(cudaMemcpyAsync(g, st.phi, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        const Fused &f = c->fused;
        HV_CUDA(cudaMemcpyAsync(g, f.phi64, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(g + G, f.phi64_prev, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(g + 2 * G, f.phi64_prev2, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(g + 3 * G, f.F4, sizeof(double) * 8 * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(g + 11 * G, st.rho, sizeof(double) * 2 * G, cudaMemcpyDeviceToDevice, c->stream));
        const int nw = fused_ctl_words();
        HV_CUDA(cudaMemcpyAsync(a->ck_ctl + (size_t)nw * s, fused_ctl(c), sizeof(int) * nw, cudaMemcpyDeviceToDevice,
                                c->stream));
    }
    if ((int)a->ck_step.size() <= s) {
        a->ck_step.resize(s + 1);
        a->ck_mhint.resize(s + 1);
        a->ck_excited.resize(s + 1);
        a->ck_boundary.resize(s + 1);
    }
    a->ck_step[s] = c->step_index;
    a->ck_mhint[s] = c->fused.m_hint;
    a->ck_excited[s] = c->excited;
    a->ck_boundary[s] = c->boundary_set;
    return HV_OK;
}

hv_status load_ckpt(hv_ctx *c, int s) {
    Adjoint *a = c->adjoint;
    State<double> &st = c->d64;
    const size_t N = c->total, G = c->geom.G;
    const bool fz = fused_layout(a->path);
    const double *src = a->ckpt + ck_stride(c, a->path) * s;
    double *dst[9] = {st.x, st.y, st.z, st.kx, st.ky, st.kz, st.fx, st.fy, st.fz};
    for (int k = 0; k < 9; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(dst[k], src + k * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    const double *g = src + 9 * N;
    if (!fz) {
        HV_CUDA(cudaMemcpyAsync(st.phi, g, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        Fused &f = c->fused;
        HV_CUDA(cudaMemcpyAsync(f.phi64, g, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(f.phi64_prev, g + G, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(f.phi64_prev2, g + 2 * G, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(f.F4, g + 3 * G, sizeof(double) * 8 * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(st.rho, g + 11 * G, sizeof(double) * 2 * G, cudaMemcpyDeviceToDevice, c->stream));
        // the plain view of phi, as a fused run's end leaves it
        HV_CUDA(cudaMemcpyAsync(st.phi, g, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
        const int nw = fused_ctl_words();
        HV_CUDA(cudaMemcpyAsync(fused_ctl(c), a->ck_ctl + (size_t)nw * s, sizeof(int) * nw, cudaMemcpyDeviceToDevice,
                                c->stream));
        f.f4_current = true;
        f.m_hint = a->ck_mhint[s];
    }
    if (N) HV_CUDA(cudaMemcpyAsync(c->perm, a->perm, sizeof(int) * N, cudaMemcpyDeviceToDevice, c->stream));
    c->permuted = a->permuted;
    c->step_index = a->ck_step[s];
    c->excited = a->ck_excited[s];
    c->boundary_set = a->ck_boundary[s];
    return HV_OK;
}

// Positions, forces and smoothed density after a step, into segment slot j.
hv_status save_slot(hv_ctx *c, int j) {
    State<double> &st = c->d64;
    const hv_step_path path = c->adjoint->path;
    const size_t N = c->total, G = c->geom.G;
    double *d = c->adjoint->seg + seg_stride(c, path) * j;
    const double *src3[3] = {st.x, st.y, st.z};
    for (int k = 0; k < 3; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(d + k * N, src3[k], sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    if (fused_layout(path)) {
        HV_CUDA(cudaMemcpyAsync(d + 3 * N, c->fused.F4, sizeof(double) * 8 * G, cudaMemcpyDeviceToDevice, c->stream));
        HV_CUDA(cudaMemcpyAsync(d + 3 * N + 8 * G, st.rho, sizeof(double) * 2 * G, cudaMemcpyDeviceToDevice,
                                c->stream));
        return HV_OK;
    }
    const double *srcF[4] = {st.Fx, st.Fy, st.Fz, st.rho};
    for (int k = 0; k < 4; k++)
        HV_CUDA(cudaMemcpyAsync(d + 3 * N + k * 2 * G, srcF[k], sizeof(double) * 2 * G, cudaMemcpyDeviceToDevice,
                                c->stream));
    return HV_OK;
}

// lam_x += dforce(x)^T lam_f at the point stored in slot j; the parameter
// derivatives are added to acc.
// After a transposed solve on the persistent kernel: its iterations and
// whether it stopped unconverged, added to cnt[0] and cnt[1] (status words:
// [1] iterations, [2] converged).
__global__ void k_adj_sor_count(const int *__restrict__ status, int *cnt) {
    if (threadIdx.x == 0) {
        cnt[0] += status[1];
        cnt[1] += status[2] ? 0 : 1;
    }
}

hv_status force_adjoint(hv_ctx *c, int j) {
    Adjoint *a = c->adjoint;
    const Geom &g = c->geom;
    const size_t N = c->total, G = g.G;
    const bool fz = fused_layout(a->path);
    const double *d = a->seg + seg_stride(c, a->path) * j;
    const double *x = d, *y = d + N, *z = d + 2 * N;
    // the force field: separate arrays, or (Fx, Fy, Fz, 0) per node
    const double *F = d + 3 * N;
    const double *Fx = F, *Fy = fz ? F + 1 : F + 2 * G, *Fz = fz ? F + 2 : F + 4 * G;
    const long long fs = fz ? 4 : 1;
    const double *rho = fz ? F + 8 * G : F + 6 * G;
    double *lx = a->lam, *ly = lx + N, *lz = ly + N;
    const double *lf = a->lam + 6 * N;
    double *LFx = a->LF, *LFy = LFx + 2 * G, *LFz = LFy + 2 * G;
    // gather^T in the field
    HV_CUDA(cudaMemsetAsync(a->LF, 0, sizeof(double) * 6 * G, c->stream));
    if (N)
        k_adj_gather_field<<<nblocks(N), kBlock, 0, c->stream>>>(g, c->protons, c->total, x, y, z, lf, lf + N,
                                                                lf + 2 * N, LFx, LFy, LFz);
    // (-grad)^T
    const double dx = 2.0 * g.dmx / g.nx, dy = 2.0 * g.dmy / g.ny, dz = 2.0 * g.dmz / g.nz;
    k_adj_fdm<<<nblocks(2 * G), kBlock, 0, c->stream>>>(g, dx, dy, dz, LFx, LFy, LFz, a->LU);
    // Skyrme^T and its parameter derivatives
    const hv_skyrme &sk = c->params.skyrme;
    k_adj_skyrme<<<a->nb_sky, kBlock, 0, c->stream>>>((long long)G, sk.A, sk.B, sk.C, sk.gamma, rho, a->LU, a->Lrho,
                                                     a->partials);
    k_adj_accumulate<<<1, 32, 0, c->stream>>>(a->partials, a->nb_sky, a->acc);
    // Coulomb: the proton potential's phi term, through the transposed solve
    const double cc = 4.0 * kPi * kE2;
    k_adj_coulomb_src<<<nblocks(G), kBlock, 0, c->stream>>>((long long)G, 1.0 / cc, a->LU, a->src);
    HV_CUDA(cudaGetLastError());
    if (fz) {
        // on the persistent kernel, started from the extrapolation of the
        // previous reversed steps' mu; counted on the device
        HV_TRY(sor_fast_launch_adjoint(c, a->src, a->mu, a->mu_hist, a->mu_hist + G, a->actl));
        k_adj_sor_count<<<1, 32, 0, c->stream>>>(sor_fast_status_words(c), a->actl + 8);
    } else {
        int its = 0;
        double metric = 0.0;
        hv_status st = launch_sor_plain<double>(c, a->mu, a->src, &its, &metric);
        if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
        a->adj_sor_its += its;
        if (st == HV_ERR_NOT_CONVERGED) a->adj_sor_unconverged++;
    }
    k_adj_coulomb_add<<<nblocks(G), kBlock, 0, c->stream>>>((long long)G, cc, a->mu, a->Lrho);
    // smoothing^T = smoothing
    HV_TRY(launch_smooth<double>(c, a->Lrho, a->Lraw));
    // deposit^T and gather^T in the positions
    if (N)
        k_adj_weights<<<nblocks(N), kBlock, 0, c->stream>>>(g, c->protons, c->total, x, y, z, lf, lf + N, lf + 2 * N,
                                                           Fx, Fy, Fz, fs, a->Lraw, lx, ly, lz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

// Slot re-sorting paused while an adjoint pass runs fused steps: the adjoint
// state is indexed by particle slot, so every step of a forward run and of its
// backward pass must see one slot order.
struct SortPause {
    hv_ctx *c;
    int saved;
    explicit SortPause(hv_ctx *c_) : c(c_), saved(c_->fast.sort_every) { c->fast.sort_every = 0; }
    ~SortPause() { c->fast.sort_every = saved; }
};

// The persistent solver's error word after a stretch of fused steps and
// transposed solves (synchronous): a bounded wait that ran out leaves the
// fused copies and the fields stale.
hv_status fused_pass_status(hv_ctx *c) {
    int st0 = 0;
    HV_CUDA(cudaMemcpyAsync(&st0, sor_fast_status_words(c), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    if (!st0) return HV_OK;
    c->fields_valid = false;
    fused_invalidate(c);
    set_last_error("SOR: a bounded device-side wait timed out");
    return HV_ERR_TIMEOUT;
}

// The forward run on the fused FP64 path: one hv_run(HV_PATH_FUSED) per
// segment, with a checkpoint before each and the final state after the last.
hv_status forward_fused(hv_ctx *c, int n_steps, hv_observables *obs) {
    Adjoint *a = c->adjoint;
    // forces and phi into the fused buffers, the solution history cleared
    HV_TRY(fused_adjoint_begin(c, 0));
    for (int sgi = 0; sgi < a->nseg; sgi++) {
        const int s0 = sgi * a->every, k = std::min(a->every, n_steps - s0);
        HV_TRY(save_ckpt(c, sgi));
        HV_TRY(fused_run(c, k, obs ? obs + s0 : nullptr));
    }
    return save_ckpt(c, a->nseg);
}

// Recomputes steps s0..s1-1 from the checkpoint the context holds, keeping
// what the reversed steps need.
hv_status recompute_segment(hv_ctx *c, int s0, int s1) {
    if (fused_layout(c->adjoint->path)) {
        HV_TRY(fused_adjoint_begin(c, s1 - s0));
        for (int n = s0; n < s1; n++) {
            HV_TRY(fused_adjoint_step(c));
            HV_TRY(save_slot(c, n - s0));
        }
        return HV_OK;
    }
    for (int n = s0; n < s1; n++) {
        HV_TRY(plain_step_f64(c, nullptr));
        HV_TRY(save_slot(c, n - s0));
    }
    return HV_OK;
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" {

hv_status hv_adjoint_forward_path(hv_ctx *c, int path, int n_steps, int checkpoint_every, hv_observables *obs) {
    if (!c || n_steps < 1 || checkpoint_every < 1) return HV_ERR_BAD_ARG;
    if (path != HV_PATH_PLAIN && path != HV_PATH_FUSED) return HV_ERR_BAD_ARG;
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    HV_CUDA(cudaSetDevice(c->device));
    const hv_step_path p = (hv_step_path)path;
    if (p == HV_PATH_FUSED) {
        // the fused path solves missing fields with its own kernels
        if (!c->fields_valid) HV_TRY(fused_run(c, 0, nullptr));
        hv_status st = fused_prepare(c);
        if (st != HV_OK) {
            fused_release(c);
            return st;
        }
    } else if (!c->fields_valid) {
        HV_TRY(hv_initial_solve(c, nullptr));
    }
    fused_invalidate(c);
    const int every = checkpoint_every < n_steps ? checkpoint_every : n_steps;
    if (c->adjoint) c->adjoint->ready = false;
    HV_TRY(adjoint_alloc(c, n_steps, every, p));
    Adjoint *a = c->adjoint;
    a->ready = false;
    a->path = p;
    a->steps = n_steps;
    a->every = every;
    a->nseg = (n_steps + every - 1) / every;
    if (c->total) HV_CUDA(cudaMemcpyAsync(a->perm, c->perm, sizeof(int) * c->total, cudaMemcpyDeviceToDevice, c->stream));
    a->permuted = c->permuted;
    if (p == HV_PATH_FUSED) {
        SortPause pause(c);
        HV_TRY(forward_fused(c, n_steps, obs));
    } else {
        for (int n = 0; n < n_steps; n++) {
            if (n % every == 0) HV_TRY(save_ckpt(c, n / every));
            hv_observables *row = obs ? &obs[n] : nullptr;
            if (row) std::memset(row, 0, sizeof(*row));
            HV_TRY(plain_step_f64(c, row));
        }
        HV_TRY(save_ckpt(c, a->nseg));  // the final state, restored after a backward pass
    }
    HV_CUDA(cudaStreamSynchronize(c->stream));
    a->ready = true;
    return HV_OK;
}

hv_status hv_adjoint_forward(hv_ctx *c, int n_steps, int checkpoint_every, hv_observables *obs) {
    return hv_adjoint_forward_path(c, HV_PATH_PLAIN, n_steps, checkpoint_every, obs);
}

hv_status hv_adjoint_backward(hv_ctx *c, const double *dJ_dD, const double theta[4], double grad_theta[4],
                              double grad_skyrme[4]) {
    if (!c || !dJ_dD || !theta || !grad_theta) return HV_ERR_BAD_ARG;
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    Adjoint *a = c->adjoint;
    if (!a || !a->ready) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    const bool fz = fused_layout(a->path);
    SortPause pause(c);
    fused_invalidate(c);
    const size_t N = c->total, G = c->geom.G;
    const double dt = c->params.dt;
    const double ka = dt / (2.0 * kHbarC), kb = dt * kHbarC / kMc2;
    const double zz = c->params.z, nn = c->params.n, dfac = nn * zz / (nn + zz);
    double *lx = a->lam, *ly = lx + N, *lz = ly + N, *lkx = lz + N, *lky = lkx + N, *lkz = lky + N;
    double *lfx = lkz + N, *lfy = lfx + N, *lfz = lfy + N;
    HV_CUDA(cudaMemsetAsync(a->lam, 0, sizeof(double) * 9 * (N ? N : 1), c->stream));
    HV_CUDA(cudaMemsetAsync(a->mu, 0, sizeof(double) * G, c->stream));
    HV_CUDA(cudaMemsetAsync(a->acc, 0, sizeof(double) * 4, c->stream));
    if (fz) {
        // the transposed solves' control words: no earlier solution held, a
        // first cycle of 8 iterations; their iteration and unconverged counts
        const int h_ctl[10] = {0, 8, 0, 0, 0, 0, 0, 0, 0, 0};
        HV_CUDA(cudaMemsetAsync(a->mu_hist, 0, sizeof(double) * 2 * G, c->stream));
        HV_CUDA(cudaMemcpyAsync(a->actl, h_ctl, sizeof(h_ctl), cudaMemcpyHostToDevice, c->stream));
        HV_CUDA(cudaStreamSynchronize(c->stream));
    }
    a->adj_sor_its = 0;
    a->adj_sor_unconverged = 0;
    const int nbp = nblocks(N);
    for (int sgi = a->nseg - 1; sgi >= 0; sgi--) {
        const int s0 = sgi * a->every, s1 = std::min(s0 + a->every, a->steps);
        // recompute the segment, keeping what the reversed steps need
        HV_TRY(load_ckpt(c, sgi));
        HV_TRY(recompute_segment(c, s0, s1));
        for (int n = s1 - 1; n >= s0; n--) {
            if (!N) continue;
            k_axpy3d<<<nbp, kBlock, 0, c->stream>>>(c->total, ka, lfx, lfy, lfz, lkx, lky, lkz);
            HV_TRY(force_adjoint(c, n - s0));
            k_axpy3d<<<nbp, kBlock, 0, c->stream>>>(c->total, kb, lkx, lky, lkz, lx, ly, lz);
            const double ld = dJ_dD[n] * dfac;
            k_adj_observe<<<nbp, kBlock, 0, c->stream>>>(c->protons, c->total, c->protons ? ld / c->protons : 0.0,
                                                        c->neutrons ? ld / c->neutrons : 0.0, lz);
            k_scale3d<<<nbp, kBlock, 0, c->stream>>>(c->total, ka, lfx, lfy, lfz, lkx, lky, lkz);
            HV_CUDA(cudaGetLastError());
        }
        if (fz) HV_TRY(fused_pass_status(c));
    }
    // the forces of the starting state were solved from theta too
    HV_TRY(load_ckpt(c, 0));
    if (fz) {
        // checkpoint 0 holds the forces and smoothed density of x_0
        HV_TRY(save_slot(c, 0));
    } else {
        int its = 0;
        hv_status st = plain_fields_f64(c, &its);
        if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
        HV_TRY(save_slot(c, 0));
    }
    if (N) HV_TRY(force_adjoint(c, 0));
    double acc[4];
    int cnt[2] = {0, 0};
    HV_CUDA(cudaMemcpyAsync(acc, a->acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
    if (fz) HV_CUDA(cudaMemcpyAsync(cnt, a->actl + 8, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    if (fz) HV_TRY(fused_pass_status(c));
    // back to the state the forward run ended in
    HV_TRY(load_ckpt(c, a->nseg));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    if (fz) {
        a->adj_sor_its = cnt[0];
        a->adj_sor_unconverged = cnt[1];
    }
    c->fields_valid = false;
    fused_invalidate(c);
    // (A, B, gamma, C) -> (t0, t3, sigma, a_sym), the map of hv_skyrme_from_t0t3
    const double t3 = theta[1], sg = theta[2];
    const double r0s = std::pow(kRho0, sg + 1.0);
    grad_theta[0] = acc[0] * 0.75 * kRho0;
    grad_theta[1] = acc[1] * (sg + 2.0) / 16.0 * r0s;
    grad_theta[2] = acc[1] * t3 * r0s * (1.0 / 16.0 + (sg + 2.0) / 16.0 * std::log(kRho0)) + acc[2];
    grad_theta[3] = acc[3];
    if (grad_skyrme) {
        grad_skyrme[0] = acc[0];
        grad_skyrme[1] = acc[1];
        grad_skyrme[2] = acc[3];
        grad_skyrme[3] = acc[2];
    }
    return HV_OK;
}

hv_status hv_adjoint_stats(const hv_ctx *c, int *path, int *adjoint_sor_iterations, int *adjoint_sor_unconverged) {
    if (!c || !c->adjoint) return HV_ERR_BAD_ARG;
    const Adjoint *a = c->adjoint;
    if (path) *path = a->path;
    if (adjoint_sor_iterations) *adjoint_sor_iterations = a->adj_sor_its;
    if (adjoint_sor_unconverged) *adjoint_sor_unconverged = a->adj_sor_unconverged;
    return HV_OK;
}

}  // extern "C"
