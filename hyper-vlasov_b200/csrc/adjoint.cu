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
__global__ void k_adj_weights(Geom g, int protons, int total, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ z,
                              const double *__restrict__ lfx, const double *__restrict__ lfy,
                              const double *__restrict__ lfz, const double *__restrict__ Fx,
                              const double *__restrict__ Fy, const double *__restrict__ Fz,
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
                const double v = Fx[id] * fx + Fy[id] * fy + Fz[id] * fz + lraw[id];
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
    // checkpoints: [nseg + 1] x (9 N particle state + G phi); the last is the final state
    double *ckpt = nullptr;
    std::vector<int> ck_step;
    std::vector<char> ck_excited, ck_boundary;
    // per-step data of a recomputed segment: [every] x (3 N positions + 6 G forces + 2 G density)
    double *seg = nullptr;
    // adjoints of the particle state (9 N: x, k, f) and grid work arrays
    double *lam = nullptr;
    double *LF = nullptr;    // 3 x 2G
    double *LU = nullptr;    // 2G
    double *Lrho = nullptr;  // 2G
    double *Lraw = nullptr;  // 2G
    double *src = nullptr;   // G
    double *mu = nullptr;    // G, zero on the boundary
    double *partials = nullptr;
    double *acc = nullptr;   // 4: dJ/d(A, B, gamma, C)
    // the slot-to-caller permutation of the checkpointed particle state (the
    // plain steps of a forward run keep the slot order, so one copy serves all
    // checkpoints); restored with them, since a fused run between forward and
    // backward may re-sort the slots
    int *perm = nullptr;
    bool permuted = false;
    int nb_sky = 0;
    int adj_sor_its = 0;     // iterations of the transposed solves of the last backward pass
    bool ready = false;      // a forward run's checkpoints are held
};

void adjoint_release(hv_ctx *c) {
    Adjoint *a = c->adjoint;
    if (!a) return;
    double *bufs[] = {a->ckpt, a->seg, a->lam, a->LF, a->LU, a->Lrho, a->Lraw, a->src, a->mu, a->partials, a->acc};
    for (double *p : bufs)
        if (p) cudaFree(p);
    if (a->perm) cudaFree(a->perm);
    delete a;
    c->adjoint = nullptr;
}

namespace {

size_t ck_stride(const hv_ctx *c) { return (size_t)9 * c->total + (size_t)c->geom.G; }
size_t seg_stride(const hv_ctx *c) { return (size_t)3 * c->total + (size_t)8 * c->geom.G; }

hv_status adjoint_alloc(hv_ctx *c, int steps, int every) {
    const int nseg = (steps + every - 1) / every;
    Adjoint *a = c->adjoint;
    if (a && a->cap_every >= every && (a->cap_steps + a->cap_every - 1) / a->cap_every >= nseg) return HV_OK;
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
    HV_TRY(alloc(&a->ckpt, ck_stride(c) * (nseg + 1)));
    HV_TRY(alloc(&a->seg, seg_stride(c) * every));
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
    if (cudaMalloc((void **)&a->perm, sizeof(int) * (N > 0 ? N : 1)) != cudaSuccess) {
        cudaGetLastError();
        return HV_ERR_OOM;
    }
    a->cap_steps = steps;
    a->cap_every = every;
    return HV_OK;
}

// Particle state (x..kz, fx..fz) and phi to / from checkpoint slot s.
hv_status save_ckpt(hv_ctx *c, int s) {
    Adjoint *a = c->adjoint;
    State<double> &st = c->d64;
    const size_t N = c->total, G = c->geom.G;
    double *dst = a->ckpt + ck_stride(c) * s;
    double *src[9] = {st.x, st.y, st.z, st.kx, st.ky, st.kz, st.fx, st.fy, st.fz};
    for (int k = 0; k < 9; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(dst + k * N, src[k], sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    HV_CUDA(cudaMemcpyAsync(dst + 9 * N, st.phi, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
    if ((int)a->ck_step.size() <= s) {
        a->ck_step.resize(s + 1);
        a->ck_excited.resize(s + 1);
        a->ck_boundary.resize(s + 1);
    }
    a->ck_step[s] = c->step_index;
    a->ck_excited[s] = c->excited;
    a->ck_boundary[s] = c->boundary_set;
    return HV_OK;
}

hv_status load_ckpt(hv_ctx *c, int s) {
    Adjoint *a = c->adjoint;
    State<double> &st = c->d64;
    const size_t N = c->total, G = c->geom.G;
    const double *src = a->ckpt + ck_stride(c) * s;
    double *dst[9] = {st.x, st.y, st.z, st.kx, st.ky, st.kz, st.fx, st.fy, st.fz};
    for (int k = 0; k < 9; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(dst[k], src + k * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    HV_CUDA(cudaMemcpyAsync(st.phi, src + 9 * N, sizeof(double) * G, cudaMemcpyDeviceToDevice, c->stream));
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
    const size_t N = c->total, G = c->geom.G;
    double *d = c->adjoint->seg + seg_stride(c) * j;
    const double *src3[3] = {st.x, st.y, st.z};
    for (int k = 0; k < 3; k++)
        if (N) HV_CUDA(cudaMemcpyAsync(d + k * N, src3[k], sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    const double *srcF[4] = {st.Fx, st.Fy, st.Fz, st.rho};
    for (int k = 0; k < 4; k++)
        HV_CUDA(cudaMemcpyAsync(d + 3 * N + k * 2 * G, srcF[k], sizeof(double) * 2 * G, cudaMemcpyDeviceToDevice,
                                c->stream));
    return HV_OK;
}

// lam_x += dforce(x)^T lam_f at the point stored in slot j; the parameter
// derivatives are added to acc.
hv_status force_adjoint(hv_ctx *c, int j) {
    Adjoint *a = c->adjoint;
    const Geom &g = c->geom;
    const size_t N = c->total, G = g.G;
    const double *d = a->seg + seg_stride(c) * j;
    const double *x = d, *y = d + N, *z = d + 2 * N;
    const double *Fx = d + 3 * N, *Fy = Fx + 2 * G, *Fz = Fy + 2 * G, *rho = Fz + 2 * G;
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
    int its = 0;
    double metric = 0.0;
    hv_status st = launch_sor_plain<double>(c, a->mu, a->src, &its, &metric);
    if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
    a->adj_sor_its += its;
    k_adj_coulomb_add<<<nblocks(G), kBlock, 0, c->stream>>>((long long)G, cc, a->mu, a->Lrho);
    // smoothing^T = smoothing
    HV_TRY(launch_smooth<double>(c, a->Lrho, a->Lraw));
    // deposit^T and gather^T in the positions
    if (N)
        k_adj_weights<<<nblocks(N), kBlock, 0, c->stream>>>(g, c->protons, c->total, x, y, z, lf, lf + N, lf + 2 * N,
                                                           Fx, Fy, Fz, a->Lraw, lx, ly, lz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" {

hv_status hv_adjoint_forward(hv_ctx *c, int n_steps, int checkpoint_every, hv_observables *obs) {
    if (!c || n_steps < 1 || checkpoint_every < 1) return HV_ERR_BAD_ARG;
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    HV_CUDA(cudaSetDevice(c->device));
    if (!c->fields_valid) HV_TRY(hv_initial_solve(c, nullptr));
    fused_invalidate(c);
    const int every = checkpoint_every < n_steps ? checkpoint_every : n_steps;
    HV_TRY(adjoint_alloc(c, n_steps, every));
    Adjoint *a = c->adjoint;
    a->ready = false;
    a->steps = n_steps;
    a->every = every;
    a->nseg = (n_steps + every - 1) / every;
    if (c->total) HV_CUDA(cudaMemcpyAsync(a->perm, c->perm, sizeof(int) * c->total, cudaMemcpyDeviceToDevice, c->stream));
    a->permuted = c->permuted;
    for (int n = 0; n < n_steps; n++) {
        if (n % every == 0) HV_TRY(save_ckpt(c, n / every));
        hv_observables *row = obs ? &obs[n] : nullptr;
        if (row) std::memset(row, 0, sizeof(*row));
        HV_TRY(plain_step_f64(c, row));
    }
    HV_TRY(save_ckpt(c, a->nseg));  // the final state, restored after a backward pass
    HV_CUDA(cudaStreamSynchronize(c->stream));
    a->ready = true;
    return HV_OK;
}

hv_status hv_adjoint_backward(hv_ctx *c, const double *dJ_dD, const double theta[4], double grad_theta[4],
                              double grad_skyrme[4]) {
    if (!c || !dJ_dD || !theta || !grad_theta) return HV_ERR_BAD_ARG;
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    Adjoint *a = c->adjoint;
    if (!a || !a->ready) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
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
    a->adj_sor_its = 0;
    const int nbp = nblocks(N);
    for (int sgi = a->nseg - 1; sgi >= 0; sgi--) {
        const int s0 = sgi * a->every, s1 = std::min(s0 + a->every, a->steps);
        // recompute the segment, keeping what the reversed steps need
        HV_TRY(load_ckpt(c, sgi));
        for (int n = s0; n < s1; n++) {
            HV_TRY(plain_step_f64(c, nullptr));
            HV_TRY(save_slot(c, n - s0));
        }
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
    }
    // the forces of the starting state were solved from theta too
    HV_TRY(load_ckpt(c, 0));
    int its = 0;
    hv_status st = plain_fields_f64(c, &its);
    if (st != HV_OK && st != HV_ERR_NOT_CONVERGED) return st;
    HV_TRY(save_slot(c, 0));
    if (N) HV_TRY(force_adjoint(c, 0));
    double acc[4];
    HV_CUDA(cudaMemcpyAsync(acc, a->acc, sizeof(acc), cudaMemcpyDeviceToHost, c->stream));
    // back to the state the forward run ended in
    HV_TRY(load_ckpt(c, a->nseg));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    c->fields_valid = false;
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

}  // extern "C"
