// Plain-path kernels: one kernel per reference routine, in the reference's
// operation order.  This translation unit is compiled with --fmad=false so
// that a*b+c stays two rounded operations, as in the reference built with
// -ffp-contract=off; with identical inputs the HV_F64 results of deposit
// (sorted mode), FDM, merge, SOR, gather and push are bit-identical to it.
#include <cub/device/device_radix_sort.cuh>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kBlock = 256;

// Integer cell coordinate and fractional offset of one axis,
// distribute_volumetric_particles_cic (include/tools.hpp:50-60).
template <typename T>
struct Axis {
    T c;  // (n/2) (x/d_max + 1)
};

template <typename T>
__device__ __forceinline__ T cell_coord(T pos, T dmax, int n) {
    return (n / T(2.0)) * (pos / dmax + T(1.0));
}

template <typename T>
__device__ __forceinline__ bool in_grid(T cx, T cy, T cz, int nx, int ny, int nz) {
    return !(cx < T(0.0) || cy < T(0.0) || cz < T(0.0) || cx >= nx || cy >= ny || cz >= nz);
}

// ---- CIC deposit, atomic (include/tools.hpp:35-96) -----------------------
template <typename T>
__global__ void k_deposit_atomic(Geom g, int protons, int total, const T *__restrict__ x,
                                 const T *__restrict__ y, const T *__restrict__ z, T *rho) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    T cx = cell_coord<T>(x[i], T(g.dmx), nx);
    T cy = cell_coord<T>(y[i], T(g.dmy), ny);
    T cz = cell_coord<T>(z[i], T(g.dmz), nz);
    if (!in_grid<T>(cx, cy, cz, nx, ny, nz)) return;
    int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    T d_x = cx - x0, d_y = cy - y0, d_z = cz - z0;
    T t_x = T(1.0) - d_x, t_y = T(1.0) - d_y, t_z = T(1.0) - d_z;
    long long off = (i < protons) ? 0 : g.G;
    long long sy = nz, sx = (long long)ny * nz;
    T *b = rho + off;
    atomicAdd(b + x0 * sx + y0 * sy + z0, t_x * t_y * t_z);
    if (x1 < nx) atomicAdd(b + x1 * sx + y0 * sy + z0, d_x * t_y * t_z);
    if (y1 < ny) atomicAdd(b + x0 * sx + y1 * sy + z0, t_x * d_y * t_z);
    if (x1 < nx && y1 < ny) atomicAdd(b + x1 * sx + y1 * sy + z0, d_x * d_y * t_z);
    if (z1 < nz) atomicAdd(b + x0 * sx + y0 * sy + z1, t_x * t_y * d_z);
    if (x1 < nx && z1 < nz) atomicAdd(b + x1 * sx + y0 * sy + z1, d_x * t_y * d_z);
    if (y1 < ny && z1 < nz) atomicAdd(b + x0 * sx + y1 * sy + z1, t_x * d_y * d_z);
    if (x1 < nx && y1 < ny && z1 < nz) atomicAdd(b + x1 * sx + y1 * sy + z1, d_x * d_y * d_z);
}

// ---- CIC deposit, sorted / deterministic ---------------------------------
// Key of a particle = species * G + linear cell (x0, y0, z0); particles outside
// the grid get key 2G and sort last.
template <typename T>
__global__ void k_cell_keys(Geom g, int protons, int total, const T *__restrict__ x,
                            const T *__restrict__ y, const T *__restrict__ z, unsigned int *keys,
                            int *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    T cx = cell_coord<T>(x[i], T(g.dmx), g.nx);
    T cy = cell_coord<T>(y[i], T(g.dmy), g.ny);
    T cz = cell_coord<T>(z[i], T(g.dmz), g.nz);
    unsigned int key;
    if (!in_grid<T>(cx, cy, cz, g.nx, g.ny, g.nz)) {
        key = (unsigned int)(2 * g.G);
    } else {
        long long cell = ((long long)(int)cx * g.ny + (int)cy) * g.nz + (int)cz;
        key = (unsigned int)(cell + ((i < protons) ? 0 : g.G));
    }
    keys[i] = key;
    vals[i] = i;
}

// cell_start[k] = first sorted position whose key >= k, k in [0, 2G].
__global__ void k_cell_start(const unsigned int *__restrict__ keys, int total, long long ncells,
                             int *cell_start) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > ncells) return;
    int lo = 0, hi = total;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((long long)keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    cell_start[k] = lo;
}

// One thread per node: merges the particle lists of the (up to) eight cells
// that touch the node, in increasing particle index, and sums their CIC
// weights sequentially from 0 -- the order of a single-threaded run of the
// reference's deposit loop (include/tools.hpp:46-95).
template <typename T>
__global__ void k_deposit_merge(Geom g, const T *__restrict__ x, const T *__restrict__ y,
                                const T *__restrict__ z, const int *__restrict__ sorted_idx,
                                const int *__restrict__ cell_start, T *rho) {
    long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= 2 * g.G) return;
    const long long s_off = node >= g.G ? g.G : 0;
    const long long n0 = node - s_off;
    const int iz = (int)(n0 % g.nz), iy = (int)((n0 / g.nz) % g.ny), ix = (int)(n0 / ((long long)g.ny * g.nz));
    int pos[8], end[8], cor[8];
    int nl = 0;
    for (int c = 0; c < 8; c++) {
        int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
        int cx = ix - dx, cy = iy - dy, cz = iz - dz;
        if (cx < 0 || cy < 0 || cz < 0) continue;
        long long cell = ((long long)cx * g.ny + cy) * g.nz + cz + s_off;
        int s = cell_start[cell], e = cell_start[cell + 1];
        if (s < e) {
            pos[nl] = s;
            end[nl] = e;
            cor[nl] = c;
            nl++;
        }
    }
    T acc = T(0.0);
    const T dmx = T(g.dmx), dmy = T(g.dmy), dmz = T(g.dmz);
    while (true) {
        int best = -1, bidx = 0x7fffffff;
        for (int l = 0; l < nl; l++) {
            if (pos[l] < end[l]) {
                int p = sorted_idx[pos[l]];
                if (p < bidx) {
                    bidx = p;
                    best = l;
                }
            }
        }
        if (best < 0) break;
        pos[best]++;
        int c = cor[best];
        T cx = cell_coord<T>(x[bidx], dmx, g.nx);
        T cy = cell_coord<T>(y[bidx], dmy, g.ny);
        T cz = cell_coord<T>(z[bidx], dmz, g.nz);
        T d_x = cx - (int)cx, d_y = cy - (int)cy, d_z = cz - (int)cz;
        // node = cell + corner; corner bit 1 means the "1" side (weight d)
        T wx = ((c >> 2) & 1) ? d_x : T(1.0) - d_x;
        T wy = ((c >> 1) & 1) ? d_y : T(1.0) - d_y;
        T wz = (c & 1) ? d_z : T(1.0) - d_z;
        acc += wx * wy * wz;
    }
    rho[node] = acc;
}

// ---- smoothing (include/physics.hpp:202-234) -----------------------------
template <typename T>
__global__ void k_smooth_direct(Geom g, int ntaps, int lx, int ly, int lz, const int *__restrict__ taps,
                                const T *__restrict__ w, T term, const T *__restrict__ src, T *dst) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * g.G) return;
    const long long off = i >= g.G ? g.G : 0;
    const long long node = i - off;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int iz = (int)(node % nz), iy = (int)((node / nz) % ny), ix = (int)(node / ((long long)ny * nz));
    const T *s = src + off;
    T rho_f = T(0.0);
    const bool interior = ix >= lx && ix < nx - lx && iy >= ly && iy < ny - ly && iz >= lz && iz < nz - lz;
    if (interior) {
        for (int t = 0; t < ntaps; t++) {
            int p = __ldg(taps + t);
            int a = (p >> 20) - 512, b = ((p >> 10) & 1023) - 512, c = (p & 1023) - 512;
            long long j = node + ((long long)a * ny + b) * nz + c;
            rho_f += s[j] * __ldg(w + t);
        }
    } else {
        for (int t = 0; t < ntaps; t++) {
            int p = __ldg(taps + t);
            int a = (p >> 20) - 512, b = ((p >> 10) & 1023) - 512, c = (p & 1023) - 512;
            int jx = ix + a, jy = iy + b, jz = iz + c;
            if (jx < 0 || jx >= nx || jy < 0 || jy >= ny || jz < 0 || jz >= nz) continue;
            rho_f += s[((long long)jx * ny + jy) * nz + jz] * __ldg(w + t);
        }
    }
    dst[i] = rho_f * term;  // physics.hpp:229-232
}

// ---- Skyrme (include/physics.hpp:272-281, physics_formulas.hpp:70-77) ------
template <typename T>
__device__ __forceinline__ T skyrme_u(T A, T B, T C, T gamma, T rho_p, T rho_n, T tau) {
    T rho = rho_p + rho_n;
    T t = rho / T(0.16);
    return A * t + B * pow(t, gamma) + T(2.0) * tau * C * ((rho_n - rho_p) / T(0.16));
}

template <typename T>
__global__ void k_skyrme(long long G, T A, T B, T C, T gamma, const T *__restrict__ rho, T *U) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    T rp = rho[i], rn = rho[i + G];
    U[i] = skyrme_u<T>(A, B, C, gamma, rp, rn, T(-1.0));
    U[i + G] = skyrme_u<T>(A, B, C, gamma, rp, rn, T(+1.0));
}

// ---- Coulomb boundary (include/tools.hpp:283-300) -------------------------
template <typename T>
__device__ __forceinline__ T node_pos(T dmax, int i, int n) {
    return dmax * (T(2.0) * (T)i / (T)n - T(1.0));
}

template <typename T, typename A>  // A: arithmetic type of the monopole
__global__ void k_boundary(Geom g, int Z, T *phi) {
    long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= g.G) return;
    const int nz = g.nz, ny = g.ny, nx = g.nx;
    const int k = (int)(id % nz), j = (int)((id / nz) % ny), i = (int)(id / ((long long)ny * nz));
    if (!(i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1)) return;
    A v0 = node_pos<A>(A(g.dmx), i, nx), v1 = node_pos<A>(A(g.dmy), j, ny), v2 = node_pos<A>(A(g.dmz), k, nz);
    A r = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    phi[id] = (T)(A(1.44) * Z / r);
}

// ---- red-black SOR half sweep (include/physics.hpp:99-157) ----------------
__device__ __forceinline__ void atomic_max_bits(unsigned long long *m, double v) {
    atomicMax(m, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_bits(unsigned long long *m, float v) {
    atomicMax(m, (unsigned long long)__float_as_uint(v));
}

template <typename T>
__global__ void k_sor_half(Geom g, int color, T omega, T inv_dx2, T hx2, T hy2, T hz2, T src_c,
                           T *phi, const T *__restrict__ rho, unsigned long long *maxbits) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int half = (nz - 1) / 2;  // upper bound of colour points per (i, j) line
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long lines = (long long)(nx - 2) * (ny - 2);
    T diff = T(0.0);
    if (t < lines * half) {
        int kk = (int)(t % half);
        long long l = t / half;
        int j = 1 + (int)(l % (ny - 2)), i = 1 + (int)(l / (ny - 2));
        int k = 1 + ((i + j + 1 + color) & 1) + 2 * kk;
        if (k < nz - 1) {
            const long long sx = (long long)ny * nz, sy = nz;
            long long id = i * sx + j * sy + k;
            T r = rho[id];
            T phi_x = (phi[id + sx] + phi[id - sx]) / hx2;
            T phi_y = (phi[id + sy] + phi[id - sy]) / hy2;
            T phi_z = (phi[id + 1] + phi[id - 1]) / hz2;
            T phi_star = (phi_x + phi_y + phi_z + src_c * r) * inv_dx2;
            T phi_old = phi[id];
            T nv = (T(1.0) - omega) * phi_old + omega * phi_star;
            phi[id] = nv;
            diff = fabs(nv - phi_old);
        }
    }
    // block max, then one atomic per block (max is order independent)
    __shared__ T red[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) {
        T other = __shfl_xor_sync(0xffffffffu, diff, o);
        diff = (other > diff || other != other) ? other : diff;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = diff;
    __syncthreads();
    if (threadIdx.x == 0) {
        T m = red[0];
        for (int w = 1; w < kBlock / 32; w++) m = (red[w] > m || red[w] != red[w]) ? red[w] : m;
        atomic_max_bits(maxbits, m);
    }
}

// ||b + lap_h phi||^2 and ||b||^2 over interior nodes, in double; one partial
// pair per block (fixed grid, fixed order: deterministic).
template <typename T>
__global__ void k_residual_partials(Geom g, double ix2, double iy2, double iz2, double src_c,
                                    const T *__restrict__ phi, const T *__restrict__ rho,
                                    double *partials) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const long long n_int = (long long)(nx - 2) * (ny - 2) * (nz - 2);
    const double diag = 2.0 * ix2 + 2.0 * iy2 + 2.0 * iz2;
    double rr = 0.0, bb = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_int;
         t += (long long)gridDim.x * blockDim.x) {
        int k = 1 + (int)(t % (nz - 2));
        long long l = t / (nz - 2);
        int j = 1 + (int)(l % (ny - 2)), i = 1 + (int)(l / (ny - 2));
        long long id = i * sx + j * sy + k;
        double b = src_c * (double)rho[id];
        double lap = ((double)phi[id + sx] + (double)phi[id - sx]) * ix2 +
                     ((double)phi[id + sy] + (double)phi[id - sy]) * iy2 +
                     ((double)phi[id + 1] + (double)phi[id - 1]) * iz2 - diag * (double)phi[id];
        double r = b + lap;
        rr += r * r;
        bb += b * b;
    }
    __shared__ double s_rr[kBlock], s_bb[kBlock];
    s_rr[threadIdx.x] = rr;
    s_bb[threadIdx.x] = bb;
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_rr[threadIdx.x] += s_rr[threadIdx.x + o];
            s_bb[threadIdx.x] += s_bb[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = s_rr[0];
        partials[2 * blockIdx.x + 1] = s_bb[0];
    }
}

// Sums `width`-wide rows of partials (nblocks rows) in fixed order.
__global__ void k_sum_partials(const double *__restrict__ partials, int nblocks, int width,
                               double *out) {
    int c = threadIdx.x;
    if (c >= width) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; b++) s += partials[(long long)b * width + c];
    out[c] = s;
}

// ---- merge, FDM, gather, push, excite ------------------------------------
template <typename T>
__global__ void k_merge(long long G, T *U, const T *__restrict__ phi) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) U[i] += phi[i];
}

// compute_volumetric_forces_fdm (include/physics.hpp:159-200)
template <typename T>
__global__ void k_fdm(Geom g, T dx, T dy, T dz, const T *__restrict__ Uall, T *Fx, T *Fy, T *Fz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * g.G) return;
    const long long off = i >= g.G ? g.G : 0;
    const long long id = i - off;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const int k = (int)(id % nz), j = (int)((id / nz) % ny), ii = (int)(id / sx);
    const T *U = Uall + off;
    T gx, gy, gz;
    if (ii == 0) gx = (U[id + sx] - U[id]) / dx;
    else if (ii == nx - 1) gx = (U[id] - U[id - sx]) / dx;
    else gx = (U[id + sx] - U[id - sx]) / (T(2.0) * dx);
    if (j == 0) gy = (U[id + sy] - U[id]) / dy;
    else if (j == ny - 1) gy = (U[id] - U[id - sy]) / dy;
    else gy = (U[id + sy] - U[id - sy]) / (T(2.0) * dy);
    if (k == 0) gz = (U[id + 1] - U[id]) / dz;
    else if (k == nz - 1) gz = (U[id] - U[id - 1]) / dz;
    else gz = (U[id + 1] - U[id - 1]) / (T(2.0) * dz);
    Fx[i] = -gx;
    Fy[i] = -gy;
    Fz[i] = -gz;
}

// distribute_forces_to_particles_cic (include/tools.hpp:98-168)
template <typename T>
__global__ void k_gather(Geom g, int protons, int total, const T *__restrict__ x,
                         const T *__restrict__ y, const T *__restrict__ z, const T *__restrict__ Fx,
                         const T *__restrict__ Fy, const T *__restrict__ Fz, T *fx, T *fy, T *fz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    T cx = cell_coord<T>(x[i], T(g.dmx), nx);
    T cy = cell_coord<T>(y[i], T(g.dmy), ny);
    T cz = cell_coord<T>(z[i], T(g.dmz), nz);
    if (!in_grid<T>(cx, cy, cz, nx, ny, nz)) {
        fx[i] = T(0.0);
        fy[i] = T(0.0);
        fz[i] = T(0.0);
        return;
    }
    int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    T d_x = cx - x0, d_y = cy - y0, d_z = cz - z0;
    T t_x = T(1.0) - d_x, t_y = T(1.0) - d_y, t_z = T(1.0) - d_z;
    const long long off = (i < protons) ? 0 : g.G;
    const long long sx = (long long)ny * nz, sy = nz;
    T ax = T(0.0), ay = T(0.0), az = T(0.0);
    auto acc = [&](int a, int b, int c, T w) {
        long long id = a * sx + b * sy + c + off;
        ax += w * Fx[id];
        ay += w * Fy[id];
        az += w * Fz[id];
    };
    acc(x0, y0, z0, t_x * t_y * t_z);
    if (x1 < nx) acc(x1, y0, z0, d_x * t_y * t_z);
    if (y1 < ny) acc(x0, y1, z0, t_x * d_y * t_z);
    if (x1 < nx && y1 < ny) acc(x1, y1, z0, d_x * d_y * t_z);
    if (z1 < nz) acc(x0, y0, z1, t_x * t_y * d_z);
    if (x1 < nx && z1 < nz) acc(x1, y0, z1, d_x * t_y * d_z);
    if (y1 < ny && z1 < nz) acc(x0, y1, z1, t_x * d_y * d_z);
    if (x1 < nx && y1 < ny && z1 < nz) acc(x1, y1, z1, d_x * d_y * d_z);
    fx[i] = ax;
    fy[i] = ay;
    fz[i] = az;
}

// update_momenta_half / update_positions_full (include/physics.hpp:248-270):
// a += fact * b on three arrays.
template <typename T>
__global__ void k_axpy3(int total, T fact, T *a0, T *a1, T *a2, const T *__restrict__ b0,
                        const T *__restrict__ b1, const T *__restrict__ b2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    a0[i] += fact * b0[i];
    a1[i] += fact * b1[i];
    a2[i] += fact * b2[i];
}

// nuclear_excitation (include/physics.hpp:236-246)
template <typename T>
__global__ void k_excite(int protons, int total, T dp, T dn, T *kz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    if (i < protons) kz[i] += dp;
    else kz[i] -= dn;
}

// center_of_mass / mean_squared_radius partials (include/tools.hpp:302-338):
// per block {sum z_p, sum z_n, sum r2_p, sum r2_n, n_in_p, n_in_n}.
template <typename T>
__global__ void k_observe_partials(Geom g, int protons, int total, const T *__restrict__ x,
                                   const T *__restrict__ y, const T *__restrict__ z, double *partials) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    const T dmx = T(g.dmx), dmy = T(g.dmy), dmz = T(g.dmz);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int s = i < protons ? 0 : 1;
        T xi = x[i], yi = y[i], zi = z[i];
        v[s] += (double)zi;
        if (xi < -dmx || xi > +dmx || yi < -dmy || yi > +dmy || zi < -dmz || zi > +dmz) continue;
        T r2 = xi * xi + yi * yi + zi * zi;
        v[2 + s] += (double)r2;
        v[4 + s] += 1.0;
    }
    __shared__ double sh[6][kBlock];
    for (int c = 0; c < 6; c++) sh[c][threadIdx.x] = v[c];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int c = 0; c < 6; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 6) partials[6 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

inline int blocks_for(long long n) { return div_up(n > 0 ? n : 1, kBlock); }

}  // namespace

// ======================= launchers ========================================

template <typename T>
hv_status launch_deposit_atomic(hv_ctx *c, const T *x, const T *y, const T *z, T *rho) {
    HV_CUDA(cudaMemsetAsync(rho, 0, sizeof(T) * 2 * c->geom.G, c->stream));
    if (c->total > 0)
        k_deposit_atomic<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->geom, c->protons, c->total, x, y, z, rho);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_deposit_sorted(hv_ctx *c, const T *x, const T *y, const T *z, T *rho) {
    const long long ncell = 2 * c->geom.G;
    Scratch &s = c->scratch;
    if (c->total == 0) {
        HV_CUDA(cudaMemsetAsync(rho, 0, sizeof(T) * ncell, c->stream));
        return HV_OK;
    }
    k_cell_keys<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->geom, c->protons, c->total, x, y, z, s.keys, s.vals);
    HV_CUDA(cudaGetLastError());
    int end_bit = 1;
    while ((1ull << end_bit) <= (unsigned long long)ncell) end_bit++;
    size_t bytes = s.cub_tmp_bytes;
    HV_CUDA(cub::DeviceRadixSort::SortPairs(s.cub_tmp, bytes, s.keys, s.keys_alt, s.vals, s.vals_alt,
                                            c->total, 0, end_bit, c->stream));
    k_cell_start<<<blocks_for(ncell + 1), kBlock, 0, c->stream>>>(s.keys_alt, c->total, ncell, s.cell_start);
    HV_CUDA(cudaGetLastError());
    k_deposit_merge<T><<<blocks_for(ncell), kBlock, 0, c->stream>>>(c->geom, x, y, z, s.vals_alt, s.cell_start, rho);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

// Bytes of CUB temporary storage for a sort of `total` keys.
size_t sorted_deposit_tmp_bytes(int total) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs((void *)nullptr, bytes, (unsigned int *)nullptr, (unsigned int *)nullptr,
                                    (int *)nullptr, (int *)nullptr, total > 0 ? total : 1, 0, 32);
    return bytes;
}

template <typename T>
hv_status launch_smooth(hv_ctx *c, const T *rho_raw, T *rho) {
    const hv_run_params &p = c->params;
    // normalisation term in T, evaluated as the reference does (physics.hpp:229)
    const T sig = T(p.sigma_r);
    const T term = (T(1.0) / p.part_per_nucleon) *
                   (T(1.0) / std::pow(T(2.0) * T(kPi) * sig * sig, T(1.5)));
    const T *w = reinterpret_cast<const T *>(sizeof(T) == 8 ? (void *)c->d64.taps_w : (void *)c->d32.taps_w);
    k_smooth_direct<T><<<blocks_for(2 * c->geom.G), kBlock, 0, c->stream>>>(
        c->geom, c->taps_count, c->taps.lim[0], c->taps.lim[1], c->taps.lim[2], c->taps_dev, w, term, rho_raw, rho);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_skyrme(hv_ctx *c, const T *rho, T *U) {
    const hv_skyrme &s = c->params.skyrme;
    k_skyrme<T><<<blocks_for(c->geom.G), kBlock, 0, c->stream>>>(c->geom.G, T(s.A), T(s.B), T(s.C), T(s.gamma), rho, U);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_boundary(hv_ctx *c, T *phi) {
    k_boundary<T, T><<<blocks_for(c->geom.G), kBlock, 0, c->stream>>>(c->geom, c->params.z, phi);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_sor_plain(hv_ctx *c, T *phi, const T *rho, int *iters, double *metric) {
    const Geom &g = c->geom;
    const hv_sor_params &sp = c->params.sor;
    const T dx = T(2.0) * T(g.dmx) / g.nx, dy = T(2.0) * T(g.dmy) / g.ny, dz = T(2.0) * T(g.dmz) / g.nz;
    const T hx2 = dx * dx, hy2 = dy * dy, hz2 = dz * dz;
    const T inv_dx2 = T(1.0) / (T(2.0) / hx2 + T(2.0) / hy2 + T(2.0) / hz2);
    const T omega = T(sp.omega);
    const T src_c = T(4.0) * T(kPi) * T(1.44);
    const long long lines = (long long)(g.nx - 2) * (g.ny - 2);
    const int half = (g.nz - 1) / 2;
    const int nb = blocks_for(lines * half);
    // residual in double from double spacings
    const double ddx = 2.0 * g.dmx / g.nx, ddy = 2.0 * g.dmy / g.ny, ddz = 2.0 * g.dmz / g.nz;
    const int rb = 2 * c->sm_count;
    double m = 0.0;
    int it = 0;
    bool converged = false;
    for (it = 0; it < sp.max_iter;) {
        if (sp.criterion == HV_SOR_MAX_UPDATE)
            HV_CUDA(cudaMemsetAsync(c->scratch.maxbits, 0, sizeof(unsigned long long), c->stream));
        for (int color = 0; color < 2; color++) {
            k_sor_half<T><<<nb, kBlock, 0, c->stream>>>(g, color, omega, inv_dx2, hx2, hy2, hz2, src_c, phi, rho,
                                                       c->scratch.maxbits);
        }
        HV_CUDA(cudaGetLastError());
        it++;
        if (sp.criterion == HV_SOR_MAX_UPDATE) {
            unsigned long long bits = 0;
            HV_CUDA(cudaMemcpyAsync(&bits, c->scratch.maxbits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
            HV_CUDA(cudaStreamSynchronize(c->stream));
            T md;
            if (sizeof(T) == 8) {
                double d;
                memcpy(&d, &bits, 8);
                md = (T)d;
            } else {
                unsigned int u = (unsigned int)bits;
                float f;
                memcpy(&f, &u, 4);
                md = (T)f;
            }
            m = (double)md;
            if (md != md) {
                if (iters) *iters = it;
                if (metric) *metric = m;
                return HV_ERR_NONFINITE;
            }
            if (md < T(sp.tol)) {  // physics.hpp:152
                converged = true;
                break;
            }
        } else {
            k_residual_partials<T><<<rb, kBlock, 0, c->stream>>>(g, 1.0 / (ddx * ddx), 1.0 / (ddy * ddy),
                                                                 1.0 / (ddz * ddz), 4.0 * kPi * 1.44, phi, rho,
                                                                 c->scratch.partials);
            k_sum_partials<<<1, 32, 0, c->stream>>>(c->scratch.partials, rb, 2, c->scratch.result);
            HV_CUDA(cudaGetLastError());
            HV_CUDA(cudaMemcpyAsync(c->scratch.h_result, c->scratch.result, 2 * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
            HV_CUDA(cudaStreamSynchronize(c->stream));
            double rr = c->scratch.h_result[0], bb = c->scratch.h_result[1];
            m = bb > 0.0 ? std::sqrt(rr / bb) : std::sqrt(rr);
            if (m != m) {
                if (iters) *iters = it;
                if (metric) *metric = m;
                return HV_ERR_NONFINITE;
            }
            if (m <= sp.tol) {
                converged = true;
                break;
            }
        }
    }
    if (iters) *iters = it;
    if (metric) *metric = m;
    return converged ? HV_OK : HV_ERR_NOT_CONVERGED;
}

template <typename T>
hv_status launch_merge(hv_ctx *c, T *U, const T *phi) {
    k_merge<T><<<blocks_for(c->geom.G), kBlock, 0, c->stream>>>(c->geom.G, U, phi);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_fdm(hv_ctx *c, const T *U, T *Fx, T *Fy, T *Fz) {
    const Geom &g = c->geom;
    const T dx = T(2.0) * T(g.dmx) / g.nx, dy = T(2.0) * T(g.dmy) / g.ny, dz = T(2.0) * T(g.dmz) / g.nz;
    k_fdm<T><<<blocks_for(2 * g.G), kBlock, 0, c->stream>>>(g, dx, dy, dz, U, Fx, Fy, Fz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_gather(hv_ctx *c, const T *x, const T *y, const T *z, const T *Fx, const T *Fy, const T *Fz,
                        T *fx, T *fy, T *fz) {
    if (c->total == 0) return HV_OK;
    k_gather<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->geom, c->protons, c->total, x, y, z, Fx, Fy, Fz,
                                                               fx, fy, fz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_kick(hv_ctx *c, T *kx, T *ky, T *kz, const T *fx, const T *fy, const T *fz, double dt) {
    if (c->total == 0) return HV_OK;
    const T fact = T(dt) / (T(2.0) * T(kHbarC));  // physics.hpp:251
    k_axpy3<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->total, fact, kx, ky, kz, fx, fy, fz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_drift(hv_ctx *c, T *x, T *y, T *z, const T *kx, const T *ky, const T *kz, double dt) {
    if (c->total == 0) return HV_OK;
    const T fact = (T(dt) * T(kHbarC)) / T(kMc2);  // physics.hpp:263
    k_axpy3<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->total, fact, x, y, z, kx, ky, kz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_excite(hv_ctx *c, T *kz, double eta) {
    if (c->total == 0) return HV_OK;
    const T zz = T(c->params.z), nn = T(c->params.n), e = T(eta);
    const T dp = e * nn / (zz + nn), dn = e * zz / (zz + nn);  // physics.hpp:241,244
    k_excite<T><<<blocks_for(c->total), kBlock, 0, c->stream>>>(c->protons, c->total, dp, dn, kz);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status launch_observe(hv_ctx *c, const T *x, const T *y, const T *z, hv_observables *out) {
    const int nb = 2 * c->sm_count;
    k_observe_partials<T><<<nb, kBlock, 0, c->stream>>>(c->geom, c->protons, c->total, x, y, z, c->scratch.partials);
    k_sum_partials<<<1, 32, 0, c->stream>>>(c->scratch.partials, nb, 6, c->scratch.result);
    HV_CUDA(cudaGetLastError());
    HV_CUDA(cudaMemcpyAsync(c->scratch.h_result, c->scratch.result, 6 * sizeof(double), cudaMemcpyDeviceToHost,
                            c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    const double *v = c->scratch.h_result;
    out->zcm_p = v[0] / (double)c->protons;
    out->zcm_n = v[1] / (double)c->neutrons;
    out->rms_p = std::sqrt(v[2] / v[4]);
    out->rms_n = std::sqrt(v[3] / v[5]);
    const double zz = c->params.z, nn = c->params.n;
    out->dipole = (nn * zz) / (nn + zz) * (out->zcm_p - out->zcm_n);
    return HV_OK;
}

#define HV_INST(T)                                                                                         \
    template hv_status launch_deposit_atomic<T>(hv_ctx *, const T *, const T *, const T *, T *);           \
    template hv_status launch_deposit_sorted<T>(hv_ctx *, const T *, const T *, const T *, T *);           \
    template hv_status launch_smooth<T>(hv_ctx *, const T *, T *);                                         \
    template hv_status launch_skyrme<T>(hv_ctx *, const T *, T *);                                         \
    template hv_status launch_boundary<T>(hv_ctx *, T *);                                                  \
    template hv_status launch_sor_plain<T>(hv_ctx *, T *, const T *, int *, double *);                     \
    template hv_status launch_merge<T>(hv_ctx *, T *, const T *);                                          \
    template hv_status launch_fdm<T>(hv_ctx *, const T *, T *, T *, T *);                                  \
    template hv_status launch_gather<T>(hv_ctx *, const T *, const T *, const T *, const T *, const T *,   \
                                        const T *, T *, T *, T *);                                         \
    template hv_status launch_kick<T>(hv_ctx *, T *, T *, T *, const T *, const T *, const T *, double);   \
    template hv_status launch_drift<T>(hv_ctx *, T *, T *, T *, const T *, const T *, const T *, double);  \
    template hv_status launch_excite<T>(hv_ctx *, T *, double);                                            \
    template hv_status launch_observe<T>(hv_ctx *, const T *, const T *, const T *, hv_observables *);

HV_INST(double)
HV_INST(float)

}  // namespace hv
