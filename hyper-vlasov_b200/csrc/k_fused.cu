// Fused fast path (HV_PATH_FUSED): one particle kernel per step, the field
// kernels, the persistent SOR, replayed from a CUDA graph.
//
// The reference's step (src/hyper_vlasov.cpp:86-103) is
//   [observe] [excite once] kick/2(f_n) drift deposit ... gather(f_{n+1}) kick/2(f_{n+1}).
// The particle kernel of step n does, per particle, everything between two
// field solves with the same arithmetic sequence:
//   gather f_n -> [closing kick/2 of step n-1] -> observe x_n -> [excite]
//   -> opening kick/2 of step n -> drift -> deposit x_{n+1},
// so x and k are read and written once per step (48 B per particle in
// float).  The closing half kick of the last step is applied by
// k_close_kick when hv_run returns, leaving the state the plain path leaves.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "hv_internal.h"

namespace hv {

hv_status sor_fast_plan(hv_ctx *c);
void sor_fast_release(hv_ctx *c);
template <typename T>
hv_status sor_fast_launch(hv_ctx *c, const T *rho, int *ctl, int *its_ring, int ring, bool step_solve);
hv_status sor_fast_clear_error(hv_ctx *c);
hv_status smooth_fast_plan(hv_ctx *c);
void smooth_fast_release(hv_ctx *c);
hv_status smooth_fast_launch(hv_ctx *c, const float *rho_raw, float *rho, const int *wcount);
bool smooth_fft_runs(const hv_ctx *c);

namespace {

constexpr int kPBlock = 256;      // default threads per block of the particle step
constexpr int kPBlockMax = 512;   // largest of the autotuner's candidates
constexpr int kPGridMax = 16;     // most blocks per SM of the particle step
constexpr int kForceRows = 8;     // y rows per thread of the forces kernel on every row
constexpr int kForceRowsGated = 4; // the same where only rows holding raw density are computed:
                                   // shorter walks, as few blocks work (an eighth on 208Pb 128^3)
constexpr int kRing = 64;  // observable rows kept on the device

// control words (Fused::ctl)
enum { CTL_STEP = 0, CTL_MHINT = 1, CTL_PREV = 2, CTL_EXCITE = 3, CTL_CLOSE = 4, CTL_N = 8 };

template <typename T>
__device__ __forceinline__ void load_f4(const T *F4, long long node, T &fx, T &fy, T &fz);
template <>
__device__ __forceinline__ void load_f4<float>(const float *F4, long long node, float &fx, float &fy, float &fz) {
    float4 v = __ldg(reinterpret_cast<const float4 *>(F4) + node);
    fx = v.x;
    fy = v.y;
    fz = v.z;
}
template <>
__device__ __forceinline__ void load_f4<double>(const double *F4, long long node, double &fx, double &fy, double &fz) {
    const double2 *p = reinterpret_cast<const double2 *>(F4) + 2 * node;
    double2 a = __ldg(p), b = __ldg(p + 1);
    fx = a.x;
    fy = a.y;
    fz = b.x;
}

// Grid coordinates of a position, (n / 2) (p / d_max + 1) per axis
// (include/tools.hpp:35-96 and :98-168).  In float the division is a product
// by the axis's reciprocal d_max, formed once per launch: the particle step
// would otherwise make six IEEE divisions per particle.  A coordinate then
// moves by at most about an ulp; a particle that lies on a cell face may land
// in the neighbouring cell with a weight of ~0 there, which the continuity of
// the CIC weights makes harmless.  The double form keeps the division.
template <typename T>
struct CellMap {
    T hx, hy, hz;  // n / 2
    T ix, iy, iz;  // 1 / d_max (float form)
    T dx, dy, dz;  // d_max (double form)
};

template <typename T>
__device__ __forceinline__ CellMap<T> cell_map(const Geom &g) {
    return CellMap<T>{g.nx / T(2.0),      g.ny / T(2.0),      g.nz / T(2.0), T(1.0) / T(g.dmx), T(1.0) / T(g.dmy),
                      T(1.0) / T(g.dmz), T(g.dmx),           T(g.dmy),      T(g.dmz)};
}

template <typename T>
__device__ __forceinline__ void cell_coords(const CellMap<T> &m, T px, T py, T pz, T &cx, T &cy, T &cz) {
    if constexpr (sizeof(T) == 4) {
        cx = m.hx * (px * m.ix + T(1.0));
        cy = m.hy * (py * m.iy + T(1.0));
        cz = m.hz * (pz * m.iz + T(1.0));
    } else {
        cx = m.hx * (px / m.dx + T(1.0));
        cy = m.hy * (py / m.dy + T(1.0));
        cz = m.hz * (pz / m.dz + T(1.0));
    }
}

// CIC force gather at (px,py,pz) (distribute_forces_to_particles_cic,
// include/tools.hpp:98-168; corner order and corner drop as there).
template <typename T>
__device__ __forceinline__ void gather_at(const Geom &g, const CellMap<T> &m, const T *F4, long long off, T px, T py,
                                          T pz, T &ax, T &ay, T &az) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    ax = ay = az = T(0);
    T cx, cy, cz;
    cell_coords<T>(m, px, py, pz, cx, cy, cz);
    if (cx < T(0) || cy < T(0) || cz < T(0) || cx >= nx || cy >= ny || cz >= nz) return;
    int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    T dx = cx - x0, dy = cy - y0, dz = cz - z0;
    T tx = T(1) - dx, ty = T(1) - dy, tz = T(1) - dz;
    const bool bx = x0 + 1 < nx, by = y0 + 1 < ny, bz = z0 + 1 < nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const long long n0 = off + x0 * sx + y0 * sy + z0;
    T fx, fy, fz, w;
#define HV_G(COND, DNODE, W)                    \
    if (COND) {                                 \
        load_f4<T>(F4, n0 + (DNODE), fx, fy, fz); \
        w = (W);                                \
        ax += w * fx;                           \
        ay += w * fy;                           \
        az += w * fz;                           \
    }
    HV_G(true, 0, tx * ty * tz)
    HV_G(bx, sx, dx * ty * tz)
    HV_G(by, sy, tx * dy * tz)
    HV_G(bx && by, sx + sy, dx * dy * tz)
    HV_G(bz, 1, tx * ty * dz)
    HV_G(bx && bz, sx + 1, dx * ty * dz)
    HV_G(by && bz, sy + 1, tx * dy * dz)
    HV_G(bx && by && bz, sx + sy + 1, dx * dy * dz)
#undef HV_G
}

// CIC deposit of one particle (distribute_volumetric_particles_cic,
// include/tools.hpp:35-96), atomically.
template <typename T>
__device__ __forceinline__ void deposit_at(const Geom &g, const CellMap<T> &m, T *rho, long long off, T px, T py,
                                           T pz) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    T cx, cy, cz;
    cell_coords<T>(m, px, py, pz, cx, cy, cz);
    if (cx < T(0) || cy < T(0) || cz < T(0) || cx >= nx || cy >= ny || cz >= nz) return;
    int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
    T dx = cx - x0, dy = cy - y0, dz = cz - z0;
    T tx = T(1) - dx, ty = T(1) - dy, tz = T(1) - dz;
    const bool bx = x0 + 1 < nx, by = y0 + 1 < ny, bz = z0 + 1 < nz;
    const long long sx = (long long)ny * nz, sy = nz;
    T *b = rho + off + x0 * sx + y0 * sy + z0;
    if constexpr (sizeof(T) == 4) {
        // nz even (so the row and plane strides are even) and an even base
        // index: each z-pair of corners is one 8-byte-aligned float2, added
        // by one vector atomic
        if (bz && (nz & 1) == 0 && ((off + x0 * sx + y0 * sy + z0) & 1) == 0) {
            float2 *b2 = reinterpret_cast<float2 *>(b);
            const long long sx2 = sx / 2, sy2 = sy / 2;
            atomicAdd(b2, make_float2(tx * ty * tz, tx * ty * dz));
            if (bx) atomicAdd(b2 + sx2, make_float2(dx * ty * tz, dx * ty * dz));
            if (by) atomicAdd(b2 + sy2, make_float2(tx * dy * tz, tx * dy * dz));
            if (bx && by) atomicAdd(b2 + sx2 + sy2, make_float2(dx * dy * tz, dx * dy * dz));
            return;
        }
        // nz a multiple of 4 and the base index 1 mod 4: the z-pair is the
        // middle of a 16-byte-aligned float4 whose outer two elements (inside
        // the row: z0 - 1 >= 0, z0 + 2 < nz) receive exact zeros
        if (bz && (nz & 3) == 0 && ((off + x0 * sx + y0 * sy + z0) & 3) == 1) {
            float4 *b4 = reinterpret_cast<float4 *>(b - 1);
            const long long sx4 = sx / 4, sy4 = sy / 4;
            atomicAdd(b4, make_float4(0.0f, tx * ty * tz, tx * ty * dz, 0.0f));
            if (bx) atomicAdd(b4 + sx4, make_float4(0.0f, dx * ty * tz, dx * ty * dz, 0.0f));
            if (by) atomicAdd(b4 + sy4, make_float4(0.0f, tx * dy * tz, tx * dy * dz, 0.0f));
            if (bx && by) atomicAdd(b4 + sx4 + sy4, make_float4(0.0f, dx * dy * tz, dx * dy * dz, 0.0f));
            return;
        }
    }
    atomicAdd(b, tx * ty * tz);
    if (bx) atomicAdd(b + sx, dx * ty * tz);
    if (by) atomicAdd(b + sy, tx * dy * tz);
    if (bx && by) atomicAdd(b + sx + sy, dx * dy * tz);
    if (bz) atomicAdd(b + 1, tx * ty * dz);
    if (bx && bz) atomicAdd(b + sx + 1, dx * ty * dz);
    if (by && bz) atomicAdd(b + sy + 1, tx * dy * dz);
    if (bx && by && bz) atomicAdd(b + sx + sy + 1, dx * dy * dz);
}

// The z-pair-wise vector atomics of deposit_at for one base node n0 (index in
// the stacked grid) and eight corner weights w[c], c = dx + 2 dy + 4 dz
// (corners with an index equal to n already zeroed or skipped by bx/by/bz).
__device__ __forceinline__ void add_corners(const Geom &g, float *rho, long long n0, bool bx, bool by, bool bz,
                                            const float (&w)[8]) {
    const int nz = g.nz;
    const long long sx = (long long)g.ny * nz, sy = nz;
    float *b = rho + n0;
    if (bz && (nz & 1) == 0 && (n0 & 1) == 0) {
        float2 *b2 = reinterpret_cast<float2 *>(b);
        const long long sx2 = sx / 2, sy2 = sy / 2;
        atomicAdd(b2, make_float2(w[0], w[4]));
        if (bx) atomicAdd(b2 + sx2, make_float2(w[1], w[5]));
        if (by) atomicAdd(b2 + sy2, make_float2(w[2], w[6]));
        if (bx && by) atomicAdd(b2 + sx2 + sy2, make_float2(w[3], w[7]));
        return;
    }
    if (bz && (nz & 3) == 0 && (n0 & 3) == 1) {
        float4 *b4 = reinterpret_cast<float4 *>(b - 1);
        const long long sx4 = sx / 4, sy4 = sy / 4;
        atomicAdd(b4, make_float4(0.0f, w[0], w[4], 0.0f));
        if (bx) atomicAdd(b4 + sx4, make_float4(0.0f, w[1], w[5], 0.0f));
        if (by) atomicAdd(b4 + sy4, make_float4(0.0f, w[2], w[6], 0.0f));
        if (bx && by) atomicAdd(b4 + sx4 + sy4, make_float4(0.0f, w[3], w[7], 0.0f));
        return;
    }
    atomicAdd(b, w[0]);
    if (bx) atomicAdd(b + sx, w[1]);
    if (by) atomicAdd(b + sy, w[2]);
    if (bx && by) atomicAdd(b + sx + sy, w[3]);
    if (bz) atomicAdd(b + 1, w[4]);
    if (bx && bz) atomicAdd(b + sx + 1, w[5]);
    if (by && bz) atomicAdd(b + sy + 1, w[6]);
    if (bx && by && bz) atomicAdd(b + sx + sy + 1, w[7]);
}

// CIC deposit of one particle per lane of a warp (all 32 lanes call it;
// valid false for a lane past the last particle), aggregated over runs of
// consecutive lanes with the same base node: the slots are re-sorted by cell
// every few steps, so neighbouring lanes mostly share one.  A ballot marks
// each run's last lane, a segmented suffix sum over shuffles gives the run's
// first lane the sums of its lanes' eight corner weights, and that lane alone
// issues the atomics (distribute_volumetric_particles_cic,
// include/tools.hpp:35-96: the same cells, weights and corner drops; only the
// order of the float additions differs).
__device__ __forceinline__ void deposit_warp(const Geom &g, const CellMap<float> &m, float *rho, long long off,
                                             float px, float py, float pz, bool valid) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int lane = threadIdx.x & 31;
    float cx, cy, cz;
    cell_coords<float>(m, px, py, pz, cx, cy, cz);
    const bool in = valid && !(cx < 0.0f || cy < 0.0f || cz < 0.0f || cx >= nx || cy >= ny || cz >= nz);
    int x0 = 0, y0 = 0, z0 = 0;
    float w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long key = -1;
    if (in) {
        x0 = (int)cx;
        y0 = (int)cy;
        z0 = (int)cz;
        const float dx = cx - x0, dy = cy - y0, dz = cz - z0;
        const float tx = 1.0f - dx, ty = 1.0f - dy, tz = 1.0f - dz;
        w[0] = tx * ty * tz;
        w[1] = dx * ty * tz;
        w[2] = tx * dy * tz;
        w[3] = dx * dy * tz;
        w[4] = tx * ty * dz;
        w[5] = dx * ty * dz;
        w[6] = tx * dy * dz;
        w[7] = dx * dy * dz;
        key = off + ((long long)x0 * ny + y0) * nz + z0;
    }
    const long long knext = __shfl_down_sync(0xffffffffu, key, 1);
    const long long kprev = __shfl_up_sync(0xffffffffu, key, 1);
    const bool last = lane == 31 || knext != key;
    const bool first = lane == 0 || kprev != key;
    const unsigned ends = __ballot_sync(0xffffffffu, last);
    if (ends != 0xffffffffu) {  // some run is longer than one lane
        const int run_end = lane + __ffs(ends >> lane) - 1;
        const unsigned longest = __reduce_max_sync(0xffffffffu, (unsigned)(run_end - lane + 1));
        for (int d = 1; d < (int)longest; d <<= 1) {
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const float o = __shfl_down_sync(0xffffffffu, w[c], d);
                if (lane + d <= run_end) w[c] += o;
            }
        }
    }
    if (!first || key < 0) return;
    add_corners(g, rho, key, x0 + 1 < nx, y0 + 1 < ny, z0 + 1 < nz, w);
}

template <typename T>
struct PArgs {
    Geom g;
    int protons, total;
    T *x, *y, *z, *kx, *ky, *kz;
    const T *F4;
    T *rho_raw;
    T h, fd, dp, dn;
    int deposit;  // 1: atomic CIC deposit of x_{n+1} here; 0: the sorted deposit follows
    int aggregate;  // float atomic deposit aggregated over warp runs of equal base nodes
    // the FFT smoothing's wrap list (null: not kept): particles whose deposit
    // reaches within the stencil half-widths wA, wB, wW of a face
    float4 *wlist;
    int *wcount;
    int wcap, wA, wB, wW;
    const int *ctl;
    double *obs;  // [kRing][blocks][6]
};

// Lists the particles whose CIC corners reach within the FFT smoothing's
// stencil of a face, where the circular convolution wraps their deposit
// around: grid coordinates (as the deposit forms them) and species, a warp's
// entries appended with one atomic.  Every lane calls it; past the list's
// capacity entries are counted but not stored (the smoothing then takes the
// direct form).
__device__ __forceinline__ void list_wrap(const PArgs<float> &a, const CellMap<float> &m, float px, float py,
                                          float pz, long long off, bool valid) {
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    float cx, cy, cz;
    cell_coords<float>(m, px, py, pz, cx, cy, cz);
    bool want = false;
    if (valid && !(cx < 0.0f || cy < 0.0f || cz < 0.0f || cx >= nx || cy >= ny || cz >= nz)) {
        const int x0 = (int)cx, y0 = (int)cy, z0 = (int)cz;
        want = x0 < a.wA || x0 >= nx - a.wA - 1 || y0 < a.wB || y0 >= ny - a.wB - 1 || z0 < a.wW ||
               z0 >= nz - a.wW - 1;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(a.wcount, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        const int pos = base + __popc(mask & ((1u << lane) - 1u));
        if (pos < a.wcap) a.wlist[pos] = make_float4(cx, cy, cz, off ? 1.0f : 0.0f);
    }
}

// One particle of one step: gather f_n, the closing kick/2 of the previous
// step, observables of x_n, the excitation, the opening kick/2 and the drift;
// returns x_{n+1} and the particle's species offset in the stacked grids.
// The state (x_n, k) of one particle, loaded ahead of its update.
template <typename T>
struct PState {
    T px, py, pz, qx, qy, qz;
};

template <typename T>
__device__ __forceinline__ PState<T> load_state(const PArgs<T> &a, int i) {
    return PState<T>{a.x[i], a.y[i], a.z[i], a.kx[i], a.ky[i], a.kz[i]};
}

// The observable sums of one thread, per species (v[s], v[2 + s], v[4 + s]
// with s the species): indexed by constants only, so that they stay in
// registers (an index by the particle's species put them in local memory).
struct ObsSums {
    double z0, z1, r0, r1;
    int n0, n1;  // counts, exact in an int
};

template <typename T>
__device__ __forceinline__ void particle_update(const PArgs<T> &a, const CellMap<T> &m, int i, const PState<T> &st,
                                                bool close, bool excite, T dmx, T dmy, T dmz, ObsSums &v, T &px,
                                                T &py, T &pz, long long &off) {
    const int s = i < a.protons ? 0 : 1;
    off = s ? a.g.G : 0;
    px = st.px;
    py = st.py;
    pz = st.pz;
    T qx = st.qx, qy = st.qy, qz = st.qz;
    T fx, fy, fz;
    gather_at<T>(a.g, m, a.F4, off, px, py, pz, fx, fy, fz);
    if (close) {  // closing kick/2 of the previous step (physics.hpp:248-258)
        qx += a.h * fx;
        qy += a.h * fy;
        qz += a.h * fz;
    }
    // observables of x_n (tools.hpp:302-338)
    const bool inside = !(px < -dmx || px > dmx || py < -dmy || py > dmy || pz < -dmz || pz > dmz);
    const double zd = (double)pz;
    const double r2 = inside ? (double)(px * px + py * py + pz * pz) : 0.0;
    if (s == 0) {
        v.z0 += zd;
        if (inside) {
            v.r0 += r2;
            v.n0 += 1;
        }
    } else {
        v.z1 += zd;
        if (inside) {
            v.r1 += r2;
            v.n1 += 1;
        }
    }
    if (excite) qz += s ? -a.dn : a.dp;  // physics.hpp:236-246
    qx += a.h * fx;                      // opening kick/2
    qy += a.h * fy;
    qz += a.h * fz;
    px += a.fd * qx;  // drift (physics.hpp:260-270)
    py += a.fd * qy;
    pz += a.fd * qz;
    a.x[i] = px;
    a.y[i] = py;
    a.z[i] = pz;
    a.kx[i] = qx;
    a.ky[i] = qy;
    a.kz[i] = qz;
}

// One step of every particle; observables of x_n into the ring row of step n.
// Float: at most 64 registers a thread (1024 threads resident per SM), with
// no spills; the step is bound by the latency of its gathers, so resident
// warps count.  The double form would spill under that bound and is left
// unbounded (its step is dominated by the double solve).
template <typename T, int kB>
__global__ void __launch_bounds__(kB, sizeof(T) == 4 ? 1024 / kB : 1) k_particle_step(PArgs<T> a) {
    const int step = a.ctl[CTL_STEP];
    const bool close = a.ctl[CTL_CLOSE] != 0;
    const bool excite = a.ctl[CTL_EXCITE] == step;
    const T dmx = T(a.g.dmx), dmy = T(a.g.dmy), dmz = T(a.g.dmz);
    const CellMap<T> m = cell_map<T>(a.g);
    ObsSums v{0.0, 0.0, 0.0, 0.0, 0, 0};
    // Each block takes one contiguous chunk of the slots (a multiple of 32):
    // the slots are sorted by cell every few steps, so a block's particles
    // lie in a few rows of cells and their force gathers hit in L1.  Warp-
    // uniform trip count (the aggregated deposit needs every lane); the next
    // particle's state is loaded before this one's gathers and atomics, so
    // that its memory round trip overlaps them.
    const int chunk = (int)((((long long)a.total + gridDim.x - 1) / gridDim.x + 31) & ~31ll);
    const int begin = (int)min((long long)blockIdx.x * chunk, (long long)a.total);
    const int end = (int)min((long long)begin + chunk, (long long)a.total);
    const int stride = blockDim.x;
    const int i_first = begin + threadIdx.x;
    PState<T> next{};
    if (i_first < end) next = load_state(a, i_first);
    for (int i0 = begin + (threadIdx.x & ~31); i0 < end; i0 += stride) {
        const int i = i0 + (threadIdx.x & 31);
        const bool valid = i < end;
        const PState<T> cur = next;
        if (i + stride < end) next = load_state(a, i + stride);
        T px = T(0), py = T(0), pz = T(0);
        long long off = 0;
        if (valid) particle_update<T>(a, m, i, cur, close, excite, dmx, dmy, dmz, v, px, py, pz, off);
        if (!a.deposit) continue;
        if constexpr (sizeof(T) == 4) {
            if (a.wlist) list_wrap(a, m, px, py, pz, off, valid);
            if (a.aggregate) {
                deposit_warp(a.g, m, reinterpret_cast<float *>(a.rho_raw), off, px, py, pz, valid);
                continue;
            }
        }
        if (valid) deposit_at<T>(a.g, m, a.rho_raw, off, px, py, pz);
    }
    // deterministic block reduction of the six sums
    __shared__ double sh[6][kB / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const double vs[6] = {v.z0, v.z1, v.r0, v.r1, (double)v.n0, (double)v.n1};
#pragma unroll
    for (int c = 0; c < 6; c++) {
        double u = vs[c];
        for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
        if (l == 0) sh[c][w] = u;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double u = 0.0;
        for (int q = 0; q < kB / 32; q++) u += sh[threadIdx.x][q];
        a.obs[((long long)(step % kRing) * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = u;
    }
}

// Closing kick/2 with the forces of the final positions; stores f.
template <typename T>
__global__ void k_close_kick(Geom g, int protons, int total, const T *__restrict__ x, const T *__restrict__ y,
                             const T *__restrict__ z, T *kx, T *ky, T *kz, T *fx, T *fy, T *fz, const T *F4, T h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    T ax, ay, az;
    gather_at<T>(g, cell_map<T>(g), F4, i < protons ? 0 : g.G, x[i], y[i], z[i], ax, ay, az);
    kx[i] += h * ax;
    ky[i] += h * ay;
    kz[i] += h * az;
    fx[i] = ax;
    fy[i] = ay;
    fz[i] = az;
}

// Skyrme potential (include/physics.hpp:272-281, physics_formulas.hpp:70-77).
// In float, t^gamma is CUDA's fast power intrinsic (exp2 of gamma log2 t on
// the special-function units) and the divisions by rho0 are products by its
// reciprocal: the accurate pow and two divisions made this kernel compute-
// bound (58 % SM, 11 % DRAM in ncu).  The results move by float rounding;
// the FP32 form's accuracy is checked on D(t).  The double form (the fused
// FP64 path) keeps pow and the divisions.
template <typename T>
__device__ __forceinline__ void skyrme_node(T A, T B, T C, T gamma, T rp, T rn, T &up, T &un) {
    if constexpr (sizeof(T) == 4) {
        const float inv_rho0 = 1.0f / 0.16f;
        const float t = (rp + rn) * inv_rho0;
        const float base = A * t + B * __powf(t, gamma);
        const float iso = 2.0f * C * ((rn - rp) * inv_rho0);
        up = base - iso;
        un = base + iso;
    } else {
        const T t = (rp + rn) / T(0.16);
        const T base = A * t + B * pow(t, gamma);
        const T iso = T(2.0) * C * ((rn - rp) / T(0.16));
        up = base - iso;
        un = base + iso;
    }
}

// The smoothed density is also clamped at zero here, in place: the FFT
// smoothing's wrap correction subtracts from the edge slabs after the
// transform's own clamp, and may leave rounding-level negatives there (the
// exact sum is non-negative; rho^gamma has no value below zero).  A node is
// stored back only when it was negative.
__device__ __forceinline__ bool clamp4(float4 &v) {
    const bool neg = v.x < 0.0f || v.y < 0.0f || v.z < 0.0f || v.w < 0.0f;
    if (neg) v = make_float4(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f), fmaxf(v.w, 0.0f));
    return neg;
}

template <typename T>
__global__ void k_skyrme_fast(long long G, T A, T B, T C, T gamma, T *rho, T *U) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (sizeof(T) == 4) {
        // four nodes per thread with 16-byte loads and stores (G a multiple
        // of 4): enough bytes in flight per thread for the memory system
        if ((G & 3) == 0) {
            if (4 * i >= G) return;
            float4 p = reinterpret_cast<const float4 *>(rho)[i];
            float4 n = reinterpret_cast<const float4 *>(rho + G)[i];
            if (clamp4(p)) reinterpret_cast<float4 *>(rho)[i] = p;
            if (clamp4(n)) reinterpret_cast<float4 *>(rho + G)[i] = n;
            float4 up, un;
            skyrme_node<T>(A, B, C, gamma, p.x, n.x, up.x, un.x);
            skyrme_node<T>(A, B, C, gamma, p.y, n.y, up.y, un.y);
            skyrme_node<T>(A, B, C, gamma, p.z, n.z, up.z, un.z);
            skyrme_node<T>(A, B, C, gamma, p.w, n.w, up.w, un.w);
            reinterpret_cast<float4 *>(U)[i] = up;
            reinterpret_cast<float4 *>(U + G)[i] = un;
            return;
        }
    }
    if (i >= G) return;
    T p = rho[i], n = rho[i + G];
    if (p < T(0)) rho[i] = p = T(0);
    if (n < T(0)) rho[i + G] = n = T(0);
    skyrme_node<T>(A, B, C, gamma, p, n, U[i], U[i + G]);
}

// threads of k_skyrme_fast: one per node, or one per four in float
template <typename T>
inline long long skyrme_threads(long long G) {
    return (sizeof(T) == 4 && (G & 3) == 0) ? G / 4 : G;
}

// -grad(U + phi_p) with the reference's one-sided faces
// (compute_volumetric_forces_fdm, include/physics.hpp:159-200), the Coulomb
// merge (include/tools.hpp:377-384) folded in, written as (Fx,Fy,Fz,0).
//
// raw (float steps): the raw CIC density of the positions the next gather
// reads.  A gather weights the force at a node by the same CIC weight the
// deposit of that position added to the node, so the only forces read with a
// nonzero weight are those at nodes of nonzero raw density.  A block whose
// rows hold no raw density (most of the grid: 12.8 % of the groups of four
// rows hold density on 208Pb 2.08 M, 128^3) leaves its forces as they were; the
// gather multiplies any such finite value by a zero weight.  The end of a run
// computes every row again for the plain-path view of the fields (raw null).
// occ (128^3 FFT smoothing, rows = 4): the same test, already made by the
// smoothing's forward pass while it read the raw densities, one bit per
// group of four rows.
template <typename T>
__global__ void k_forces_f4(Geom g, T idx, T idy, T idz, const T *__restrict__ U, const double *__restrict__ phi,
                            T *F4, int *advance, const T *__restrict__ raw, int rows,
                            const unsigned *__restrict__ occ) {
    // the step's last kernel also advances the step counter (advance: the
    // control words; null for the initial solve)
    if (advance && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) {
        advance[CTL_STEP] += 1;
        advance[CTL_CLOSE] = 1;
    }
    // block (row group, x plane, species), threads along z: each thread walks
    // `rows` consecutive y rows at its z, keeping the y-1, y and y+1 values
    // of U + phi in registers, so a node loads five values, not seven
    const int ii = blockIdx.y;
    const bool prot = blockIdx.z == 0;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long sx = (long long)ny * nz, sy = nz;
    const T *Us = U + (prot ? 0 : g.G);
    auto u = [&](long long q) { return prot ? Us[q] + (T)phi[q] : Us[q]; };
    const int j0 = blockIdx.x * rows, j1 = min(j0 + rows, ny);
    if (occ) {
        if (!((occ[blockIdx.z * nx + ii] >> blockIdx.x) & 1u)) return;
    } else if (raw) {
        // the block's rows are contiguous: (j1 - j0) nz values of its species
        const T *r = raw + (prot ? 0 : g.G) + (long long)ii * sx + (long long)j0 * sy;
        int any = 0;
        for (int e = threadIdx.x; e < (j1 - j0) * nz; e += blockDim.x) any |= r[e] != T(0);
        if (!__syncthreads_or(any)) return;
    }
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        long long id = (long long)ii * sx + (long long)j0 * sy + k;
        T um = j0 > 0 ? u(id - sy) : T(0);
        T uc = u(id);
        for (int j = j0; j < j1; j++, id += sy) {
            const T up = j + 1 < ny ? u(id + sy) : T(0);
            T gx, gy, gz;
            if (ii == 0) gx = (u(id + sx) - uc) * idx;
            else if (ii == nx - 1) gx = (uc - u(id - sx)) * idx;
            else gx = (u(id + sx) - u(id - sx)) * (T(0.5) * idx);
            if (j == 0) gy = (up - uc) * idy;
            else if (j == ny - 1) gy = (uc - um) * idy;
            else gy = (up - um) * (T(0.5) * idy);
            if (k == 0) gz = (u(id + 1) - uc) * idz;
            else if (k == nz - 1) gz = (uc - u(id - 1)) * idz;
            else gz = (u(id + 1) - u(id - 1)) * (T(0.5) * idz);
            const long long i = (prot ? 0 : g.G) + id;
            if constexpr (sizeof(T) == 4) {
                reinterpret_cast<float4 *>(F4)[i] = make_float4(-gx, -gy, -gz, 0.0f);
            } else {
                T *o = F4 + 4 * i;
                o[0] = -gx;
                o[1] = -gy;
                o[2] = -gz;
                o[3] = T(0);
            }
            um = uc;
            uc = up;
        }
    }
}

// k_forces_f4's launch: one block per (group of `rows` y rows, x plane,
// species), threads along z
inline dim3 forces_grid(const Geom &g, int rows) {
    return dim3((unsigned)((g.ny + rows - 1) / rows), (unsigned)g.nx, 2u);
}
inline dim3 forces_block(const Geom &g) { return dim3((unsigned)std::min(128, (g.nz + 31) / 32 * 32)); }

template <typename T>
__global__ void k_pack_f4(long long n, const T *__restrict__ Fx, const T *__restrict__ Fy, const T *__restrict__ Fz,
                          T *F4) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    F4[4 * i] = Fx[i];
    F4[4 * i + 1] = Fy[i];
    F4[4 * i + 2] = Fz[i];
    F4[4 * i + 3] = T(0);
}

template <typename T>
__global__ void k_unpack_f4(long long n, const T *__restrict__ F4, T *Fx, T *Fy, T *Fz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fx[i] = F4[4 * i];
    Fy[i] = F4[4 * i + 1];
    Fz[i] = F4[4 * i + 2];
}

// POTENTIAL with the Coulomb term merged and phi in T, as the plain path leaves them.
template <typename T>
__global__ void k_merge_out(long long G, const double *__restrict__ phi64, T *U, T *phi) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    const T p = (T)phi64[i];
    U[i] += p;
    phi[i] = p;
}

template <typename T>
__global__ void k_widen(long long n, const T *__restrict__ in, double *out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}

// rows[r] = sums over blocks (fixed order) of the ring row of step s0 + r
__global__ void k_reduce_rows(const double *__restrict__ obs, int blocks, int s0, int nrows, double *rows) {
    const int r = blockIdx.x, c = threadIdx.x;
    if (r >= nrows || c >= 6) return;
    const long long base = (long long)((s0 + r) % kRing) * blocks * 6;
    double u = 0.0;
    for (int b = 0; b < blocks; b++) u += obs[base + (long long)b * 6 + c];
    rows[r * 8 + c] = u;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

template <typename T>
State<T> &st(hv_ctx *c);
template <>
State<double> &st<double>(hv_ctx *c) { return c->d64; }
template <>
State<float> &st<float>(hv_ctx *c) { return c->d32; }

int *ctl_of(hv_ctx *c) { return c->fused.sor_its + kRing; }

// CUDA-event pair around one kernel launch when profiling is on.
struct ProfScope {
    hv_ctx *c;
    int pair = -1;
    ProfScope(hv_ctx *cc, int kid) : c(cc) {
        Profile &p = c->prof;
        if (!p.on) return;
        pair = (int)p.kernel.size();
        while (p.events.size() < 2 * (size_t)pair + 2) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) {
                pair = -1;
                return;
            }
            p.events.push_back(e);
        }
        p.kernel.push_back(kid);
        cudaEventRecord(p.events[2 * pair], c->stream);
    }
    ~ProfScope() {
        if (pair >= 0) cudaEventRecord(c->prof.events[2 * pair + 1], c->stream);
    }
};

// Adds the recorded pairs (the stream must be synchronised) to the totals.
void prof_collect(hv_ctx *c) {
    Profile &p = c->prof;
    for (size_t i = 0; i < p.kernel.size(); i++) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.events[2 * i], p.events[2 * i + 1]) == cudaSuccess) {
            p.ms[p.kernel[i]] += ms;
            p.launches[p.kernel[i]] += 1;
        }
    }
    p.kernel.clear();
    cudaGetLastError();
}

// Enqueues one fused step on the context stream (graph-capturable).
// A step in three parts, so that several contexts can interleave them (the
// batched driver): A = particle step, smoothing, Skyrme; the SOR; C = forces
// and the step counter.
template <typename T>
hv_status enqueue_phase_a(hv_ctx *c) {
    State<T> &s = st<T>(c);
    Fused &f = c->fused;
    const Geom &g = c->geom;
    const hv_run_params &p = c->params;
    int *ctl = ctl_of(c);
    const bool sorted = p.deposit_mode == HV_DEPOSIT_SORTED;
    // the raw density and, after it, the wrap list's count
    if (!sorted) HV_CUDA(cudaMemsetAsync(s.rho_raw, 0, sizeof(T) * (2 * g.G + 4), c->stream));
    int *wcount = nullptr;
    PArgs<T> a;
    a.g = g;
    a.protons = c->protons;
    a.total = c->total;
    a.x = s.x;
    a.y = s.y;
    a.z = s.z;
    a.kx = s.kx;
    a.ky = s.ky;
    a.kz = s.kz;
    a.F4 = reinterpret_cast<const T *>(f.F4);
    a.rho_raw = s.rho_raw;
    a.h = T(p.dt) / (T(2.0) * T(kHbarC));
    a.fd = (T(p.dt) * T(kHbarC)) / T(kMc2);
    const T zz = T(p.z), nn = T(p.n), e = T(p.eta_exc);
    a.dp = e * nn / (zz + nn);
    a.dn = e * zz / (zz + nn);
    a.deposit = sorted ? 0 : 1;
    a.aggregate = c->fast.deposit_aggregate;
    a.wlist = nullptr;
    a.wcount = nullptr;
    a.wcap = kWrapParticles;
    a.wA = f.smooth.A;
    a.wB = f.smooth.B;
    a.wW = f.smooth.W;
    if (sizeof(T) == 4 && !sorted && smooth_fft_runs(c)) {
        wcount = reinterpret_cast<int *>(s.rho_raw + 2 * g.G);
        a.wlist = reinterpret_cast<float4 *>(f.smooth.wlist);
        a.wcount = wcount;
    }
    a.ctl = ctl;
    a.obs = f.obs_partials;
    if (c->total > 0) {
        ProfScope ps(c, HV_K_PARTICLE);
        switch (f.pblock) {
            case 128: k_particle_step<T, 128><<<f.obs_blocks, 128, 0, c->stream>>>(a); break;
            case 512: k_particle_step<T, 512><<<f.obs_blocks, 512, 0, c->stream>>>(a); break;
            default: k_particle_step<T, kPBlock><<<f.obs_blocks, kPBlock, 0, c->stream>>>(a); break;
        }
    } else {
        HV_CUDA(cudaMemsetAsync(f.obs_partials, 0, sizeof(double) * kRing * f.obs_blocks * 6, c->stream));
    }
    HV_CUDA(cudaGetLastError());
    // deterministic mode: every node sums its particles in slot order
    // (distribute_volumetric_particles_cic's single-thread order when the
    // slots are not permuted)
    if (sorted) {
        ProfScope ps(c, HV_K_PARTICLE);
        HV_TRY(launch_deposit_sorted<T>(c, s.x, s.y, s.z, s.rho_raw));
    }
    {
        ProfScope ps(c, HV_K_SMOOTH);
        if (sizeof(T) == 4 && f.smooth.ok)
            HV_TRY(smooth_fast_launch(c, reinterpret_cast<const float *>(s.rho_raw), reinterpret_cast<float *>(s.rho),
                                      wcount));
        else
            HV_TRY(launch_smooth<T>(c, s.rho_raw, s.rho));
    }
    const hv_skyrme &sk = p.skyrme;
    {
        ProfScope ps(c, HV_K_SKYRME);
        k_skyrme_fast<T><<<nblk(skyrme_threads<T>(g.G), 256), 256, 0, c->stream>>>(g.G, T(sk.A), T(sk.B), T(sk.C),
                                                                                   T(sk.gamma), s.rho, s.U);
    }
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status enqueue_phase_c(hv_ctx *c) {
    State<T> &s = st<T>(c);
    Fused &f = c->fused;
    const Geom &g = c->geom;
    int *ctl = ctl_of(c);
    const T idx = T(1.0) / (T(2.0) * T(g.dmx) / g.nx), idy = T(1.0) / (T(2.0) * T(g.dmy) / g.ny),
            idz = T(1.0) / (T(2.0) * T(g.dmz) / g.nz);
    // float steps with the particle step's own atomic deposit: forces only on
    // the rows holding raw density.  The deterministic deposit forms its cells
    // with the reference's division, which can put a particle on a cell face
    // into the neighbouring cell of the gather's (a product by the reciprocal),
    // so its steps compute every row.
    const T *raw = (sizeof(T) == 4 && c->params.deposit_mode != HV_DEPOSIT_SORTED) ? s.rho_raw : nullptr;
    {
        ProfScope ps(c, HV_K_FORCES);
        const int rows = raw ? kForceRowsGated : kForceRows;
        // the 128^3 FFT smoothing's occupancy bits: 32 groups of four rows
        const unsigned *occ = (raw && f.smooth.fft128 && f.smooth.occ && smooth_fft_runs(c) &&
                               g.ny == 32 * kForceRowsGated)
                                  ? f.smooth.occ
                                  : nullptr;
        k_forces_f4<T><<<forces_grid(g, rows), forces_block(g), 0, c->stream>>>(g, idx, idy, idz, s.U, f.phi64,
                                                                        reinterpret_cast<T *>(f.F4), ctl, raw,
                                                                        rows, occ);
    }
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

template <typename T>
hv_status enqueue_step(hv_ctx *c) {
    HV_TRY(enqueue_phase_a<T>(c));
    {
        ProfScope ps(c, HV_K_SOR);
        HV_TRY(sor_fast_launch<T>(c, st<T>(c).rho, ctl_of(c), c->fused.sor_its, kRing, true));
    }
    return enqueue_phase_c<T>(c);
}

// Starting phi of the fused path's first solve inside the grid: the field of
// a uniformly charged sphere of the protons (radius 1.2 A^(1/3) fm, centred
// like the monopole boundary): 1.44 Z / r outside, 1.44 Z (3 R^2 - r^2) /
// (2 R^3) inside.  The boundary nodes keep their values; the solve's stopping
// rule is unchanged, so only its iteration count depends on this guess.
__global__ void k_sphere_guess(Geom g, int Z, double R, double *phi) {
    const int j = blockIdx.x, i = blockIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i == 0 || j == 0 || i == nx - 1 || j == ny - 1) return;
    const double x = g.dmx * (2.0 * i / nx - 1.0), y = g.dmy * (2.0 * j / ny - 1.0);
    for (int k = 1 + threadIdx.x; k < nz - 1; k += blockDim.x) {
        const double z = g.dmz * (2.0 * k / nz - 1.0);
        const double r = sqrt(x * x + y * y + z * z);
        const double v = r >= R ? 1.44 * Z / r : 1.44 * Z * (3.0 * R * R - r * r) / (2.0 * R * R * R);
        phi[((long long)i * ny + j) * nz + k] = v;
    }
}

// The initial field solve of cpu_simulate (src/hyper_vlasov.cpp:53-62) on the
// fused kernels: deposit, smoothing, Coulomb boundary (double monopole,
// include/tools.hpp:283-300), Skyrme, SOR from phi = 0 inside, forces, and the
// gather into f.
template <typename T>
hv_status initial_typed(hv_ctx *c) {
    State<T> &s = st<T>(c);
    Fused &f = c->fused;
    const Geom &g = c->geom;
    const hv_run_params &p = c->params;
    int *ctl = ctl_of(c);
    if (p.deposit_mode == HV_DEPOSIT_SORTED)
        HV_TRY(launch_deposit_sorted<T>(c, s.x, s.y, s.z, s.rho_raw));
    else
        HV_TRY(launch_deposit_atomic<T>(c, s.x, s.y, s.z, s.rho_raw));
    // no wrap list here (the deposit is not the particle step's): density at
    // a face takes the direct form
    if (sizeof(T) == 4 && f.smooth.ok)
        HV_TRY(smooth_fast_launch(c, reinterpret_cast<const float *>(s.rho_raw), reinterpret_cast<float *>(s.rho),
                                  nullptr));
    else
        HV_TRY(launch_smooth<T>(c, s.rho_raw, s.rho));
    const hv_skyrme &sk = p.skyrme;
    k_skyrme_fast<T><<<nblk(skyrme_threads<T>(g.G), 256), 256, 0, c->stream>>>(g.G, T(sk.A), T(sk.B), T(sk.C),
                                                                               T(sk.gamma), s.rho, s.U);
    HV_CUDA(cudaGetLastError());
    // the boundary counts as set only once the solve has succeeded: a solve
    // that gave up leaves phi64 unfinished and the plain phi without the
    // monopole boundary, so the next attempt must start from the boundary again
    bool set_boundary = false;
    if (!c->boundary_set) {
        HV_CUDA(cudaMemsetAsync(f.phi64, 0, sizeof(double) * g.G, c->stream));
        HV_TRY(launch_boundary<double>(c, f.phi64));
        const double R = 1.2 * std::cbrt((double)(c->params.z + c->params.n));
        k_sphere_guess<<<dim3((unsigned)g.ny, (unsigned)g.nx), 128, 0, c->stream>>>(g, c->params.z, R, f.phi64);
        HV_CUDA(cudaGetLastError());
        set_boundary = true;
    } else {
        k_widen<T><<<nblk(g.G, 256), 256, 0, c->stream>>>(g.G, s.phi, f.phi64);
    }
    int h_ctl[3] = {c->step_index, f.m_hint, 0};
    HV_CUDA(cudaMemcpyAsync(ctl, h_ctl, sizeof(int) * 3, cudaMemcpyHostToDevice, c->stream));
    // from phi = 0: neither extrapolated nor recorded as an earlier solution
    HV_TRY(sor_fast_clear_error(c));
    HV_TRY(sor_fast_launch<T>(c, s.rho, ctl, nullptr, kRing, false));
    const T idx = T(1.0) / (T(2.0) * T(g.dmx) / g.nx), idy = T(1.0) / (T(2.0) * T(g.dmy) / g.ny),
            idz = T(1.0) / (T(2.0) * T(g.dmz) / g.nz);
    k_forces_f4<T><<<forces_grid(g, kForceRows), forces_block(g), 0, c->stream>>>(
        g, idx, idy, idz, s.U, f.phi64, reinterpret_cast<T *>(f.F4), nullptr, nullptr, kForceRows, nullptr);
    HV_CUDA(cudaGetLastError());
    int status[3] = {0, 0, 0};
    HV_CUDA(cudaMemcpyAsync(status, f.sor.status, sizeof(int) * 3, cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    if (status[0]) {
        set_last_error("SOR: a bounded device-side wait timed out");
        return HV_ERR_TIMEOUT;
    }
    if (set_boundary) c->boundary_set = true;
    // f of the initial positions; the plain buffers get the same fields
    if (c->total > 0)
        k_close_kick<T><<<nblk(c->total, 256), 256, 0, c->stream>>>(g, c->protons, c->total, s.x, s.y, s.z, s.kx, s.ky,
                                                                    s.kz, s.fx, s.fy, s.fz,
                                                                    reinterpret_cast<const T *>(f.F4), T(0));
    k_unpack_f4<T><<<nblk(2 * g.G, 256), 256, 0, c->stream>>>(2 * g.G, reinterpret_cast<const T *>(f.F4), s.Fx, s.Fy, s.Fz);
    k_merge_out<T><<<nblk(g.G, 256), 256, 0, c->stream>>>(g.G, f.phi64, s.U, s.phi);
    HV_CUDA(cudaGetLastError());
    HV_CUDA(cudaStreamSynchronize(c->stream));
    f.f4_current = true;
    c->fields_valid = true;
    return HV_OK;
}

template <typename T>
hv_status enqueue_steps(hv_ctx *c, int n) {
    for (int i = 0; i < n; i++) HV_TRY(enqueue_step<T>(c));
    return HV_OK;
}

// Before n_steps fused steps: the fused state brought up to date with the plain
// buffers and the control words set; returns the excitation step (or -1).
template <typename T>
hv_status run_begin(hv_ctx *c, int n_steps, int *exc_out) {
    State<T> &s = st<T>(c);
    Fused &f = c->fused;
    const Geom &g = c->geom;
    int *ctl = ctl_of(c);
    // bring the fused state up to date with the plain buffers
    if (!f.f4_current) {
        k_pack_f4<T><<<nblk(2 * g.G, 256), 256, 0, c->stream>>>(2 * g.G, s.Fx, s.Fy, s.Fz, reinterpret_cast<T *>(f.F4));
        k_widen<T><<<nblk(g.G, 256), 256, 0, c->stream>>>(g.G, s.phi, f.phi64);
        HV_CUDA(cudaGetLastError());
        int zero = 0;
        HV_CUDA(cudaMemcpyAsync(ctl + CTL_PREV, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        f.f4_current = true;
    }
    // excitation step: first n with n dt >= t_exc (hyper_vlasov.cpp:86), in T
    int exc = -1;
    if (!c->excited) {
        for (int n = c->step_index; n < c->step_index + n_steps; n++)
            if (T(n) * T(c->params.dt) >= T(c->params.t_exc)) {
                exc = n;
                break;
            }
    }
    int h_ctl[5] = {c->step_index, f.m_hint, 0, exc, 0};
    HV_TRY(sor_fast_clear_error(c));
    HV_CUDA(cudaMemcpyAsync(ctl + CTL_STEP, &h_ctl[0], sizeof(int), cudaMemcpyHostToDevice, c->stream));
    HV_CUDA(cudaMemcpyAsync(ctl + CTL_EXCITE, &h_ctl[3], sizeof(int) * 2, cudaMemcpyHostToDevice, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    *exc_out = exc;
    return HV_OK;
}

// After k steps that started at step s0: their observable rows (obs[0..k)),
// and the SOR status; synchronous.
// The rows of k steps from step s0 into host memory (pinned for an
// asynchronous copy): k x 8 doubles, then the solver's per-step iteration
// ring (kRing ints); stream-ordered, no synchronisation.
hv_status rows_enqueue(hv_ctx *c, int s0, int k, double *rows, int *its) {
    Fused &f = c->fused;
    k_reduce_rows<<<k, 32, 0, c->stream>>>(f.obs_partials, f.obs_blocks, s0, k, f.obs_rows_dev);
    HV_CUDA(cudaGetLastError());
    HV_CUDA(cudaMemcpyAsync(rows, f.obs_rows_dev, sizeof(double) * 8 * k, cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaMemcpyAsync(its, f.sor_its, sizeof(int) * kRing, cudaMemcpyDeviceToHost, c->stream));
    return HV_OK;
}

// Decodes k rows copied by rows_enqueue (the stream synchronised since).
template <typename T>
void rows_decode(hv_ctx *c, int s0, int k, const double *rows, const int *its, hv_observables *obs) {
    const double zz = c->params.z, nn = c->params.n;
    for (int r = 0; r < k; r++) {
        hv_observables &o = obs[r];
        const double *v = &rows[(size_t)r * 8];
        std::memset(&o, 0, sizeof(o));
        o.t = (double)(T(s0 + r) * T(c->params.dt));
        o.zcm_p = v[0] / (double)c->protons;
        o.zcm_n = v[1] / (double)c->neutrons;
        o.rms_p = std::sqrt(v[2] / v[4]);
        o.rms_n = std::sqrt(v[3] / v[5]);
        o.dipole = (nn * zz) / (nn + zz) * (o.zcm_p - o.zcm_n);
        const int it = its[(s0 + r) % kRing];
        o.sor_iterations = it < 0 ? -it : it;
        if (it < 0) o.flags |= HV_OBS_SOR_NOT_CONVERGED;
    }
}

// A timed-out solve (the sticky error word): the steps ran on an unfinished
// potential, and the next run solves the fields of the current positions again.
hv_status rows_status(hv_ctx *c, int status0) {
    if (!status0) return HV_OK;
    c->fields_valid = false;
    fused_invalidate(c);
    set_last_error("SOR: a bounded device-side wait timed out");
    return HV_ERR_TIMEOUT;
}

template <typename T>
hv_status run_rows(hv_ctx *c, int s0, int k, hv_observables *obs) {
    Fused &f = c->fused;
    std::vector<double> rows((size_t)k * 8);
    std::vector<int> its(kRing);
    HV_TRY(rows_enqueue(c, s0, k, rows.data(), its.data()));
    int status[3] = {0, 0, 0};
    HV_CUDA(cudaMemcpyAsync(status, f.sor.status, sizeof(int) * 3, cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    prof_collect(c);
    if (status[0]) {
        // the steps ran on an unfinished potential: the next run solves the
        // fields of the current positions again
        c->fields_valid = false;
        fused_invalidate(c);
        set_last_error("SOR: a bounded device-side wait timed out");
        return HV_ERR_TIMEOUT;
    }
    if (obs) {
        const double zz = c->params.z, nn = c->params.n;
        for (int r = 0; r < k; r++) {
            hv_observables &o = obs[r];
            const double *v = &rows[(size_t)r * 8];
            std::memset(&o, 0, sizeof(o));
            o.t = (double)(T(s0 + r) * T(c->params.dt));
            o.zcm_p = v[0] / (double)c->protons;
            o.zcm_n = v[1] / (double)c->neutrons;
            o.rms_p = std::sqrt(v[2] / v[4]);
            o.rms_n = std::sqrt(v[3] / v[5]);
            o.dipole = (nn * zz) / (nn + zz) * (o.zcm_p - o.zcm_n);
            int it = its[(s0 + r) % kRing];
            o.sor_iterations = it < 0 ? -it : it;
            if (it < 0) o.flags |= HV_OBS_SOR_NOT_CONVERGED;
        }
    }
    return HV_OK;
}

template <typename T>
hv_status run_end(hv_ctx *c, int n_steps, int exc);

template <typename T>
hv_status run_typed(hv_ctx *c, int n_steps, hv_observables *obs) {
    Fused &f = c->fused;
    int exc = -1;
    HV_TRY(run_begin<T>(c, n_steps, &exc));
    const int chunk = c->fast.graph_steps > 0 ? std::min(c->fast.graph_steps, kRing) : std::min(8, kRing);
    int done = 0;
    // the rows go to the context's pinned staging memory chunk by chunk
    // without a synchronisation per chunk (profiled runs synchronise per
    // chunk to read their events)
    const bool async_rows = !c->prof.on;
    const int max_chunks = (n_steps + chunk - 1) / chunk;
    double *host_rows = nullptr;
    int *host_its = nullptr;
    int nchunk = 0;
    std::vector<int> chunk_start;
    if (async_rows) {
        const size_t need = sizeof(double) * 8 * (size_t)n_steps + sizeof(int) * ((size_t)max_chunks * kRing + 4);
        if (c->staging_bytes < need) {
            // room for runs of 4096 steps at least, so that the pinned buffer
            // is not reallocated run after run
            const size_t least = sizeof(double) * 8 * 4096 + sizeof(int) * ((size_t)4096 * kRing + 4);
            if (c->staging) cudaFreeHost(c->staging);
            c->staging = nullptr;
            c->staging_bytes = 0;
            HV_CUDA(cudaMallocHost(&c->staging, std::max(need, least)));
            c->staging_bytes = std::max(need, least);
        }
        host_rows = static_cast<double *>(c->staging);
        host_its = reinterpret_cast<int *>(host_rows + (size_t)8 * n_steps);
    }
    while (done < n_steps) {
        const int k = std::min(chunk, n_steps - done);
        // slot re-sort by cell every sort_every steps (at most once per
        // chunk), outside the graph: its kernels keep their pointers
        const int step_now = c->step_index + done;
        if (c->fast.sort_every > 0 && step_now - f.last_sort >= c->fast.sort_every) {
            HV_TRY(fused_sort_slots(c));
            f.last_sort = step_now;
        }
        bool launched = false;
        if (c->fast.graph_steps > 0 && k == chunk && !c->prof.on) {
            if (!f.graph || f.graph_len != k) {
                if (f.graph) {
                    cudaGraphExecDestroy(f.graph);
                    f.graph = nullptr;
                }
                cudaGraph_t gr = nullptr;
                if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                    hv_status es = enqueue_steps<T>(c, k);
                    cudaError_t ce = cudaStreamEndCapture(c->stream, &gr);
                    if (es == HV_OK && ce == cudaSuccess && gr &&
                        cudaGraphInstantiate(&f.graph, gr, 0) == cudaSuccess) {
                        f.graph_len = k;
                    } else {
                        f.graph = nullptr;
                        c->fast.graph_steps = 0;  // capture not possible here: launch directly
                    }
                    if (gr) cudaGraphDestroy(gr);
                    cudaGetLastError();
                }
            }
            if (f.graph) {
                HV_CUDA(cudaGraphLaunch(f.graph, c->stream));
                launched = true;
            }
        }
        if (!launched) HV_TRY(enqueue_steps<T>(c, k));
        if (async_rows) {
            HV_TRY(rows_enqueue(c, c->step_index + done, k, host_rows + (size_t)done * 8, host_its + (size_t)nchunk * kRing));
            chunk_start.push_back(done);
            nchunk++;
        } else {
            HV_TRY(run_rows<T>(c, c->step_index + done, k, obs ? obs + done : nullptr));
        }
        done += k;
    }
    if (async_rows) {
        // one synchronisation for the whole run: the rows, then the error word
        int *status = host_its + (size_t)nchunk * kRing;
        HV_CUDA(cudaMemcpyAsync(status, f.sor.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        HV_CUDA(cudaStreamSynchronize(c->stream));
        HV_TRY(rows_status(c, *status));
        if (obs)
            for (int q = 0; q < nchunk; q++) {
                const int d0 = chunk_start[q], kk = (q + 1 < nchunk ? chunk_start[q + 1] : n_steps) - d0;
                rows_decode<T>(c, c->step_index + d0, kk, host_rows + (size_t)d0 * 8, host_its + (size_t)q * kRing,
                               obs + d0);
            }
    }
    return run_end<T>(c, n_steps, exc);
}

// After a run of n_steps: step counter, excitation flag, the closing kick/2
// and the plain-path view of the fields.
template <typename T>
hv_status run_end(hv_ctx *c, int n_steps, int exc) {
    Fused &f = c->fused;
    const Geom &g = c->geom;
    int *ctl = ctl_of(c);
    if (exc >= 0) c->excited = true;
    c->step_index += n_steps;
    State<T> &S = st<T>(c);
    if (sizeof(T) == 4 && n_steps > 0) {
        // the float steps computed forces only where the next gather reads
        // them: the plain-path view of the fields gets every row, from the
        // same U and phi (before the merge below adds phi to U)
        const T idx = T(1.0) / (T(2.0) * T(g.dmx) / g.nx), idy = T(1.0) / (T(2.0) * T(g.dmy) / g.ny),
                idz = T(1.0) / (T(2.0) * T(g.dmz) / g.nz);
        k_forces_f4<T><<<forces_grid(g, kForceRows), forces_block(g), 0, c->stream>>>(
            g, idx, idy, idz, S.U, f.phi64, reinterpret_cast<T *>(f.F4), nullptr, nullptr, kForceRows, nullptr);
    }
    if (c->total > 0)
        k_close_kick<T><<<nblk(c->total, 256), 256, 0, c->stream>>>(g, c->protons, c->total, S.x, S.y, S.z, S.kx, S.ky,
                                                                    S.kz, S.fx, S.fy, S.fz,
                                                                    reinterpret_cast<const T *>(f.F4),
                                                                    T(c->params.dt) / (T(2.0) * T(kHbarC)));
    k_unpack_f4<T><<<nblk(2 * g.G, 256), 256, 0, c->stream>>>(2 * g.G, reinterpret_cast<const T *>(f.F4), S.Fx, S.Fy, S.Fz);
    k_merge_out<T><<<nblk(g.G, 256), 256, 0, c->stream>>>(g.G, f.phi64, S.U, S.phi);
    HV_CUDA(cudaGetLastError());
    int mh = 0;
    HV_CUDA(cudaMemcpyAsync(&mh, ctl + CTL_MHINT, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    f.m_hint = mh > 0 ? mh : f.m_hint;
    return HV_OK;
}

}  // namespace

hv_status fused_prepare(hv_ctx *c) {
    Fused &f = c->fused;
    if (f.ready) return HV_OK;
    const Geom &g = c->geom;
    const size_t es = c->prec == HV_F64 ? 8 : 4;
    HV_CUDA(cudaMalloc((void **)&f.phi64, sizeof(double) * g.G));
    HV_CUDA(cudaMalloc((void **)&f.phi64_prev, sizeof(double) * g.G));
    HV_CUDA(cudaMalloc((void **)&f.phi64_prev2, sizeof(double) * g.G));
    HV_CUDA(cudaMemsetAsync(f.phi64, 0, sizeof(double) * g.G, c->stream));
    HV_CUDA(cudaMemsetAsync(f.phi64_prev, 0, sizeof(double) * g.G, c->stream));
    HV_CUDA(cudaMemsetAsync(f.phi64_prev2, 0, sizeof(double) * g.G, c->stream));
    HV_CUDA(cudaMalloc(&f.F4, es * 4 * 2 * g.G));
    f.obs_blocks = 4 * c->sm_count;
    f.pblock = kPBlock;
    // partial rows for the largest grid the autotuner may choose
    HV_CUDA(cudaMalloc((void **)&f.obs_partials, sizeof(double) * kRing * kPGridMax * c->sm_count * 6));
    HV_CUDA(cudaMalloc((void **)&f.obs_rows_dev, sizeof(double) * kRing * 8));
    HV_CUDA(cudaMalloc((void **)&f.sor_its, sizeof(int) * (kRing + CTL_N)));
    HV_CUDA(cudaMemsetAsync(f.sor_its, 0, sizeof(int) * (kRing + CTL_N), c->stream));
    f.obs_rows = kRing;
    HV_TRY(sor_fast_plan(c));
    if (!f.sor.ok) {
        set_last_error("fused path: the SOR correction of this grid does not fit on chip");
        return HV_ERR_UNSUPPORTED;
    }
    if (c->prec == HV_F32) HV_TRY(smooth_fast_plan(c));
    HV_CUDA(cudaStreamSynchronize(c->stream));
    f.ready = true;
    return HV_OK;
}

hv_status fused_release(hv_ctx *c) {
    Fused &f = c->fused;
    if (f.graph) cudaGraphExecDestroy(f.graph);
    void *ptrs[] = {f.phi64, f.phi64_prev, f.phi64_prev2, f.F4, f.obs_partials, f.obs_rows_dev, f.sor_its};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    sor_fast_release(c);
    smooth_fast_release(c);
    f = Fused();
    return HV_OK;
}

hv_status fused_initial_solve(hv_ctx *c) {
    hv_status st = fused_prepare(c);
    if (st != HV_OK) {
        fused_release(c);
        return st;
    }
    return c->prec == HV_F64 ? initial_typed<double>(c) : initial_typed<float>(c);
}

hv_status fused_run(hv_ctx *c, int n_steps, hv_observables *obs) {
    if (!c->fields_valid) HV_TRY(fused_initial_solve(c));
    if (n_steps == 0) return HV_OK;
    hv_status st = fused_prepare(c);
    if (st != HV_OK) {
        fused_release(c);
        return st;
    }
    return c->prec == HV_F64 ? run_typed<double>(c, n_steps, obs) : run_typed<float>(c, n_steps, obs);
}

// ---- autotuner of a single run ---------------------------------------------
namespace {

// Device milliseconds per launch of kernel `kid` over `trial` fused steps
// (direct launches with CUDA events, after one untimed step that loads the
// configuration's kernels).
hv_status time_kernel(hv_ctx *c, int kid, int trial, double *ms) {
    HV_TRY(fused_run(c, 1, nullptr));
    HV_TRY(hv_ctx_set_profiling(c, 1));
    const hv_status st = fused_run(c, trial, nullptr);
    const double total = c->prof.ms[kid];
    const int n = c->prof.launches[kid];
    HV_TRY(hv_ctx_set_profiling(c, 0));
    HV_TRY(st);
    *ms = n > 0 ? total / n : 0.0;
    return HV_OK;
}

void drop_graph(hv_ctx *c) {
    if (c->fused.graph) cudaGraphExecDestroy(c->fused.graph);
    c->fused.graph = nullptr;
    c->fused.graph_len = 0;
}

}  // namespace

// Chooses the particle step's block size and grid, then the SOR tile, by
// timing each candidate's kernel over trial steps (coordinate descent: the
// particle candidates with the planned tile, then the tiles with the chosen
// particle configuration).  The trial steps advance the run.
hv_status fused_autotune(hv_ctx *c, int trial, hv_autotune_report *rep) {
    HV_TRY(fused_run(c, 0, nullptr));  // initial solve and plans, if not done
    HV_TRY(fused_prepare(c));
    Fused &f = c->fused;
    int count = 0;
    double best_ms = 0.0, ms = 0.0;
    const int blocks[3] = {128, 256, 512}, grids[4] = {2, 4, 8, 16};
    int best_b = f.pblock, best_g = f.obs_blocks;
    for (int pb : blocks)
        for (int pg : grids) {
            f.pblock = pb;
            f.obs_blocks = pg * c->sm_count;
            drop_graph(c);
            HV_TRY(time_kernel(c, HV_K_PARTICLE, trial, &ms));
            count++;
            if (count == 1 || ms < best_ms) {
                best_ms = ms;
                best_b = pb;
                best_g = f.obs_blocks;
            }
        }
    f.pblock = best_b;
    f.obs_blocks = best_g;
    const double particle_ms = best_ms;
    // SOR tiles: the plan's first few candidates
    int ntile = 0, best_rank = 0;
    double sor_best = 0.0;
    for (int rank = 0; rank < 4; rank++) {
        if (rank > 0 && rank >= ntile) break;
        HV_TRY(sor_fast_replan_rank(c, rank, &ntile));
        drop_graph(c);
        if (!f.sor.ok) continue;
        HV_TRY(time_kernel(c, HV_K_SOR, trial, &ms));
        count++;
        if (rank == 0 || ms < sor_best) {
            sor_best = ms;
            best_rank = rank;
        }
    }
    HV_TRY(sor_fast_replan_rank(c, best_rank, &ntile));
    drop_graph(c);
    if (!f.sor.ok) {
        set_last_error("autotune: the chosen SOR tile does not fit on chip");
        return HV_ERR_UNSUPPORTED;
    }
    if (rep) {
        rep->particle_block = f.pblock;
        rep->particle_grid = f.obs_blocks;
        rep->sor_planes = f.sor.P;
        rep->sor_rows = f.sor.R;
        rep->sor_blocks = f.sor.nblocks;
        rep->sor_tile_rank = best_rank;
        rep->candidates = count;
        rep->particle_ms = particle_ms;
        rep->sor_ms = sor_best;
    }
    return HV_OK;
}

// ---- batched driver support (batch.cu): float contexts, parts of a step on a
// caller's stream
namespace {
struct StreamSwap {
    hv_ctx *c;
    cudaStream_t saved;
    StreamSwap(hv_ctx *c_, cudaStream_t s) : c(c_), saved(c_->stream) { c->stream = s; }
    ~StreamSwap() { c->stream = saved; }
};
}  // namespace

hv_status fused_batch_ready(hv_ctx *c) {
    if (c->prec != HV_F32) return HV_ERR_UNSUPPORTED;
    if (!c->fields_valid) HV_TRY(fused_initial_solve(c));
    hv_status st = fused_prepare(c);
    if (st != HV_OK) fused_release(c);
    return st;
}
hv_status fused_batch_begin(hv_ctx *c, int n_steps, int *exc) { return run_begin<float>(c, n_steps, exc); }
hv_status fused_batch_phase_a(hv_ctx *c, cudaStream_t s) {
    StreamSwap sw(c, s);
    return enqueue_phase_a<float>(c);
}
hv_status fused_batch_phase_c(hv_ctx *c, cudaStream_t s) {
    StreamSwap sw(c, s);
    return enqueue_phase_c<float>(c);
}
hv_status fused_batch_rows(hv_ctx *c, cudaStream_t s, int s0, int k, hv_observables *obs) {
    StreamSwap sw(c, s);
    return run_rows<float>(c, s0, k, obs);
}
hv_status fused_batch_end(hv_ctx *c, int n_steps, int exc) { return run_end<float>(c, n_steps, exc); }
void fused_batch_sor_inputs(hv_ctx *c, const float **rho, int **ctl, int **its_ring, int *ring) {
    *rho = c->d32.rho;
    *ctl = ctl_of(c);
    *its_ring = c->fused.sor_its;
    *ring = kRing;
}

// ---- adjoint support (adjoint.cu): fused FP64 steps one at a time
hv_status fused_adjoint_begin(hv_ctx *c, int n_steps) {
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    int exc = -1;
    return run_begin<double>(c, n_steps, &exc);
}
hv_status fused_adjoint_step(hv_ctx *c) { return enqueue_step<double>(c); }
int *fused_ctl(hv_ctx *c) { return ctl_of(c); }
int fused_ctl_words() { return CTL_N; }

// Marks the fused copies stale after the plain path or an upload changed the state.
void fused_invalidate(hv_ctx *c) {
    c->fused.f4_current = false;
    c->fused.prev_valid = false;
    // the step counter may have been rewound (an adjoint pass restores
    // checkpoints): the next fused run re-sorts at its first chunk
    c->fused.last_sort = Fused().last_sort;
}

}  // namespace hv
