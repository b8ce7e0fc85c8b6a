// Persistent red-black SOR for the fused path.
//
// Solves lap_h phi = -4 pi 1.44 rho_p with the reference's red-black SOR
// update (include/physics.hpp:99-157) as mixed-precision iterative
// refinement: phi is held in double; every cycle computes the double residual
// r = b + lap_h phi, tests the stopping rule on it, and then runs m red+black
// iterations of the same SOR update on a correction delta (type S) with r as
// source, starting from delta = 0, before folding phi += delta.  In exact
// arithmetic this is the SOR iteration on phi itself; holding delta rather
// than phi in float removes the float rounding floor of the residual (a float
// phi stalls near 1e-4 relative residual on a 64^3 grid).
//
// One cooperative launch per solve.  Block b owns P interior x-planes by R
// rows (all z).  Its delta and, when it fits, its source live in shared
// memory for the whole solve, in a colour-split layout: within a plane all
// red nodes of a row are contiguous, then all black nodes, so a colour sweep
// reads and writes unit-stride runs; the global mirror of delta has the same
// layout ([x][colour][y][z/2]).  A colour sweep is:
//   wait for the (up to four) neighbouring blocks' phase counters,
//   update the own nodes of the colour -- own neighbours from shared memory,
//     the neighbouring blocks' from their global mirror rows -- writing each
//     result to shared memory and to the own mirror row,
//   bump the own phase counter.
// The mirror rows of the Dirichlet planes and rows are never written and
// stay zero, so no neighbour load needs a boundary test.  Grid-wide barriers
// are used only around the double residual.  Every wait is bounded: on
// timeout the block records an error word and returns, and the host reports
// HV_ERR_TIMEOUT.
//
// Tagged exchange (float corrections): instead of phase counters, every
// mirror entry is a 64-bit word holding the float value and the number of
// the half-sweep that wrote it.  A block reads a neighbour's row by polling
// the words themselves until they carry the half-sweep it needs, so a row can
// be consumed as soon as it is written, without a block-wide release and a
// separate flag.  One mirror copy is enough: a block overwrites its entry of
// half-sweep s with that of s + 2 only after reading the neighbour's entry of
// s + 1 at the same position, which the neighbour computed from the entry of
// s.  Tags restart at 1 in every solve (the mirror rows are cleared on entry);
// the first red sweep of each cycle reads no mirror, its neighbours' black
// corrections being zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kSorThreads = 1024;
// relaxation of the sweeps after each coarse-grid correction (default of
// hv_fast_options.sor_coarse_omega).  In a NumPy model of the kernel's cycle
// on successive 208Pb densities (quadratic start, rule 1e-6), 12 sweeps at
// 1.7 ended every solve in two cycles on 48^3, 64^3, 96^3 and 128^3 grids
// (final residual 2.3e-7 to 4.8e-7), where 16 sweeps at 1.8 took two cycles
// at 128^3 (2.9e-7) and three on the other grids; measured on the GPU at
// 128^3, 13 sweeps at 1.8 took three cycles in 999 of 1000 solves.
constexpr double kCoarseOmega = 1.7;
// default bounds of the device-side waits (hv_fast_options.sor_wait_limit
// replaces both): polls of a grid barrier or a neighbour's phase counter before
// the wait gives up (~1 s), and polls of one tagged mirror entry
constexpr long long kDefaultSpin = 1ll << 24;
constexpr long long kDefaultPoll = 1ll << 22;
#ifndef HV_SOR_POLL_NS
#define HV_SOR_POLL_NS 64
#endif
constexpr unsigned kPollSleepNs = HV_SOR_POLL_NS;  // back-off after a poll that missed

using u64 = unsigned long long;

template <typename T, typename S>
struct SorArgs {
    int nx, ny, nz, nz2, P, R, bxn, byn, nblocks, src_smem, vec4;
    int nq_shift;           // log2(nz2 / 4) when a power of two, else -1
    u64 *tmirror;           // tagged mirror [x][colour][y][nz2]: value bits | half-sweep << 32
    S cx, cy, cz, cself;    // omega h^-2 / diag per axis, 1 - omega: the update's coefficients
    double dhx2i, dhy2i, dhz2i, ddiag, src_c;
    double src_scale;       // omega / diag: the residual is stored pre-scaled
    double tol;
    int max_iter, criterion, inner_min, inner_max;
    long long max_spin, max_poll;  // bounds of the waits (kDefaultSpin, kDefaultPoll)
    int extrapolate;        // initial guess: 0 previous phi, else extrapolation of this order (1, 2)
    const T *rho;
    double *phi64, *phi64_prev, *phi64_prev2;
    double *resid;          // FP64 residual of phi per node, carried between checks
    S *delta, *src;         // global mirrors, [x][colour][y][nz2]
    double *partials;       // [nblocks][4]: rr, bb, max|ddelta|, -
    unsigned *phase;        // [nblocks]
    unsigned *bar;          // [0] arrivals, [1] generation
    int *status;            // [0] error, [1] iterations, [2] converged, [3] cycles
    double *metric;
    int *ctl;               // [0] step counter, [1] iterations of the previous solve, [2] phi history held
    int *its_ring;          // per-step iterations, indexed by step % ring
    int ring;
    // coarse-grid correction (staged float form): coarsening factor F, interior
    // extents of the coarse grid (its nodes sit at every F-th fine node, with
    // zero corrections at 0 and n / F), red+black iterations per cycle, and
    // the restriction's buffers t1 [nx][ny][cmz] and t2 [cmx][cmy][cmz]
    int coarse, cf, cmx, cmy, cmz, csweeps;
    float *t1, *t2;
    double hx, hy, hz;      // fine grid spacings
    // several solves in one launch: block -> instance, first block of an
    // instance, and the instances' arguments (null for a single solve)
    const SorArgs *batch;
    const int *binst, *bfirst;
};

__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// Grid barrier for co-resident blocks; false when a wait timed out or another
// block reported an error.
__device__ bool grid_barrier(unsigned *bar, int nblocks, int *err, long long max_spin) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned gen = ld_relaxed(bar + 1);
        fence_acq_rel();
        unsigned arrived = atomicAdd(bar, 1u) + 1u;
        if (arrived == (unsigned)nblocks) {
            atomicExch(bar, 0u);
            st_release(bar + 1, gen + 1u);
        } else {
            long long spin = 0;
            while (ld_relaxed(bar + 1) == gen) {
                if (++spin > max_spin || ld_volatile(err)) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
            }
        }
        fence_acq_rel();
    }
    __syncthreads();
    return ok;
}

// Waits until every neighbouring block has published `target` phases: lane q
// of warp 0 polls neighbour q with relaxed loads, then one acquire fence; the
// block barrier extends the ordering to every thread.
template <typename T, typename S>
__device__ bool wait_neighbours(const SorArgs<T, S> &a, int bx, int by, unsigned target) {
    __shared__ int ok;
    if (threadIdx.x < 32) {
        const int q = threadIdx.x;
        int nb = -1;
        if (q == 0 && bx > 0) nb = by * a.bxn + bx - 1;
        if (q == 1 && bx + 1 < a.bxn) nb = by * a.bxn + bx + 1;
        if (q == 2 && by > 0) nb = (by - 1) * a.bxn + bx;
        if (q == 3 && by + 1 < a.byn) nb = (by + 1) * a.bxn + bx;
        int good = 1;
        if (nb >= 0) {
            long long spin = 0;
            while (ld_relaxed(a.phase + nb) < target) {
                if (++spin > a.max_spin || ld_volatile(a.status)) {
                    atomicExch(a.status, 1);
                    good = 0;
                    break;
                }
            }
        }
        good = __all_sync(0xffffffffu, good);
        if (q == 0) {
            fence_acq_rel();
            ok = good;
        }
    }
    __syncthreads();
    return ok;
}

// Publishes `value` after every thread's prior stores: the block barrier
// orders them before thread 0's release store at gpu scope.
__device__ __forceinline__ void publish(unsigned *phase_slot, unsigned value) {
    __syncthreads();
    if (threadIdx.x == 0) st_release(phase_slot, value);
}

// Deterministic block sum of two doubles (fixed shuffle tree, fixed warp order);
// the result is valid in thread 0.
__device__ void block_sum2(double &u, double &v) {
    __shared__ double su[kSorThreads / 32], sv[kSorThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        u += __shfl_xor_sync(0xffffffffu, u, o);
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        su[w] = u;
        sv[w] = v;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        u = l < nw ? su[l] : 0.0;
        v = l < nw ? sv[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            u += __shfl_xor_sync(0xffffffffu, u, o);
            v += __shfl_xor_sync(0xffffffffu, v, o);
        }
    }
}

template <typename S>
__device__ S block_max(S m) {
    __shared__ S sm[kSorThreads / 32];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm[w] = m;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        m = l < nw ? sm[l] : S(0);
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    return m;
}

// One SOR update of a node: the reference's phi* and relaxation
// (include/physics.hpp:114-125) applied to the correction,
//   self + omega ((xs hx^-2 + ys hy^-2 + zs hz^-2 + r) / diag - self),
// regrouped as four fused multiply-adds with the source s = omega r / diag
// stored pre-scaled by the residual pass.
template <typename S, typename T>
__device__ __forceinline__ S sor_update(const SorArgs<T, S> &a, S self, S xs, S ys, S zs, S s, bool valid) {
    const S v = fma(a.cx, xs, fma(a.cy, ys, fma(a.cz, zs, fma(a.cself, self, s))));
    return valid ? v : self;
}

// Geometry of one block, shared by the sweeps.
struct Block {
    int x0, y0, np, nr, nz2, hp, ny;
    __device__ long long mirror(int x, int c, int y) const { return (((long long)x * 2 + c) * ny + y) * nz2; }
};

// Neighbour row pointers of own row (p, j), other colour cp.
template <typename S>
__device__ __forceinline__ void neighbour_rows(const Block &B, S *sd, const S *mirror, int p, int j, int cp,
                                               const S *&xm, const S *&xp, const S *&ym, const S *&yp) {
    const S *orow = sd + ((p * 2 + cp) * B.nr + j) * B.nz2;
    const int x = B.x0 + p, y = B.y0 + j;
    xm = p > 0 ? orow - 2 * B.hp : mirror + B.mirror(x - 1, cp, y);
    xp = p + 1 < B.np ? orow + 2 * B.hp : mirror + B.mirror(x + 1, cp, y);
    ym = j > 0 ? orow - B.nz2 : mirror + B.mirror(x, cp, y - 1);
    yp = j + 1 < B.nr ? orow + B.nz2 : mirror + B.mirror(x, cp, y + 1);
}

template <typename S>
__device__ __forceinline__ float4 load4(const S *p, int q, bool global) {
    const float4 *v = reinterpret_cast<const float4 *>(p) + q;
    return global ? __ldcg(v) : *v;
}

// Colour sweep, four consecutive same-colour nodes per thread (float
// correction, nz/2 a multiple of 4, source in shared memory).  Lane i of quad
// q is the node k = kc + 2 (4 q + i); its z neighbours are the other colour's
// entries 4 q + i + kc - 1 and 4 q + i + kc of the same row.
template <typename S, typename T>
__device__ __forceinline__ void sweep_quads(const SorArgs<T, S> &a, const Block &B, int c, S *sd, const S *ss,
                                            int q_own, int r_start, int rows_step, int j_start, int p_start, int dj,
                                            int dp, bool track, S &last_max) {
    const int nz2 = a.nz2, nq = nz2 / 4, ny = a.ny, nz = a.nz, cp = c ^ 1;
    if (q_own >= nq) return;
    int j = j_start, p = p_start;
    for (int l = r_start; l < B.np * B.nr; l += rows_step) {
        const int x = B.x0 + p, y = B.y0 + j;
        if (y >= 1 && y <= ny - 2) {
            const int kc = (c - x - y) & 1;
            const int roff = ((p * 2 + c) * B.nr + j) * nz2;
            S *row = sd + roff;
            const S *orow = sd + ((p * 2 + cp) * B.nr + j) * nz2;
            const S *xmr, *xpr, *ymr, *ypr;
            neighbour_rows(B, sd, a.delta, p, j, cp, xmr, xpr, ymr, ypr);
            const float4 xm = load4(xmr, q_own, p == 0), xp = load4(xpr, q_own, p + 1 == B.np);
            const float4 ym = load4(ymr, q_own, j == 0), yp = load4(ypr, q_own, j + 1 == B.nr);
            const float4 self = reinterpret_cast<const float4 *>(row)[q_own];
            const float4 o = reinterpret_cast<const float4 *>(orow)[q_own];
            const float4 s = reinterpret_cast<const float4 *>(ss + roff)[q_own];
            float z0, z1, z2, z3;  // zm + zp per lane
            if (kc == 0) {
                const float left = q_own > 0 ? orow[4 * q_own - 1] : 0.0f;
                z0 = left + o.x;
                z1 = o.x + o.y;
                z2 = o.y + o.z;
                z3 = o.z + o.w;
            } else {
                const float right = q_own + 1 < nq ? orow[4 * q_own + 4] : 0.0f;
                z0 = o.x + o.y;
                z1 = o.y + o.z;
                z2 = o.z + o.w;
                z3 = o.w + right;
            }
            const int kb = kc + 8 * q_own;  // k of lane 0; lanes step by 2
            float4 nv;
            nv.x = sor_update<S, T>(a, self.x, xm.x + xp.x, ym.x + yp.x, z0, s.x, kb >= 1 && kb <= nz - 2);
            nv.y = sor_update<S, T>(a, self.y, xm.y + xp.y, ym.y + yp.y, z1, s.y, kb + 2 <= nz - 2);
            nv.z = sor_update<S, T>(a, self.z, xm.z + xp.z, ym.z + yp.z, z2, s.z, kb + 4 <= nz - 2);
            nv.w = sor_update<S, T>(a, self.w, xm.w + xp.w, ym.w + yp.w, z3, s.w, kb + 6 <= nz - 2);
            reinterpret_cast<float4 *>(row)[q_own] = nv;
            __stcg(reinterpret_cast<float4 *>(a.delta + B.mirror(x, c, y)) + q_own, nv);
            if (track)
                last_max = fmax(last_max, fmax(fmax(fabs(nv.x - self.x), fabs(nv.y - self.y)),
                                               fmax(fabs(nv.z - self.z), fabs(nv.w - self.w))));
        }
        j += dj;
        p += dp;
        if (j >= B.nr) {
            j -= B.nr;
            p++;
        }
    }
}

// double corrections never take the quad path
template <>
__device__ __forceinline__ void sweep_quads<double, double>(const SorArgs<double, double> &, const Block &, int,
                                                            double *, const double *, int, int, int, int, int, int,
                                                            int, bool, double &) {}

__device__ __forceinline__ u64 tag_word(float v, unsigned tag) {
    return (u64)__float_as_uint(v) | ((u64)tag << 32);
}

// Four consecutive tagged entries (one quad), written with two 16-byte
// relaxed stores; each 64-bit word is single-copy atomic.
__device__ __forceinline__ void st_tagged4(u64 *p, float4 v, unsigned tag) {
    asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(p), "l"(tag_word(v.x, tag)),
                 "l"(tag_word(v.y, tag))
                 : "memory");
    asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(p + 2), "l"(tag_word(v.z, tag)),
                 "l"(tag_word(v.w, tag))
                 : "memory");
}

// Two ghost quads of one work item (the two neighbours along one axis),
// polled together: both sources are loaded, then all tags are checked, and
// only a miss repeats the loads, so a row whose ghosts are already written
// costs one L2 round trip.  A null source is not read (its value is zero).
// Bounded: after max_poll polls, or when another block has reported an error,
// it records the error, sets `failed` and returns what it read; a thread that
// has failed once reads each further source once without waiting.
__device__ __forceinline__ void poll_pair(const u64 *g0, const u64 *g1, unsigned tag, int *status,
                                          long long max_poll, bool &failed, float4 &v0, float4 &v1) {
    u64 w[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    const u64 *g[2] = {g0, g1};
    long long n = 0;
    while (true) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (!g[i]) continue;
            asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];"
                         : "=l"(w[i][0]), "=l"(w[i][1])
                         : "l"(g[i])
                         : "memory");
            asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];"
                         : "=l"(w[i][2]), "=l"(w[i][3])
                         : "l"(g[i] + 2)
                         : "memory");
        }
        bool ok = true;
#pragma unroll
        for (int i = 0; i < 2; i++)
            if (g[i])
                ok = ok && (unsigned)(w[i][0] >> 32) == tag && (unsigned)(w[i][1] >> 32) == tag &&
                     (unsigned)(w[i][2] >> 32) == tag && (unsigned)(w[i][3] >> 32) == tag;
        if (ok || failed) break;
        if ((++n & 63) == 0 && (n > max_poll || ld_volatile(status))) {
            failed = true;
            atomicExch(status, 1);
            break;
        }
        // a waiting warp yields its issue slots to the warps that compute
        if (kPollSleepNs) __nanosleep(kPollSleepNs);
    }
    v0 = make_float4(__uint_as_float((unsigned)w[0][0]), __uint_as_float((unsigned)w[0][1]),
                     __uint_as_float((unsigned)w[0][2]), __uint_as_float((unsigned)w[0][3]));
    v1 = make_float4(__uint_as_float((unsigned)w[1][0]), __uint_as_float((unsigned)w[1][1]),
                     __uint_as_float((unsigned)w[1][2]), __uint_as_float((unsigned)w[1][3]));
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// Colour sweep with the tagged exchange (float corrections, nz/2 a multiple
// of 4, source in shared memory).  Work item w is quad w % nq (four
// consecutive same-colour nodes) of row order[w / nq] (p << 16 | j); the order lists the
// block's face rows -- those that read or feed another block -- before its
// inner rows, so the rows the neighbours wait for are written first and the
// ghosts this block needs have the inner rows' time to arrive.  Rows of other
// blocks are polled for half-sweep `tag_in` (0: they are zero, the first red
// sweep of a cycle); Dirichlet planes and rows are zero.  Face rows are
// written to the mirror with `tag_out`.
template <typename T>
__device__ __forceinline__ void sweep_quads_tagged(const SorArgs<T, float> &a, const Block &B, int c, float *sd,
                                                   const float *ss, const unsigned *order, bool track,
                                                   float &last_max, unsigned tag_out, unsigned tag_in, bool &failed) {
    const int nz2 = a.nz2, nq = nz2 / 4, nx = a.nx, ny = a.ny, nz = a.nz, cp = c ^ 1;
    const int items = B.np * B.nr * nq;
    const long long cstride = (long long)ny * nz2;  // one colour of one plane in the mirror
    for (int w = threadIdx.x; w < items; w += blockDim.x) {
        const int r = a.nq_shift >= 0 ? w >> a.nq_shift : w / nq, q = w - r * nq;
        const unsigned e = order[r];
        const int p = (int)(e >> 16), j = (int)(e & 0xffffu);
        const int x = B.x0 + p, y = B.y0 + j;
        if (y < 1 || y > ny - 2) continue;
        const int kc = (c - x - y) & 1;
        const int roff = ((p * 2 + c) * B.nr + j) * nz2;
        float *row = sd + roff;
        const float *orow = sd + ((p * 2 + cp) * B.nr + j) * nz2;
        // ghost sources: xm, xp, ym, yp rows of other blocks (null: own or zero)
        const bool gx0 = p == 0 && x - 1 >= 1, gx1 = p + 1 == B.np && x + 1 <= nx - 2;
        const bool gy0 = j == 0 && y - 1 >= 1, gy1 = j + 1 == B.nr && y + 1 <= ny - 2;
        // mirror entry of quad q in row (x, y), other colour
        const u64 *gq = a.tmirror + ((2ll * x + cp) * cstride + (long long)y * nz2 + 4 * q);
        float4 m4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), p4 = m4;
        if (tag_in && (gx0 || gx1))
            poll_pair(gx0 ? gq - 2 * cstride : nullptr, gx1 ? gq + 2 * cstride : nullptr, tag_in, a.status,
                      a.max_poll, failed, m4, p4);
        if (p > 0) m4 = reinterpret_cast<const float4 *>(orow - 2 * B.hp)[q];
        if (p + 1 < B.np) p4 = reinterpret_cast<const float4 *>(orow + 2 * B.hp)[q];
        const float4 xs = add4(m4, p4);
        m4 = p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (tag_in && (gy0 || gy1))
            poll_pair(gy0 ? gq - nz2 : nullptr, gy1 ? gq + nz2 : nullptr, tag_in, a.status, a.max_poll, failed, m4,
                      p4);
        if (j > 0) m4 = reinterpret_cast<const float4 *>(orow - nz2)[q];
        if (j + 1 < B.nr) p4 = reinterpret_cast<const float4 *>(orow + nz2)[q];
        const float4 ys = add4(m4, p4);
        const float4 self = reinterpret_cast<const float4 *>(row)[q];
        const float4 o = reinterpret_cast<const float4 *>(orow)[q];
        const float4 s = reinterpret_cast<const float4 *>(ss + roff)[q];
        float z0, z1, z2, z3;  // zm + zp per lane
        if (kc == 0) {
            const float left = q > 0 ? orow[4 * q - 1] : 0.0f;
            z0 = left + o.x;
            z1 = o.x + o.y;
            z2 = o.y + o.z;
            z3 = o.z + o.w;
        } else {
            const float right = q + 1 < nq ? orow[4 * q + 4] : 0.0f;
            z0 = o.x + o.y;
            z1 = o.y + o.z;
            z2 = o.z + o.w;
            z3 = o.w + right;
        }
        const int kb = kc + 8 * q;
        float4 nv;
        nv.x = sor_update<float, T>(a, self.x, xs.x, ys.x, z0, s.x, kb >= 1 && kb <= nz - 2);
        nv.y = sor_update<float, T>(a, self.y, xs.y, ys.y, z1, s.y, kb + 2 <= nz - 2);
        nv.z = sor_update<float, T>(a, self.z, xs.z, ys.z, z2, s.z, kb + 4 <= nz - 2);
        nv.w = sor_update<float, T>(a, self.w, xs.w, ys.w, z3, s.w, kb + 6 <= nz - 2);
        reinterpret_cast<float4 *>(row)[q] = nv;
        if (gx0 || gx1 || gy0 || gy1) st_tagged4(const_cast<u64 *>(gq) + (c - cp) * cstride, nv, tag_out);
        if (track)
            last_max = fmax(last_max, fmax(fmax(fabs(nv.x - self.x), fabs(nv.y - self.y)),
                                           fmax(fabs(nv.z - self.z), fabs(nv.w - self.w))));
    }
}

__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

// ---- staged tagged sweep -------------------------------------------------
// A sweep first updates the block's perimeter rows, from shared memory and a
// shared-memory buffer of ghost rows (the neighbouring blocks' rows across the
// block's faces), writing those that a neighbouring block reads to the
// mirror.  After a block barrier, threads [0, kGhostThreads) poll the
// neighbours' perimeter rows just written for this sweep into the ghost
// buffer, for the next sweep, while the other threads update the inner rows
// (off the block's perimeter), which read only this block's shared memory.
// The fetch's L2 round trip is thus spent under the inner rows' updates.
constexpr int kGhostThreads = 256;
// rows of the residual check whose loads one thread issues together
constexpr int kCheckRows = 2;

// Shared-memory tables behind delta | src, sized by the plan's P x R block.
struct Staged {
    unsigned *order;  // [P R] rows, face rows first (generic tagged sweep)
    unsigned *ftab;   // [P R] perimeter rows: p << 16 | j
    unsigned *fgi;    // [P R][2] ghost-buffer rows: xm | xp << 16, ym | yp << 16 (0xffff: none)
    unsigned *gsrc;   // [2 (P + R)] mirror index of each ghost row (colour 0)
    float *gbuf;      // [2 (P + R)][nz2] ghost values of the current sweep
    __host__ __device__ static size_t bytes(int P, int R, int nz2) {
        const size_t pr = (size_t)P * R, g = 2 * ((size_t)P + R);
        return 16 * ((pr * 4 + 15) / 16 + (pr * 4 + 15) / 16 + (pr * 8 + 15) / 16 + (g * 4 + 15) / 16) +
               g * nz2 * 4;
    }
    __device__ Staged(void *base, int P, int R) {
        const size_t pr = (size_t)P * R, g = 2 * ((size_t)P + R);
        unsigned char *p = reinterpret_cast<unsigned char *>(base);
        order = reinterpret_cast<unsigned *>(p);
        p += 16 * ((pr * 4 + 15) / 16);
        ftab = reinterpret_cast<unsigned *>(p);
        p += 16 * ((pr * 4 + 15) / 16);
        fgi = reinterpret_cast<unsigned *>(p);
        p += 16 * ((pr * 8 + 15) / 16);
        gsrc = reinterpret_cast<unsigned *>(p);
        p += 16 * ((g * 4 + 15) / 16);
        gbuf = reinterpret_cast<float *>(p);
    }
};

enum : unsigned {
    kQActive = 1u,     // an interior row of the grid
    kQOwnXm = 2u,      // neighbour rows in this block's shared memory
    kQOwnXp = 4u,
    kQOwnYm = 8u,
    kQOwnYp = 16u,
    kQGhXm = 32u,      // neighbour rows of another block (ghost buffer)
    kQGhXp = 64u,
    kQGhYm = 128u,
    kQGhYp = 256u,
    kQKc0 = 512u,      // parity of the row's first colour-0 node
    kQFirst = 1024u,   // first / last quad of the row
    kQLast = 2048u,
};
constexpr int kQLanes = 12;  // bits 12..15: lanes inside the z range for kc = 0; 16..19 for kc = 1
constexpr int kQShift = 24;  // bits 24..31: the quad index q
constexpr unsigned kQGhAny = kQGhXm | kQGhXp | kQGhYm | kQGhYp;

struct Quad {        // a quad of an inner row
    int roff;        // shared-memory offset of the quad in colour 0 of its row
    unsigned flags;
};
struct FaceQuad {    // a quad of a perimeter row
    int roff;
    unsigned flags;
    unsigned gq;     // mirror index of the quad in colour 0 of its row
    unsigned gx, gy; // ghost-buffer rows xm | xp << 16, ym | yp << 16
};
struct GhostQuad {   // a quad of a ghost row
    unsigned src;    // mirror index (colour 0)
    int dst;         // ghost-buffer offset; < 0: none
};

// Flags shared by inner and perimeter quads: parity, z-range lanes, row ends.
__device__ __forceinline__ unsigned quad_flags(int x, int y, int q, int nq, int nz) {
    unsigned f = kQActive | (unsigned)q << kQShift;
    if ((-x - y) & 1) f |= kQKc0;
    if (q == 0) f |= kQFirst;
    if (q + 1 == nq) f |= kQLast;
    for (int kc = 0; kc < 2; kc++)
        for (int i = 0; i < 4; i++) {
            const int k = kc + 8 * q + 2 * i;
            if (k >= 1 && k <= nz - 2) f |= 1u << (kQLanes + 4 * kc + i);
        }
    return f;
}

// The SOR update of a quad from its neighbour sums (lanes outside the z range
// keep their value), written to shared memory; returns the new quad.
template <typename T>
__device__ __forceinline__ float4 update_quad(const SorArgs<T, float> &a, unsigned f, int c, float *rowq,
                                              const float *orq, const float *srq, float4 xs, float4 ys, bool track,
                                              float &last_max) {
    const int kc = ((f & kQKc0) ? 1 : 0) ^ c;
    const float4 self = lds4(rowq), o = lds4(orq), s = lds4(srq);
    float z0, z1, z2, z3;  // zm + zp per lane
    if (kc == 0) {
        const float left = (f & kQFirst) ? 0.0f : orq[-1];
        z0 = left + o.x;
        z1 = o.x + o.y;
        z2 = o.y + o.z;
        z3 = o.z + o.w;
    } else {
        const float right = (f & kQLast) ? 0.0f : orq[4];
        z0 = o.x + o.y;
        z1 = o.y + o.z;
        z2 = o.z + o.w;
        z3 = o.w + right;
    }
    const unsigned lanes = f >> (kQLanes + 4 * kc);
    float4 nv;
    nv.x = sor_update<float, T>(a, self.x, xs.x, ys.x, z0, s.x, lanes & 1u);
    nv.y = sor_update<float, T>(a, self.y, xs.y, ys.y, z1, s.y, lanes & 2u);
    nv.z = sor_update<float, T>(a, self.z, xs.z, ys.z, z2, s.z, lanes & 4u);
    nv.w = sor_update<float, T>(a, self.w, xs.w, ys.w, z3, s.w, lanes & 8u);
    *reinterpret_cast<float4 *>(rowq) = nv;
    if (track)
        last_max = fmax(last_max, fmax(fmax(fabs(nv.x - self.x), fabs(nv.y - self.y)),
                                       fmax(fabs(nv.z - self.z), fabs(nv.w - self.w))));
    return nv;
}

template <typename T>
__device__ __forceinline__ void sweep_inner(const SorArgs<T, float> &a, const Quad &it, int c, int hp, float *sd,
                                            const float *ss, bool track, float &last_max) {
    if (!(it.flags & kQActive)) return;
    const int nz2 = a.nz2;
    float *rowq = sd + it.roff + c * hp;
    const float *orq = sd + it.roff + (c ^ 1) * hp;
    const float4 xs = add4(lds4(orq - 2 * hp), lds4(orq + 2 * hp));
    const float4 ys = add4(lds4(orq - nz2), lds4(orq + nz2));
    update_quad<T>(a, it.flags, c, rowq, orq, ss + it.roff + c * hp, xs, ys, track, last_max);
}

template <typename T>
__device__ __forceinline__ void sweep_face(const SorArgs<T, float> &a, const FaceQuad &it, int c, int hp,
                                           long long cstride, float *sd, const float *ss, const float *gbuf,
                                           unsigned tag_out, bool track, float &last_max) {
    const unsigned f = it.flags;
    if (!(f & kQActive)) return;
    const int nz2 = a.nz2, q4 = 4 * (int)(f >> kQShift);
    float *rowq = sd + it.roff + c * hp;
    const float *orq = sd + it.roff + (c ^ 1) * hp;
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 xm = (f & kQOwnXm) ? lds4(orq - 2 * hp) : (f & kQGhXm) ? lds4(gbuf + (it.gx & 0xffffu) * nz2 + q4) : zero4;
    const float4 xp = (f & kQOwnXp) ? lds4(orq + 2 * hp) : (f & kQGhXp) ? lds4(gbuf + (it.gx >> 16) * nz2 + q4) : zero4;
    const float4 ym = (f & kQOwnYm) ? lds4(orq - nz2) : (f & kQGhYm) ? lds4(gbuf + (it.gy & 0xffffu) * nz2 + q4) : zero4;
    const float4 yp = (f & kQOwnYp) ? lds4(orq + nz2) : (f & kQGhYp) ? lds4(gbuf + (it.gy >> 16) * nz2 + q4) : zero4;
    const float4 nv =
        update_quad<T>(a, f, c, rowq, orq, ss + it.roff + c * hp, add4(xm, xp), add4(ym, yp), track, last_max);
    if (f & kQGhAny) st_tagged4(a.tmirror + it.gq + c * cstride, nv, tag_out);
}

// Polls the thread's ghost quads (colour offset coff) until all carry `tag`
// and copies them to the ghost buffer; tag 0 stores zeros (the first red
// sweep of a cycle).  All loads are issued before any tag is checked, and only
// a miss repeats them.  Bounded like poll_pair.
template <int kG>
__device__ __forceinline__ void fetch_ghosts(const u64 *tm, const GhostQuad (&g)[kG], long long coff, unsigned tag,
                                             float *gbuf, int *status, long long max_poll, bool &failed) {
    u64 w[kG][4];
#pragma unroll
    for (int i = 0; i < kG; i++) w[i][0] = w[i][1] = w[i][2] = w[i][3] = 0;
    if (tag) {
        long long n = 0;
        while (true) {
#pragma unroll
            for (int i = 0; i < kG; i++) {
                if (g[i].dst < 0) continue;
                const u64 *p = tm + g[i].src + coff;
                asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];"
                             : "=l"(w[i][0]), "=l"(w[i][1])
                             : "l"(p)
                             : "memory");
                asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];"
                             : "=l"(w[i][2]), "=l"(w[i][3])
                             : "l"(p + 2)
                             : "memory");
            }
            bool ok = true;
#pragma unroll
            for (int i = 0; i < kG; i++)
                if (g[i].dst >= 0)
                    ok = ok && (unsigned)(w[i][0] >> 32) == tag && (unsigned)(w[i][1] >> 32) == tag &&
                         (unsigned)(w[i][2] >> 32) == tag && (unsigned)(w[i][3] >> 32) == tag;
            if (ok || failed) break;
            if ((++n & 63) == 0 && (n > max_poll || ld_volatile(status))) {
                failed = true;
                atomicExch(status, 1);
                break;
            }
            if (kPollSleepNs) __nanosleep(kPollSleepNs);
        }
    }
#pragma unroll
    for (int i = 0; i < kG; i++)
        if (g[i].dst >= 0)
            *reinterpret_cast<float4 *>(gbuf + g[i].dst) =
                make_float4(__uint_as_float((unsigned)w[i][0]), __uint_as_float((unsigned)w[i][1]),
                            __uint_as_float((unsigned)w[i][2]), __uint_as_float((unsigned)w[i][3]));
}

// Correction of a neighbouring block's node from its mirror entry (either
// layout); called after a grid barrier, when every entry is final.
template <bool kTag, typename T, typename S>
__device__ __forceinline__ double mirror_value(const SorArgs<T, S> &a, long long idx) {
    if constexpr (kTag) return (double)__uint_as_float((unsigned)__ldcg(a.tmirror + idx));
    else return (double)__ldcg(a.delta + idx);
}

// Colour sweep, one node per thread per row (any size and type).
template <typename S, typename T>
__device__ __forceinline__ void sweep_scalar(const SorArgs<T, S> &a, const Block &B, int c, S *sd, const S *ss,
                                             int t_own, int r_start, int rows_step, int j_start, int p_start, int dj,
                                             int dp, bool track, S &last_max) {
    const int nz2 = a.nz2, ny = a.ny, nz = a.nz, cp = c ^ 1;
    if (t_own >= nz2) return;
    int j = j_start, p = p_start;
    for (int l = r_start; l < B.np * B.nr; l += rows_step) {
        const int x = B.x0 + p, y = B.y0 + j;
        const int kc = (c - x - y) & 1, k = kc + 2 * t_own;
        if (y >= 1 && y <= ny - 2 && k >= 1 && k <= nz - 2) {
            const int roff = ((p * 2 + c) * B.nr + j) * nz2;
            S *row = sd + roff;
            const S *orow = sd + ((p * 2 + cp) * B.nr + j) * nz2;
            const S *xmr, *xpr, *ymr, *ypr;
            neighbour_rows(B, sd, a.delta, p, j, cp, xmr, xpr, ymr, ypr);
            const S xm = p == 0 ? __ldcg(xmr + t_own) : xmr[t_own];
            const S xp = p + 1 == B.np ? __ldcg(xpr + t_own) : xpr[t_own];
            const S ym = j == 0 ? __ldcg(ymr + t_own) : ymr[t_own];
            const S yp = j + 1 == B.nr ? __ldcg(ypr + t_own) : ypr[t_own];
            const S s = ss ? ss[roff + t_own] : __ldcg(a.src + B.mirror(x, c, y) + t_own);
            const S self = row[t_own];
            const S zs = orow[t_own + kc - 1] + orow[t_own + kc];
            const S nv = sor_update<S, T>(a, self, xm + xp, ym + yp, zs, s, true);
            row[t_own] = nv;
            __stcg(a.delta + B.mirror(x, c, y) + t_own, nv);
            if (track) last_max = fmax(last_max, fabs(nv - self));
        }
        j += dj;
        p += dp;
        if (j >= B.nr) {
            j -= B.nr;
            p++;
        }
    }
}

// ---- coarse-grid correction --------------------------------------------
// Each cycle of the staged float solve starts its correction from the
// solution of the correction equation on a coarse grid, instead of from zero.
// The red-black sweeps damp the rough part of the error within a few
// iterations, but its smooth part decays by less than 1 % per iteration on a
// 128^3 grid; the coarse grid removes that part in one step.  The coarse grid
// has every F-th fine node per axis (F a power of two, chosen so that its
// interior has at most 15 nodes per axis); the fine grid's n nodes per axis
// are treated as n intervals whose last node (n) carries a zero correction
// like the Dirichlet node n - 1, so every level spans the same box.  Transfers
// are the standard pair: restriction by full weighting composed over the log2
// F levels -- per axis the triangle (F - |d|) / F^2, |d| < F -- and trilinear
// prolongation.  The coarse equation lap_H e = -R r (7-point, spacing F h per
// axis, zero boundary) is solved exactly by a discrete sine transform per axis
// (S_jk = sin(pi (j+1)(k+1) / (m+1)), S S = (m+1)/2 I), redundantly in every
// block's shared memory, so that no block waits for another to solve it.
// Restriction is separable: stage 1 filters each block's own z rows (its
// residual source is in shared memory); after a grid barrier, all blocks
// share the y and x filters of the interior coarse nodes; after another,
// every block reads the restricted residual.
constexpr int kCoarseMax = 15;

struct Coarse {
    float *ec, *tmp;       // [mx][my][mz]: the coarse field and a transform buffer
    float *sx, *sy, *sz;   // sine matrices [m][m]
    float *lam;            // [mx + my + mz] eigenvalues of the 1-D coarse operators
    float *prof;           // [rows][mz + 2] z-profiles of own and ghost rows
    float *den;            // [mx][my][mz]: -8 / ((mx+1)(my+1)(mz+1) (lam_x + lam_y + lam_z)) per mode
    __host__ __device__ static size_t bytes(int mx, int my, int mz, int rows) {
        const size_t M = (size_t)mx * my * mz;
        return 4 * (3 * M + (size_t)mx * mx + (size_t)my * my + (size_t)mz * mz + mx + my + mz +
                    (size_t)rows * (mz + 2)) + 64;
    }
    __device__ Coarse(void *base, int mx, int my, int mz) {
        const size_t M = (size_t)mx * my * mz;
        float *p = reinterpret_cast<float *>(base);
        ec = p;
        tmp = ec + M;
        sx = tmp + M;
        sy = sx + mx * mx;
        sz = sy + my * my;
        lam = sz + mz * mz;
        prof = lam + mx + my + mz;
        den = prof;  // set by coarse_tables' caller: after the profiles (see bytes)
    }
    // the mode factors follow the profiles of `rows` rows
    __device__ void place_den(int mz, int rows) { den = prof + (size_t)rows * (mz + 2); }
};

// Sine matrices and the eigenvalues (2 cos(pi (j+1) / (m+1)) - 2) / H^2 of
// the 1-D coarse operators, H = F h per axis.
template <typename T, typename S>
__device__ void coarse_tables(const SorArgs<T, S> &a, const Coarse &cs) {
    const int ms[3] = {a.cmx, a.cmy, a.cmz};
    float *mats[3] = {cs.sx, cs.sy, cs.sz};
    const double hs[3] = {a.hx, a.hy, a.hz};
    int loff = 0;
    for (int ax = 0; ax < 3; ax++) {
        const int m = ms[ax];
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int j = e / m, k = e - j * m;
            mats[ax][e] = (float)sinpi((double)((j + 1) * (k + 1)) / (double)(m + 1));
        }
        const double H = a.cf * hs[ax];
        for (int j = threadIdx.x; j < m; j += blockDim.x)
            cs.lam[loff + j] = (float)((2.0 * cospi((double)(j + 1) / (double)(m + 1)) - 2.0) / (H * H));
        loff += m;
    }
    __syncthreads();
    // the solve's per-mode factor: e^ = -f^ 8 / ((mx+1)(my+1)(mz+1)) / (lam_x + lam_y + lam_z)
    const int mx = a.cmx, my = a.cmy, mz = a.cmz;
    const float norm = 8.0f / (float)((mx + 1) * (my + 1) * (mz + 1));
    for (int o = threadIdx.x; o < mx * my * mz; o += blockDim.x) {
        const int K = o % mz, J = (o / mz) % my, I = o / (my * mz);
        cs.den[o] = -norm / (cs.lam[I] + cs.lam[mx + J] + cs.lam[mx + my + K]);
    }
}

// Stage 1: the triangle filter along z of the block's own rows of the
// pre-scaled residual (shared memory), at the coarse z nodes, into t1.  A
// half-warp takes a row (no index division per element), lane K its coarse
// node.
template <typename T, typename S>
__device__ void coarse_stage1(const SorArgs<T, S> &a, const Block &B, const S *ss) {
    const int F = a.cf, mz = a.cmz, nz2 = a.nz2, nz = a.nz, ny = a.ny;
    const float w0 = 1.0f / (float)(F * F);
    const int lane = threadIdx.x & 15, half = threadIdx.x >> 4, halves = blockDim.x >> 4;
    const int rows = B.np * B.nr;
    for (int r = half; r < rows; r += halves) {
        const int p = r / B.nr, j = r - p * B.nr, x = B.x0 + p, y = B.y0 + j;
        if (lane >= mz) continue;
        float acc = 0.0f;
        if (y >= 1 && y <= ny - 2) {
            const int kc = F * (lane + 1);
            const S *row0 = ss + ((p * 2) * B.nr + j) * nz2, *row1 = row0 + B.nr * nz2;
            for (int d0 = 1 - F; d0 < F; d0 += 8) {
                float v[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int d = d0 + q, k = kc + d;
                    const S *row = ((x + y + k) & 1) ? row1 : row0;
                    v[q] = (d < F && k >= 1 && k <= nz - 2) ? (float)row[k >> 1] : 0.0f;
                }
#pragma unroll
                for (int q = 0; q < 8; q++) acc = fmaf((float)max(F - abs(d0 + q), 0), v[q], acc);
            }
        }
        __stcg(a.t1 + ((long long)x * ny + y) * mz + lane, acc * w0);
    }
}

// Stages 2 and 3 (every block's share of the outputs): the filters along y
// and x of t1 at each interior coarse node, into t2[I][J][K].  A group of
// lanes (the power of two covering the 2F - 1 taps) shares a node: lane l
// sums its tap x = F (I + 1) + l - (F - 1) over the 2F - 1 y taps with all
// loads issued together, and the group adds its lanes with shuffles.
template <typename T, typename S>
__device__ void coarse_stage23(const SorArgs<T, S> &a, int b) {
    const int F = a.cf, my = a.cmy, mz = a.cmz, nx = a.nx, ny = a.ny, taps = 2 * F - 1;
    int lanes = 1;
    while (lanes < taps) lanes <<= 1;
    const int M = a.cmx * my * mz;
    const float w0 = 1.0f / ((float)F * F * F * F);
    const int lane = threadIdx.x & 31, sub = lane & (lanes - 1);
    const long long groups_per_warp = 32 / lanes;
    const long long gw = ((long long)b * blockDim.x + threadIdx.x) / 32;  // this warp's index
    const long long warps = (long long)a.nblocks * (blockDim.x / 32);
    for (long long g0 = gw * groups_per_warp; g0 < M; g0 += warps * groups_per_warp) {
        const long long o = g0 + lane / lanes;  // this lane's coarse node
        float acc = 0.0f;
        if (o < M && sub < taps) {
            const int K = (int)(o % mz), J = (int)((o / mz) % my), I = (int)(o / ((long long)my * mz));
            const int dx = sub - (F - 1), x = F * (I + 1) + dx;
            if (x >= 1 && x <= nx - 2) {
                const int yc = F * (J + 1);
                const float *col = a.t1 + (long long)x * ny * mz + K;
                // eight taps' loads at a time, issued before their sums
                for (int q0 = 0; q0 < taps; q0 += 8) {
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        const int y = yc + q0 + q - (F - 1);
                        v[q] = (q0 + q < taps && y >= 1 && y <= ny - 2) ? __ldcg(col + (long long)y * mz) : 0.0f;
                    }
#pragma unroll
                    for (int q = 0; q < 8; q++) acc = fmaf((float)max(F - abs(q0 + q - (F - 1)), 0), v[q], acc);
                }
                acc *= (float)(F - abs(dx));
            }
        }
        for (int off = lanes / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (sub == 0 && o < M) __stcg(a.t2 + o, acc * w0);
    }
}

// out = S applied along one axis of in ([mx][my][mz], z fastest), times
// scale[element] when scale is given.  Eight threads take a line: thread k
// keeps rows k and k + 8 of S in registers and produces elements k and k + 8,
// so each input element loaded (the eight read the same one: a shared-memory
// broadcast) feeds two multiply-adds.  (Measured against two threads per
// line with eight outputs each, whose 450 threads left each pass latency-
// bound at twice the time, and one thread per output and line, at 1.3x.)
__device__ __forceinline__ void dst_pass(const float *in, float *out, const float *Sm, int m, int axis, int mx, int my,
                                         int mz, const float *scale) {
    const int k0 = threadIdx.x & 7, k1 = k0 + 8, lg = threadIdx.x >> 3, lgs = blockDim.x >> 3;
    float s0[kCoarseMax], s1[kCoarseMax];
#pragma unroll
    for (int j = 0; j < kCoarseMax; j++) {
        s0[j] = (k0 < m && j < m) ? Sm[k0 * m + j] : 0.0f;
        s1[j] = (k1 < m && j < m) ? Sm[k1 * m + j] : 0.0f;
    }
    const int stride = axis == 2 ? 1 : axis == 1 ? mz : my * mz;
    const int L = axis == 2 ? mx * my : axis == 1 ? mx * mz : my * mz;
    for (int line = lg; line < L; line += lgs) {
        int base;
        if (axis == 2) base = line * mz;
        else if (axis == 1) base = (line / mz) * (my * mz) + line % mz;
        else base = line;
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int j = 0; j < kCoarseMax; j++)
            if (j < m) {
                const float v = in[base + j * stride];
                a0 = fmaf(s0[j], v, a0);
                a1 = fmaf(s1[j], v, a1);
            }
        if (k0 < m) {
            const int e = base + k0 * stride;
            out[e] = scale ? a0 * scale[e] : a0;
        }
        if (k1 < m) {
            const int e = base + k1 * stride;
            out[e] = scale ? a1 * scale[e] : a1;
        }
    }
}

// The coarse solve: the restricted residual (t2, every block reads all of
// it), scaled back from the pre-scaled residual to r, then
// e = S_x S_y S_z (-(S_x S_y S_z R r) / (lam_x + lam_y + lam_z)) 8 / ((mx+1)(my+1)(mz+1)).
template <typename T, typename S>
__device__ void coarse_solve(const SorArgs<T, S> &a, const Coarse &cs) {
    const int mx = a.cmx, my = a.cmy, mz = a.cmz, M = mx * my * mz;
    const float w0 = (float)(1.0 / a.src_scale);
    for (int o = threadIdx.x; o < M; o += blockDim.x) cs.ec[o] = __ldcg(a.t2 + o) * w0;
    __syncthreads();
    dst_pass(cs.ec, cs.tmp, cs.sz, mz, 2, mx, my, mz, nullptr);
    __syncthreads();
    dst_pass(cs.tmp, cs.ec, cs.sy, my, 1, mx, my, mz, nullptr);
    __syncthreads();
    dst_pass(cs.ec, cs.tmp, cs.sx, mx, 0, mx, my, mz, cs.den);  // with the per-mode factor
    __syncthreads();
    dst_pass(cs.tmp, cs.ec, cs.sz, mz, 2, mx, my, mz, nullptr);
    __syncthreads();
    dst_pass(cs.ec, cs.tmp, cs.sy, my, 1, mx, my, mz, nullptr);
    __syncthreads();
    dst_pass(cs.tmp, cs.ec, cs.sx, mx, 0, mx, my, mz, nullptr);
    __syncthreads();
}

// The coarse field at coarse node (I, J, K) of the full grid, zero on its faces.
__device__ __forceinline__ float coarse_at(const Coarse &cs, int mx, int my, int mz, int I, int J, int K) {
    if (I < 1 || J < 1 || K < 1 || I > mx || J > my || K > mz) return 0.0f;
    return cs.ec[((I - 1) * my + (J - 1)) * mz + (K - 1)];
}

// Trilinear prolongation of the coarse field into the block's own
// correction (both colours, every node; zero on the Dirichlet rows and
// z ends) and into the ghost buffer (the other blocks' black values across
// the block's faces, read by the cycle's first red sweep).  Separable: the
// (x, y) interpolation of each row's coarse z profile first (a warp per row,
// a lane per coarse z node), then z (a warp per row and colour, lanes along
// the half-row; F is a power of two, so no division per node).
template <typename T>
__device__ void coarse_prolong(const SorArgs<T, float> &a, const Block &B, const Coarse &cs, float *sd, float *gbuf,
                               const unsigned *gsrc, int ng) {
    const int F = a.cf, mx = a.cmx, my = a.cmy, mz = a.cmz, ny = a.ny, nz = a.nz, nz2 = a.nz2;
    const int own_rows = B.np * B.nr, rows = own_rows + ng, pw = mz + 2;
    const int lf = __ffs(F) - 1;
    const float inv = 1.0f / (float)F;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    auto row_xy = [&](int r, int &x, int &y) {
        if (r < own_rows) {
            const int p = r / B.nr;
            x = B.x0 + p;
            y = B.y0 + (r - p * B.nr);
        } else {
            const unsigned g = gsrc[r - own_rows];
            y = (int)((g / (unsigned)nz2) % (unsigned)ny);
            x = (int)(g / (unsigned)(2 * ny * nz2));
        }
    };
    for (int r = warp; r < rows; r += warps) {
        int x, y;
        row_xy(r, x, y);
        if (lane >= pw) continue;
        float v = 0.0f;
        if (y >= 1 && y <= ny - 2) {
            const int I = x >> lf, J = y >> lf, Kp = lane;
            const float tx = (float)(x & (F - 1)) * inv, ty = (float)(y & (F - 1)) * inv;
            v = (1.0f - tx) * ((1.0f - ty) * coarse_at(cs, mx, my, mz, I, J, Kp) +
                               ty * coarse_at(cs, mx, my, mz, I, J + 1, Kp)) +
                tx * ((1.0f - ty) * coarse_at(cs, mx, my, mz, I + 1, J, Kp) +
                      ty * coarse_at(cs, mx, my, mz, I + 1, J + 1, Kp));
        }
        cs.prof[r * pw + lane] = v;
    }
    __syncthreads();
    // z: value at node k of row r
    auto zval = [&](const float *pr, int k) -> float {
        if (k < 1 || k > nz - 2) return 0.0f;
        const int K = k >> lf;
        const float t = (float)(k & (F - 1)) * inv;
        return (1.0f - t) * pr[K] + t * pr[K + 1];
    };
    for (int task = warp; task < own_rows * 2; task += warps) {
        const int r = task >> 1, c = task & 1;
        const int p = r / B.nr, j = r - p * B.nr, x = B.x0 + p, y = B.y0 + j;
        const int kc = (c - x - y) & 1;
        const float *pr = cs.prof + r * pw;
        float *row = sd + ((p * 2 + c) * B.nr + j) * nz2;
        for (int kh = lane; kh < nz2; kh += 32) row[kh] = zval(pr, kc + 2 * kh);
    }
    for (int g = warp; g < ng; g += warps) {
        int x, y;
        row_xy(own_rows + g, x, y);
        const int kc = (1 - x - y) & 1;
        const float *pr = cs.prof + (own_rows + g) * pw;
        for (int kh = lane; kh < nz2; kh += 32) gbuf[g * nz2 + kh] = zval(pr, kc + 2 * kh);
    }
    __syncthreads();
}

// kTag: tagged exchange (float corrections in quads).  kInner, kFace,
// kGhost > 0: staged sweep with at most that many inner quads per compute
// thread, perimeter quads per thread and ghost quads per fetch thread, decoded
// once per solve; kInner = 0: the generic tagged sweep.
template <typename T, typename S, bool kTag, int kInner, int kFace, int kGhost>
__device__ __forceinline__ void sor_body(const SorArgs<T, S> &a, const int b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_tot[3];
    __shared__ int s_m;

    const int tid = threadIdx.x, nth = blockDim.x;
    const int bx = b % a.bxn, by = b / a.bxn;
    const int x0 = 1 + bx * a.P, x1 = min(x0 + a.P, a.nx - 1);
    const int y0 = by * a.R, y1 = min(y0 + a.R, a.ny);
    const int np = x1 - x0, nr = y1 - y0;
    const int ny = a.ny, nz = a.nz, nz2 = a.nz2;
    const long long sxy = (long long)ny * nz;
    const int hp = nr * nz2;   // one colour of one own plane
    const int own = np * 2 * hp;
    int *err = a.status;
    const Block B{x0, y0, np, nr, nz2, hp, ny};

    // shared memory: delta | src (when it fits)
    S *sd = reinterpret_cast<S *>(smem_raw);
    S *ss = a.src_smem ? sd + own : nullptr;
    // tagged sweeps: row tables and the ghost buffer
    const Staged st(sd + (size_t)a.P * 2 * a.R * nz2 * (a.src_smem ? 2 : 1), a.P, a.R);
    unsigned *order = st.order;
    // coarse-grid correction: its arrays follow the ghost buffer
    Coarse cs(st.gbuf + (size_t)2 * (a.P + a.R) * nz2, a.cmx, a.cmy, a.cmz);
    cs.place_den(a.cmz, a.P * a.R + 2 * (a.P + a.R));
    int ng_rows = 0;  // ghost rows listed in st.gsrc (staged sweeps)
    auto SD = [&](int p, int c, int j, int t) -> S & { return sd[((p * 2 + c) * nr + j) * nz2 + t]; };
    unsigned my_phase = 0;
    // colour sweeps: thread -> half-line position t_own, rows r_start, +rows_step
    const int rows_step = max(1, nth / nz2);
    const int r_start = tid / nz2;
    const int t_own = r_start < rows_step ? tid % nz2 : nz2;  // nz2 = idle thread
    const int j_start = r_start % nr, p_start = r_start / nr, dj = rows_step % nr, dp = rows_step / nr;
    // float4 colour sweeps: thread -> quad q_own (4 same-colour nodes) per row
    const int nq = nz2 / 4;
    const int rows_step4 = max(1, nq > 0 ? nth / nq : 1);
    const int r4_start = nq > 0 ? tid / nq : 0;
    const int q_own = (nq > 0 && r4_start < rows_step4) ? tid % nq : nq;
    const int j4_start = r4_start % nr, p4_start = r4_start / nr, dj4 = rows_step4 % nr, dp4 = rows_step4 / nr;
    // residual checks: thread -> z position k_own, rows rz_start, +zrows_step
    const int zrows_step = max(1, nth / nz);
    const int rz_start = tid / nz;
    const int k_own = rz_start < zrows_step ? tid % nz : nz;
    const int jz_start = rz_start % nr, pz_start = rz_start / nr, djz = zrows_step % nr, dpz = zrows_step / nr;

    constexpr bool kStaged = kTag && kInner > 0;
    if constexpr (kTag && !kStaged) {
        if (tid == 0) {
            int n = 0;
            for (int pass = 0; pass < 2; pass++)
                for (int l = 0; l < np * nr; l++) {
                    const int p = l / nr, j = l - p * nr, x = x0 + p, y = y0 + j;
                    const bool face = (p == 0 && x - 1 >= 1) || (p + 1 == np && x + 1 <= a.nx - 2) ||
                                      (j == 0 && y - 1 >= 1) || (j + 1 == nr && y + 1 <= ny - 2);
                    if (face == (pass == 0)) order[n++] = (unsigned)p << 16 | (unsigned)j;
                }
        }
    }
    [[maybe_unused]] Quad inner[kStaged ? kInner : 1];
    [[maybe_unused]] FaceQuad face[kStaged ? kFace : 1];
    [[maybe_unused]] GhostQuad ghost[kStaged ? kGhost : 1];
    if constexpr (kStaged) {
        __shared__ int s_nf, s_ng;
        if (tid < 32) {
            // Perimeter rows and their ghost rows, and (in `order`) the inner
            // rows, each listed by the parity of x + y first: a row's parity
            // fixes which end of its other-colour half-row a quad reads, so
            // warps whose rows share it take one path.  Warp 0 lists 32 rows
            // at a time; ballots and a scan of the ghost counts give each
            // lane its slots, in row order.
            const unsigned below = (1u << tid) - 1u;
            int nf = 0, ng = 0, ni = 0;
            for (int base = 0; base < 2 * np * nr; base += 32) {
                const int l = base + tid;
                int p = 0, j = 0, x = 0, y = 0;
                bool sel = false, perim = false;
                if (l < 2 * np * nr) {
                    const int par = l / (np * nr), lr = l - par * np * nr;
                    p = lr / nr;
                    j = lr - p * nr;
                    x = x0 + p;
                    y = y0 + j;
                    sel = ((x + y) & 1) == par;
                    perim = p == 0 || p + 1 == np || j == 0 || j + 1 == nr;
                }
                const bool is_in = sel && !perim, is_f = sel && perim;
                const bool active = is_f && y >= 1 && y <= ny - 2;
                const bool need[4] = {active && p == 0 && x - 1 >= 1, active && p + 1 == np && x + 1 <= a.nx - 2,
                                      active && j == 0 && y - 1 >= 1, active && j + 1 == nr && y + 1 <= ny - 2};
                const int cnt = (int)need[0] + (int)need[1] + (int)need[2] + (int)need[3];
                int inc = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (tid >= o) inc += v;
                }
                const unsigned bi = __ballot_sync(0xffffffffu, is_in), bf = __ballot_sync(0xffffffffu, is_f);
                if (is_in) order[ni + __popc(bi & below)] = (unsigned)p << 16 | (unsigned)j;
                if (is_f) {
                    int g = ng + inc - cnt;
                    unsigned gi[4] = {0xffffu, 0xffffu, 0xffffu, 0xffffu};
                    const int sx[4] = {x - 1, x + 1, x, x}, sy[4] = {y, y, y - 1, y + 1};
                    for (int d = 0; d < 4; d++)
                        if (need[d]) {
                            st.gsrc[g] = (unsigned)(((2ll * sx[d]) * ny + sy[d]) * nz2);
                            gi[d] = (unsigned)g++;
                        }
                    const int f = nf + __popc(bf & below);
                    st.ftab[f] = (unsigned)p << 16 | (unsigned)j;
                    st.fgi[2 * f] = gi[0] | gi[1] << 16;
                    st.fgi[2 * f + 1] = gi[2] | gi[3] << 16;
                }
                ni += __popc(bi);
                nf += __popc(bf);
                ng += __shfl_sync(0xffffffffu, inc, 31);
            }
            if (tid == 0) {
                s_nf = nf;
                s_ng = ng;
            }
        }
        __syncthreads();
        ng_rows = s_ng;
        const int nq = nz2 / 4, nfq = s_nf * nq, ngq = s_ng * nq;
        const int ip = max(np - 2, 0), ir = max(nr - 2, 0), niq = ip * ir * nq;
        const int nct = nth - kGhostThreads;
#pragma unroll
        for (int k = 0; k < kInner; k++) {
            const int w = tid - kGhostThreads + k * nct;
            inner[k] = Quad{0, 0u};
            if (tid >= kGhostThreads && w < niq) {
                const int r = w / nq, q = w - r * nq;
                const int p = (int)(order[r] >> 16), j = (int)(order[r] & 0xffffu);
                inner[k].roff = (p * 2 * nr + j) * nz2 + 4 * q;
                inner[k].flags = quad_flags(x0 + p, y0 + j, q, nq, nz);
            }
        }
#pragma unroll
        for (int k = 0; k < kFace; k++) {
            const int w = tid + k * nth;
            face[k] = FaceQuad{0, 0u, 0u, 0u, 0u};
            if (w < nfq) {
                const int r = w / nq, q = w - r * nq;
                const unsigned e = st.ftab[r];
                const int p = (int)(e >> 16), j = (int)(e & 0xffffu), x = x0 + p, y = y0 + j;
                if (y >= 1 && y <= ny - 2) {
                    unsigned f = quad_flags(x, y, q, nq, nz);
                    const unsigned gx = st.fgi[2 * r], gy = st.fgi[2 * r + 1];
                    if (p > 0) f |= kQOwnXm;
                    else if ((gx & 0xffffu) != 0xffffu) f |= kQGhXm;
                    if (p + 1 < np) f |= kQOwnXp;
                    else if ((gx >> 16) != 0xffffu) f |= kQGhXp;
                    if (j > 0) f |= kQOwnYm;
                    else if ((gy & 0xffffu) != 0xffffu) f |= kQGhYm;
                    if (j + 1 < nr) f |= kQOwnYp;
                    else if ((gy >> 16) != 0xffffu) f |= kQGhYp;
                    face[k] = FaceQuad{(p * 2 * nr + j) * nz2 + 4 * q, f,
                                       (unsigned)(((2ll * x) * ny + y) * nz2 + 4 * q), gx, gy};
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kGhost; k++) {
            const int g = tid + k * kGhostThreads;
            ghost[k] = GhostQuad{0u, -1};
            if (tid < kGhostThreads && g < ngq) {
                const int r = g / nq, q = g - r * nq;
                ghost[k] = GhostQuad{st.gsrc[r] + 4u * q, r * nz2 + 4 * q};
            }
        }
        // the first sweep reads zero ghosts
        for (int e = tid; e < 2 * (a.P + a.R) * nz2; e += nth) st.gbuf[e] = 0.0f;
        if (a.coarse) coarse_tables(a, cs);
    }

    // ---- entry: zero delta (shared and own global mirror) -----------------
    for (int e = tid; e < own; e += nth) sd[e] = S(0);
    for (int p = 0; p < np; p++)
        for (int c = 0; c < 2; c++)
            for (int e = tid; e < hp; e += nth) {
                if constexpr (kTag) a.tmirror[B.mirror(x0 + p, c, y0) + e] = 0ull;
                else a.delta[B.mirror(x0 + p, c, y0) + e] = S(0);
            }
    const int step = a.ctl[0];
    // initial guess from the phi of earlier steps (ctl[2]: how many are held)
    const int hist = a.extrapolate ? a.ctl[2] : 0;
    if (a.extrapolate) {
        // polynomial extrapolation in time of the highest order the history
        // allows: 2 p0 - p1 (linear), 3 (p0 - p1) + p2 (quadratic).  A cubic
        // guess measured worse: it amplifies the step-to-step particle noise.
        // Four nodes per thread at a time, their loads ahead of the stores.
        const int ord = min(a.extrapolate, hist), ne = np * nr * nz;
        constexpr int kU = 4;
        for (int e0 = tid; e0 < ne; e0 += kU * nth) {
            long long idv[kU];
            double cur[kU], prev[kU], prev2[kU];
            bool ok[kU];
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const int e = e0 + u * nth, k = e % nz, l = e / nz, j = l % nr, p = l / nr;
                const int y = y0 + j;
                ok[u] = e < ne && y >= 1 && y <= ny - 2 && k >= 1 && k <= nz - 2;
                idv[u] = (x0 + p) * sxy + (long long)y * nz + k;
                cur[u] = prev[u] = prev2[u] = 0.0;
                if (ok[u]) {
                    cur[u] = a.phi64[idv[u]];
                    prev[u] = a.phi64_prev[idv[u]];
                    if (ord == 2) prev2[u] = a.phi64_prev2[idv[u]];
                }
            }
#pragma unroll
            for (int u = 0; u < kU; u++) {
                if (!ok[u]) continue;
                if (ord == 2) a.phi64[idv[u]] = 3.0 * (cur[u] - prev[u]) + prev2[u];
                else if (ord == 1) a.phi64[idv[u]] = 2.0 * cur[u] - prev[u];
                if (a.extrapolate >= 2) a.phi64_prev2[idv[u]] = prev[u];
                a.phi64_prev[idv[u]] = cur[u];
            }
        }
    }

    // first cycle: 7/8 of the previous solve's iteration count (ctl[1]), so
    // that a solve like the last one takes one long cycle and a short
    // correction, three residual checks in all; the cycles after it follow the
    // observed rate, clamped to [inner_min, inner_max]
    int its = 0, m_prev = 0, cycles = 0, m = max(1, min(a.inner_max, (7 * a.ctl[1]) / 8));
    double rel_prev = -1.0, rel = 0.0, maxd = 0.0;
    bool converged = false;
    S last_max = S(0);

    while (true) {
        if (its > 0) {
            S bm = block_max<S>(last_max);
            if (tid == 0) a.partials[4 * b + 2] = (double)bm;
        }
        // delta of every block is final in global memory after this barrier
        if (!grid_barrier(a.bar, a.nblocks, err, a.max_spin)) return;

        // ---- FP64 residual of phi + delta on own interior nodes ----------
        // The first check of a solve evaluates b + L phi from phi's stencil
        // (delta is zero there).  Later ones carry it: the residual of
        // phi + delta is r + L delta, with r the FP64 residual kept per node
        // since the last check and delta read as floats (exact in double), so
        // no block reads another block's phi and phi += delta folds in the
        // same pass.  The source of the next cycle is the new residual,
        // pre-scaled.
        double rr = 0.0;
        const int k = k_own;
        const bool kin = k >= 1 && k <= nz - 2;
        if (its == 0) {
            double bb = 0.0;
            // kCheckRows rows at a time: their stencil loads go out together
            for (int l = rz_start; kin && l < np * nr; l += kCheckRows * zrows_step) {
                long long idr[kCheckRows];
                double v[kCheckRows][7];
                T rh[kCheckRows];
                bool okr[kCheckRows];
#pragma unroll
                for (int u = 0; u < kCheckRows; u++) {
                    const int lu = l + u * zrows_step;
                    const int p = lu / nr, j = lu - p * nr, y = y0 + j;
                    okr[u] = lu < np * nr && y >= 1 && y <= ny - 2;
                    const long long id = (x0 + p) * sxy + (long long)y * nz + k;
                    idr[u] = id;
                    rh[u] = T(0);
#pragma unroll
                    for (int q = 0; q < 7; q++) v[u][q] = 0.0;
                    if (okr[u]) {
                        v[u][0] = __ldcg(a.phi64 + id);
                        v[u][1] = __ldcg(a.phi64 + id - sxy);
                        v[u][2] = __ldcg(a.phi64 + id + sxy);
                        v[u][3] = __ldcg(a.phi64 + id - nz);
                        v[u][4] = __ldcg(a.phi64 + id + nz);
                        v[u][5] = __ldcg(a.phi64 + id - 1);
                        v[u][6] = __ldcg(a.phi64 + id + 1);
                        rh[u] = __ldg(a.rho + id);
                    }
                }
#pragma unroll
                for (int u = 0; u < kCheckRows; u++) {
                    if (!okr[u]) continue;
                    const int lu = l + u * zrows_step;
                    const int p = lu / nr, j = lu - p * nr, x = x0 + p, y = y0 + j;
                    const double bv = a.src_c * (double)rh[u];
                    const double r = bv + (v[u][2] + v[u][1]) * a.dhx2i + (v[u][4] + v[u][3]) * a.dhy2i +
                                     (v[u][6] + v[u][5]) * a.dhz2i - a.ddiag * v[u][0];
                    a.resid[idr[u]] = r;
                    rr += r * r;
                    bb += bv * bv;
                    const int kh = k >> 1, c0 = (x + y + k) & 1;
                    if (ss) ss[((p * 2 + c0) * nr + j) * nz2 + kh] = (S)(r * a.src_scale);
                    else a.src[B.mirror(x, c0, y) + kh] = (S)(r * a.src_scale);
                }
            }
            block_sum2(rr, bb);
            if (tid == 0) {
                a.partials[4 * b + 0] = rr;
                a.partials[4 * b + 1] = bb;  // kept for the later checks
            }
        } else {
            // kCheckRows rows at a time: their loads go out before any store
            for (int l = rz_start; kin && l < np * nr; l += kCheckRows * zrows_step) {
                long long idr[kCheckRows];
                double rv[kCheckRows], pv[kCheckRows];
                S mv[kCheckRows][4];
                int pr[kCheckRows], jr[kCheckRows];
                bool okr[kCheckRows];
#pragma unroll
                for (int u = 0; u < kCheckRows; u++) {
                    const int lu = l + u * zrows_step;
                    const int p = lu / nr, j = lu - p * nr, x = x0 + p, y = y0 + j;
                    pr[u] = p;
                    jr[u] = j;
                    okr[u] = lu < np * nr && y >= 1 && y <= ny - 2;
                    idr[u] = x * sxy + (long long)y * nz + k;
                    rv[u] = pv[u] = 0.0;
                    mv[u][0] = mv[u][1] = mv[u][2] = mv[u][3] = S(0);
                    if (okr[u]) {
                        rv[u] = a.resid[idr[u]];
                        pv[u] = __ldcg(a.phi64 + idr[u]);
                        // other blocks' delta from their mirrors (zero on the
                        // Dirichlet planes and rows)
                        const int kh = k >> 1, c1 = ((x + y + k) & 1) ^ 1;
                        if (p == 0) mv[u][0] = (S)mirror_value<kTag>(a, B.mirror(x - 1, c1, y) + kh);
                        if (p + 1 == np) mv[u][1] = (S)mirror_value<kTag>(a, B.mirror(x + 1, c1, y) + kh);
                        if (j == 0) mv[u][2] = (S)mirror_value<kTag>(a, B.mirror(x, c1, y - 1) + kh);
                        if (j + 1 == nr) mv[u][3] = (S)mirror_value<kTag>(a, B.mirror(x, c1, y + 1) + kh);
                    }
                }
#pragma unroll
                for (int u = 0; u < kCheckRows; u++) {
                    if (!okr[u]) continue;
                    const int p = pr[u], j = jr[u], x = x0 + p, y = y0 + j;
                    const int kh = k >> 1, c0 = (x + y + k) & 1, c1 = c0 ^ 1;
                    const double dc = (double)SD(p, c0, j, kh);
                    const double dzm = (double)SD(p, c1, j, (k - 1) >> 1), dzp = (double)SD(p, c1, j, (k + 1) >> 1);
                    const double dxm = p > 0 ? (double)SD(p - 1, c1, j, kh) : (double)mv[u][0];
                    const double dxp = p + 1 < np ? (double)SD(p + 1, c1, j, kh) : (double)mv[u][1];
                    const double dym = j > 0 ? (double)SD(p, c1, j - 1, kh) : (double)mv[u][2];
                    const double dyp = j + 1 < nr ? (double)SD(p, c1, j + 1, kh) : (double)mv[u][3];
                    const double r = rv[u] + (dxp + dxm) * a.dhx2i + (dyp + dym) * a.dhy2i + (dzp + dzm) * a.dhz2i -
                                     a.ddiag * dc;
                    a.resid[idr[u]] = r;
                    a.phi64[idr[u]] = pv[u] + dc;
                    rr += r * r;
                    if (ss) ss[((p * 2 + c0) * nr + j) * nz2 + kh] = (S)(r * a.src_scale);
                    else a.src[B.mirror(x, c0, y) + kh] = (S)(r * a.src_scale);
                }
            }
            double none = 0.0;
            block_sum2(rr, none);
            if (tid == 0) a.partials[4 * b + 0] = rr;
        }
        if constexpr (kStaged) {
            if (a.coarse) {
                __syncthreads();  // every own row's residual source is in shared memory
                coarse_stage1(a, B, ss);
            }
        }
        if (!grid_barrier(a.bar, a.nblocks, err, a.max_spin)) return;

        // ---- every block sums the partials in the same fixed order ------
        if (tid < 32) {
            double u = 0.0, v = 0.0, w = 0.0;
            for (int q = tid; q < a.nblocks; q += 32) {
                u += __ldcg(a.partials + 4 * q);
                v += __ldcg(a.partials + 4 * q + 1);
                w = fmax(w, __ldcg(a.partials + 4 * q + 2));
            }
            for (int o = 16; o > 0; o >>= 1) {
                u += __shfl_xor_sync(0xffffffffu, u, o);
                v += __shfl_xor_sync(0xffffffffu, v, o);
                w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
            }
            if (tid == 0) {
                s_tot[0] = u;
                s_tot[1] = v;
                s_tot[2] = w;
            }
        }
        __syncthreads();
        rel = s_tot[1] > 0.0 ? sqrt(s_tot[0] / s_tot[1]) : sqrt(s_tot[0]);
        maxd = s_tot[2];
        cycles++;

        // ---- the next cycle starts from delta = 0 (or the coarse grid's
        // correction, which overwrites every own node) -----------------------
        if (!a.coarse)
            for (int e = tid; e < own; e += nth) sd[e] = S(0);
        if constexpr (!kTag)
            for (int p = 0; p < np; p++)
                for (int c = 0; c < 2; c++)
                    for (int e = tid; e < hp; e += nth) a.delta[B.mirror(x0 + p, c, y0) + e] = S(0);

        if (a.criterion == HV_SOR_REL_RESIDUAL) converged = rel <= a.tol;
        else converged = its > 0 && maxd < a.tol;
        if (converged || its >= a.max_iter || !(rel == rel)) break;

        // ---- next inner cycle length: predicted from the observed rate ---
        if (tid == 0) {
            int mm = m;
            if (a.coarse) {
                // a fixed number of iterations after each coarse correction
                mm = a.csweeps;
            } else if (a.criterion == HV_SOR_REL_RESIDUAL && rel_prev > 0.0 && rel < rel_prev && m_prev > 0) {
                double q = pow(rel / rel_prev, 1.0 / m_prev);
                double pred = log(a.tol / rel) / log(q);
                mm = pred < 1e6 ? (int)ceil(pred) : a.inner_max;
            }
            mm = max(a.inner_min, min(a.inner_max, mm));
            mm = min(mm, a.max_iter - its);
            s_m = max(mm, 1);
        }
        __syncthreads();
        m_prev = m = s_m;
        rel_prev = rel;
        last_max = S(0);

        // ---- m red+black iterations on delta, tagged exchange -------------
        if constexpr (kStaged) {
            if (a.coarse) {
                // restriction stages 2 and 3, the coarse solve and its
                // prolongation, which the sweeps below start from
                coarse_stage23(a, b);
                if (!grid_barrier(a.bar, a.nblocks, err, a.max_spin)) return;
                coarse_solve(a, cs);
                coarse_prolong<T>(a, B, cs, sd, st.gbuf, st.gsrc, ng_rows);
            }
        }
        if constexpr (kTag) {
            bool failed = false;
            for (int it = 0; it < m; it++) {
                const unsigned t = (unsigned)(its + it);
                for (int c = 0; c < 2; c++) {
                    // red(t) is half-sweep 2t+1, black(t) 2t+2; red reads black(t-1)
                    const unsigned tag_in = c == 0 ? (it == 0 ? 0u : 2u * t) : 2u * t + 1u;
                    const unsigned tag_out = 2u * t + 1u + (unsigned)c;
                    if constexpr (kStaged) {
                        // perimeter rows first, from the ghosts fetched during the
                        // previous sweep; then the inner rows while the fetch threads
                        // poll the neighbours' perimeter rows of this sweep for the next
                        // one (zeros after a cycle's last sweep: the next cycle starts
                        // from zero corrections)
                        const long long cstride = (long long)ny * nz2;
                        const bool track = it == m - 1;
#pragma unroll
                        for (int k = 0; k < kFace; k++)
                            sweep_face<T>(a, face[k], c, hp, cstride, sd, ss, st.gbuf, tag_out, track, last_max);
                        __syncthreads();
                        if (tid < kGhostThreads) {
                            const unsigned tag_next = (c == 1 && it == m - 1) ? 0u : tag_out;
                            fetch_ghosts<kGhost>(a.tmirror, ghost, c * cstride, tag_next, st.gbuf, a.status, a.max_poll,
                                                failed);
                        } else {
#pragma unroll
                            for (int k = 0; k < kInner; k++) sweep_inner<T>(a, inner[k], c, hp, sd, ss, track, last_max);
                        }
                    } else {
                        sweep_quads_tagged<T>(a, B, c, sd, ss, order, it == m - 1, last_max, tag_out, tag_in,
                                              failed);
                    }
                    if (__syncthreads_or(failed)) return;
                }
            }
            its += m;
            continue;
        }

        // ---- m red+black iterations on delta, phase counters --------------
        publish(a.phase + b, ++my_phase);
        for (int it = 0; it < m; it++) {
            for (int c = 0; c < 2; c++) {
                if (!wait_neighbours(a, bx, by, my_phase)) return;
                const bool track = (it == m - 1);
                if (a.vec4)
                    sweep_quads<S>(a, B, c, sd, ss, q_own, r4_start, rows_step4, j4_start, p4_start, dj4, dp4, track,
                                   last_max);
                else
                    sweep_scalar<S>(a, B, c, sd, ss, t_own, r_start, rows_step, j_start, p_start, dj, dp, track,
                                    last_max);
                publish(a.phase + b, ++my_phase);
            }
        }
        its += m;
    }

    if (b == 0 && tid == 0) {
        a.status[1] = its;
        a.status[2] = converged ? 1 : 0;
        a.status[3] = cycles;
        a.metric[0] = a.criterion == HV_SOR_REL_RESIDUAL ? rel : maxd;
        a.ctl[1] = max(its, 1);
        if (a.extrapolate) a.ctl[2] = min(a.ctl[2] + 1, 2);
        if (a.its_ring) a.its_ring[step % a.ring] = converged ? its : -its;
    }
}

// One solve (kBatch false: the arguments are the kernel parameter), or several
// independent solves in one cooperative launch (kBatch: block blockIdx.x works
// on instance binst[blockIdx.x], as its block blockIdx.x - bfirst[instance];
// barriers, residual sums and the exchange stay within an instance, and an
// instance that has converged leaves while the others go on).
template <typename T, typename S, bool kTag, int kInner, int kFace, int kGhost, bool kBatch = false>
__global__ void __launch_bounds__(kSorThreads, 1) k_sor_fast(SorArgs<T, S> p) {
    if constexpr (kBatch) {
        __shared__ SorArgs<T, S> s_inst;
        const int inst = p.binst[blockIdx.x];
        if (threadIdx.x == 0) s_inst = p.batch[inst];
        __syncthreads();
        sor_body<T, S, kTag, kInner, kFace, kGhost>(s_inst, (int)blockIdx.x - p.bfirst[inst]);
    } else {
        sor_body<T, S, kTag, kInner, kFace, kGhost>(p, (int)blockIdx.x);
    }
}

}  // namespace

template <typename S>
static hv_status plan_for(hv_ctx *c, int max_blocks, int rank = 0) {
    SorFast &f = c->fused.sor;
    const Geom &g = c->geom;
    cudaDeviceProp prop;
    HV_CUDA(cudaGetDeviceProperties(&prop, c->device));
    const size_t static_smem = 2048;
    const size_t limit = prop.sharedMemPerBlockOptin > static_smem ? prop.sharedMemPerBlockOptin - static_smem : 0;
    // blocks of one solve: all SMs, or fewer when the solve shares a launch
    const long long cap = max_blocks > 0 ? std::min(max_blocks, prop.multiProcessorCount) : prop.multiProcessorCount;
    const int nz2 = (g.nz + 1) / 2;
    const int interior = g.nx - 2;
    f.ok = false;
    // coarse-grid correction of the float solve: the smallest power-of-two
    // factor F that divides every axis and leaves at most kCoarseMax interior
    // coarse nodes per axis (at least one)
    int cf = 0, cm[3] = {0, 0, 0};
    // grids of fewer nodes converge in a few dozen plain iterations, less than
    // the correction's fixed cost per cycle repays
    const long long coarse_min_nodes = 48ll * 48 * 48;
    if (sizeof(S) == 4 && g.G >= coarse_min_nodes) {
        const int n3[3] = {g.nx, g.ny, g.nz};
        for (int F = 2; F <= 256 && !cf; F *= 2) {
            bool ok = true;
            for (int ax = 0; ax < 3; ax++) {
                const int m = n3[ax] / F - 1;
                ok = ok && n3[ax] % F == 0 && m >= 1 && m <= kCoarseMax;
                cm[ax] = m;
            }
            if (ok) cf = F;
            else if (n3[0] / F - 1 < 1 || n3[1] / F - 1 < 1 || n3[2] / F - 1 < 1) break;
        }
    }
    if (sizeof(S) == 4 && nz2 % 4 == 0) {
        // float corrections in quads: blocks of P planes x R rows with the
        // source in shared memory, ranked by the fewest quads per thread, then
        // the smallest total face (blocks x (P + R): the rows exchanged per
        // sweep), then the fewest blocks; the plan takes candidate `rank` of
        // that order (0, the first, unless the autotuner chose another)
        const long long nq = nz2 / 4;
        struct Cand {
            long long key[3];
            int P, R, bxn, byn;
            size_t smem;
        };
        std::vector<Cand> cands;
        for (int P = 1; P <= interior; P++)
            for (int R = 1; R <= g.ny; R++) {
                const size_t own = (size_t)P * 2 * R * nz2;
                const size_t smem = sizeof(S) * own * 2 + Staged::bytes(P, R, nz2) +
                                    (cf ? Coarse::bytes(cm[0], cm[1], cm[2], P * R + 2 * (P + R)) : 0);
                if (smem > limit) break;
                const long long bxn = (interior + P - 1) / P, byn = (g.ny + R - 1) / R;
                if (bxn * byn > cap) continue;
                cands.push_back(Cand{{((long long)P * R * nq + kSorThreads - 1) / kSorThreads, bxn * byn * (P + R),
                                      bxn * byn},
                                     P, R, (int)bxn, (int)byn, smem});
            }
        std::stable_sort(cands.begin(), cands.end(), [](const Cand &u, const Cand &v) {
            return std::lexicographical_compare(u.key, u.key + 3, v.key, v.key + 3);
        });
        f.tile_candidates = (int)cands.size();
        if (!cands.empty()) {
            const Cand &b = cands[rank < (int)cands.size() ? rank : 0];
            f.P = b.P;
            f.R = b.R;
            f.bx = b.bxn;
            f.by = b.byn;
            f.nblocks = b.bxn * b.byn;
            f.smem = b.smem;
            f.src_smem = true;
            f.tables = true;
            f.ok = true;
        }
    }
    // otherwise smallest blocks first (most parallel), the source in shared
    // memory when it fits, a y split only when a plane does not fit
    for (int pass = 0; pass < 2 && !f.ok; pass++) {
        const bool with_src = pass == 0;
        for (int R = g.ny; R >= 1 && !f.ok; R = (R == 1) ? 0 : (R + 1) / 2) {
            for (int P = 1; P <= interior; P++) {
                const size_t own = (size_t)P * 2 * R * nz2;
                const size_t smem = sizeof(S) * own * (with_src ? 2 : 1);
                if (smem > limit) break;
                const int bxn = (interior + P - 1) / P, byn = (g.ny + R - 1) / R;
                if ((long long)bxn * byn > cap) continue;
                f.P = P;
                f.R = R;
                f.bx = bxn;
                f.by = byn;
                f.nblocks = bxn * byn;
                f.smem = smem;
                f.src_smem = with_src;
                f.tables = false;
                f.ok = true;
                break;
            }
        }
    }
    if (!f.ok) return HV_OK;  // the fused path reports HV_ERR_UNSUPPORTED
    f.nz2 = nz2;
    f.threads = kSorThreads;
    const void *kerns[4] = {(const void *)k_sor_fast<S, S, false, 0, 0, 0>, nullptr, nullptr, nullptr};
    if constexpr (sizeof(S) == 4) {
        kerns[1] = (const void *)k_sor_fast<S, S, true, 0, 0, 0>;
        kerns[2] = (const void *)k_sor_fast<S, S, true, 1, 1, 2>;
        kerns[3] = (const void *)k_sor_fast<S, S, true, 2, 1, 3>;
    }
    for (const void *kern : kerns) {
        if (!kern) continue;
        HV_TRY(allow_max_dynamic_smem(kern, c->device));
        int per_sm = 0;
        HV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, f.threads, f.smem));
        if (per_sm < 1 || (long long)per_sm * prop.multiProcessorCount < f.nblocks) {
            f.ok = false;
            return HV_OK;
        }
    }
    // mirrors cover every plane and row, so the Dirichlet ones stay zero; 8
    // bytes per entry, which also holds the tagged words of a float solve
    const size_t n = (size_t)g.nx * 2 * g.ny * nz2;
    HV_CUDA(cudaMalloc(&f.delta, n * 8));
    HV_CUDA(cudaMalloc(&f.src, n * sizeof(S)));
    HV_CUDA(cudaMalloc((void **)&f.resid, sizeof(double) * g.G));
    HV_CUDA(cudaMemsetAsync(f.delta, 0, n * 8, c->stream));
    HV_CUDA(cudaMemsetAsync(f.src, 0, n * sizeof(S), c->stream));
    HV_CUDA(cudaMalloc((void **)&f.partials, sizeof(double) * 4 * f.nblocks));
    HV_CUDA(cudaMemsetAsync(f.partials, 0, sizeof(double) * 4 * f.nblocks, c->stream));
    HV_CUDA(cudaMalloc((void **)&f.phase, sizeof(unsigned) * (f.nblocks + 2)));
    HV_CUDA(cudaMemsetAsync(f.phase, 0, sizeof(unsigned) * (f.nblocks + 2), c->stream));
    f.bar = f.phase + f.nblocks;
    HV_CUDA(cudaMalloc((void **)&f.status, sizeof(int) * 8));
    HV_CUDA(cudaMalloc((void **)&f.metric, sizeof(double) * 2));
    HV_CUDA(cudaMemsetAsync(f.status, 0, sizeof(int) * 8, c->stream));
    if (cf && f.tables) {
        f.cf = cf;
        f.cmx = cm[0];
        f.cmy = cm[1];
        f.cmz = cm[2];
        const size_t n1 = (size_t)g.nx * g.ny * cm[2], n2 = (size_t)g.nx * cm[1] * cm[2];
        HV_CUDA(cudaMalloc((void **)&f.t1, sizeof(float) * n1));
        HV_CUDA(cudaMalloc((void **)&f.t2, sizeof(float) * n2));
        HV_CUDA(cudaMemsetAsync(f.t1, 0, sizeof(float) * n1, c->stream));
        HV_CUDA(cudaMemsetAsync(f.t2, 0, sizeof(float) * n2, c->stream));
    }
    return HV_OK;
}

// Clears the error word of the fused solver before a run's solves.
// Also zeroes the barrier and phase counters: a solve that ended normally
// leaves the tagged forms' arrival counter at zero, so their steps need no
// reset of their own, but one that gave up may not.
hv_status sor_fast_clear_error(hv_ctx *c) {
    const SorFast &f = c->fused.sor;
    HV_CUDA(cudaMemsetAsync(f.status, 0, sizeof(int) * 4, c->stream));
    HV_CUDA(cudaMemsetAsync(f.phase, 0, sizeof(unsigned) * (f.nblocks + 2), c->stream));
    return HV_OK;
}

hv_status sor_fast_plan(hv_ctx *c) {
    return c->prec == HV_F64 ? plan_for<double>(c, 0) : plan_for<float>(c, 0);
}


void sor_fast_release(hv_ctx *c) {
    SorFast &f = c->fused.sor;
    void *ptrs[] = {f.delta, f.src, f.resid, f.partials, f.phase, f.status, f.metric, f.t1, f.t2};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    f = SorFast();
}

hv_status sor_fast_replan(hv_ctx *c, int max_blocks) {
    sor_fast_release(c);
    return c->prec == HV_F64 ? plan_for<double>(c, max_blocks) : plan_for<float>(c, max_blocks);
}

// Re-plans with the tile of the given rank among the ranked candidates of a
// float solve (see plan_for); *count receives the number of candidates.
hv_status sor_fast_replan_rank(hv_ctx *c, int rank, int *count) {
    sor_fast_release(c);
    const hv_status st = c->prec == HV_F64 ? plan_for<double>(c, 0, rank) : plan_for<float>(c, 0, rank);
    if (count) *count = c->fused.sor.tile_candidates;
    c->fused.sor.tile_rank = rank < c->fused.sor.tile_candidates ? rank : 0;
    return st;
}

// The update's coefficients for the cycles the arguments run: the sweeps of
// a coarse-corrected cycle smooth what the coarse solve leaves (kCoarseOmega
// unless set); plain cycles relax at the run's omega (or its override).
template <typename T, typename S>
static void set_relaxation(const hv_ctx *c, SorArgs<T, S> &a) {
    const double omega = a.coarse ? (c->fast.sor_coarse_omega > 0.0 ? c->fast.sor_coarse_omega : kCoarseOmega)
                                  : (c->fast.sor_omega > 0.0 ? c->fast.sor_omega : c->params.sor.omega);
    a.cx = (S)(omega * a.dhx2i / a.ddiag);
    a.cy = (S)(omega * a.dhy2i / a.ddiag);
    a.cz = (S)(omega * a.dhz2i / a.ddiag);
    a.cself = (S)(1.0 - omega);
    a.src_scale = omega / a.ddiag;
}

// The arguments of one solve and its kernel form: 0 phase counters, 1 the
// generic tagged sweep, 2 and 3 the staged sweep for at most (1, 1, 2) and
// (2, 1, 3) inner / perimeter / ghost quads per thread.
template <typename T>
static int sor_fast_args(hv_ctx *c, const T *rho, int *ctl, int *its_ring, int ring, SorArgs<T, T> &a) {
    using S = T;
    SorFast &f = c->fused.sor;
    const Geom &g = c->geom;
    const hv_sor_params &sp = c->params.sor;
    std::memset(&a, 0, sizeof(a));
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.nz2 = f.nz2;
    a.P = f.P;
    a.R = f.R;
    a.bxn = f.bx;
    a.byn = f.by;
    a.nblocks = f.nblocks;
    a.src_smem = f.src_smem ? 1 : 0;
    a.vec4 = (sizeof(S) == 4 && f.nz2 % 4 == 0 && f.src_smem) ? 1 : 0;
    a.nq_shift = -1;
    for (int sh = 0; sh < 30; sh++)
        if ((f.nz2 / 4) == (1 << sh)) a.nq_shift = sh;
    const double dx = 2.0 * g.dmx / g.nx, dy = 2.0 * g.dmy / g.ny, dz = 2.0 * g.dmz / g.nz;
    a.dhx2i = 1.0 / (dx * dx);
    a.dhy2i = 1.0 / (dy * dy);
    a.dhz2i = 1.0 / (dz * dz);
    a.ddiag = 2.0 * (a.dhx2i + a.dhy2i + a.dhz2i);
    a.src_c = 4.0 * kPi * kE2;
    a.tol = sp.tol;
    a.max_iter = sp.max_iter;
    a.criterion = sp.criterion;
    a.inner_min = c->fast.sor_inner_min;
    a.inner_max = c->fast.sor_inner_max;
    a.max_spin = c->fast.sor_wait_limit > 0 ? c->fast.sor_wait_limit : kDefaultSpin;
    a.max_poll = c->fast.sor_wait_limit > 0 ? c->fast.sor_wait_limit : kDefaultPoll;
    a.extrapolate = c->fast.sor_warm_start == HV_WARM_EXTRAPOLATE ? 1
                    : c->fast.sor_warm_start == HV_WARM_QUADRATIC ? 2 : 0;
    a.rho = rho;
    a.phi64 = c->fused.phi64;
    a.phi64_prev = c->fused.phi64_prev;
    a.phi64_prev2 = c->fused.phi64_prev2;
    a.resid = f.resid;
    a.delta = reinterpret_cast<S *>(f.delta);
    a.tmirror = reinterpret_cast<u64 *>(f.delta);
    a.src = reinterpret_cast<S *>(f.src);
    a.partials = f.partials;
    a.phase = f.phase;
    a.bar = f.bar;
    a.status = f.status;
    a.metric = f.metric;
    a.ctl = ctl;
    a.its_ring = its_ring;
    a.ring = ring;
    int form = 0;
    // the tagged sweeps need their row tables in shared memory
    if (sizeof(S) == 4 && a.vec4 && f.tables && c->fast.sor_exchange == HV_SOR_EXCHANGE_AUTO) {
        // staged sweep when its per-thread quad counts fit an instantiation
        const long long nq = f.nz2 / 4, P = f.P, R = f.R;
        const long long inner = std::max(P - 2, 0ll) * std::max(R - 2, 0ll);
        const long long ni = (inner * nq + f.threads - kGhostThreads - 1) / (f.threads - kGhostThreads);
        const long long nf = ((P * R - inner) * nq + f.threads - 1) / f.threads;
        const long long ng = (2 * (P + R) * nq + kGhostThreads - 1) / kGhostThreads;
        form = 1;
        if (ni <= 1 && nf <= 1 && ng <= 2) form = 2;
        else if (ni <= 2 && nf <= 1 && ng <= 3) form = 3;
    }
    // the coarse-grid correction: staged float sweeps, relative-residual rule
    a.coarse = (f.cf > 0 && form >= 2 && c->fast.sor_coarse && sp.criterion == HV_SOR_REL_RESIDUAL) ? 1 : 0;
    a.cf = f.cf;
    a.cmx = f.cmx;
    a.cmy = f.cmy;
    a.cmz = f.cmz;
    a.csweeps = c->fast.sor_coarse_sweeps;
    a.t1 = f.t1;
    a.t2 = f.t2;
    a.hx = dx;
    a.hy = dy;
    a.hz = dz;
    set_relaxation(c, a);
    return form;
}

template <typename T, bool kBatch>
static const void *sor_kernel(int form) {
    if constexpr (sizeof(T) == 4) {
        switch (form) {
        case 1: return (const void *)k_sor_fast<T, T, true, 0, 0, 0, kBatch>;
        case 2: return (const void *)k_sor_fast<T, T, true, 1, 1, 2, kBatch>;
        case 3: return (const void *)k_sor_fast<T, T, true, 2, 1, 3, kBatch>;
        default: break;
        }
    }
    if constexpr (kBatch) return nullptr;
    else return (const void *)k_sor_fast<T, T, false, 0, 0, 0>;
}

// step_solve false: a solve whose starting phi is not a converged solution
// (the initial solve from phi = 0) starts from that phi and leaves the history
// of earlier solutions untouched.
template <typename T>
hv_status sor_fast_launch(hv_ctx *c, const T *rho, int *ctl, int *its_ring, int ring, bool step_solve) {
    SorFast &f = c->fused.sor;
    SorArgs<T, T> a;
    const int form = sor_fast_args<T>(c, rho, ctl, its_ring, ring, a);
    // the phase-counter form counts from zero in every solve; the tagged
    // forms' barrier counter is back at zero after each completed solve (the
    // run's start resets it, sor_fast_clear_error).  The error word stays set
    // from an earlier solve of the run, so that a later one cannot hide it
    if (form == 0) HV_CUDA(cudaMemsetAsync(f.phase, 0, sizeof(unsigned) * (f.nblocks + 2), c->stream));
    if (!step_solve) a.extrapolate = 0;
    void *args[] = {&a};
    HV_CUDA(cudaLaunchCooperativeKernel(sor_kernel<T, false>(form), dim3(f.nblocks), dim3(f.threads), args, f.smem,
                                        c->stream));
    return HV_OK;
}

hv_status sor_fast_launch_adjoint(hv_ctx *c, const double *src, double *mu, double *mu_prev, double *mu_prev2,
                                  int *ctl) {
    if (c->prec != HV_F64) return HV_ERR_UNSUPPORTED;
    SorFast &f = c->fused.sor;
    SorArgs<double, double> a;
    const int form = sor_fast_args<double>(c, src, ctl, nullptr, 0, a);
    a.phi64 = mu;
    a.phi64_prev = mu_prev;
    a.phi64_prev2 = mu_prev2;
    if (form == 0) HV_CUDA(cudaMemsetAsync(f.phase, 0, sizeof(unsigned) * (f.nblocks + 2), c->stream));
    void *args[] = {&a};
    HV_CUDA(cudaLaunchCooperativeKernel(sor_kernel<double, false>(form), dim3(f.nblocks), dim3(f.threads), args,
                                        f.smem, c->stream));
    return HV_OK;
}

const int *sor_fast_status_words(hv_ctx *c) { return c->fused.sor.status; }

// ---- several float solves in one cooperative launch ------------------------

hv_status sor_wave_build(SorWave &w, const std::vector<hv_ctx *> &cs, const std::vector<const float *> &rho,
                         const std::vector<int *> &ctl, const std::vector<int *> &its_ring, int ring) {
    sor_wave_release(w);
    const int n = (int)cs.size();
    std::vector<SorArgs<float, float>> args(n);
    std::vector<int> binst, bfirst(n);
    // one kernel form for all: the generic tagged sweep if any instance needs
    // it, else the staged sweep whose per-thread counts cover every instance
    bool any1 = false, all2 = true;
    size_t smem = 0;
    for (int i = 0; i < n; i++) {
        hv_ctx *c = cs[i];
        if (c->prec != HV_F32 || !c->fused.sor.ok) return HV_ERR_UNSUPPORTED;
        const int fi = sor_fast_args<float>(c, rho[i], ctl[i], its_ring[i], ring, args[i]);
        if (fi == 0) return HV_ERR_UNSUPPORTED;  // the batched form needs the tagged exchange
        any1 = any1 || fi == 1;
        all2 = all2 && fi == 2;
        bfirst[i] = (int)binst.size();
        for (int b = 0; b < c->fused.sor.nblocks; b++) binst.push_back(i);
        smem = std::max(smem, c->fused.sor.smem);
    }
    const int form = any1 ? 1 : all2 ? 2 : 3;
    // the coarse-grid correction needs the staged sweep (its ghost buffer and
    // row tables); a wave of generic tagged sweeps runs plain cycles
    if (form == 1)
        for (int i = 0; i < n; i++) {
            args[i].coarse = 0;
            set_relaxation(cs[i], args[i]);
        }
    int dev = 0;
    HV_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    HV_CUDA(cudaGetDeviceProperties(&prop, dev));
    w.kern = sor_kernel<float, true>(form);
    HV_TRY(allow_max_dynamic_smem(w.kern, dev));
    int per_sm = 0;
    HV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, w.kern, kSorThreads, smem));
    if ((long long)per_sm * prop.multiProcessorCount < (long long)binst.size()) return HV_ERR_UNSUPPORTED;
    HV_CUDA(cudaMalloc(&w.args, sizeof(SorArgs<float, float>) * n));
    HV_CUDA(cudaMalloc((void **)&w.binst, sizeof(int) * binst.size()));
    HV_CUDA(cudaMalloc((void **)&w.bfirst, sizeof(int) * n));
    HV_CUDA(cudaMemcpy(w.args, args.data(), sizeof(SorArgs<float, float>) * n, cudaMemcpyHostToDevice));
    HV_CUDA(cudaMemcpy(w.binst, binst.data(), sizeof(int) * binst.size(), cudaMemcpyHostToDevice));
    HV_CUDA(cudaMemcpy(w.bfirst, bfirst.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    // a cudaMemcpy from pageable memory may return before its DMA ends; the
    // wave's kernels run later on other streams
    HV_CUDA(cudaDeviceSynchronize());
    w.ctx = cs;
    w.nblocks = (int)binst.size();
    w.smem = smem;
    return HV_OK;
}

// The waves run tagged forms only: each instance's barrier counter is back at
// zero after its solve, and the batch's start resets it (run_begin).
hv_status sor_wave_launch(const SorWave &w, cudaStream_t st) {
    SorArgs<float, float> p;
    std::memset(&p, 0, sizeof(p));
    p.batch = reinterpret_cast<const SorArgs<float, float> *>(w.args);
    p.binst = w.binst;
    p.bfirst = w.bfirst;
    void *args[] = {&p};
    HV_CUDA(cudaLaunchCooperativeKernel(w.kern, dim3(w.nblocks), dim3(kSorThreads), args, w.smem, st));
    return HV_OK;
}

void sor_wave_release(SorWave &w) {
    if (w.args) cudaFree(w.args);
    if (w.binst) cudaFree(w.binst);
    if (w.bfirst) cudaFree(w.bfirst);
    w = SorWave();
}

template hv_status sor_fast_launch<float>(hv_ctx *, const float *, int *, int *, int, bool);
template hv_status sor_fast_launch<double>(hv_ctx *, const double *, int *, int *, int, bool);

}  // namespace hv
