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
#include <cmath>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kSorThreads = 1024;
constexpr long long kMaxSpin = 1ll << 24;  // polls before a wait gives up (~1 s)

template <typename T, typename S>
struct SorArgs {
    int nx, ny, nz, nz2, P, R, bxn, byn, nblocks, src_smem, vec4;
    S hx2i, hy2i, hz2i, inv_diag, omega;
    double dhx2i, dhy2i, dhz2i, ddiag, src_c;
    double tol;
    int max_iter, criterion, inner_min, inner_max, extrapolate;
    const T *rho;
    double *phi64, *phi64_prev;
    S *delta, *src;         // global mirrors, [x][colour][y][nz2]
    double *partials;       // [nblocks][4]: rr, bb, max|ddelta|, -
    unsigned *phase;        // [nblocks]
    unsigned *bar;          // [0] arrivals, [1] generation
    int *status;            // [0] error, [1] iterations, [2] converged, [3] cycles
    double *metric;
    int *ctl;               // [0] step counter, [1] m hint, [2] previous-phi valid
    int *its_ring;          // per-step iterations, indexed by step % ring
    int ring;
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
__device__ bool grid_barrier(unsigned *bar, int nblocks, int *err) {
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
                if (++spin > kMaxSpin || ld_volatile(err)) {
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
                if (++spin > kMaxSpin || ld_volatile(a.status)) {
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
// (include/physics.hpp:114-125) applied to the correction.
template <typename S, typename T>
__device__ __forceinline__ S sor_update(const SorArgs<T, S> &a, S self, S xs, S ys, S zs, S s, bool valid) {
    const S star = (xs * a.hx2i + ys * a.hy2i + zs * a.hz2i + s) * a.inv_diag;
    return valid ? self + a.omega * (star - self) : self;
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

template <typename T, typename S>
__global__ void __launch_bounds__(kSorThreads, 1) k_sor_fast(SorArgs<T, S> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_tot[3];
    __shared__ int s_m;

    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
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
    // residual and fold: thread -> z position k_own, rows rz_start, +zrows_step
    const int zrows_step = max(1, nth / nz);
    const int rz_start = tid / nz;
    const int k_own = rz_start < zrows_step ? tid % nz : nz;
    const int jz_start = rz_start % nr, pz_start = rz_start / nr, djz = zrows_step % nr, dpz = zrows_step / nr;

    // ---- entry: zero delta (shared and own global mirror) -----------------
    for (int e = tid; e < own; e += nth) sd[e] = S(0);
    for (int p = 0; p < np; p++)
        for (int c = 0; c < 2; c++)
            for (int e = tid; e < hp; e += nth) a.delta[B.mirror(x0 + p, c, y0) + e] = S(0);
    const int step = a.ctl[0];
    const bool extrap = a.extrapolate && a.ctl[2];
    if (a.extrapolate) {
        for (int e = tid; e < np * nr * nz; e += nth) {
            int k = e % nz, l = e / nz, j = l % nr, p = l / nr;
            int x = x0 + p, y = y0 + j;
            if (y < 1 || y > ny - 2 || k < 1 || k > nz - 2) continue;
            long long id = x * sxy + (long long)y * nz + k;
            double cur = a.phi64[id];
            if (extrap) a.phi64[id] = 2.0 * cur - a.phi64_prev[id];
            a.phi64_prev[id] = cur;
        }
    }

    int its = 0, m_prev = 0, cycles = 0, m = max(a.inner_min, min(a.inner_max, a.ctl[1]));
    double rel_prev = -1.0, rel = 0.0, maxd = 0.0;
    bool converged = false;
    S last_max = S(0);

    while (true) {
        if (its > 0) {
            S bm = block_max<S>(last_max);
            if (tid == 0) a.partials[4 * b + 2] = (double)bm;
        }
        // delta of every block is final in global memory after this barrier
        if (!grid_barrier(a.bar, a.nblocks, err)) return;

        // ---- double residual of phi + delta on own interior nodes -------
        double rr = 0.0, bb = 0.0;
        const int k = k_own;
        for (int l = rz_start, j = jz_start, p = pz_start; k >= 1 && k <= nz - 2 && l < np * nr;
             l += zrows_step, j += djz, p += dpz) {
            if (j >= nr) {
                j -= nr;
                p++;
            }
            const int x = x0 + p, y = y0 + j;
            if (y < 1 || y > ny - 2) continue;
            const long long id = x * sxy + (long long)y * nz + k;
            const int kh = k >> 1, c0 = (x + y + k) & 1, c1 = c0 ^ 1;
            // own values from shared memory, other blocks' from their mirrors
            // (zero on the Dirichlet planes and rows)
            double dc = (double)SD(p, c0, j, kh);
            double dzm = (double)SD(p, c1, j, (k - 1) >> 1), dzp = (double)SD(p, c1, j, (k + 1) >> 1);
            double dxm = p > 0 ? (double)SD(p - 1, c1, j, kh) : (double)__ldcg(a.delta + B.mirror(x - 1, c1, y) + kh);
            double dxp =
                p + 1 < np ? (double)SD(p + 1, c1, j, kh) : (double)__ldcg(a.delta + B.mirror(x + 1, c1, y) + kh);
            double dym = j > 0 ? (double)SD(p, c1, j - 1, kh) : (double)__ldcg(a.delta + B.mirror(x, c1, y - 1) + kh);
            double dyp =
                j + 1 < nr ? (double)SD(p, c1, j + 1, kh) : (double)__ldcg(a.delta + B.mirror(x, c1, y + 1) + kh);
            double pc = __ldcg(a.phi64 + id) + dc;
            double pxm = __ldcg(a.phi64 + id - sxy) + dxm;
            double pxp = __ldcg(a.phi64 + id + sxy) + dxp;
            double pym = __ldcg(a.phi64 + id - nz) + dym;
            double pyp = __ldcg(a.phi64 + id + nz) + dyp;
            double pzm = __ldcg(a.phi64 + id - 1) + dzm;
            double pzp = __ldcg(a.phi64 + id + 1) + dzp;
            double bv = a.src_c * (double)__ldg(a.rho + id);
            double r = bv + (pxp + pxm) * a.dhx2i + (pyp + pym) * a.dhy2i + (pzp + pzm) * a.dhz2i - a.ddiag * pc;
            rr += r * r;
            bb += bv * bv;
            if (ss) ss[((p * 2 + c0) * nr + j) * nz2 + kh] = (S)r;
            else a.src[B.mirror(x, c0, y) + kh] = (S)r;
        }
        block_sum2(rr, bb);
        if (tid == 0) {
            a.partials[4 * b + 0] = rr;
            a.partials[4 * b + 1] = bb;
        }
        if (!grid_barrier(a.bar, a.nblocks, err)) return;

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

        // ---- fold: phi += delta, delta = 0 -------------------------------
        for (int l = rz_start, j = jz_start, p = pz_start; k >= 1 && k <= nz - 2 && l < np * nr;
             l += zrows_step, j += djz, p += dpz) {
            if (j >= nr) {
                j -= nr;
                p++;
            }
            const int x = x0 + p, y = y0 + j;
            if (y < 1 || y > ny - 2) continue;
            const long long id = x * sxy + (long long)y * nz + k;
            a.phi64[id] += (double)SD(p, (x + y + k) & 1, j, k >> 1);
        }
        __syncthreads();
        for (int e = tid; e < own; e += nth) sd[e] = S(0);
        for (int p = 0; p < np; p++)
            for (int c = 0; c < 2; c++)
                for (int e = tid; e < hp; e += nth) a.delta[B.mirror(x0 + p, c, y0) + e] = S(0);

        if (a.criterion == HV_SOR_REL_RESIDUAL) converged = rel <= a.tol;
        else converged = its > 0 && maxd < a.tol;
        if (converged || its >= a.max_iter || !(rel == rel)) break;

        // ---- next inner cycle length: predicted from the observed rate ---
        if (tid == 0) {
            int mm = m;
            if (a.criterion == HV_SOR_REL_RESIDUAL && rel_prev > 0.0 && rel < rel_prev && m_prev > 0) {
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
        publish(a.phase + b, ++my_phase);

        // ---- m red+black iterations on delta ------------------------------
        last_max = S(0);
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
        a.ctl[1] = max(m, a.inner_min);
        if (a.extrapolate) a.ctl[2] = 1;
        if (a.its_ring) a.its_ring[step % a.ring] = converged ? its : -its;
    }
}

}  // namespace

template <typename S>
static hv_status plan_for(hv_ctx *c) {
    SorFast &f = c->fused.sor;
    const Geom &g = c->geom;
    cudaDeviceProp prop;
    HV_CUDA(cudaGetDeviceProperties(&prop, c->device));
    const size_t static_smem = 2048;
    const size_t limit = prop.sharedMemPerBlockOptin > static_smem ? prop.sharedMemPerBlockOptin - static_smem : 0;
    const int nz2 = (g.nz + 1) / 2;
    const int interior = g.nx - 2;
    f.ok = false;
    // smallest blocks first (most parallel), the source in shared memory when
    // it fits, a y split only when a plane does not fit
    for (int pass = 0; pass < 2 && !f.ok; pass++) {
        const bool with_src = pass == 0;
        for (int R = g.ny; R >= 1 && !f.ok; R = (R == 1) ? 0 : (R + 1) / 2) {
            for (int P = 1; P <= interior; P++) {
                const size_t own = (size_t)P * 2 * R * nz2;
                const size_t smem = sizeof(S) * own * (with_src ? 2 : 1);
                if (smem > limit) break;
                const int bxn = (interior + P - 1) / P, byn = (g.ny + R - 1) / R;
                if ((long long)bxn * byn > prop.multiProcessorCount) continue;
                f.P = P;
                f.R = R;
                f.bx = bxn;
                f.by = byn;
                f.nblocks = bxn * byn;
                f.smem = smem;
                f.src_smem = with_src;
                f.ok = true;
                break;
            }
        }
    }
    if (!f.ok) return HV_OK;  // the fused path reports HV_ERR_UNSUPPORTED
    f.nz2 = nz2;
    f.threads = kSorThreads;
    auto kern = c->prec == HV_F64 ? (const void *)k_sor_fast<double, double> : (const void *)k_sor_fast<float, float>;
    HV_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.smem));
    int per_sm = 0;
    HV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, f.threads, f.smem));
    if (per_sm < 1 || (long long)per_sm * prop.multiProcessorCount < f.nblocks) {
        f.ok = false;
        return HV_OK;
    }
    // mirrors cover every plane and row, so the Dirichlet ones stay zero
    const size_t n = (size_t)g.nx * 2 * g.ny * nz2;
    HV_CUDA(cudaMalloc(&f.delta, n * sizeof(S)));
    HV_CUDA(cudaMalloc(&f.src, n * sizeof(S)));
    HV_CUDA(cudaMemsetAsync(f.delta, 0, n * sizeof(S), c->stream));
    HV_CUDA(cudaMemsetAsync(f.src, 0, n * sizeof(S), c->stream));
    HV_CUDA(cudaMalloc((void **)&f.partials, sizeof(double) * 4 * f.nblocks));
    HV_CUDA(cudaMemsetAsync(f.partials, 0, sizeof(double) * 4 * f.nblocks, c->stream));
    HV_CUDA(cudaMalloc((void **)&f.phase, sizeof(unsigned) * (f.nblocks + 2)));
    f.bar = f.phase + f.nblocks;
    HV_CUDA(cudaMalloc((void **)&f.status, sizeof(int) * 8));
    HV_CUDA(cudaMalloc((void **)&f.metric, sizeof(double) * 2));
    HV_CUDA(cudaMemsetAsync(f.status, 0, sizeof(int) * 8, c->stream));
    return HV_OK;
}

hv_status sor_fast_plan(hv_ctx *c) {
    return c->prec == HV_F64 ? plan_for<double>(c) : plan_for<float>(c);
}

void sor_fast_release(hv_ctx *c) {
    SorFast &f = c->fused.sor;
    void *ptrs[] = {f.delta, f.src, f.partials, f.phase, f.status, f.metric};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    f = SorFast();
}

template <typename T>
hv_status sor_fast_launch(hv_ctx *c, const T *rho, int *ctl, int *its_ring, int ring) {
    using S = T;
    SorFast &f = c->fused.sor;
    const Geom &g = c->geom;
    const hv_sor_params &sp = c->params.sor;
    HV_CUDA(cudaMemsetAsync(f.phase, 0, sizeof(unsigned) * (f.nblocks + 2), c->stream));
    HV_CUDA(cudaMemsetAsync(f.status, 0, sizeof(int) * 4, c->stream));
    SorArgs<T, S> a;
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
    const double dx = 2.0 * g.dmx / g.nx, dy = 2.0 * g.dmy / g.ny, dz = 2.0 * g.dmz / g.nz;
    a.dhx2i = 1.0 / (dx * dx);
    a.dhy2i = 1.0 / (dy * dy);
    a.dhz2i = 1.0 / (dz * dz);
    a.ddiag = 2.0 * (a.dhx2i + a.dhy2i + a.dhz2i);
    a.hx2i = (S)a.dhx2i;
    a.hy2i = (S)a.dhy2i;
    a.hz2i = (S)a.dhz2i;
    a.inv_diag = (S)(1.0 / a.ddiag);
    a.omega = (S)sp.omega;
    a.src_c = 4.0 * kPi * kE2;
    a.tol = sp.tol;
    a.max_iter = sp.max_iter;
    a.criterion = sp.criterion;
    a.inner_min = c->fast.sor_inner_min;
    a.inner_max = c->fast.sor_inner_max;
    a.extrapolate = c->fast.sor_warm_start == HV_WARM_EXTRAPOLATE;
    a.rho = rho;
    a.phi64 = c->fused.phi64;
    a.phi64_prev = c->fused.phi64_prev;
    a.delta = reinterpret_cast<S *>(f.delta);
    a.src = reinterpret_cast<S *>(f.src);
    a.partials = f.partials;
    a.phase = f.phase;
    a.bar = f.bar;
    a.status = f.status;
    a.metric = f.metric;
    a.ctl = ctl;
    a.its_ring = its_ring;
    a.ring = ring;
    void *args[] = {&a};
    HV_CUDA(cudaLaunchCooperativeKernel((const void *)k_sor_fast<T, S>, dim3(f.nblocks), dim3(f.threads), args,
                                        f.smem, c->stream));
    return HV_OK;
}

template hv_status sor_fast_launch<float>(hv_ctx *, const float *, int *, int *, int);
template hv_status sor_fast_launch<double>(hv_ctx *, const double *, int *, int *, int);

}  // namespace hv
