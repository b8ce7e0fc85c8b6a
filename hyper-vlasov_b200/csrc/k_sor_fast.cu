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
// One launch per solve, cooperative so that all blocks are resident.  Block b
// owns P interior x-planes by R rows (all z) and keeps its delta in shared
// memory in a colour-split layout: each z-line is stored as its red half and
// its black half, so a colour sweep reads and writes unit-stride runs.  After
// each colour sweep a block publishes its updated values to global memory and
// bumps its phase counter; before the next sweep it waits only for its (up to
// four) neighbours' counters.  Grid-wide barriers are used only around the
// double residual.  Every wait is bounded: on timeout the block records an
// error word and returns, and the host reports HV_ERR_TIMEOUT.
#include <cmath>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kSorThreads = 1024;
constexpr long long kMaxSpin = 1ll << 23;  // ~0.5 s of polling before giving up

template <typename T, typename S>
struct SorArgs {
    int nx, ny, nz, nz2, P, R, bxn, byn, nblocks;
    S hx2i, hy2i, hz2i, inv_diag, omega;
    double dhx2i, dhy2i, dhz2i, ddiag, src_c;
    double tol;
    int max_iter, criterion, inner_min, inner_max, extrapolate;
    const T *rho;
    double *phi64, *phi64_prev;
    S *delta, *src;
    double *partials;       // [nblocks][4]: rr, bb, max|ddelta|, -
    unsigned *phase;        // [nblocks]
    unsigned *bar;          // [0] arrivals, [1] generation
    int *status;            // [0] error, [1] iterations, [2] converged
    double *metric;
    int *ctl;               // [0] step counter, [1] m hint, [2] previous-phi valid
    int *its_ring;          // per-step iterations, indexed by step % ring
    int ring;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// Grid barrier for co-resident blocks; false when a wait timed out or another
// block reported an error.
__device__ bool grid_barrier(unsigned *bar, int nblocks, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        unsigned gen = ld_acquire(bar + 1);
        __threadfence();
        unsigned arrived = atomicAdd(bar, 1u) + 1u;
        if (arrived == (unsigned)nblocks) {
            atomicExch(bar, 0u);
            __threadfence();
            st_release(bar + 1, gen + 1u);
        } else {
            long long spin = 0;
            while (ld_acquire(bar + 1) == gen) {
                if (++spin > kMaxSpin || ld_volatile(err)) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
}

// Waits until every neighbouring block has published `target` phases.
template <typename T, typename S>
__device__ bool wait_neighbours(const SorArgs<T, S> &a, int bx, int by, unsigned target) {
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        int nbs[4], n = 0;
        if (bx > 0) nbs[n++] = by * a.bxn + bx - 1;
        if (bx + 1 < a.bxn) nbs[n++] = by * a.bxn + bx + 1;
        if (by > 0) nbs[n++] = (by - 1) * a.bxn + bx;
        if (by + 1 < a.byn) nbs[n++] = (by + 1) * a.bxn + bx;
        for (int q = 0; q < n && ok; q++) {
            long long spin = 0;
            while (ld_acquire(a.phase + nbs[q]) < target) {
                if (++spin > kMaxSpin || ld_volatile(a.status)) {
                    atomicExch(a.status, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
}

__device__ __forceinline__ void publish(unsigned *phase_slot, unsigned value) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(phase_slot, value);
    }
}

// Deterministic block sum of two doubles (fixed shuffle tree, fixed warp order).
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

template <typename T, typename S>
__global__ void __launch_bounds__(kSorThreads, 1) k_sor_fast(SorArgs<T, S> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S *sd = reinterpret_cast<S *>(smem_raw);
    __shared__ double s_tot[3];
    __shared__ int s_m;

    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const int bx = b % a.bxn, by = b / a.bxn;
    const int x0 = 1 + bx * a.P, x1 = min(x0 + a.P, a.nx - 1);
    const int y0 = by * a.R, y1 = min(y0 + a.R, a.ny);
    const int np = x1 - x0, nr = y1 - y0;
    const int nz = a.nz, ny = a.ny, nz2 = a.nz2, line = 2 * nz2;
    const long long sxy = (long long)ny * nz;
    const int own = np * nr * line;
    int *err = a.status;
    unsigned my_phase = 0;

    // ---- entry: zero delta, optional extrapolated start ------------------
    for (int e = tid; e < own; e += nth) sd[e] = S(0);
    for (int e = tid; e < own; e += nth) {
        int l = e / line, rem = e - l * line;
        int j = l % nr, p = l / nr;
        a.delta[((long long)(x0 + p) * ny + (y0 + j)) * line + rem] = S(0);
    }
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

    int its = 0, m_prev = 0, m = max(a.inner_min, min(a.inner_max, a.ctl[1]));
    double rel_prev = -1.0, rel = 0.0, maxd = 0.0;
    bool converged = false;
    S last_max = S(0);

    while (true) {
        // delta of every block is final in global memory after this barrier
        if (its > 0) {
            S bm = block_max<S>(last_max);
            if (tid == 0) a.partials[4 * b + 2] = (double)bm;
        }
        if (!grid_barrier(a.bar, a.nblocks, err)) return;

        // ---- double residual of phi + delta on own interior nodes -------
        double rr = 0.0, bb = 0.0;
        for (int e = tid; e < np * nr * nz; e += nth) {
            int k = e % nz, l = e / nz, j = l % nr, p = l / nr;
            int x = x0 + p, y = y0 + j;
            if (y < 1 || y > ny - 2 || k < 1 || k > nz - 2) continue;
            const long long id = x * sxy + (long long)y * nz + k;
            auto dl = [&](int xx, int yy, int kk) -> double {
                // delta at (xx,yy,kk): shared memory when owned, else global
                int c = (xx + yy + kk) & 1;
                if (xx >= x0 && xx < x1 && yy >= y0 && yy < y1)
                    return (double)sd[((xx - x0) * nr + (yy - y0)) * line + c * nz2 + (kk >> 1)];
                return (double)__ldcg(a.delta + ((long long)xx * ny + yy) * line + c * nz2 + (kk >> 1));
            };
            double pc = __ldcg(a.phi64 + id) + dl(x, y, k);
            double pxm = __ldcg(a.phi64 + id - sxy) + dl(x - 1, y, k);
            double pxp = __ldcg(a.phi64 + id + sxy) + dl(x + 1, y, k);
            double pym = __ldcg(a.phi64 + id - nz) + dl(x, y - 1, k);
            double pyp = __ldcg(a.phi64 + id + nz) + dl(x, y + 1, k);
            double pzm = __ldcg(a.phi64 + id - 1) + dl(x, y, k - 1);
            double pzp = __ldcg(a.phi64 + id + 1) + dl(x, y, k + 1);
            double bv = a.src_c * (double)__ldg(a.rho + id);
            double r = bv + (pxp + pxm) * a.dhx2i + (pyp + pym) * a.dhy2i + (pzp + pzm) * a.dhz2i - a.ddiag * pc;
            rr += r * r;
            bb += bv * bv;
            a.src[((long long)x * ny + y) * line + ((x + y + k) & 1) * nz2 + (k >> 1)] = (S)r;
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

        // ---- fold: phi += delta, delta = 0 -------------------------------
        for (int e = tid; e < np * nr * nz; e += nth) {
            int k = e % nz, l = e / nz, j = l % nr, p = l / nr;
            int x = x0 + p, y = y0 + j;
            if (y < 1 || y > ny - 2 || k < 1 || k > nz - 2) continue;
            const long long id = x * sxy + (long long)y * nz + k;
            S d = sd[(p * nr + j) * line + ((x + y + k) & 1) * nz2 + (k >> 1)];
            a.phi64[id] += (double)d;
        }
        __syncthreads();
        for (int e = tid; e < own; e += nth) {
            sd[e] = S(0);
            int l = e / line, rem = e - l * line;
            int j = l % nr, p = l / nr;
            a.delta[((long long)(x0 + p) * ny + (y0 + j)) * line + rem] = S(0);
        }

        if (a.criterion == HV_SOR_REL_RESIDUAL) converged = rel <= a.tol;
        else converged = its > 0 && maxd < a.tol;
        if (converged || its >= a.max_iter || !(rel == rel)) break;

        // ---- next inner cycle length: predicted from the observed rate ---
        if (tid == 0) {
            int mm = m;
            if (a.criterion == HV_SOR_REL_RESIDUAL && rel_prev > 0.0 && rel < rel_prev && m_prev > 0) {
                double q = pow(rel / rel_prev, 1.0 / m_prev);
                double pred = log(a.tol / rel) / log(q);
                mm = (int)ceil(pred);
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
                const int cp = c ^ 1;
                const bool track = (it == m - 1);
                for (int e = tid; e < np * nr * nz2; e += nth) {
                    const int t = e % nz2, l = e / nz2, j = l % nr, p = l / nr;
                    const int x = x0 + p, y = y0 + j;
                    if (y < 1 || y > ny - 2) continue;
                    const int k = ((c - x - y) & 1) + 2 * t;
                    if (k < 1 || k > nz - 2) continue;
                    const int base = (p * nr + j) * line;
                    const int kk = k >> 1;
                    const S self = sd[base + c * nz2 + t];
                    const S zm = sd[base + cp * nz2 + ((k - 1) >> 1)];
                    const S zp = sd[base + cp * nz2 + ((k + 1) >> 1)];
                    S ym, yp, xm, xp;
                    if (y - 1 == 0) ym = S(0);
                    else if (j > 0) ym = sd[base - line + cp * nz2 + kk];
                    else ym = __ldcg(a.delta + ((long long)x * ny + y - 1) * line + cp * nz2 + kk);
                    if (y + 1 == ny - 1) yp = S(0);
                    else if (j + 1 < nr) yp = sd[base + line + cp * nz2 + kk];
                    else yp = __ldcg(a.delta + ((long long)x * ny + y + 1) * line + cp * nz2 + kk);
                    if (x - 1 == 0) xm = S(0);
                    else if (p > 0) xm = sd[base - nr * line + cp * nz2 + kk];
                    else xm = __ldcg(a.delta + ((long long)(x - 1) * ny + y) * line + cp * nz2 + kk);
                    if (x + 1 == a.nx - 1) xp = S(0);
                    else if (p + 1 < np) xp = sd[base + nr * line + cp * nz2 + kk];
                    else xp = __ldcg(a.delta + ((long long)(x + 1) * ny + y) * line + cp * nz2 + kk);
                    const long long gi = ((long long)x * ny + y) * line + c * nz2 + t;
                    const S s = a.src[gi];
                    const S star = ((xm + xp) * a.hx2i + (ym + yp) * a.hy2i + (zm + zp) * a.hz2i + s) * a.inv_diag;
                    const S nv = self + a.omega * (star - self);
                    sd[base + c * nz2 + t] = nv;
                    a.delta[gi] = nv;
                    if (track) last_max = fmax(last_max, fabs(nv - self));
                }
                publish(a.phase + b, ++my_phase);
            }
        }
        its += m;
    }

    if (b == 0 && tid == 0) {
        a.status[1] = its;
        a.status[2] = converged ? 1 : 0;
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
    const size_t line = 2 * (size_t)nz2 * sizeof(S);
    const int interior = g.nx - 2;
    f.ok = false;
    for (int R = g.ny; R >= 1 && !f.ok; R = (R + 1) / 2 == R ? 0 : (R + 1) / 2) {
        for (int P = 1; P <= interior; P++) {
            const size_t smem = (size_t)P * R * line;
            if (smem > limit) break;
            const int bxn = (interior + P - 1) / P, byn = (g.ny + R - 1) / R;
            if ((long long)bxn * byn > prop.multiProcessorCount) continue;
            f.P = P;
            f.R = R;
            f.bx = bxn;
            f.by = byn;
            f.nblocks = bxn * byn;
            f.smem = smem;
            f.ok = true;
            break;
        }
        if (R == 1) break;
    }
    if (!f.ok) return HV_OK;  // the fused path falls back to the plain SOR
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
    const size_t n = (size_t)g.nx * g.ny * 2 * nz2;
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
    HV_CUDA(cudaMemsetAsync(f.status, 0, sizeof(int) * 3, c->stream));
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
