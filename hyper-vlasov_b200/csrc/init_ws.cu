// Woods-Saxon self-consistent initialisation of the test particles,
// initialize_particles (include/physics.hpp:34-97), on the device.
//
// One pass of the reference's loop, each step here a device phase:
//   1. 2M temporary particles (M = max_test_part per species): positions and
//      then momenta drawn in the cube and kept inside the balls r_max and k_max
//      (generate_random_particles, include/tools.hpp:234-254);
//   2. their energies (compute_energy, tools.hpp:205-224) counted against the
//      Fermi levels and eps +- 0.5 (physics.hpp:46-62), and the host's update of
//      the levels (physics.hpp:63-72);
//   3. the particles of the run drawn as (r, k) pairs in the cube, kept when
//      their energy lies below the level of the species being filled, and
//      stored with their mirror (-r, -k) (generate_checking_particles,
//      tools.hpp:256-281);
//   4. their densities (compute_particle_densities, pdens.cu);
//   5. the Woods-Saxon fit of each species (minim_woods_saxon,
//      include/fit_algorithm.hpp:95-137) and the relaxation (relax_woods_saxon,
//      tools.hpp:368-375).
//
// Rejection sampling runs as batches of candidates: a kernel tests every
// candidate of a batch, a scan numbers the accepted ones in candidate order,
// and a second kernel stores the first `need` of them -- exactly the ones a
// sequential loop would keep.  The uniform numbers come either from the C
// library's rand(), drawn on the host in the reference's order (HV_RNG_LIBC:
// batches never hold more candidates than are still needed, so no number
// past the reference's last one is drawn and the stream continues as the
// reference's would), or from Philox4x32-10 on the device (HV_RNG_PHILOX).
//
// The fit: the reference calls GSL's trust-region least-squares driver, which
// is not available here.  It is restated as Levenberg-Marquardt (Madsen,
// Nielsen and Tingleff 2004, algorithm 3.16) with More's scaling and the step
// and gradient tests of GSL's manual (xtol = gtol = 1e-4, at most 100
// iterations, as fit_algorithm.hpp:125 passes them; the relative-decrease test
// on ftol is not applied, so a fit runs until its step or gradient is small);
// each iteration is one
// pass over the species' particles that forms f^T f, J^T J and J^T f in double
// with a deterministic two-level reduction.  The residuals and Jacobian rows
// are evaluated in the context's precision from parameters rounded to it, as
// woods_saxon_f / woods_saxon_df do (fit_algorithm.hpp:49-94).
//
// Compiled with --fmad=false: the energies, the sampling arithmetic and the
// residuals keep the reference's operation order without contraction, so in
// double the kept candidates are the reference's.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kBlock = 256;
constexpr long long kBatchCap = 1ll << 23;      // candidates per batch (flags and positions: 64 MB)
constexpr long long kBatchCapLibc = 1ll << 20;  // HV_RNG_LIBC: 6 rand() values each, pinned on the host
constexpr long long kGiveUp = 1ll << 28;       // candidates drawn in a row, none kept, before giving up

// ---- uniform numbers -----------------------------------------------------

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): ten rounds of two 32-bit multiplies with the
// Weyl-sequence key schedule.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

struct Source {
    const int *raw;     // HV_RNG_LIBC: rand() values, kU per candidate; null: Philox
    uint2 key;          // Philox key (the seed)
    unsigned stream;    // Philox stream: pass << 2 | purpose
    long long c0;       // stream index of the batch's first candidate
};

template <typename T>
__device__ __forceinline__ T unit_philox(unsigned u);
template <>
__device__ __forceinline__ double unit_philox<double>(unsigned u) {
    return (double)u * 0x1.0p-32;
}
template <>
__device__ __forceinline__ float unit_philox<float>(unsigned u) {
    return (float)(u >> 8) * 0x1.0p-24f;
}

// kU values rand_val(-m_j, m_j) (include/math_functions.hpp:29-40) of
// candidate i of the batch: min + s (max - min), s = rand() / RAND_MAX.
template <typename T, int kU>
__device__ __forceinline__ void draw(const Source &s, long long i, T rand_max, const T (&m)[kU], T (&v)[kU]) {
    T u[kU];
    if (s.raw) {
#pragma unroll
        for (int j = 0; j < kU; j++) u[j] = (T)s.raw[i * kU + j] / rand_max;
    } else {
        const unsigned long long c = (unsigned long long)(s.c0 + i);
        const uint2 k = s.key;
        const uint4 a = philox(make_uint4((unsigned)c, (unsigned)(c >> 32), s.stream, 0u), k);
        unsigned w[8] = {a.x, a.y, a.z, a.w, 0u, 0u, 0u, 0u};
        if (kU > 4) {
            const uint4 b = philox(make_uint4((unsigned)c, (unsigned)(c >> 32), s.stream, 1u), k);
            w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
        }
#pragma unroll
        for (int j = 0; j < kU; j++) u[j] = unit_philox<T>(w[j]);
    }
#pragma unroll
    for (int j = 0; j < kU; j++) v[j] = -m[j] + u[j] * (m[j] - -m[j]);
}

// ---- energies ------------------------------------------------------------

template <typename T>
struct EnergyConst {
    T ekin, efluc, zc;       // kinetic_energy<T>(), fluctuation_energy(sigma_k), Z
    T V0[2], R12[2], a[2];   // Woods-Saxon of protons, neutrons
};

// compute_energy (include/tools.hpp:205-224) of a particle of species sp.
template <typename T>
__device__ __forceinline__ T energy_of(const EnergyConst<T> &c, int sp, T x, T y, T z, T kx, T ky, T kz) {
    const T r = sqrt(x * x + y * y + z * z), k = sqrt(kx * kx + ky * ky + kz * kz);
    T e = T(0);
    e += c.V0[sp] / (T(1) + exp((r - c.R12[sp]) / c.a[sp]));  // physics_formulas.hpp:64-68
    e += (k * k) * c.ekin;
    if (sp == 0) {  // coulomb_potential, physics_formulas.hpp:79-84
        const T R = c.R12[0];
        if (r <= R) e += T(1.44) * (c.zc - T(1)) / R * (T(1.5) - T(0.5) * (r / R) * (r / R));
        else e += T(1.44) * (c.zc - T(1)) / r;
    }
    e += c.efluc;
    return e;
}

// ---- candidates ----------------------------------------------------------

template <typename T>
struct Test {
    T m[6];       // half-widths of the cube: r_max (x3) or k_max (x3) for the balls; r_max x3, k_max x3 for pairs
    T m2;         // balls: m^2
    EnergyConst<T> ec;
    int sp;       // pairs: the species being filled
    T eps;        // pairs: its Fermi level
    T rand_max;
};

// kKind 0: a vector kept inside the ball (tools.hpp:238-242); 1: an (r, k)
// pair kept below the Fermi level (tools.hpp:266-280).
template <typename T, int kKind>
__device__ __forceinline__ bool candidate(const Source &s, long long i, const Test<T> &t, T (&v)[6]) {
    if (kKind == 0) {
        T w[3];
        const T m[3] = {t.m[0], t.m[1], t.m[2]};
        draw<T, 3>(s, i, t.rand_max, m, w);
        v[0] = w[0]; v[1] = w[1]; v[2] = w[2];
        return w[0] * w[0] + w[1] * w[1] + w[2] * w[2] < t.m2;
    } else {
        draw<T, 6>(s, i, t.rand_max, t.m, v);
        return energy_of<T>(t.ec, t.sp, v[0], v[1], v[2], v[3], v[4], v[5]) < t.eps;
    }
}

template <typename T, int kKind>
__global__ void k_flags(int k, Source s, Test<T> t, int *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    T v[6];
    flag[i] = candidate<T, kKind>(s, i, t, v) ? 1 : 0;
}

struct Out {
    void *o[6];
    long long base;     // first output element (balls) or pair (pairs) of this batch
};

// Stores the accepted candidates numbered below `need`; res[0] = accepted in
// the batch, res[1] = batch index of the need-th accepted one.
template <typename T, int kKind>
__global__ void k_store(int k, Source s, Test<T> t, const int *__restrict__ flag, const int *__restrict__ pos,
                        long long need, Out out, int *res) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    if (i == k - 1) res[0] = pos[i] + flag[i];
    if (!flag[i]) return;
    const int p = pos[i];
    if (p >= need) return;
    if (p == need - 1) res[1] = i;
    T v[6];
    candidate<T, kKind>(s, i, t, v);
    if (kKind == 0) {
        const long long o = out.base + p;
        for (int j = 0; j < 3; j++) ((T *)out.o[j])[o] = v[j];
    } else {
        const long long o = 2 * (out.base + p);  // the pair fills particles o and o + 1
        for (int j = 0; j < 6; j++) {
            ((T *)out.o[j])[o] = v[j];
            ((T *)out.o[j])[o + 1] = v[j] * T(-1);  // mult_vec(v, v, -1)
        }
    }
}

// Counts of the temporary particles below eps, eps + 0.5 and eps - 0.5 per
// species (physics.hpp:46-62): cnt = {equal, more, less} x {protons, neutrons}.
template <typename T>
__global__ void k_level_counts(int M, EnergyConst<T> ec, const T *__restrict__ x, const T *__restrict__ y,
                               const T *__restrict__ z, const T *__restrict__ kx, const T *__restrict__ ky,
                               const T *__restrict__ kz, T eps_p, T eps_n, T hi_p, T hi_n, T lo_p, T lo_n,
                               unsigned long long *cnt) {
    unsigned c[6] = {0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * M; i += gridDim.x * blockDim.x) {
        const int sp = i < M ? 0 : 1;
        const T e = energy_of<T>(ec, sp, x[i], y[i], z[i], kx[i], ky[i], kz[i]);
        const T eq = sp ? eps_n : eps_p, hi = sp ? hi_n : hi_p, lo = sp ? lo_n : lo_p;
        c[3 * sp] += e < eq;
        c[3 * sp + 1] += e < hi;
        c[3 * sp + 2] += e < lo;
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const unsigned w = __reduce_add_sync(0xffffffffu, c[q]);
        if ((threadIdx.x & 31) == 0 && w) atomicAdd(cnt + q, (unsigned long long)w);
    }
}

// compute_particle_energies (tools.hpp:226-232) of N particles, species by index.
template <typename T>
__global__ void k_energies(int N, int protons, EnergyConst<T> ec, const T *__restrict__ x, const T *__restrict__ y,
                           const T *__restrict__ z, const T *__restrict__ kx, const T *__restrict__ ky,
                           const T *__restrict__ kz, T *__restrict__ e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    e[i] = energy_of<T>(ec, i < protons ? 0 : 1, x[i], y[i], z[i], kx[i], ky[i], kz[i]);
}

// ---- the fit ---------------------------------------------------------------

// r_i = |r_i| and v_i = skyrme_potential of the particle's densities
// (include/physics_formulas.hpp:70-77), the fit's fixed inputs.
template <typename T>
__global__ void k_fit_inputs(int N, int protons, T A, T B, T C, T gam, const T *__restrict__ x,
                             const T *__restrict__ y, const T *__restrict__ z, const T *__restrict__ dp,
                             const T *__restrict__ dn, T *__restrict__ r, T *__restrict__ vs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    r[i] = sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
    const T tau = i < protons ? T(-1) : T(1);
    const T rho = dp[i] + dn[i], t = rho / T(0.16);
    vs[i] = A * t + B * pow(t, gam) + T(2) * tau * C * ((dn[i] - dp[i]) / T(0.16));
}

constexpr int kSums = 10;  // f^T f, J^T J (00 01 02 11 12 22), J^T f

// Per-block sums of the fit at (V0, R12, a) over n particles; fixed order.
template <typename T>
__global__ void k_fit_sums(int n, const T *__restrict__ r, const T *__restrict__ vs, double V0d, double R12d,
                           double ad, double *__restrict__ partials) {
    const T V0 = (T)V0d, R12 = (T)R12d, a = (T)ad;
    double s[kSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T e = exp((r[i] - R12) / a);
        const T f = vs[i] - V0 / (T(1) + e);
        const T e2 = (T(1) + e) * (T(1) + e);
        const double j0 = (double)(-T(1) / (T(1) + e));
        const double j1 = (double)(-(V0 * e) / (a * e2));
        const double j2 = (double)(-(V0 * (r[i] - R12) * e) / (a * a * e2));
        const double fd = (double)f;
        s[0] += fd * fd;
        s[1] += j0 * j0; s[2] += j0 * j1; s[3] += j0 * j2;
        s[4] += j1 * j1; s[5] += j1 * j2; s[6] += j2 * j2;
        s[7] += j0 * fd; s[8] += j1 * fd; s[9] += j2 * fd;
    }
    __shared__ double sh[kSums][kBlock];
#pragma unroll
    for (int q = 0; q < kSums; q++) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
#pragma unroll
            for (int q = 0; q < kSums; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < kSums) partials[blockIdx.x * kSums + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_fit_total(int nb, const double *__restrict__ partials, double *__restrict__ out) {
    const int q = threadIdx.x;
    if (q >= kSums) return;
    double v = 0.0;
    for (int b = 0; b < nb; b++) v += partials[b * kSums + q];
    out[q] = v;
}

// ---- host side ---------------------------------------------------------------

template <typename T>
struct Work {
    hv_ctx *c = nullptr;
    cudaStream_t s = nullptr;
    int kind = HV_RNG_PHILOX;
    uint2 key{0, 0};
    long long drawn = 0;
    // sampling
    long long cap = 0;
    int *flag = nullptr, *pos = nullptr, *res = nullptr, *h_res = nullptr;
    int *raw = nullptr, *h_raw = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    // particles (caller order) and fit inputs
    T *p[6] = {}, *tmp[6] = {};
    T *dp = nullptr, *dn = nullptr, *r = nullptr, *vs = nullptr;
    unsigned long long *cnt = nullptr;
    double *partials = nullptr, *sums = nullptr, *h_sums = nullptr;
    int fit_blocks = 0;

    ~Work() {
        void *dev[] = {flag, pos, res, raw, scan_tmp, dp, dn, r, vs, cnt, partials, sums,
                       p[0], p[1], p[2], p[3], p[4], p[5], tmp[0], tmp[1], tmp[2], tmp[3], tmp[4], tmp[5]};
        for (void *q : dev)
            if (q) cudaFreeAsync(q, s);
        if (h_res) cudaFreeHost(h_res);
        if (h_raw) cudaFreeHost(h_raw);
        if (h_sums) cudaFreeHost(h_sums);
        if (s) cudaStreamSynchronize(s);
    }

    hv_status alloc_sampling(long long cap_) {
        cap = cap_;
        HV_CUDA(cudaMallocAsync((void **)&flag, sizeof(int) * cap, s));
        HV_CUDA(cudaMallocAsync((void **)&pos, sizeof(int) * cap, s));
        HV_CUDA(cudaMallocAsync((void **)&res, sizeof(int) * 2, s));
        HV_CUDA(cudaMallocHost((void **)&h_res, sizeof(int) * 2));
        HV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flag, pos, (int)cap, s));
        HV_CUDA(cudaMallocAsync(&scan_tmp, scan_bytes, s));
        if (kind == HV_RNG_LIBC) {
            HV_CUDA(cudaMallocAsync((void **)&raw, sizeof(int) * 6 * cap, s));
            HV_CUDA(cudaMallocHost((void **)&h_raw, sizeof(int) * 6 * cap));
        }
        return HV_OK;
    }

    hv_status alloc_fit(int N) {
        HV_CUDA(cudaMallocAsync((void **)&dp, sizeof(T) * std::max(N, 1), s));
        HV_CUDA(cudaMallocAsync((void **)&dn, sizeof(T) * std::max(N, 1), s));
        HV_CUDA(cudaMallocAsync((void **)&r, sizeof(T) * std::max(N, 1), s));
        HV_CUDA(cudaMallocAsync((void **)&vs, sizeof(T) * std::max(N, 1), s));
        fit_blocks = std::max(1, std::min(div_up(std::max(N, 1), kBlock), 2 * c->sm_count));
        HV_CUDA(cudaMallocAsync((void **)&partials, sizeof(double) * kSums * fit_blocks, s));
        HV_CUDA(cudaMallocAsync((void **)&sums, sizeof(double) * kSums, s));
        HV_CUDA(cudaMallocHost((void **)&h_sums, sizeof(double) * kSums));
        return HV_OK;
    }

    // Keeps the first `need` accepted candidates of the stream in `out`
    // (stream position *c0 on entry and exit).
    template <int kKind>
    hv_status sample(const Test<T> &t, unsigned stream, long long *c0, long long need, Out out) {
        constexpr int kU = kKind == 0 ? 3 : 6;
        double p_est = kKind == 0 ? 0.5236 : 0.05;
        long long dry = 0;  // candidates since the last kept one
        while (need > 0) {
            long long k;
            if (kind == HV_RNG_LIBC) k = std::min(need, cap);
            else k = std::min(cap, (long long)((double)need / p_est * 1.05) + 1024);
            Source src{nullptr, key, stream, *c0};
            if (kind == HV_RNG_LIBC) {
                for (long long q = 0; q < k * kU; q++) h_raw[q] = std::rand();
                HV_CUDA(cudaMemcpyAsync(raw, h_raw, sizeof(int) * k * kU, cudaMemcpyHostToDevice, s));
                src.raw = raw;
            }
            k_flags<T, kKind><<<div_up(k, kBlock), kBlock, 0, s>>>((int)k, src, t, flag);
            HV_CUDA(cudaGetLastError());
            HV_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flag, pos, (int)k, s));
            k_store<T, kKind><<<div_up(k, kBlock), kBlock, 0, s>>>((int)k, src, t, flag, pos, need, out, res);
            HV_CUDA(cudaGetLastError());
            HV_CUDA(cudaMemcpyAsync(h_res, res, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
            HV_CUDA(cudaStreamSynchronize(s));
            const long long acc = h_res[0];
            const long long used = acc >= need ? (long long)h_res[1] + 1 : k;
            const long long taken = std::min(acc, need);
            *c0 += used;
            drawn += used;
            need -= taken;
            out.base += taken;
            if (acc > 0) {
                p_est = std::max((double)acc / (double)k, 1e-7);
                dry = 0;
            } else {
                p_est = std::max(p_est / 8.0, 1e-9);
                // the reference's loop would never end (tools.hpp:262-281)
                if ((dry += k) >= kGiveUp) return HV_ERR_NOT_CONVERGED;
            }
        }
        return HV_OK;
    }

    hv_status fit_sums(int n, const T *rr, const T *vv, const double *x, double *out) {
        k_fit_sums<T><<<fit_blocks, kBlock, 0, s>>>(n, rr, vv, x[0], x[1], x[2], partials);
        k_fit_total<<<1, 32, 0, s>>>(fit_blocks, partials, sums);
        HV_CUDA(cudaGetLastError());
        HV_CUDA(cudaMemcpyAsync(h_sums, sums, sizeof(double) * kSums, cudaMemcpyDeviceToHost, s));
        HV_CUDA(cudaStreamSynchronize(s));
        for (int q = 0; q < kSums; q++) out[q] = h_sums[q];
        return HV_OK;
    }

    // Levenberg-Marquardt fit of one species (n particles from rr / vv) from
    // x; see the file comment.  *status: 1 xtol, 2 gtol, 0 iterations
    // exhausted, -1 no acceptable step, -2 fewer than 3 particles.
    hv_status fit(int n, const T *rr, const T *vv, double x[3], int *iters, int *status) {
        const int kMaxIter = 100;
        const double xtol = 1e-4, gtol = 1e-4;
        *iters = 0;
        *status = -2;
        if (n < 3) return HV_OK;
        double sm[kSums], sn[kSums], D[3] = {0, 0, 0}, h[3];
        HV_TRY(fit_sums(n, rr, vv, x, sm));
        const int dg[3] = {1, 4, 6};
        for (int q = 0; q < 3; q++) D[q] = std::max(D[q], sm[dg[q]]);
        double mu = 1e-3, nu = 2.0;
        int st = 0, it;
        for (it = 1; it <= kMaxIter; it++) {
            // (J^T J + mu D) h = -J^T f: elimination with partial pivoting
            double M[3][4] = {{sm[1] + mu * D[0], sm[2], sm[3], -sm[7]},
                              {sm[2], sm[4] + mu * D[1], sm[5], -sm[8]},
                              {sm[3], sm[5], sm[6] + mu * D[2], -sm[9]}};
            bool singular = false;
            for (int col = 0; col < 3 && !singular; col++) {
                int pv = col;
                for (int q = col + 1; q < 3; q++)
                    if (std::fabs(M[q][col]) > std::fabs(M[pv][col])) pv = q;
                if (!(std::fabs(M[pv][col]) > 0.0)) {
                    singular = true;
                    break;
                }
                if (pv != col)
                    for (int q = 0; q < 4; q++) std::swap(M[col][q], M[pv][q]);
                for (int q = col + 1; q < 3; q++) {
                    const double m = M[q][col] / M[col][col];
                    for (int u = col; u < 4; u++) M[q][u] -= m * M[col][u];
                }
            }
            if (singular) {
                st = -1;
                break;
            }
            for (int q = 2; q >= 0; q--) {
                double v = M[q][3];
                for (int u = q + 1; u < 3; u++) v -= M[q][u] * h[u];
                h[q] = v / M[q][q];
            }
            const double xn[3] = {x[0] + h[0], x[1] + h[1], x[2] + h[2]};
            HV_TRY(fit_sums(n, rr, vv, xn, sn));
            const double pred = 0.5 * (mu * (D[0] * h[0] * h[0] + D[1] * h[1] * h[1] + D[2] * h[2] * h[2]) -
                                       (sm[7] * h[0] + sm[8] * h[1] + sm[9] * h[2]));
            const double rho = pred > 0.0 ? 0.5 * (sm[0] - sn[0]) / pred : -1.0;
            if (rho > 0.0 && std::isfinite(sn[0])) {
                for (int q = 0; q < 3; q++) x[q] = xn[q];
                for (int q = 0; q < kSums; q++) sm[q] = sn[q];
                for (int q = 0; q < 3; q++) D[q] = std::max(D[q], sm[dg[q]]);
                const double tt = 2.0 * rho - 1.0;
                mu *= std::max(1.0 / 3.0, 1.0 - tt * tt * tt);
                nu = 2.0;
                bool small_step = true;
                for (int q = 0; q < 3; q++) small_step = small_step && std::fabs(h[q]) <= xtol * (std::fabs(x[q]) + xtol);
                if (small_step) {
                    st = 1;
                    break;
                }
                double gm = 0.0;
                for (int q = 0; q < 3; q++) gm = std::max(gm, std::fabs(sm[7 + q]) * std::max(std::fabs(x[q]), 1.0));
                if (gm <= gtol * std::max(0.5 * sm[0], 1.0)) {
                    st = 2;
                    break;
                }
            } else {
                mu *= nu;
                nu *= 2.0;
                if (!(nu < 1e30)) {
                    st = -1;
                    break;
                }
            }
        }
        *iters = std::min(it, kMaxIter);
        *status = st;
        return HV_OK;
    }
};

template <typename T>
EnergyConst<T> energy_const(double sigma_k_d, int z, const T V0[2], const T R12[2], const T a[2]) {
    EnergyConst<T> e;
    const T hc2 = T(197.33) * T(197.33);
    e.ekin = hc2 / (T(2.0) * T(935.0));  // kinetic_energy (physics_formulas.hpp:34-38)
    const T sigma_k = T(sigma_k_d);
    e.efluc = T(3.0) * e.ekin * sigma_k * sigma_k;  // fluctuation_energy (physics_formulas.hpp:40-44)
    e.zc = T(z);
    for (int q = 0; q < 2; q++) {
        e.V0[q] = V0[q];
        e.R12[q] = R12[q];
        e.a[q] = a[q];
    }
    return e;
}

// nuclear_radius and max_particles (physics_formulas.hpp:27-32,47-53) in T.
template <typename T>
void init_sizes(int A, int ppn, T *r_max, int *max_part) {
    *r_max = T(1.5) * std::pow(T(A), T(1.0) / T(3.0));
    const T t = *r_max * T(1.5), ct = T(2.0) * T(kPi);
    const T psv = T(16.0) / T(9.0) * T(kPi) * T(kPi) * (t * t * t);
    *max_part = ppn * (int)std::floor(psv / (ct * ct * ct) + T(0.5));
}

template <typename T>
hv_status fit_species(Work<T> &w, int N, int protons, const T *const pos[3], const hv_skyrme &skm, T V0[2], T R12[2],
                      T a[2], int iters[2], int status[2]) {
    HV_TRY(particle_densities_at<T>(w.c, N, protons, pos[0], pos[1], pos[2], w.dp, w.dn));
    if (N > 0) {
        k_fit_inputs<T><<<div_up(N, kBlock), kBlock, 0, w.s>>>(N, protons, T(skm.A), T(skm.B), T(skm.C), T(skm.gamma),
                                                              pos[0], pos[1], pos[2], w.dp, w.dn, w.r, w.vs);
        HV_CUDA(cudaGetLastError());
    }
    for (int sp = 0; sp < 2; sp++) {
        const int start = sp == 0 ? 0 : protons, n = sp == 0 ? protons : N - protons;
        double x[3] = {(double)V0[sp], (double)R12[sp], (double)a[sp]};
        HV_TRY(w.fit(n, w.r + start, w.vs + start, x, &iters[sp], &status[sp]));
        V0[sp] = T(x[0]);
        R12[sp] = T(x[1]);
        a[sp] = T(x[2]);
    }
    return HV_OK;
}

template <typename T>
hv_status initialize(hv_ctx *c, const hv_skyrme &skm, hv_woods_saxon ws_io[2], hv_fermi *fermi,
                     const hv_init_params &ip, hv_init_report *rep, hv_init_row *rows) {
    const int Z = c->params.z, Nn = c->params.n, ppn = c->params.part_per_nucleon;
    const int total_p = c->protons, total_n = c->neutrons, total = c->total;
    if (Z < 0 || Nn < 0 || ppn <= 0 || total_p != Z * ppn || total_n != Nn * ppn || (total & 1) || Z + Nn <= 0)
        return HV_ERR_BAD_ARG;
    T r_max;
    int M;
    init_sizes<T>(Z + Nn, ppn, &r_max, &M);
    if (ip.r_max > 0.0) r_max = T(ip.r_max);
    if (ip.max_test_part > 0) M = ip.max_test_part;
    const int max_it = ip.max_iterations > 0 ? ip.max_iterations : 32;  // MAX_INIT_ITERATIONS
    const T k_max = T(1.5);                                               // k_max (sim_structs.hpp:31)

    Work<T> w;
    w.c = c;
    w.s = c->stream;
    w.kind = ip.rng;
    w.key = make_uint2((unsigned)ip.seed, (unsigned)(ip.seed >> 32));
    HV_TRY(w.alloc_sampling(ip.rng == HV_RNG_LIBC ? kBatchCapLibc : kBatchCap));
    HV_TRY(w.alloc_fit(total));
    for (int q = 0; q < 6; q++) {
        HV_CUDA(cudaMallocAsync((void **)&w.p[q], sizeof(T) * std::max(total, 1), w.s));
        HV_CUDA(cudaMallocAsync((void **)&w.tmp[q], sizeof(T) * std::max(2 * M, 1), w.s));
    }
    HV_CUDA(cudaMallocAsync((void **)&w.cnt, sizeof(unsigned long long) * 6, w.s));

    T V0[2], R12[2], a[2];
    for (int q = 0; q < 2; q++) {
        V0[q] = T(ws_io[q].V0);
        R12[q] = T(ws_io[q].R12);
        a[q] = T(ws_io[q].a);
    }
    T eps_p = T(fermi->epsilon_p), eps_n = T(fermi->epsilon_n);
    const T relax = T(0.6);
    T total_delta = T(0);
    int it = 0, fit_it[2] = {0, 0}, fit_st[2] = {0, 0};
    const int proton_pairs = (total_p + 1) / 2, pairs = total / 2;
    long long c_check = 0;
    do {
        const unsigned pass = (unsigned)it << 2;
        // 1. temporary particles: positions, then momenta
        Test<T> ball{};
        ball.rand_max = T(RAND_MAX);
        for (int q = 0; q < 3; q++) ball.m[q] = r_max;
        ball.m2 = r_max * r_max;
        long long c0 = 0;
        HV_TRY(w.template sample<0>(ball, pass | 0u, &c0, 2ll * M, Out{{w.tmp[0], w.tmp[1], w.tmp[2]}, 0}));
        for (int q = 0; q < 3; q++) ball.m[q] = k_max;
        ball.m2 = k_max * k_max;
        c0 = 0;
        HV_TRY(w.template sample<0>(ball, pass | 1u, &c0, 2ll * M, Out{{w.tmp[3], w.tmp[4], w.tmp[5]}, 0}));
        // 2. level counts and the Fermi-level update (physics.hpp:46-72)
        const EnergyConst<T> ec = energy_const<T>(ip.sigma_k, Z, V0, R12, a);
        HV_CUDA(cudaMemsetAsync(w.cnt, 0, sizeof(unsigned long long) * 6, w.s));
        if (M > 0) {
            const int nb = std::min(div_up(2ll * M, kBlock), 4 * c->sm_count);
            k_level_counts<T><<<nb, kBlock, 0, w.s>>>(M, ec, w.tmp[0], w.tmp[1], w.tmp[2], w.tmp[3], w.tmp[4],
                                                      w.tmp[5], eps_p, eps_n, eps_p + T(0.5), eps_n + T(0.5),
                                                      eps_p - T(0.5), eps_n - T(0.5), w.cnt);
            HV_CUDA(cudaGetLastError());
        }
        unsigned long long hc[6];
        HV_CUDA(cudaMemcpyAsync(hc, w.cnt, sizeof(hc), cudaMemcpyDeviceToHost, w.s));
        HV_CUDA(cudaStreamSynchronize(w.s));
        const int equal_p = 2 * (int)hc[0], more_p = 2 * (int)hc[1], less_p = 2 * (int)hc[2];
        const int equal_n = 2 * (int)hc[3], more_n = 2 * (int)hc[4], less_n = 2 * (int)hc[5];
        const T delta_part_n = total_n - equal_n;
        const T delta_part_p = total_p - equal_p;
        T delta_epsilon_n = T(0.5) * delta_part_n / (more_n - less_n);
        T delta_epsilon_p = T(0.5) * delta_part_p / (more_p - less_p);
        if (std::abs(delta_epsilon_p) > T(0.5)) delta_epsilon_p *= relax;
        if (std::abs(delta_epsilon_n) > T(0.5)) delta_epsilon_n *= relax;
        eps_p += delta_epsilon_p;
        eps_n += delta_epsilon_n;
        if (!std::isfinite((double)eps_p) || !std::isfinite((double)eps_n)) return HV_ERR_NOT_CONVERGED;
        // 3. the run's particles: proton pairs, then neutron pairs
        Test<T> pr{};
        pr.rand_max = T(RAND_MAX);
        for (int q = 0; q < 3; q++) {
            pr.m[q] = r_max;
            pr.m[3 + q] = k_max;
        }
        pr.ec = ec;
        pr.sp = 0;
        pr.eps = eps_p;
        c_check = 0;
        Out po{{w.p[0], w.p[1], w.p[2], w.p[3], w.p[4], w.p[5]}, 0};
        HV_TRY(w.template sample<1>(pr, pass | 2u, &c_check, proton_pairs, po));
        pr.sp = 1;
        pr.eps = eps_n;
        po.base = proton_pairs;
        HV_TRY(w.template sample<1>(pr, pass | 2u, &c_check, pairs - proton_pairs, po));
        // 4.-5. densities, fits, relaxation (tools.hpp:368-375)
        T V0o[2] = {V0[0], V0[1]}, R12o[2] = {R12[0], R12[1]}, ao[2] = {a[0], a[1]};
        const T *pos3[3] = {w.p[0], w.p[1], w.p[2]};
        HV_TRY(fit_species<T>(w, total, total_p, pos3, skm, V0, R12, a, fit_it, fit_st));
        for (int q = 0; q < 2; q++) {
            V0[q] = relax * V0[q] + (1.0 - relax) * V0o[q];
            R12[q] = relax * R12[q] + (1.0 - relax) * R12o[q];
            a[q] = relax * a[q] + (1.0 - relax) * ao[q];
        }
        total_delta = std::abs(delta_epsilon_n) + std::abs(delta_epsilon_p);
        if (rows) {
            hv_init_row &rw = rows[it];
            rw.equal_p = equal_p;
            rw.equal_n = equal_n;
            rw.epsilon_p = (double)eps_p;
            rw.epsilon_n = (double)eps_n;
            rw.delta_epsilon = (double)total_delta;
            for (int q = 0; q < 2; q++) {
                rw.ws[q].V0 = (double)V0[q];
                rw.ws[q].R12 = (double)R12[q];
                rw.ws[q].a = (double)a[q];
                rw.fit_iterations[q] = fit_it[q];
                rw.fit_status[q] = fit_st[q];
            }
        }
        it++;
    } while (total_delta > T(0.1) && it < max_it);  // delta_epsilon_tolerance (sim_structs.hpp:37)

    // chi_squared (tools.hpp:340-366) of the final particles and parameters
    double chi[2] = {0.0, 0.0};
    for (int sp = 0; sp < 2; sp++) {
        const int start = sp == 0 ? 0 : total_p, n = sp == 0 ? total_p : total_n;
        if (n == 0) continue;
        const double x[3] = {(double)V0[sp], (double)R12[sp], (double)a[sp]};
        double sm[kSums];
        HV_TRY(w.fit_sums(n, w.r + start, w.vs + start, x, sm));
        chi[sp] = sm[0] / ppn;
    }
    const T *src[6] = {w.p[0], w.p[1], w.p[2], w.p[3], w.p[4], w.p[5]};
    HV_TRY(store_particles<T>(c, src));
    HV_CUDA(cudaStreamSynchronize(w.s));

    for (int q = 0; q < 2; q++) {
        ws_io[q].V0 = (double)V0[q];
        ws_io[q].R12 = (double)R12[q];
        ws_io[q].a = (double)a[q];
    }
    fermi->epsilon_p = (double)eps_p;
    fermi->epsilon_n = (double)eps_n;
    if (rep) {
        rep->iterations = it;
        rep->converged = !(total_delta > T(0.1));
        rep->delta_epsilon = (double)total_delta;
        rep->chi_squared_p = chi[0];
        rep->chi_squared_n = chi[1];
        rep->candidates = w.drawn;
        rep->max_test_part = M;
        rep->r_max = (double)r_max;
    }
    return HV_OK;
}

template <typename T>
hv_status fit_context(hv_ctx *c, const hv_skyrme &skm, hv_woods_saxon ws_io[2], int iters[2], int status[2]) {
    Work<T> w;
    w.c = c;
    w.s = c->stream;
    HV_TRY(w.alloc_fit(c->total));
    State<T> &st = state<T>(c);
    T V0[2], R12[2], a[2];
    for (int q = 0; q < 2; q++) {
        V0[q] = T(ws_io[q].V0);
        R12[q] = T(ws_io[q].R12);
        a[q] = T(ws_io[q].a);
    }
    const T *pos3[3] = {st.x, st.y, st.z};
    HV_TRY(fit_species<T>(w, c->total, c->protons, pos3, skm, V0, R12, a, iters, status));
    for (int q = 0; q < 2; q++) {
        ws_io[q].V0 = (double)V0[q];
        ws_io[q].R12 = (double)R12[q];
        ws_io[q].a = (double)a[q];
    }
    return HV_OK;
}

template <typename T>
hv_status energies_context(hv_ctx *c, const hv_woods_saxon ws[2], double sigma_k, void *host) {
    T V0[2], R12[2], a[2];
    for (int q = 0; q < 2; q++) {
        V0[q] = T(ws[q].V0);
        R12[q] = T(ws[q].R12);
        a[q] = T(ws[q].a);
    }
    const EnergyConst<T> ec = energy_const<T>(sigma_k, c->params.z, V0, R12, a);
    State<T> &st = state<T>(c);
    T *e = nullptr;
    HV_CUDA(cudaMallocAsync((void **)&e, sizeof(T) * c->total, c->stream));
    k_energies<T><<<div_up(c->total, kBlock), kBlock, 0, c->stream>>>(c->total, c->protons, ec, st.x, st.y, st.z,
                                                                      st.kx, st.ky, st.kz, e);
    hv_status r = cudaGetLastError() == cudaSuccess ? HV_OK : HV_ERR_CUDA;
    if (r == HV_OK) r = download_slots(c, e, host);
    cudaFreeAsync(e, c->stream);
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return r;
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" {

void hv_init_params_default(hv_init_params *p) {
    if (!p) return;
    // sigma_k = calc_sigma(k_fwhm = 0.346), the drivers' default (auto_compute.py:54;
    // include/physics_formulas.hpp:56-60)
    p->sigma_k = 0.346 / (2.0 * std::sqrt(2.0 * std::log(2.0)));
    p->r_max = 0.0;
    p->max_test_part = 0;
    p->max_iterations = 0;
    p->rng = HV_RNG_PHILOX;
    p->seed = 128;
}

hv_status hv_initialize_particles(hv_ctx *c, const hv_skyrme *skm, hv_woods_saxon ws[2], hv_fermi *fermi,
                                  const hv_init_params *ip, hv_init_report *report, hv_init_row *rows) {
    if (!c || !ws || !fermi || !ip) return HV_ERR_BAD_ARG;
    if (ip->rng != HV_RNG_LIBC && ip->rng != HV_RNG_PHILOX) return HV_ERR_BAD_ARG;
    if (!(ip->sigma_k >= 0.0) || ip->max_test_part < 0 || ip->max_iterations < 0 || !(ip->r_max >= 0.0))
        return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    const hv_skyrme &sk = skm ? *skm : c->params.skyrme;
    return c->prec == HV_F64 ? initialize<double>(c, sk, ws, fermi, *ip, report, rows)
                             : initialize<float>(c, sk, ws, fermi, *ip, report, rows);
}

hv_status hv_fit_woods_saxon(hv_ctx *c, const hv_skyrme *skm, hv_woods_saxon ws[2], int iterations[2],
                             int status[2]) {
    if (!c || !ws) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    const hv_skyrme &sk = skm ? *skm : c->params.skyrme;
    int it[2] = {0, 0}, st[2] = {0, 0};
    const hv_status r = c->prec == HV_F64 ? fit_context<double>(c, sk, ws, it, st) : fit_context<float>(c, sk, ws, it, st);
    if (iterations) {
        iterations[0] = it[0];
        iterations[1] = it[1];
    }
    if (status) {
        status[0] = st[0];
        status[1] = st[1];
    }
    return r;
}

hv_status hv_particle_energies(hv_ctx *c, const hv_woods_saxon ws[2], double sigma_k, void *energy) {
    if (!c || !ws || (!energy && c->total)) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (c->total == 0) return HV_OK;
    return c->prec == HV_F64 ? energies_context<double>(c, ws, sigma_k, energy)
                             : energies_context<float>(c, ws, sigma_k, energy);
}

}  // extern "C"
