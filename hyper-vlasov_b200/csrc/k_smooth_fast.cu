// Decomposed Gaussian smoothing for the float fused path.
//
// compute_volumetric_densities (include/physics.hpp:202-234) sums
// rho(j) exp(-|r_i - r_j|^2 / (2 sigma^2)) over the node pairs inside the
// sphere |r_i - r_j|^2 <= 16 sigma^2.  The weight factorises over the axes,
// g(a) g(b) g(c), and for a symmetric tap set every (a, b) column of the
// sphere is a z-run |c| <= w(|a|, |b|).  So
//
//   rho_s(i,j,k) = sum_a g(a) sum_b g(b) Z_{w(|a|,|b|)}(i+a, j+b, k),
//   Z_w(i,j,k)   = sum_{|c|<=w} g(c) rho(i,j,k+c),
//
// with the same pair set as the reference.  A block owns a 16 x 16 (y, z)
// column tile of one species and one x segment, and marches along x over the
// input planes that reach it (see k_smooth_march): per input plane about
// 2 (W + 1) FMA for the z-runs of each staged row and sum_a (bm(a) + 1) pair
// sums for the disc sums of each column -- roughly 110 for the 3911-tap
// stencil of a 128^3 grid at h = 0.25 fm (A = B = W = 9), against 3911 for
// the direct sum.
//
// Used when the tap table passes the symmetry and contiguity checks in
// smooth_fast_plan (all cubic grids); otherwise the direct kernel runs.
#include <cmath>
#include <set>
#include <tuple>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kMBY = 16, kMBK = 16;         // output columns (y, z) of a block
constexpr int kMThreads = kMBY * kMBK;
constexpr int kMaxR = kSmoothMaxR;
constexpr int kMaxXSplit = 16;              // x segments per column tile: 1..16, chosen by the plan

struct MarchArgs {
    int nx, ny, nz;
    long long G;
    int A, B, W;
    int xsplit;                               // x segments per column tile
    float term;
    float gx[kMaxR + 1], gy[kMaxR + 1], gz[kMaxR + 1];
    int bm[kMaxR + 1];                        // largest |b| with a tap for each |a| (-1: none)
    int wt[(kMaxR + 1) * (kMaxR + 1)];        // w(|a|, |b|) at |a| (kMaxR + 1) + |b| (-1: none)
    const float *src;                         // 2G
    float *dst;                               // 2G
};

// Plane xi of the block's rho tile (y halo B, z halo W; zero outside the
// grid) into registers: element e = tid + i * kMThreads.
template <int R, int kPer>
__device__ __forceinline__ void load_plane(const MarchArgs &a, const float *src, int xi, int Y0, int K0,
                                           float (&v)[kPer]) {
    constexpr int rows = kMBY + 2 * R, cols = kMBK + 2 * R;
    const float *plane = src + (long long)xi * a.ny * a.nz;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        const int e = threadIdx.x + i * kMThreads;
        const int r = e / cols, cc = e - r * cols;
        const int y = Y0 - R + r, z = K0 - R + cc;
        v[i] = (e < rows * cols && xi >= 0 && xi < a.nx && y >= 0 && y < a.ny && z >= 0 && z < a.nz)
                   ? __ldg(plane + (long long)y * a.nz + z)
                   : 0.0f;
    }
}

// One block: a 16 x 16 column tile (y, z) of one species and one x segment of
// the outputs.  It marches over the input planes xi that reach the segment:
// the plane's rho tile (the next plane's loads in flight in registers during
// this plane's sums) gives the z-runs Z_w, w = 0..W, of every staged
// row; each thread then forms, for its column, the disc sums
// Y_|a| = sum_|b|<=bm(a) g(b) Z_w(|a|,|b|)(y + b) and adds g(a) Y_|a| to the
// outputs x = xi -+ a, held in a thread-private ring of 2A + 1 planes in shared
// memory.  Output plane xo is complete after plane xo + A and is written then.
// R >= A, B, W is the halo and the unrolled extent of the loops over |a|, |b|
// and w; the tables hold -1 (no tap) and zero weights beyond A, B, W.
template <int R>
__global__ void __launch_bounds__(kMThreads) k_smooth_march(const __grid_constant__ MarchArgs a) {
    extern __shared__ __align__(16) float sm[];
    constexpr int rows = kMBY + 2 * R, cols = kMBK + 2 * R;
    constexpr int kPer = (rows * cols + kMThreads - 1) / kMThreads;
    const int A = a.A, ring = 2 * A + 1;
    float *s_rho = sm;                               // rows x cols
    float *s_z = s_rho + rows * cols;                // (R + 1) x rows x kMBK
    float *s_acc = s_z + (R + 1) * rows * kMBK;      // ring x kMThreads
    const int tid = threadIdx.x;
    const int tz = (a.nz + kMBK - 1) / kMBK, ty = (a.ny + kMBY - 1) / kMBY;
    const int xlen = (a.nx + a.xsplit - 1) / a.xsplit;
    int bid = blockIdx.x;
    const int kt = bid % tz;
    bid /= tz;
    const int yt = bid % ty;
    bid /= ty;
    const int xs = bid % a.xsplit;
    const int sp = bid / a.xsplit;
    const int Y0 = yt * kMBY, K0 = kt * kMBK, X0 = xs * xlen, X1 = min(a.nx, X0 + xlen);
    if (X0 >= X1) return;
    const float *src = a.src + sp * a.G;
    const int j = tid / kMBK, k = tid % kMBK, y = Y0 + j, z = K0 + k;
    const bool out_ok = y < a.ny && z < a.nz;

    for (int s = 0; s < ring; s++) s_acc[s * kMThreads + tid] = 0.0f;
    const int xfirst = max(0, X0 - A), xlast = min(a.nx - 1, X1 - 1 + A);
    float v[kPer];
    load_plane<R, kPer>(a, src, xfirst, Y0, K0, v);
    int slot = xfirst % ring;  // ring slot of plane xi
    for (int xi = xfirst; xi <= X1 - 1 + A; xi++, slot = slot + 1 == ring ? 0 : slot + 1) {
        const bool have = xi <= xlast;
        if (have) {
#pragma unroll
            for (int i = 0; i < kPer; i++) {
                const int e = tid + i * kMThreads;
                if (e < rows * cols) s_rho[e] = v[i];
            }
        }
        __syncthreads();
        if (have) {
            // z-runs of every staged row
            for (int e = tid; e < rows * kMBK; e += kMThreads) {
                const int r = e / kMBK, kk = e - r * kMBK;
                const float *line = s_rho + r * cols + kk + R;
                float zsum = a.gz[0] * line[0];
                s_z[r * kMBK + kk] = zsum;
#pragma unroll
                for (int w = 1; w <= R; w++) {
                    zsum += a.gz[w] * (line[w] + line[-w]);
                    s_z[(w * rows + r) * kMBK + kk] = zsum;
                }
            }
        }
        // the next plane's loads overlap this plane's sums
        if (xi + 1 <= xlast) load_plane<R, kPer>(a, src, xi + 1, Y0, K0, v);
        __syncthreads();
        if (have) {
            const float *zc = s_z + (j + R) * kMBK + k;  // this column's row, width 0
            constexpr int zstride = rows * kMBK;
#pragma unroll
            for (int aa = 0; aa <= R; aa++) {
                const int bm = a.bm[aa];
                if (bm < 0) continue;
                const int xo1 = xi - aa, xo2 = xi + aa;
                const bool h1 = xo1 >= X0 && xo1 < X1, h2 = aa > 0 && xo2 >= X0 && xo2 < X1;
                if (!h1 && !h2) continue;
                const int *wr = a.wt + aa * (kMaxR + 1);
                float y0 = a.gy[0] * zc[wr[0] * zstride], y1 = 0.0f;
#pragma unroll
                for (int b = 1; b <= R; b++) {
                    if (b > bm) break;
                    const float *pb = zc + wr[b] * zstride;
                    const float t = a.gy[b] * (pb[b * kMBK] + pb[-b * kMBK]);
                    if (b & 1) y0 += t;
                    else y1 += t;
                }
                const float c = a.gx[aa] * (y0 + y1);
                const int s1 = slot - aa < 0 ? slot - aa + ring : slot - aa;
                const int s2 = slot + aa >= ring ? slot + aa - ring : slot + aa;
                if (h1) s_acc[s1 * kMThreads + tid] += c;
                if (h2) s_acc[s2 * kMThreads + tid] += c;
            }
        }
        // output plane xi - A is complete
        const int xo = xi - A;
        if (xo >= X0 && xo < X1) {
            float *acc = s_acc + (slot - A < 0 ? slot - A + ring : slot - A) * kMThreads + tid;
            if (out_ok) a.dst[sp * a.G + ((long long)xo * a.ny + y) * a.nz + z] = *acc * a.term;
            *acc = 0.0f;
        }
    }
}

const void *march_kernel(int r) {
    switch (r) {
    case 1: return (const void *)k_smooth_march<1>;
    case 2: return (const void *)k_smooth_march<2>;
    case 3: return (const void *)k_smooth_march<3>;
    case 4: return (const void *)k_smooth_march<4>;
    case 5: return (const void *)k_smooth_march<5>;
    case 6: return (const void *)k_smooth_march<6>;
    case 7: return (const void *)k_smooth_march<7>;
    case 8: return (const void *)k_smooth_march<8>;
    case 9: return (const void *)k_smooth_march<9>;
    case 10: return (const void *)k_smooth_march<10>;
    case 11: return (const void *)k_smooth_march<11>;
    case 12: return (const void *)k_smooth_march<12>;
    case 13: return (const void *)k_smooth_march<13>;
    case 14: return (const void *)k_smooth_march<14>;
    case 15: return (const void *)k_smooth_march<15>;
    case 16: return (const void *)k_smooth_march<16>;
    default: return nullptr;
    }
}

}  // namespace

// Builds the decomposition from the tap table, or leaves ok = false when the
// table is not symmetric with contiguous z-runs.
hv_status smooth_fast_plan(hv_ctx *c) {
    SmoothFast &f = c->fused.smooth;
    f.ok = false;
    const TapTable &t = c->taps;
    if (t.count == 0) return HV_OK;
    std::set<std::tuple<int, int, int>> taps;
    int A = 0, B = 0, W = 0;
    for (int i = 0; i < t.count; i++) {
        int p = t.packed[i];
        int a = (p >> 20) - 512, b = ((p >> 10) & 1023) - 512, cz = (p & 1023) - 512;
        taps.insert({a, b, cz});
        A = std::max(A, std::abs(a));
        B = std::max(B, std::abs(b));
        W = std::max(W, std::abs(cz));
    }
    if (A > kMaxR || B > kMaxR || W > kMaxR) return HV_OK;
    std::vector<int> wtab((A + 1) * (B + 1), -1);
    for (auto &e : taps) {
        int a, b, cz;
        std::tie(a, b, cz) = e;
        if (!taps.count({-a, b, cz}) || !taps.count({a, -b, cz}) || !taps.count({a, b, -cz})) return HV_OK;
        int &w = wtab[std::abs(a) * (B + 1) + std::abs(b)];
        w = std::max(w, std::abs(cz));
    }
    // each present (a,b) column must be the full run |c| <= w, and for each
    // |a| the present |b| must be 0..bm(a)
    size_t expect = 0;
    for (int a = -A; a <= A; a++)
        for (int b = -B; b <= B; b++) {
            int w = wtab[std::abs(a) * (B + 1) + std::abs(b)];
            if (w >= 0) expect += 2 * w + 1;
        }
    if (expect != taps.size()) return HV_OK;
    for (int i = 0; i <= kMaxR; i++) f.bm[i] = -1;
    for (int i = 0; i < (kMaxR + 1) * (kMaxR + 1); i++) f.wt[i] = -1;
    for (int a = 0; a <= A; a++) {
        int bm = -1;
        for (int b = 0; b <= B; b++)
            if (wtab[a * (B + 1) + b] >= 0) bm = b;
        for (int b = 0; b <= bm; b++)
            if (wtab[a * (B + 1) + b] < 0) return HV_OK;
        f.bm[a] = bm;
        for (int b = 0; b <= B; b++) f.wt[a * (kMaxR + 1) + b] = wtab[a * (B + 1) + b];
    }
    // separable weights from the same node coordinates as the table
    const hv_world &wd = c->world;
    const double sig = c->params.sigma_r, e = 1.0 / (2.0 * sig * sig);
    auto g1 = [&](int axis, int off) {
        const int n = wd.n[axis], ctr = n / 2;
        const double dm = wd.d_max[axis];
        double d = dm * (2.0 * ctr / n - 1.0) - dm * (2.0 * (ctr + off) / n - 1.0);
        return (float)std::exp(-d * d * e);
    };
    for (int i = 0; i <= kMaxR; i++) f.gx[i] = f.gy[i] = f.gz[i] = 0.0f;
    for (int a = 0; a <= A; a++) f.gx[a] = g1(0, a);
    for (int b = 0; b <= B; b++) f.gy[b] = g1(1, b);
    for (int cz = 0; cz <= W; cz++) f.gz[cz] = g1(2, cz);
    const int R = std::max(1, std::max(A, std::max(B, W)));
    const int rows = kMBY + 2 * R, cols = kMBK + 2 * R;
    f.per = R;
    f.smem = sizeof(float) * ((size_t)rows * cols + (size_t)(R + 1) * rows * kMBK + (size_t)(2 * A + 1) * kMThreads);
    HV_TRY(allow_max_dynamic_smem(march_kernel(R), c->device));
    // x segments: more blocks raise the warps per SM (the kernel is bound by
    // shared-memory latency) but each segment re-reads 2A halo planes; take
    // the split with the fewest (waves x planes per block), fewer blocks on
    // ties.  Measured at 128^3 (A = 9): 2 -> 383 us, 3 -> 338, 4 -> 320, 6 -> 374.
    {
        cudaDeviceProp prop;
        HV_CUDA(cudaGetDeviceProperties(&prop, c->device));
        int per_sm = 0;
        HV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march_kernel(R), kMThreads, f.smem));
        const long long slots = (long long)std::max(per_sm, 1) * prop.multiProcessorCount;
        const long long tiles = 2ll * ((c->geom.ny + kMBY - 1) / kMBY) * ((c->geom.nz + kMBK - 1) / kMBK);
        long long best = -1;
        f.xsplit = 1;
        for (int s = 1; s <= kMaxXSplit && s <= c->geom.nx; s++) {
            const long long waves = (tiles * s + slots - 1) / slots;
            const long long planes = (c->geom.nx + s - 1) / s + 2ll * A;
            const long long cost = waves * planes;
            if (best < 0 || cost < best) {
                best = cost;
                f.xsplit = s;
            }
        }
    }
    f.A = A;
    f.B = B;
    f.W = W;
    f.ok = true;
    return HV_OK;
}

void smooth_fast_release(hv_ctx *c) { c->fused.smooth = SmoothFast(); }

hv_status smooth_fast_launch(hv_ctx *c, const float *rho_raw, float *rho) {
    const SmoothFast &f = c->fused.smooth;
    const Geom &g = c->geom;
    const hv_run_params &p = c->params;
    MarchArgs a;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.G = g.G;
    a.A = f.A;
    a.B = f.B;
    a.W = f.W;
    a.xsplit = f.xsplit;
    const double sig = p.sigma_r;
    a.term = (float)((1.0 / p.part_per_nucleon) * (1.0 / std::pow(2.0 * kPi * sig * sig, 1.5)));
    for (int i = 0; i <= kMaxR; i++) {
        a.gx[i] = f.gx[i];
        a.gy[i] = f.gy[i];
        a.gz[i] = f.gz[i];
        a.bm[i] = f.bm[i];
    }
    for (int i = 0; i < (kMaxR + 1) * (kMaxR + 1); i++) a.wt[i] = f.wt[i];
    a.src = rho_raw;
    a.dst = rho;
    const int tz = (g.nz + kMBK - 1) / kMBK, ty = (g.ny + kMBY - 1) / kMBY;
    void *args[] = {&a};
    HV_CUDA(cudaLaunchKernel(march_kernel(f.per), dim3(2 * f.xsplit * ty * tz), dim3(kMThreads), args, f.smem,
                             c->stream));
    return HV_OK;
}

}  // namespace hv
