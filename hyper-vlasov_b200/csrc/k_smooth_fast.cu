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
// with the same pair set as the reference.  A block owns a BX x BY x BK
// output tile of one species and marches over the input x-planes that touch
// it.  Per input plane it stages the rho tile (with y and z halos) in shared
// memory, builds Z_0..Z_W for its rows incrementally (2 FMA per w), forms the
// (b)-disc sums Y_|a| for its own rows and adds g(a) Y_|a| into the
// accumulators of the output planes x = i - a.  That is about
// 1.6 x (20 + sum_a (2 B(a) + 1)) ~ 300 FMA per output node for the 3911-tap
// stencil of a 128^3 grid at h = 0.25 fm, against 3911 for the direct sum.
//
// Used when the tap table passes the symmetry and contiguity checks in
// smooth_fast_plan (all cubic grids); otherwise the direct kernel runs.
#include <cmath>
#include <set>
#include <tuple>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kBX = 32, kBY = 16, kBK = 32;
constexpr int kThreads = kBY * kBK;
constexpr int kMaxR = 16;  // largest |a|, |b| or w handled

struct SmoothArgs {
    int nx, ny, nz;
    long long G;
    int A, B, W;
    float term;
    const float *g;   // gx[A+1] gy[B+1] gz[W+1]
    const int *wtab;  // (A+1) x (B+1)
    const float *src; // 2G
    float *dst;       // 2G
};

__global__ void __launch_bounds__(kThreads) k_smooth_decomposed(SmoothArgs a) {
    extern __shared__ __align__(16) float sm[];
    const int A = a.A, B = a.B, W = a.W;
    const int rows = kBY + 2 * B, cols = kBK + 2 * W;
    float *s_rho = sm;                             // rows x cols
    float *s_z = s_rho + rows * cols;              // (W+1) x rows x kBK
    float *s_acc = s_z + (W + 1) * rows * kBK;     // kBX x kThreads
    __shared__ float s_gx[kMaxR + 1], s_gy[kMaxR + 1], s_gz[kMaxR + 1];
    __shared__ int s_w[(kMaxR + 1) * (kMaxR + 1)];
    __shared__ int s_bm[kMaxR + 1];

    const int tid = threadIdx.x;
    // block -> (species, x tile, y tile, z tile)
    const int tz = (a.nz + kBK - 1) / kBK, ty = (a.ny + kBY - 1) / kBY, tx = (a.nx + kBX - 1) / kBX;
    int bid = blockIdx.x;
    const int kt = bid % tz;
    bid /= tz;
    const int yt = bid % ty;
    bid /= ty;
    const int xt = bid % tx;
    const int sp = bid / tx;
    const int X0 = xt * kBX, Y0 = yt * kBY, K0 = kt * kBK;
    const float *src = a.src + sp * a.G;

    if (tid <= A) s_gx[tid] = a.g[tid];
    if (tid <= B) s_gy[tid] = a.g[A + 1 + tid];
    if (tid <= W) s_gz[tid] = a.g[A + 1 + B + 1 + tid];
    for (int e = tid; e < (A + 1) * (B + 1); e += kThreads) s_w[e] = a.wtab[e];
    for (int e = tid; e < kBX * kThreads; e += kThreads) s_acc[e] = 0.0f;
    __syncthreads();
    if (tid <= A) {  // largest |b| with a tap for this |a|
        int bm = -1;
        for (int b = 0; b <= B; b++)
            if (s_w[tid * (B + 1) + b] >= 0) bm = b;
        s_bm[tid] = bm;
    }

    const int j = tid / kBK, k = tid % kBK;
    const int xlo = max(0, X0 - A), xhi = min(a.nx, X0 + kBX + A);
    for (int xi = xlo; xi < xhi; xi++) {
        // 1. rho tile of plane xi with y and z halos (zero outside the grid)
        const float *plane = src + (long long)xi * a.ny * a.nz;
        for (int e = tid; e < rows * cols; e += kThreads) {
            int r = e / cols, cc = e % cols;
            int y = Y0 - B + r, z = K0 - W + cc;
            s_rho[e] = (y >= 0 && y < a.ny && z >= 0 && z < a.nz) ? __ldg(plane + (long long)y * a.nz + z) : 0.0f;
        }
        __syncthreads();
        // 2. z-runs Z_w for every staged row, w = 0..W
        for (int e = tid; e < rows * kBK; e += kThreads) {
            int r = e / kBK, kk = e % kBK;
            const float *line = s_rho + r * cols + kk + W;
            float zsum = s_gz[0] * line[0];
            s_z[r * kBK + kk] = zsum;
            for (int w = 1; w <= W; w++) {
                zsum += s_gz[w] * (line[w] + line[-w]);
                s_z[(w * rows + r) * kBK + kk] = zsum;
            }
        }
        __syncthreads();
        // 3. disc sums over b for each |a|, scattered to the output planes
        for (int aa = 0; aa <= A; aa++) {
            const int bm = s_bm[aa];
            if (bm < 0) continue;
            const int xo1 = xi - aa - X0, xo2 = xi + aa - X0;
            const bool h1 = xo1 >= 0 && xo1 < kBX, h2 = aa > 0 && xo2 >= 0 && xo2 < kBX;
            if (!h1 && !h2) continue;
            float ysum = 0.0f;
            const int *wr = s_w + aa * (B + 1);
            for (int b = -bm; b <= bm; b++) {
                const int w = wr[b < 0 ? -b : b];
                if (w < 0) continue;
                ysum += s_gy[b < 0 ? -b : b] * s_z[(w * rows + j + B + b) * kBK + k];
            }
            const float gy = s_gx[aa] * ysum;
            if (h1) s_acc[xo1 * kThreads + tid] += gy;
            if (h2) s_acc[xo2 * kThreads + tid] += gy;
        }
        __syncthreads();
    }
    const int y = Y0 + j, z = K0 + k;
    if (y < a.ny && z < a.nz) {
        for (int xo = 0; xo < kBX && X0 + xo < a.nx; xo++)
            a.dst[sp * a.G + ((long long)(X0 + xo) * a.ny + y) * a.nz + z] = s_acc[xo * kThreads + tid] * a.term;
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
    // each present (a,b) column must be the full run |c| <= w
    size_t expect = 0;
    for (int a = -A; a <= A; a++)
        for (int b = -B; b <= B; b++) {
            int w = wtab[std::abs(a) * (B + 1) + std::abs(b)];
            if (w >= 0) expect += 2 * w + 1;
        }
    if (expect != taps.size()) return HV_OK;
    // separable weights from the same node coordinates as the table
    const hv_world &wd = c->world;
    const double sig = c->params.sigma_r, e = 1.0 / (2.0 * sig * sig);
    auto g1 = [&](int axis, int off) {
        const int n = wd.n[axis], ctr = n / 2;
        const double dm = wd.d_max[axis];
        double d = dm * (2.0 * ctr / n - 1.0) - dm * (2.0 * (ctr + off) / n - 1.0);
        return (float)std::exp(-d * d * e);
    };
    std::vector<float> g;
    for (int a = 0; a <= A; a++) g.push_back(g1(0, a));
    for (int b = 0; b <= B; b++) g.push_back(g1(1, b));
    for (int cz = 0; cz <= W; cz++) g.push_back(g1(2, cz));
    HV_CUDA(cudaMalloc((void **)&f.g, sizeof(float) * g.size()));
    HV_CUDA(cudaMalloc((void **)&f.w, sizeof(int) * wtab.size()));
    HV_CUDA(cudaMemcpyAsync(f.g, g.data(), sizeof(float) * g.size(), cudaMemcpyHostToDevice, c->stream));
    HV_CUDA(cudaMemcpyAsync(f.w, wtab.data(), sizeof(int) * wtab.size(), cudaMemcpyHostToDevice, c->stream));
    const size_t smem = sizeof(float) * ((size_t)(kBY + 2 * B) * (kBK + 2 * W) + (size_t)(W + 1) * (kBY + 2 * B) * kBK +
                                         (size_t)kBX * kThreads);
    HV_CUDA(cudaFuncSetAttribute(k_smooth_decomposed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    f.A = A;
    f.B = B;
    f.W = W;
    f.ok = true;
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return HV_OK;
}

void smooth_fast_release(hv_ctx *c) {
    SmoothFast &f = c->fused.smooth;
    if (f.g) cudaFree(f.g);
    if (f.w) cudaFree(f.w);
    f = SmoothFast();
}

hv_status smooth_fast_launch(hv_ctx *c, const float *rho_raw, float *rho) {
    const SmoothFast &f = c->fused.smooth;
    const Geom &g = c->geom;
    const hv_run_params &p = c->params;
    SmoothArgs a;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    a.G = g.G;
    a.A = f.A;
    a.B = f.B;
    a.W = f.W;
    const double sig = p.sigma_r;
    a.term = (float)((1.0 / p.part_per_nucleon) * (1.0 / std::pow(2.0 * kPi * sig * sig, 1.5)));
    a.g = f.g;
    a.wtab = f.w;
    a.src = rho_raw;
    a.dst = rho;
    const int tz = (g.nz + kBK - 1) / kBK, ty = (g.ny + kBY - 1) / kBY, tx = (g.nx + kBX - 1) / kBX;
    const size_t smem = sizeof(float) * ((size_t)(kBY + 2 * f.B) * (kBK + 2 * f.W) +
                                         (size_t)(f.W + 1) * (kBY + 2 * f.B) * kBK + (size_t)kBX * kThreads);
    k_smooth_decomposed<<<2 * tx * ty * tz, kThreads, smem, c->stream>>>(a);
    HV_CUDA(cudaGetLastError());
    return HV_OK;
}

}  // namespace hv
