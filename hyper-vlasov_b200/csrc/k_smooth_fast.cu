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
#include <algorithm>
#include <cmath>
#include <set>
#include <tuple>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kMBY = 16, kMBK = 16;         // output columns (y, z) of a block
constexpr int kMThreads = kMBY * kMBK;
constexpr int kMaxR = kSmoothMaxR;
constexpr int kMaxXSplit = 16;              // x segments per column tile: 1..16, chosen by the plan

// Edge flags summed over the x planes (every thread of the block gets it; the
// block's first warp sums).
__device__ __forceinline__ int edge_total(const int *edge, int nx) {
    __shared__ int s_total;
    if (threadIdx.x < 32) {
        int v = 0;
        for (int i = threadIdx.x; i < nx; i += 32) v += edge[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) s_total = v;
    }
    __syncthreads();
    return s_total;
}

// The wrap correction applies to this step's smoothing: density lies within
// the stencil of a face (flags > 0), and the particles that put it there are
// listed, 1..wcap of them.
__device__ __forceinline__ bool wrap_active(int flags, const int *wcount, int wcap) {
    if (flags == 0 || !wcount) return false;
    const int n = *wcount;
    return n >= 1 && n <= wcap;
}

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
    const int *edge;                          // [nx] edge flags of the FFT form: run only if one
                                              // is set and the wrap correction does not apply
                                              // (null: always run)
    const int *wcount;                        // the wrap list's count (null: no list)
    int wcap;
    const float4 *wlist;                      // the wrap list (particle step)
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

// The wrap correction of the FFT form, run by the march kernel's blocks after
// the transform's last pass when it applies (wrap_active).  The circular
// convolution adds, to nodes within the stencil of a face, the weights of
// density near the opposite face whose offset wraps around the grid; the
// reference's truncated sum (compute_volumetric_densities,
// include/physics.hpp:202-234) has no such pairs.  The deposit of every
// listed particle is taken again -- the same grid coordinates, weights and
// corner drops -- and its wrapped pairs are subtracted from the output.  Work
// items are (particle, x plane of the box its corners' stencils cover), a
// warp each, its lanes over the plane's (y, z) targets that lie outside the
// grid.  For such an unwrapped target T, the sum over the corners c whose
// offset T - c is a tap of w_c g(a) g(b) g(c), times term, is subtracted at T
// taken modulo the axes, where the transform put it: one atomic per target of
// a particle.  The output may then dip below zero by the transform's
// rounding; the Skyrme kernel, which reads it next, clamps it.  Each axis
// holds at least twice its half-width plus two nodes (a plan condition), so a
// target leaves the grid on one side of an axis at most, and one shift brings
// it back.
__device__ void wrap_correct(const MarchArgs &a) {
    __shared__ float s_g[3][kMaxR + 1];
    __shared__ int s_bm[kMaxR + 1], s_wt[(kMaxR + 1) * (kMaxR + 1)];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    for (int i = threadIdx.x; i <= kMaxR; i += blockDim.x) {
        s_g[0][i] = a.gx[i];
        s_g[1][i] = a.gy[i];
        s_g[2][i] = a.gz[i];
        s_bm[i] = a.bm[i];
    }
    for (int i = threadIdx.x; i < (kMaxR + 1) * (kMaxR + 1); i += blockDim.x) s_wt[i] = a.wt[i];
    __syncthreads();
    const int np = *a.wcount, bxn = 2 * a.A + 2, byn = 2 * a.B + 2, bzn = 2 * a.W + 2;
    // q / bzn for q below byn bzn (at most 34^2) as a product: exact for divisors below 56
    const unsigned inv_bzn = (65536u + bzn - 1) / bzn;
    const int lane = threadIdx.x & 31;
    const long long items = (long long)np * bxn, nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long it = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < items; it += nwarps) {
        const int p = (int)(it / bxn), ix = (int)(it - (long long)p * bxn);
        const float4 e = a.wlist[p];
        const int x0 = (int)e.x, y0 = (int)e.y, z0 = (int)e.z;
        const int X = x0 - a.A + ix;
        const bool xout = X < 0 || X >= nx;
        // no target of this x row lies outside the grid
        if (!xout && y0 - a.B >= 0 && y0 + 1 + a.B < ny && z0 - a.W >= 0 && z0 + 1 + a.W < nz) continue;
        const float dx = e.x - x0, dy = e.y - y0, dz = e.z - z0;
        // the two x corners: tap extent in y, weight (a corner with an index
        // equal to n is dropped, as by the deposit)
        const int ua0 = abs(X - x0), ua1 = abs(X - x0 - 1);
        const int bm0 = ua0 <= a.A ? s_bm[ua0] : -1, bm1 = (x0 + 1 < nx && ua1 <= a.A) ? s_bm[ua1] : -1;
        if (bm0 < 0 && bm1 < 0) continue;
        const float wx0 = bm0 >= 0 ? (1.0f - dx) * s_g[0][ua0] : 0.0f, wx1 = bm1 >= 0 ? dx * s_g[0][ua1] : 0.0f;
        const int cyn = y0 + 1 < ny ? 2 : 1, czn = z0 + 1 < nz ? 2 : 1;
        float *out = a.dst + (e.w != 0.0f ? a.G : 0);
        const int Xt = X + (X < 0 ? nx : (X >= nx ? -nx : 0));
        // the plane's targets outside the grid: every one when X is outside;
        // otherwise the rows whose Y is outside (ylo below, yhi above), and
        // in the other rows the z offsets whose Z is outside (zlo, zhi)
        const int ylo = xout ? 0 : max(0, a.B - y0), yhi = xout ? 0 : max(0, y0 + 1 + a.B - (ny - 1));
        const int zlo = xout ? 0 : max(0, a.W - z0), zhi = xout ? 0 : max(0, z0 + 1 + a.W - (nz - 1));
        const int nrow = xout ? byn : ylo + yhi, nzo = zlo + zhi;
        const int nfull = nrow * bzn, ntarget = nfull + (xout ? 0 : (byn - nrow) * nzo);
        for (int q = lane; q < ntarget; q += 32) {
            int iy, iz;
            if (q < nfull) {
                const int r = (int)(((unsigned)q * inv_bzn) >> 16);
                iz = q - r * bzn;
                iy = r < ylo || xout ? r : byn - yhi + (r - ylo);
            } else {
                const int qq = q - nfull, r = qq / nzo, c = qq - r * nzo;
                iy = ylo + r;
                iz = c < zlo ? c : bzn - zhi + (c - zlo);
            }
            const int Y = y0 - a.B + iy, Z = z0 - a.W + iz;
            float v = 0.0f;
#pragma unroll
            for (int cb = 0; cb < 2; cb++) {
                if (cb >= cyn) break;
                const int ub = abs(Y - y0 - cb);
                if (ub > a.B) continue;
                const float wy = (cb ? dy : 1.0f - dy) * s_g[1][ub];
#pragma unroll
                for (int ca = 0; ca < 2; ca++) {
                    if (ub > (ca ? bm1 : bm0)) continue;
                    const int w = s_wt[(ca ? ua1 : ua0) * (kMaxR + 1) + ub];
                    const float wxy = (ca ? wx1 : wx0) * wy;
#pragma unroll
                    for (int cc = 0; cc < 2; cc++) {
                        if (cc >= czn) break;
                        const int uc = abs(Z - z0 - cc);
                        if (uc <= w) v += wxy * (cc ? dz : 1.0f - dz) * s_g[2][uc];
                    }
                }
            }
            if (v == 0.0f) continue;
            const int Yt = Y + (Y < 0 ? ny : (Y >= ny ? -ny : 0)), Zt = Z + (Z < 0 ? nz : (Z >= nz ? -nz : 0));
            atomicAdd(out + ((long long)Xt * ny + Yt) * nz + Zt, -v * a.term);
        }
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
    if (a.edge) {
        // after the FFT form: needed only where neither the transform nor
        // its wrap correction is exact
        const int flags = edge_total(a.edge, a.nx);
        if (flags == 0) return;
        if (wrap_active(flags, a.wcount, a.wcap)) {
            wrap_correct(a);
            return;
        }
    }
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

// ---- FFT form --------------------------------------------------------------
//
// The smoothing is a convolution by a fixed symmetric stencil, so on a grid of
// power-of-two axes it is also a pointwise product in Fourier space.  The
// circular convolution equals the reference's truncated sum when no density
// lies within the stencil's half-widths (A, B, W) of a face: the only wrapped
// inputs come from those edge slabs.  The first pass flags any density there;
// the march kernel then runs (and overwrites the result) only when a flag is
// set.  Both species go through one complex transform, rho_p + i rho_n: the
// stencil's spectrum is real (the stencil is even), so the product keeps them
// apart.  Three passes over a complex work grid:
//   1. per x plane: load both species (rows in bit-reversed y order), flag
//      the edge slabs, transform along z (decimation in frequency: z leaves
//      in bit-reversed order) and along y (decimation in time: y leaves in
//      natural order);
//   2. per y: transform along x (decimation in time from a bit-reversed
//      load), multiply by the spectrum, inverse along x (decimation in
//      frequency, stored back from bit-reversed order);
//   3. per x plane: inverse along z (bit-reversed in, natural out) and along
//      y (natural in, bit-reversed out), both species stored from the
//      permuted rows, clamped at 0.
// Only whole rows are permuted in shared memory, so no pass scatters single
// elements across banks.  The spectrum keeps z in bit-reversed order between
// the passes, and so does khat.
constexpr int kFThreads = 1024;
constexpr int kFMaxN = 128;        // longest axis of the FFT form
constexpr int kFMaxPlane = 16384;  // complex elements of a plane or column slab (128 KB)
constexpr int kFftAutoHalfWidth = 6;  // smooth_fft = 1: stencils at least this wide

struct FftArgs {
    int nx, ny, nz, lx, ly, lz;  // axis lengths and their log2
    int A, B, W;                 // stencil half-widths: the edge slabs
    long long G;
    const float *src;            // 2G: protons, neutrons
    float *dst;                  // 2G
    float2 *work;                // G complex
    const float *khat;           // G: spectrum x term / G, z in bit-reversed order
    const float2 *tw;            // kFMaxN / 2 twiddles exp(-2 pi i m / kFMaxN)
    int *edge;                   // [nx]: nonzero densities within the stencil of a face, per x plane
    unsigned *occ;               // 128^3 forward pass: [2][nx] row-group occupancy of the raw
                                 // densities (bit q: rows 4q..4q+3), null when not wanted
    float post;                  // current term / the term folded into khat
};

__device__ __forceinline__ int bit_reverse(int v, int l) { return (int)(__brev((unsigned)v) >> (32 - l)); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Stages over `lines` = 2^ll transforms of length n = 2^l (l >= 1) in shared
// memory, element m of line q at s[q * qs + m * ms].  kDit: bit-reversed input,
// natural output (decimation in time); otherwise natural input, bit-reversed
// output (decimation in frequency).  inv: conjugate twiddles (no 1/n; the
// spectrum carries it).  Two radix-2 stages at a time: a thread takes the four
// elements i, i + h, i + 2h, i + 3h and applies both stages' butterflies in
// registers, so a length-128 transform is one radix-2 pass and three radix-4
// passes.  Rows (ms = 1) give consecutive threads consecutive butterflies of a
// line; columns give them consecutive lines, so a warp's accesses are
// contiguous either way.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a W_4: a * (-i) forward, a * (+i) inverse
__device__ __forceinline__ float2 cmul_w4(float2 a, bool inv) {
    return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

__device__ __forceinline__ void fft_radix2(float2 *s, int l, int ll, int qs, int ms, const float2 *tw, int tstep,
                                           int h, bool dit, bool inv) {
    const int half = 1 << (l - 1), total = half << ll;
    const int wstep = (half / h) * tstep;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int q, j;
        if (ms == 1) {
            j = t & (half - 1);
            q = t >> (l - 1);
        } else {
            q = t & ((1 << ll) - 1);
            j = t >> ll;
        }
        const int k = j & (h - 1), i = ((j - k) << 1) + k;
        float2 w = tw[k * wstep];
        if (inv) w.y = -w.y;
        float2 *p0 = s + q * qs + i * ms, *p1 = p0 + h * ms;
        const float2 u = *p0, v = *p1;
        if (dit) {
            const float2 vw = cmul(v, w);
            *p0 = cadd(u, vw);
            *p1 = csub(u, vw);
        } else {
            *p0 = cadd(u, v);
            *p1 = cmul(csub(u, v), w);
        }
    }
    __syncthreads();
}

// The radix-2 stages of spans h and 2h (dit) or 2h and h (dif) in one pass.
__device__ __forceinline__ void fft_radix4(float2 *s, int l, int ll, int qs, int ms, const float2 *tw, int tstep,
                                           int h, bool dit, bool inv) {
    const int quarter = 1 << (l - 2), total = quarter << ll, n = 1 << l;
    const int w1step = (n / (2 * h)) * tstep, w2step = (n / (4 * h)) * tstep;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int q, j;
        if (ms == 1) {
            j = t & (quarter - 1);
            q = t >> (l - 2);
        } else {
            q = t & ((1 << ll) - 1);
            j = t >> ll;
        }
        const int k = j & (h - 1), i = ((j - k) << 2) + k;
        float2 w1 = tw[k * w1step], w2 = tw[k * w2step];  // W_2h^k, W_4h^k
        if (inv) {
            w1.y = -w1.y;
            w2.y = -w2.y;
        }
        float2 *p0 = s + q * qs + i * ms;
        const int d = h * ms;
        const float2 x0 = p0[0], x1 = p0[d], x2 = p0[2 * d], x3 = p0[3 * d];
        if (dit) {
            // span h: (x0, x1), (x2, x3) by W_2h^k; span 2h: (a0, a2) by
            // W_4h^k, (a1, a3) by W_4h^(k + h) = W_4h^k W_4
            const float2 t1 = cmul(x1, w1), t3 = cmul(x3, w1);
            const float2 a0 = cadd(x0, t1), a1 = csub(x0, t1), a2 = cadd(x2, t3), a3 = csub(x2, t3);
            const float2 b2 = cmul(a2, w2), b3 = cmul_w4(cmul(a3, w2), inv);
            p0[0] = cadd(a0, b2);
            p0[2 * d] = csub(a0, b2);
            p0[d] = cadd(a1, b3);
            p0[3 * d] = csub(a1, b3);
        } else {
            // span 2h: (x0, x2) by W_4h^k, (x1, x3) by W_4h^(k + h); span h:
            // (a0, a1), (a2, a3) by W_2h^k
            const float2 a0 = cadd(x0, x2), a2 = cmul(csub(x0, x2), w2);
            const float2 a1 = cadd(x1, x3), a3 = cmul_w4(cmul(csub(x1, x3), w2), inv);
            p0[0] = cadd(a0, a1);
            p0[d] = cmul(csub(a0, a1), w1);
            p0[2 * d] = cadd(a2, a3);
            p0[3 * d] = cmul(csub(a2, a3), w1);
        }
    }
    __syncthreads();
}

template <bool kDit>
__device__ void fft_stages(float2 *s, int n, int l, int ll, int qs, int ms, const float2 *tw, bool inv) {
    const int tstep = kFMaxN / n;
    if (kDit) {
        int st = 0;
        if (l & 1) {
            fft_radix2(s, l, ll, qs, ms, tw, tstep, 1, true, inv);
            st = 1;
        }
        for (; st + 1 < l; st += 2) fft_radix4(s, l, ll, qs, ms, tw, tstep, 1 << st, true, inv);
    } else {
        int st = l - 1;  // the span 2^st comes first
        for (; st >= 1; st -= 2) fft_radix4(s, l, ll, qs, ms, tw, tstep, 1 << (st - 1), false, inv);
        if (st == 0) fft_radix2(s, l, ll, qs, ms, tw, tstep, 1, false, inv);
    }
}

__global__ void __launch_bounds__(kFThreads) k_fft_plane_fwd(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];  // ny x nz
    __shared__ float2 stw[kFMaxN / 2];
    const int x = blockIdx.x, tid = threadIdx.x, P = a.ny * a.nz;
    if (tid < kFMaxN / 2) stw[tid] = a.tw[tid];
    const float *sp = a.src + (long long)x * P, *sn = sp + a.G;
    const bool xedge = x < a.A || x >= a.nx - a.A;
    int edge = 0;
    for (int e = tid; e < P; e += kFThreads) {
        const int y = e >> a.lz, z = e & (a.nz - 1);
        const float rp = __ldg(sp + e), rn = __ldg(sn + e);
        if ((rp != 0.0f || rn != 0.0f) && (xedge || y < a.B || y >= a.ny - a.B || z < a.W || z >= a.nz - a.W))
            edge = 1;
        fs[(bit_reverse(y, a.ly) << a.lz) + z] = make_float2(rp, rn);
    }
    edge = __syncthreads_or(edge);
    if (tid == 0) a.edge[x] = edge;
    fft_stages<false>(fs, a.nz, a.lz, a.ly, a.nz, 1, stw, false);
    fft_stages<true>(fs, a.ny, a.ly, a.lz, 1, a.nz, stw, false);
    float2 *out = a.work + (long long)x * P;
    for (int e = tid; e < P; e += kFThreads) out[e] = fs[e];
}

__global__ void __launch_bounds__(kFThreads) k_fft_columns(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];  // nx x nz
    __shared__ float2 stw[kFMaxN / 2];
    const int y = blockIdx.x, tid = threadIdx.x, P = a.ny * a.nz, L = a.nx * a.nz;
    if (tid < kFMaxN / 2) stw[tid] = a.tw[tid];
    for (int e = tid; e < L; e += kFThreads) {
        const int x = e >> a.lz, z = e & (a.nz - 1);
        fs[(bit_reverse(x, a.lx) << a.lz) + z] = a.work[(long long)x * P + y * a.nz + z];
    }
    __syncthreads();
    fft_stages<true>(fs, a.nx, a.lx, a.lz, 1, a.nz, stw, false);
    for (int e = tid; e < L; e += kFThreads) {
        const int x = e >> a.lz, z = e & (a.nz - 1);
        const float kh = __ldg(a.khat + (long long)x * P + y * a.nz + z);
        fs[e] = make_float2(fs[e].x * kh, fs[e].y * kh);
    }
    __syncthreads();
    fft_stages<false>(fs, a.nx, a.lx, a.lz, 1, a.nz, stw, true);
    for (int e = tid; e < L; e += kFThreads) {
        const int x = e >> a.lz, z = e & (a.nz - 1);
        a.work[(long long)x * P + y * a.nz + z] = fs[(bit_reverse(x, a.lx) << a.lz) + z];
    }
}

__global__ void __launch_bounds__(kFThreads) k_fft_plane_inv(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];  // ny x nz
    __shared__ float2 stw[kFMaxN / 2];
    const int x = blockIdx.x, tid = threadIdx.x, P = a.ny * a.nz;
    if (tid < kFMaxN / 2) stw[tid] = a.tw[tid];
    const float2 *in = a.work + (long long)x * P;
    for (int e = tid; e < P; e += kFThreads) fs[e] = in[e];
    __syncthreads();
    fft_stages<true>(fs, a.nz, a.lz, a.ly, a.nz, 1, stw, true);
    fft_stages<false>(fs, a.ny, a.ly, a.lz, 1, a.nz, stw, true);
    float *dp = a.dst + (long long)x * P, *dn = dp + a.G;
    for (int e = tid; e < P; e += kFThreads) {
        const int y = e >> a.lz, z = e & (a.nz - 1);
        const float2 v = fs[(bit_reverse(y, a.ly) << a.lz) + z];
        // the exact sum is non-negative; the transform's rounding (~1e-7 of
        // the maximum) must not leave negative densities, where the Skyrme
        // term rho^gamma has no value
        dp[e] = fmaxf(v.x * a.post, 0.0f);
        dn[e] = fmaxf(v.y * a.post, 0.0f);
    }
}

// khat(kx, ky, zrev(kz)) = sum_a cx[a][kx] Y_a(ky, kz): the last sum of the
// stencil's spectrum, one node per thread, in double.  zrev = 0 keeps z in
// natural order (the 128^3 form below).
__global__ void k_fft_khat(int nx, int P, int nz, int lz, int na, const double *cx, const double *ya, float *khat,
                           int zrev) {
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= (long long)nx * P) return;
    const int kx = (int)(id / P), q = (int)(id - (long long)kx * P);
    double acc = 0.0;
    for (int a = 0; a < na; a++) acc += cx[a * nx + kx] * ya[(size_t)a * P + q];
    const int ky = q >> lz, kz = q & (nz - 1);
    khat[(long long)kx * P + ((long long)ky << lz) + (zrev ? bit_reverse(kz, lz) : kz)] = (float)acc;
}

// ---- The 128^3 form: 128-point transforms as 16 x 8 in registers ----------
//
// A block transforms 128 lines of 128 points, eight threads a line (thread j
// of a line holds points j + 8c, c = 0..15).  With n = 8a + b and
// k = k1 + 16 k2 (a, k1 < 16; b, k2 < 8):
//   X[k1 + 16 k2] = sum_b W8^(b k2) W128^(b k1) sum_a x[8a + b] W16^(a k1).
// Thread j computes the inner 16-point transform of its points in registers
// and multiplies by W128^(j k1); the 16 x 8 values of a line then cross once
// through shared memory (position 8 k1 + b), and thread j takes k1 = j and
// j + 8 for two 8-point transforms over b.  It ends holding X[j + 8c], the
// layout it started from, so a forward and an inverse transform chain in
// registers.  The warps of a block hold 32 consecutive lines each (thread
// index = j * 128 + line), so a warp's 32 accesses of any step go to 32
// lines: consecutive addresses along a column, or rows 129 complex apart,
// which spreads them over every bank.  An inverse is conj(forward(conj(.))).
// Per kernel the plane crosses shared memory four times (twice per axis)
// instead of once per radix-4 stage.
constexpr int kF128 = 128;
constexpr int kFRow = 129;  // row stride of a shared plane, in complex elements
constexpr size_t kF128Smem = sizeof(float2) * kF128 * kFRow;

__host__ __device__ constexpr int brev4(int i) { return ((i & 1) << 3) | ((i & 2) << 1) | ((i & 4) >> 1) | ((i & 8) >> 3); }
__host__ __device__ constexpr int brev3(int i) { return ((i & 1) << 2) | (i & 2) | ((i & 4) >> 2); }

// v W16^e for e in [0, 8): W16 = exp(-2 pi i / 16); cos and sin of pi/8,
// pi/4 and 3 pi/8
__device__ __forceinline__ float2 mul_w16(float2 v, int e) {
    constexpr float c1 = 0.923879532511286756f, s1 = 0.382683432365089772f, r2 = 0.707106781186547524f;
    switch (e) {
        case 1: return make_float2(c1 * v.x + s1 * v.y, c1 * v.y - s1 * v.x);
        case 2: return make_float2(r2 * (v.x + v.y), r2 * (v.y - v.x));
        case 3: return make_float2(s1 * v.x + c1 * v.y, s1 * v.y - c1 * v.x);
        case 4: return make_float2(v.y, -v.x);
        case 5: return make_float2(c1 * v.y - s1 * v.x, -s1 * v.y - c1 * v.x);
        case 6: return make_float2(r2 * (v.y - v.x), -r2 * (v.x + v.y));
        case 7: return make_float2(s1 * v.y - c1 * v.x, -c1 * v.y - s1 * v.x);
        default: return v;
    }
}

// In-place decimation-in-frequency transform of N = 16 or 8 points in
// registers (natural in, bit-reversed out); every index and twiddle exponent
// is a constant once unrolled.
template <int N>
__device__ __forceinline__ void dft_regs(float2 (&a)[N]) {
#pragma unroll
    for (int h = N / 2; h >= 1; h >>= 1) {
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (i & h) continue;
            const float2 u = a[i], v = a[i + h];
            a[i] = cadd(u, v);
            a[i + h] = mul_w16(csub(u, v), (i & (h - 1)) * (8 / h));
        }
    }
}

// The 128-point transform of one line (see above): r holds points j + 8c in,
// X[j + 8c] out.  xb[p * ps] is the line's exchange area (p < 128), tw the
// 128 powers of W128.  Every thread of the block calls it at once.
__device__ __forceinline__ void fft128_line(float2 (&r)[16], int j, float2 *xb, int ps, const float2 *tw) {
    dft_regs<16>(r);  // r[brev4(k1)] = sum_a x[8a + j] W16^(a k1)
#pragma unroll
    for (int k1 = 1; k1 < 16; k1++) r[brev4(k1)] = cmul(r[brev4(k1)], tw[(j * k1) & 127]);
    __syncthreads();  // the exchange area may still hold inputs being read
#pragma unroll
    for (int k1 = 0; k1 < 16; k1++) xb[(8 * k1 + j) * ps] = r[brev4(k1)];
    __syncthreads();
    float2 e0[8], e1[8];
#pragma unroll
    for (int b = 0; b < 8; b++) {
        e0[b] = xb[(8 * j + b) * ps];
        e1[b] = xb[(64 + 8 * j + b) * ps];
    }
    dft_regs<8>(e0);  // e0[brev3(k2)] = X[j + 16 k2]
    dft_regs<8>(e1);  // e1[brev3(k2)] = X[j + 8 + 16 k2]
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) {
        r[2 * k2] = e0[brev3(k2)];
        r[2 * k2 + 1] = e1[brev3(k2)];
    }
}

__device__ __forceinline__ float2 cconj(float2 v) { return make_float2(v.x, -v.y); }

__device__ __forceinline__ void load_tw128(const float2 *tw64, float2 *tw) {
    if (threadIdx.x < 64) {
        const float2 w = tw64[threadIdx.x];
        tw[threadIdx.x] = w;
        tw[threadIdx.x + 64] = make_float2(-w.x, -w.y);  // W128^(m + 64) = -W128^m
    }
}

// Pass 1 at 128^3, per x plane: forward along y (lines are z columns, loaded
// straight from the densities: consecutive lanes, consecutive z), then along
// z (lines are rows of the shared plane), stored through the plane so that
// the store is coalesced.  Flags density within the stencil of a face, and
// records which groups of four y rows of the plane hold raw density of each
// species (the forces kernel computes only those).
__global__ void __launch_bounds__(kFThreads, 1) k_fft128_plane_fwd(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];  // 128 rows of kFRow
    __shared__ float2 tw[kF128];
    __shared__ unsigned s_occ[2];
    const int x = blockIdx.x, tid = threadIdx.x, line = tid & 127, j = tid >> 7, P = kF128 * kF128;
    load_tw128(a.tw, tw);
    if (tid < 2) s_occ[tid] = 0u;
    const float *sp = a.src + (long long)x * P, *sn = sp + a.G;
    const bool zx_edge = x < a.A || x >= kF128 - a.A || line < a.W || line >= kF128 - a.W;
    int edge = 0;
    // row groups y / 4 holding nonzero values of the warp's rows (a warp
    // shares j, so its rows are those of every lane: warp-uniform masks)
    unsigned op = 0u, on = 0u;
    float2 r[16];
#pragma unroll
    for (int c = 0; c < 16; c++) {
        const int y = j + 8 * c;
        const float rp = __ldg(sp + y * kF128 + line), rn = __ldg(sn + y * kF128 + line);
        if ((rp != 0.0f || rn != 0.0f) && (zx_edge || y < a.B || y >= kF128 - a.B)) edge = 1;
        if (__any_sync(0xffffffffu, rp != 0.0f)) op |= 1u << (y >> 2);
        if (__any_sync(0xffffffffu, rn != 0.0f)) on |= 1u << (y >> 2);
        r[c] = make_float2(rp, rn);
    }
    edge = __syncthreads_or(edge);  // also publishes tw and the cleared s_occ
    if (tid == 0) a.edge[x] = edge;
    if (a.occ && (tid & 31) == 0) {
        if (op) atomicOr(&s_occ[0], op);
        if (on) atomicOr(&s_occ[1], on);
    }
    fft128_line(r, j, fs + line, kFRow, tw);  // r[c] = V[ky = j + 8c][z = line]
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) fs[(j + 8 * c) * kFRow + line] = r[c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) r[c] = fs[line * kFRow + j + 8 * c];
    fft128_line(r, j, fs + line * kFRow, 1, tw);  // r[c] = Z[ky = line][kz = j + 8c]
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) fs[line * kFRow + j + 8 * c] = r[c];
    __syncthreads();
    float2 *out = a.work + (long long)x * P;
    for (int e = tid; e < P; e += kFThreads) out[e] = fs[(e >> 7) * kFRow + (e & 127)];
    if (a.occ && tid < 2) a.occ[tid * kF128 + x] = s_occ[tid];  // complete: barriers since the atomics
}

// Pass 2 at 128^3, per y: forward along x (lines are z columns, loaded and
// stored straight: consecutive lanes, consecutive z), the product by the
// spectrum (natural order), and the inverse along x.
__global__ void __launch_bounds__(kFThreads, 1) k_fft128_columns(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];
    __shared__ float2 tw[kF128];
    const int y = blockIdx.x, tid = threadIdx.x, line = tid & 127, j = tid >> 7, P = kF128 * kF128;
    load_tw128(a.tw, tw);
    float2 *col = a.work + (long long)y * kF128 + line;
    const float *kh = a.khat + (long long)y * kF128 + line;
    float2 r[16];
#pragma unroll
    for (int c = 0; c < 16; c++) r[c] = col[(long long)(j + 8 * c) * P];
    __syncthreads();  // tw
    fft128_line(r, j, fs + line, kFRow, tw);  // r[c] = F[kx = j + 8c]
#pragma unroll
    for (int c = 0; c < 16; c++) {
        const float k = __ldg(kh + (long long)(j + 8 * c) * P);
        r[c] = cconj(make_float2(r[c].x * k, r[c].y * k));
    }
    fft128_line(r, j, fs + line, kFRow, tw);
#pragma unroll
    for (int c = 0; c < 16; c++) col[(long long)(j + 8 * c) * P] = cconj(r[c]);
}

// Pass 3 at 128^3, per x plane: inverse along y (lines are z columns, loaded
// straight), then along z (rows), both species stored through the plane,
// scaled and clamped at 0.
__global__ void __launch_bounds__(kFThreads, 1) k_fft128_plane_inv(const __grid_constant__ FftArgs a) {
    extern __shared__ __align__(16) float2 fs[];
    __shared__ float2 tw[kF128];
    const int x = blockIdx.x, tid = threadIdx.x, line = tid & 127, j = tid >> 7, P = kF128 * kF128;
    load_tw128(a.tw, tw);
    const float2 *in = a.work + (long long)x * P + line;
    float2 r[16];
#pragma unroll
    for (int c = 0; c < 16; c++) r[c] = cconj(in[(j + 8 * c) * kF128]);
    __syncthreads();  // tw
    fft128_line(r, j, fs + line, kFRow, tw);  // r[c]: y = j + 8c, z = line (conjugated domain)
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) fs[(j + 8 * c) * kFRow + line] = r[c];
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) r[c] = fs[line * kFRow + j + 8 * c];
    fft128_line(r, j, fs + line * kFRow, 1, tw);  // r[c]: y = line, z = j + 8c
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 16; c++) fs[line * kFRow + j + 8 * c] = r[c];
    __syncthreads();
    float *dp = a.dst + (long long)x * P, *dn = dp + a.G;
    for (int e = tid; e < P; e += kFThreads) {
        const float2 v = cconj(fs[(e >> 7) * kFRow + (e & 127)]);
        // the exact sum is non-negative; rounding must not leave negative
        // densities, where rho^gamma has no value
        dp[e] = fmaxf(v.x * a.post, 0.0f);
        dn[e] = fmaxf(v.y * a.post, 0.0f);
    }
}

int log2_exact(int n) {
    int l = 0;
    while ((1 << l) < n) l++;
    return (1 << l) == n ? l : -1;
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

    // FFT form: power-of-two axes of 2..128 whose planes fit in shared memory
    const Geom &gg = c->geom;
    const int lx = log2_exact(gg.nx), ly = log2_exact(gg.ny), lz = log2_exact(gg.nz);
    if (lx < 1 || ly < 1 || lz < 1 || gg.nx > kFMaxN || gg.ny > kFMaxN || gg.nz > kFMaxN ||
        gg.ny * gg.nz > kFMaxPlane || gg.nx * gg.nz > kFMaxPlane || 2 * A + 2 > gg.nx || 2 * B + 2 > gg.ny ||
        2 * W + 2 > gg.nz)
        return HV_OK;
    // The stencil's spectrum, in double: with the taps symmetric per axis,
    //   K(kx,ky,kz) = sum_a m_a g(a) cos(2 pi a kx / nx) Y_|a|(ky, kz),
    //   Y_a(ky,kz)  = sum_{b <= bm(a)} m_b g(b) cos(2 pi b ky / ny) Z_w(a,b)(kz),
    //   Z_w(kz)     = sum_{|c| <= w} g(c) cos(2 pi c kz / nz),
    // m = 1 at 0 and 2 elsewhere; scaled by term / G (the inverse transform's 1/G).
    const int nx = gg.nx, ny = gg.ny, nz = gg.nz, P = ny * nz;
    f.fft128 = nx == kF128 && ny == kF128 && nz == kF128;
    std::vector<double> gxd(A + 1), gyd(B + 1), gzd(W + 1);
    auto g1d = [&](int axis, int off) {
        const int n = wd.n[axis], ctr = n / 2;
        const double dm = wd.d_max[axis];
        double d = dm * (2.0 * ctr / n - 1.0) - dm * (2.0 * (ctr + off) / n - 1.0);
        return std::exp(-d * d * e);
    };
    for (int a = 0; a <= A; a++) gxd[a] = g1d(0, a);
    for (int b = 0; b <= B; b++) gyd[b] = g1d(1, b);
    for (int cz = 0; cz <= W; cz++) gzd[cz] = g1d(2, cz);
    const double twopi = 2.0 * kPi;
    std::vector<double> zw((size_t)(W + 1) * nz);
    for (int kz = 0; kz < nz; kz++) {
        double acc = gzd[0];
        zw[kz] = acc;
        for (int w = 1; w <= W; w++) {
            acc += 2.0 * gzd[w] * std::cos(twopi * w * kz / nz);
            zw[(size_t)w * nz + kz] = acc;
        }
    }
    std::vector<double> ya((size_t)(A + 1) * P, 0.0);
    for (int a = 0; a <= A; a++) {
        if (f.bm[a] < 0) continue;
        for (int b = 0; b <= f.bm[a]; b++) {
            const int w = f.wt[a * (kMaxR + 1) + b];
            const double mb = b ? 2.0 : 1.0;
            for (int ky = 0; ky < ny; ky++) {
                const double cy = mb * gyd[b] * std::cos(twopi * b * ky / ny);
                double *row = &ya[(size_t)a * P + (size_t)ky * nz];
                const double *zr = &zw[(size_t)w * nz];
                for (int kz = 0; kz < nz; kz++) row[kz] += cy * zr[kz];
            }
        }
    }
    const hv_run_params &pr = c->params;
    f.fft_term = (1.0 / pr.part_per_nucleon) * (1.0 / std::pow(2.0 * kPi * sig * sig, 1.5));
    const double scale = f.fft_term / (double)gg.G;
    // cx[a][kx] = m_a g(a) cos(2 pi a kx / nx) x term / G (zero for |a| without taps)
    std::vector<double> cxv((size_t)(A + 1) * nx, 0.0);
    for (int a = 0; a <= A; a++) {
        if (f.bm[a] < 0) continue;
        for (int kx = 0; kx < nx; kx++)
            cxv[(size_t)a * nx + kx] = (a ? 2.0 : 1.0) * gxd[a] * std::cos(twopi * a * kx / nx) * scale;
    }
    std::vector<float2> tw(kFMaxN / 2);
    for (int m = 0; m < kFMaxN / 2; m++)
        tw[m] = make_float2((float)std::cos(twopi * m / kFMaxN), (float)-std::sin(twopi * m / kFMaxN));
    HV_CUDA(cudaMalloc(&f.fwork, sizeof(float2) * gg.G));
    HV_CUDA(cudaMalloc((void **)&f.khat, sizeof(float) * gg.G));
    HV_CUDA(cudaMalloc(&f.tw, sizeof(float2) * tw.size()));
    HV_CUDA(cudaMalloc((void **)&f.edge, sizeof(int) * nx));
    HV_CUDA(cudaMalloc((void **)&f.occ, sizeof(unsigned) * 2 * nx));
    // the wrap correction's particle list
    HV_CUDA(cudaMalloc(&f.wlist, sizeof(float4) * kWrapParticles));
    // copies ordered on the context stream before the kernels that read
    // them (a cudaMemcpy from pageable memory may return before its DMA ends)
    HV_CUDA(cudaMemcpyAsync(f.tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice, c->stream));
    {
        double *dcx = nullptr, *dya = nullptr;
        HV_CUDA(cudaMalloc((void **)&dcx, sizeof(double) * cxv.size()));
        if (cudaMalloc((void **)&dya, sizeof(double) * ya.size()) != cudaSuccess) {
            cudaFree(dcx);
            set_last_error("smoothing plan: device allocation failed");
            return HV_ERR_CUDA;
        }
        cudaError_t ce =
            cudaMemcpyAsync(dcx, cxv.data(), sizeof(double) * cxv.size(), cudaMemcpyHostToDevice, c->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(dya, ya.data(), sizeof(double) * ya.size(), cudaMemcpyHostToDevice, c->stream);
        if (ce == cudaSuccess) {
            k_fft_khat<<<(unsigned)((gg.G + 255) / 256), 256, 0, c->stream>>>(nx, P, nz, lz, A + 1, dcx, dya,
                                                                             f.khat, f.fft128 ? 0 : 1);
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->stream);
        cudaFree(dcx);
        cudaFree(dya);
        HV_CUDA(ce);
    }
    const size_t plane = sizeof(float2) * (size_t)std::max(P, nx * nz);
    for (const void *k : {(const void *)k_fft_plane_fwd, (const void *)k_fft_columns, (const void *)k_fft_plane_inv})
        HV_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane));
    for (const void *k :
         {(const void *)k_fft128_plane_fwd, (const void *)k_fft128_columns, (const void *)k_fft128_plane_inv})
        HV_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kF128Smem));
    f.fft = true;
    return HV_OK;
}

void smooth_fast_release(hv_ctx *c) {
    SmoothFast &f = c->fused.smooth;
    void *ptrs[] = {f.fwork, f.khat, f.tw, f.edge, f.occ, f.wlist};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    f = SmoothFast();
}

bool smooth_fft_runs(const hv_ctx *c) {
    const SmoothFast &f = c->fused.smooth;
    // auto: the transform pays off against the direct sum for wide stencils
    const bool wide = std::max(f.A, std::max(f.B, f.W)) >= kFftAutoHalfWidth;
    return f.ok && f.fft && (c->fast.smooth_fft == 2 || (c->fast.smooth_fft == 1 && wide));
}

hv_status smooth_fast_launch(hv_ctx *c, const float *rho_raw, float *rho, const int *wcount) {
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
    const double term = (1.0 / p.part_per_nucleon) * (1.0 / std::pow(2.0 * kPi * sig * sig, 1.5));
    a.term = (float)term;
    for (int i = 0; i <= kMaxR; i++) {
        a.gx[i] = f.gx[i];
        a.gy[i] = f.gy[i];
        a.gz[i] = f.gz[i];
        a.bm[i] = f.bm[i];
    }
    for (int i = 0; i < (kMaxR + 1) * (kMaxR + 1); i++) a.wt[i] = f.wt[i];
    a.src = rho_raw;
    a.dst = rho;
    a.edge = nullptr;
    a.wcount = nullptr;
    a.wcap = kWrapParticles;
    a.wlist = nullptr;
    if (smooth_fft_runs(c)) {
        FftArgs q;
        q.nx = g.nx;
        q.ny = g.ny;
        q.nz = g.nz;
        q.lx = log2_exact(g.nx);
        q.ly = log2_exact(g.ny);
        q.lz = log2_exact(g.nz);
        q.A = f.A;
        q.B = f.B;
        q.W = f.W;
        q.G = g.G;
        q.src = rho_raw;
        q.dst = rho;
        q.work = reinterpret_cast<float2 *>(f.fwork);
        q.khat = f.khat;
        q.tw = reinterpret_cast<const float2 *>(f.tw);
        q.edge = f.edge;
        q.occ = f.fft128 ? f.occ : nullptr;
        q.post = (float)(term / f.fft_term);
        a.edge = f.edge;
        // the wrap correction (in the march kernel's launch): the particle
        // step's list; none in the deterministic deposit mode, whose
        // smoothing stays deterministic by the direct form
        a.wcount = p.deposit_mode == HV_DEPOSIT_SORTED ? nullptr : wcount;
        a.wlist = reinterpret_cast<const float4 *>(f.wlist);
        if (f.fft128) {
            k_fft128_plane_fwd<<<kF128, kFThreads, kF128Smem, c->stream>>>(q);
            k_fft128_columns<<<kF128, kFThreads, kF128Smem, c->stream>>>(q);
            k_fft128_plane_inv<<<kF128, kFThreads, kF128Smem, c->stream>>>(q);
        } else {
            const size_t plane = sizeof(float2) * (size_t)g.ny * g.nz, slab = sizeof(float2) * (size_t)g.nx * g.nz;
            k_fft_plane_fwd<<<g.nx, kFThreads, plane, c->stream>>>(q);
            k_fft_columns<<<g.ny, kFThreads, slab, c->stream>>>(q);
            k_fft_plane_inv<<<g.nx, kFThreads, plane, c->stream>>>(q);
        }
        HV_CUDA(cudaGetLastError());
    }
    const int tz = (g.nz + kMBK - 1) / kMBK, ty = (g.ny + kMBY - 1) / kMBY;
    void *args[] = {&a};
    HV_CUDA(cudaLaunchKernel(march_kernel(f.per), dim3(2 * f.xsplit * ty * tz), dim3(kMThreads), args, f.smem,
                             c->stream));
    return HV_OK;
}

}  // namespace hv
