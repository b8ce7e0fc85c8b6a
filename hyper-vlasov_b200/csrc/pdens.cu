// Per-particle densities of the initialisation, compute_particle_densities
// (include/tools.hpp:170-203), with cell lists.
//
// The reference sums, for every particle, exp(-d^2 / (2 sigma_r^2)) over all
// particles within d^2 <= 16 sigma_r^2 -- an O(N^2) double loop.  Here the
// particles are binned into cubic cells of edge sigma_r over their bounding
// box and sorted by cell (CUB radix sort); a particle scans, per (x, y) row of
// cells within the cutoff, the z run of cells that the cutoff sphere reaches.
// One thread per particle, in sorted order: the threads of a warp share a
// cell, hence scan nearly the same cells, and their partner loads are
// broadcasts.  The per-particle sums keep the reference's arithmetic type;
// only their order differs (cell by cell instead of index order).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kBlock = 256;
constexpr int kMaxCells = 1 << 22;  // cells of the bounding box (coarser cells beyond)

inline int nb(long long n) { return div_up(n > 0 ? n : 1, kBlock); }

template <typename T>
__global__ void k_bbox_partials(int total, const T *__restrict__ x, const T *__restrict__ y,
                                const T *__restrict__ z, double *partials) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const double v[3] = {(double)x[i], (double)y[i], (double)z[i]};
        for (int a = 0; a < 3; a++) {
            lo[a] = fmin(lo[a], v[a]);
            hi[a] = fmax(hi[a], v[a]);
        }
    }
    __shared__ double sh[6][kBlock];
    for (int a = 0; a < 3; a++) {
        sh[a][threadIdx.x] = lo[a];
        sh[3 + a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int a = 0; a < 3; a++) {
                sh[a][threadIdx.x] = fmin(sh[a][threadIdx.x], sh[a][threadIdx.x + o]);
                sh[3 + a][threadIdx.x] = fmax(sh[3 + a][threadIdx.x], sh[3 + a][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) partials[6 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

struct Cells {
    double lo[3];
    double inv;  // 1 / cell edge
    int n[3];
};

__device__ __forceinline__ int cell_axis(double v, double lo, double inv, int n) {
    int c = (int)((v - lo) * inv);
    return c < 0 ? 0 : c >= n ? n - 1 : c;
}

template <typename T>
__global__ void k_cell_of(int total, Cells cl, const T *__restrict__ x, const T *__restrict__ y,
                          const T *__restrict__ z, unsigned *keys, int *idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int cx = cell_axis((double)x[i], cl.lo[0], cl.inv, cl.n[0]);
    const int cy = cell_axis((double)y[i], cl.lo[1], cl.inv, cl.n[1]);
    const int cz = cell_axis((double)z[i], cl.lo[2], cl.inv, cl.n[2]);
    keys[i] = (unsigned)((cx * cl.n[1] + cy) * cl.n[2] + cz);
    idx[i] = i;
}

// start[c] = first sorted slot of cell c, start[ncells] = total.
__global__ void k_cell_ranges(int total, int ncells, const unsigned *__restrict__ keys, int *start) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > total) return;
    const int k = s < total ? (int)keys[s] : ncells;
    const int prev = s > 0 ? (int)keys[s - 1] : -1;
    for (int c = prev + 1; c <= k; c++) start[c] = s;
}

// Sorted positions packed with the species: (x, y, z, 1 for a proton, 0 for
// a neutron), one vector load per partner.
template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
    using type = float4;
};
template <>
struct Vec4<double> {
    using type = double4;
};

template <typename T>
__global__ void k_sorted_positions(int total, int protons, const int *__restrict__ idx, const T *__restrict__ x,
                                   const T *__restrict__ y, const T *__restrict__ z, typename Vec4<T>::type *sp) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    const int i = idx[s];
    typename Vec4<T>::type v;
    v.x = x[i];
    v.y = y[i];
    v.z = z[i];
    v.w = i < protons ? T(1) : T(0);
    sp[s] = v;
}

// exp(-d2 * e): in float as exp2f(d2 * c) with c = -e log2(e), in double exp.
__device__ __forceinline__ float gauss(float d2, float e, float c) { return exp2f(d2 * c); }
__device__ __forceinline__ double gauss(double d2, double e, double) { return exp(-d2 * e); }

// Sums over the cells that the cutoff sphere of particle s (sorted order)
// reaches, results to the particle's own slot.  Per (x, y) row of cells, only
// the z range of cells within `reach` of the particle is scanned (a sorted,
// contiguous slot range); reach is the cutoff radius with a margin for the
// rounding of d^2 in T, whose test decides.
template <typename T>
__global__ void k_pair_densities(int total, Cells cl, double edge, double reach, T exp_term, T exp2_term, T cutoff,
                                 T term, const int *__restrict__ idx, const int *__restrict__ start,
                                 const typename Vec4<T>::type *__restrict__ sp, T *dp, T *dn) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    const typename Vec4<T>::type me = sp[s];
    const T xi = me.x, yi = me.y, zi = me.z;
    const double px = (double)xi, py = (double)yi, pz = (double)zi, r2 = reach * reach;
    const int x0 = cell_axis(px - reach, cl.lo[0], cl.inv, cl.n[0]), x1 = cell_axis(px + reach, cl.lo[0], cl.inv, cl.n[0]);
    const int y0 = cell_axis(py - reach, cl.lo[1], cl.inv, cl.n[1]), y1 = cell_axis(py + reach, cl.lo[1], cl.inv, cl.n[1]);
    T a = T(0), b = T(0);
    for (int ix = x0; ix <= x1; ix++) {
        const double clo = cl.lo[0] + ix * edge, chi = clo + edge;
        const double dx = px < clo ? clo - px : px > chi ? px - chi : 0.0;
        for (int iy = y0; iy <= y1; iy++) {
            const double rlo = cl.lo[1] + iy * edge, rhi = rlo + edge;
            const double dy = py < rlo ? rlo - py : py > rhi ? py - rhi : 0.0;
            const double rem = r2 - dx * dx - dy * dy;
            if (rem < 0.0) continue;
            const double dz = sqrt(rem);
            const int z0 = cell_axis(pz - dz, cl.lo[2], cl.inv, cl.n[2]), z1 = cell_axis(pz + dz, cl.lo[2], cl.inv, cl.n[2]);
            const int row = (ix * cl.n[1] + iy) * cl.n[2];
            const int j0 = start[row + z0], j1 = start[row + z1 + 1];
            for (int j = j0; j < j1; j++) {
                const typename Vec4<T>::type o = sp[j];
                const T ex = xi - o.x, ey = yi - o.y, ez = zi - o.z;
                const T d2 = ex * ex + ey * ey + ez * ez;
                if (d2 > cutoff) continue;
                const T f = gauss(d2, exp_term, exp2_term);
                a += o.w * f;        // protons
                b += f - o.w * f;    // neutrons
            }
        }
    }
    const int i = idx[s];
    dp[i] = a * term;
    dn[i] = b * term;
}

}  // namespace

template <typename T>
hv_status particle_densities_at(hv_ctx *c, int N, int protons, const T *px, const T *py, const T *pz, T *dp_dev,
                                T *dn_dev) {
    if (N == 0) return HV_OK;
    cudaStream_t s = c->stream;
    // bounding box
    const int bb = std::min(nb(N), 4 * c->sm_count);
    double *part = nullptr;
    HV_CUDA(cudaMallocAsync((void **)&part, sizeof(double) * 6 * bb, s));
    k_bbox_partials<T><<<bb, kBlock, 0, s>>>(N, px, py, pz, part);
    std::vector<double> hp((size_t)6 * bb);
    HV_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(double) * 6 * bb, cudaMemcpyDeviceToHost, s));
    HV_CUDA(cudaFreeAsync(part, s));
    HV_CUDA(cudaStreamSynchronize(s));
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int b = 0; b < bb; b++)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], hp[6 * b + a]);
            hi[a] = std::max(hi[a], hp[6 * b + 3 + a]);
        }
    // cells of a quarter of the cutoff radius 4 sigma_r (coarser when the
    // bounding box would need more than kMaxCells)
    const double sig = c->params.sigma_r;
    double edge = sig;
    Cells cl;
    for (;;) {
        long long cells = 1;
        for (int a = 0; a < 3; a++) {
            cl.n[a] = (int)std::floor((hi[a] - lo[a]) / edge) + 1;
            cells *= cl.n[a];
        }
        if (cells <= kMaxCells) break;
        edge *= 2.0;
    }
    for (int a = 0; a < 3; a++) cl.lo[a] = lo[a];
    cl.inv = 1.0 / edge;
    const int ncells = cl.n[0] * cl.n[1] * cl.n[2];
    // sort particles by cell
    unsigned *keys = nullptr, *keys2 = nullptr;
    int *idx = nullptr, *idx2 = nullptr, *start = nullptr;
    typename Vec4<T>::type *sp = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int bits = 1;
    while ((1ll << bits) < ncells + 1) bits++;
    HV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, idx, idx2, N, 0, bits, s));
    HV_CUDA(cudaMallocAsync((void **)&keys, sizeof(unsigned) * N, s));
    HV_CUDA(cudaMallocAsync((void **)&keys2, sizeof(unsigned) * N, s));
    HV_CUDA(cudaMallocAsync((void **)&idx, sizeof(int) * N, s));
    HV_CUDA(cudaMallocAsync((void **)&idx2, sizeof(int) * N, s));
    HV_CUDA(cudaMallocAsync((void **)&start, sizeof(int) * (ncells + 1), s));
    HV_CUDA(cudaMallocAsync((void **)&sp, sizeof(typename Vec4<T>::type) * N, s));
    HV_CUDA(cudaMallocAsync(&tmp, tmp_bytes, s));
    k_cell_of<T><<<nb(N), kBlock, 0, s>>>(N, cl, px, py, pz, keys, idx);
    HV_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, idx, idx2, N, 0, bits, s));
    k_cell_ranges<<<nb(N + 1), kBlock, 0, s>>>(N, ncells, keys2, start);
    k_sorted_positions<T><<<nb(N), kBlock, 0, s>>>(N, protons, idx2, px, py, pz, sp);
    const T sr = T(sig);
    const T exp_term = T(1.0) / (T(2.0) * sr * sr), cutoff = T(16.0) * sr * sr;
    const T exp2_term = T(-1.4426950408889634) * exp_term;  // -log2(e) / (2 sigma_r^2)
    const T term = (T(1.0) / c->params.part_per_nucleon) * (T(1.0) / std::pow(T(2.0) * T(kPi) * sr * sr, T(1.5)));
    const double reach = 4.0 * sig * (1.0 + 1e-5);
    k_pair_densities<T><<<nb(N), kBlock, 0, s>>>(N, cl, edge, reach, exp_term, exp2_term, cutoff, term, idx2, start, sp, dp_dev,
                                                 dn_dev);
    HV_CUDA(cudaGetLastError());
    void *bufs[] = {keys, keys2, idx, idx2, start, sp, tmp};
    for (void *p : bufs) HV_CUDA(cudaFreeAsync(p, s));
    return HV_OK;
}

template hv_status particle_densities_at<double>(hv_ctx *, int, int, const double *, const double *, const double *,
                                                 double *, double *);
template hv_status particle_densities_at<float>(hv_ctx *, int, int, const float *, const float *, const float *,
                                                float *, float *);

}  // namespace hv

using namespace hv;

extern "C" hv_status hv_particle_densities(hv_ctx *c, void *density_p, void *density_n) {
    if (!c || (!density_p && c->total) || (!density_n && c->total)) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    if (c->total == 0) return HV_OK;
    const size_t es = c->prec == HV_F64 ? 8 : 4, bytes = es * c->total;
    void *dp = nullptr, *dn = nullptr;
    HV_CUDA(cudaMallocAsync(&dp, bytes, c->stream));
    HV_CUDA(cudaMallocAsync(&dn, bytes, c->stream));
    hv_status st = c->prec == HV_F64
                       ? particle_densities_at<double>(c, c->total, c->protons, c->d64.x, c->d64.y, c->d64.z,
                                                       (double *)dp, (double *)dn)
                       : particle_densities_at<float>(c, c->total, c->protons, c->d32.x, c->d32.y, c->d32.z,
                                                      (float *)dp, (float *)dn);
    if (st == HV_OK) st = download_slots(c, dp, density_p);
    if (st == HV_OK) st = download_slots(c, dn, density_n);
    cudaFreeAsync(dp, c->stream);
    cudaFreeAsync(dn, c->stream);
    HV_CUDA(cudaStreamSynchronize(c->stream));
    return st;
}
