// hv_observe_noalloc: the observables reduction (centre of mass and mean
// squared radius per species, and D) for callers that cannot allocate device
// memory.
//
// Some callers of this library must not call cudaMalloc: a host framework
// that has reserved the GPU's memory for its own allocator, or code that runs
// in a region where allocation is not permitted.  They can still pass their
// particle arrays (device memory they own) and receive the result, because
// the only scratch this reduction needs -- one row of partial sums per block
// and the final sums -- lives in the file-scope array below instead of a
// context.  That array is held by every GPU that loads the library until the
// process exits (kMaxBlocks + 1 rows of 8 doubles, 256 KiB), and it limits
// one call to kMaxBlocks * kPerBlock particles.  Every call shares it and it
// keeps the last call's contents; each call rewrites every row it reads, so
// nothing has to be cleared.  Calls whose work overlaps on the GPU (on
// different streams, or from different host threads) race on the array.
#include <cmath>

#include "hv_internal.h"

namespace hv {
namespace {

constexpr int kThreads = 256;
constexpr int kPerBlock = 1024;    // particles per block
constexpr int kMaxBlocks = 4096;   // rows of partial sums
constexpr int kWidth = 8;          // doubles per row (6 used)

// Scratch of hv_observe_noalloc: rows 0..kMaxBlocks-1 hold per-block partial
// sums, row kMaxBlocks the final sums.
static __device__ __align__(256) double g_noalloc_scratch[(kMaxBlocks + 1) * kWidth];

// x^2 + y^2 + z^2 rounded after every operation (no contraction into FMA), as
// the dot product of include/math_functions.hpp:45-48 and hv_observe compute it.
__device__ __forceinline__ float dot3(float x, float y, float z) {
    return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}
__device__ __forceinline__ double dot3(double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Per-block sums {z_p, z_n, r2_p, r2_n, n_in_p, n_in_n} of particles
// [b * kPerBlock, (b + 1) * kPerBlock) (include/tools.hpp:302-338), reduced
// in a fixed order.
template <typename T>
__global__ void k_observe_rows(Geom g, int protons, int total, const T *__restrict__ x, const T *__restrict__ y,
                               const T *__restrict__ z, double *scratch) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    const T dmx = T(g.dmx), dmy = T(g.dmy), dmz = T(g.dmz);
    const int end = min(total, (blockIdx.x + 1) * kPerBlock);
    for (int i = blockIdx.x * kPerBlock + threadIdx.x; i < end; i += kThreads) {
        const int s = i < protons ? 0 : 1;
        const T xi = x[i], yi = y[i], zi = z[i];
        v[s] += (double)zi;
        if (xi < -dmx || xi > +dmx || yi < -dmy || yi > +dmy || zi < -dmz || zi > +dmz) continue;
        v[2 + s] += (double)dot3(xi, yi, zi);
        v[4 + s] += 1.0;
    }
    __shared__ double sh[6][kThreads / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int c = 0; c < 6; c++) {
        double u = v[c];
        for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
        if (l == 0) sh[c][w] = u;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double u = 0.0;
        for (int q = 0; q < kThreads / 32; q++) u += sh[threadIdx.x][q];
        scratch[blockIdx.x * kWidth + threadIdx.x] = u;
    }
}

// Final sums over the rows of the first nblocks blocks, in block order.
__global__ void k_observe_final(int nblocks, double *scratch) {
    const int c = threadIdx.x;
    if (c >= 6) return;
    double u = 0.0;
    for (int b = 0; b < nblocks; b++) u += scratch[b * kWidth + c];
    scratch[kMaxBlocks * kWidth + c] = u;
}

// Device address of the scratch array on the current device.  The name
// g_noalloc_scratch in host code is only a host-side stand-in, so every call
// asks the runtime for the address on the device that is current (the lookup
// allocates nothing).  Not caching it keeps the address right after the
// device's context has been reset and created again.
hv_status scratch_address(double **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
    *out = static_cast<double *>(p);
    return HV_OK;
}

template <typename T>
hv_status observe_typed(const Geom &g, int protons, int total, const void *x, const void *y, const void *z,
                        cudaStream_t stream, double *scratch, int nblocks, double sums[6]) {
    if (total > 0)
        k_observe_rows<T><<<nblocks, kThreads, 0, stream>>>(g, protons, total, static_cast<const T *>(x),
                                                            static_cast<const T *>(y), static_cast<const T *>(z),
                                                            scratch);
    k_observe_final<<<1, 32, 0, stream>>>(total > 0 ? nblocks : 0, scratch);
    HV_CUDA(cudaGetLastError());
    HV_CUDA(cudaMemcpyAsync(sums, scratch + kMaxBlocks * kWidth, 6 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    HV_CUDA(cudaStreamSynchronize(stream));
    return HV_OK;
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" hv_status hv_observe_noalloc(const hv_world *world, int protons, int neutrons, int nucleus_z,
                                        int nucleus_n, hv_precision prec, const void *x, const void *y,
                                        const void *z, void *stream, hv_observables *out) {
    if (!world || !out || protons < 0 || neutrons < 0 || nucleus_z < 0 || nucleus_n < 0 ||
        nucleus_z + nucleus_n <= 0 || (prec != HV_F64 && prec != HV_F32))
        return HV_ERR_BAD_ARG;
    for (int a = 0; a < 3; a++)
        if (world->n[a] < 1 || !(world->d_max[a] > 0.0)) return HV_ERR_BAD_ARG;
    const long long total = (long long)protons + neutrons;
    if (total > (long long)kMaxBlocks * kPerBlock) {
        set_last_error("hv_observe_noalloc: more than 4194304 particles; the fixed scratch has 4096 blocks of 1024");
        return HV_ERR_BAD_ARG;
    }
    if (total > 0 && (!x || !y || !z)) return HV_ERR_BAD_ARG;
    double *scratch = nullptr;
    HV_TRY(scratch_address(&scratch));
    const int nblocks = total > 0 ? (int)((total + kPerBlock - 1) / kPerBlock) : 0;
    double v[6] = {0, 0, 0, 0, 0, 0};
    const Geom g = make_geom(*world);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HV_TRY(prec == HV_F64 ? observe_typed<double>(g, protons, (int)total, x, y, z, s, scratch, nblocks, v)
                          : observe_typed<float>(g, protons, (int)total, x, y, z, s, scratch, nblocks, v));
    hv_observables o;
    o.t = 0.0;
    o.zcm_p = v[0] / (double)protons;
    o.zcm_n = v[1] / (double)neutrons;
    o.rms_p = std::sqrt(v[2] / v[4]);
    o.rms_n = std::sqrt(v[3] / v[5]);
    const double zz = nucleus_z, nn = nucleus_n;
    o.dipole = (nn * zz) / (nn + zz) * (o.zcm_p - o.zcm_n);
    o.sor_iterations = 0;
    o.flags = 0;
    *out = o;
    return HV_OK;
}
