// VTK frames of a context's fields in the reference's format
// (output_vtk_header_start, output_vector_field, output_scalar_field:
// include/init.hpp:159-254, written in the order of
// src/hyper_vlasov.cpp:79-82): an ASCII STRUCTURED_POINTS header, then
// big-endian float32 blocks with x varying fastest.  The transposition, the
// cast to float and the byte swap run on the device, one pass per block;
// the bytes stream to the file through pinned memory.
#include <cstdio>
#include <vector>

#include "hv_internal.h"

namespace hv {
namespace {

__device__ __forceinline__ unsigned bswap_float(float f) { return __byte_perm(__float_as_uint(f), 0, 0x0123); }

// write index w = (k ny + j) nx + i  <-  field index (i ny + j) nz + k
template <typename T>
__global__ void k_vtk_scalars(Geom g, const T *__restrict__ v, unsigned *p, unsigned *n, unsigned *t) {
    long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= g.G) return;
    const int i = (int)(w % g.nx), j = (int)((w / g.nx) % g.ny), k = (int)(w / ((long long)g.nx * g.ny));
    const long long id = ((long long)i * g.ny + j) * g.nz + k;
    const T a = v[id], b = v[id + g.G];
    p[w] = bswap_float(static_cast<float>(a));
    n[w] = bswap_float(static_cast<float>(b));
    t[w] = bswap_float(static_cast<float>(a + b));  // init.hpp:207: the sum in T, then the cast
}

template <typename T>
__global__ void k_vtk_vectors(Geom g, const T *__restrict__ fx, const T *__restrict__ fy, const T *__restrict__ fz,
                              unsigned *p, unsigned *n) {
    long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= g.G) return;
    const int i = (int)(w % g.nx), j = (int)((w / g.nx) % g.ny), k = (int)(w / ((long long)g.nx * g.ny));
    const long long id = ((long long)i * g.ny + j) * g.nz + k;
    p[3 * w] = bswap_float(static_cast<float>(fx[id]));
    p[3 * w + 1] = bswap_float(static_cast<float>(fy[id]));
    p[3 * w + 2] = bswap_float(static_cast<float>(fz[id]));
    n[3 * w] = bswap_float(static_cast<float>(fx[id + g.G]));
    n[3 * w + 1] = bswap_float(static_cast<float>(fy[id + g.G]));
    n[3 * w + 2] = bswap_float(static_cast<float>(fz[id + g.G]));
}

template <typename T>
hv_status write_typed(hv_ctx *c, const State<T> &s, FILE *out) {
    const Geom &g = c->geom;
    const size_t G = (size_t)g.G;
    // header (init.hpp:160-168), with the world in T as the reference holds it
    const T d0 = T(g.dmx), d1 = T(g.dmy), d2 = T(g.dmz);
    std::fprintf(out, "# vtk DataFile Version 3.0\n");
    std::fprintf(out, "Volumetric data\n");
    std::fprintf(out, "BINARY\n");
    std::fprintf(out, "DATASET STRUCTURED_POINTS\n");
    std::fprintf(out, "DIMENSIONS %d %d %d\n", g.nx, g.ny, g.nz);
    std::fprintf(out, "ORIGIN %lf %lf %lf\n", (double)-d0, (double)-d1, (double)-d2);
    std::fprintf(out, "SPACING %lf %lf %lf\n", 2.0 * (double)d0 / g.nx, 2.0 * (double)d1 / g.ny,
                 2.0 * (double)d2 / g.nz);
    std::fprintf(out, "POINT_DATA %d\n", (int)G);
    unsigned *dev = nullptr, *host = nullptr;
    const size_t words = 6 * G;  // the largest pair of blocks (forces of both species)
    HV_CUDA(cudaMallocAsync((void **)&dev, words * sizeof(unsigned), c->stream));
    if (cudaMallocHost((void **)&host, words * sizeof(unsigned)) != cudaSuccess) {
        cudaFreeAsync(dev, c->stream);
        return cuda_status(cudaErrorMemoryAllocation, "cudaMallocHost");
    }
    const int nb = div_up((long long)G, 256);
    auto fetch = [&](size_t n) -> hv_status {
        HV_CUDA(cudaGetLastError());
        HV_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
        HV_CUDA(cudaStreamSynchronize(c->stream));
        return HV_OK;
    };
    hv_status st = HV_OK;
    // forces (init.hpp:215-254)
    k_vtk_vectors<T><<<nb, 256, 0, c->stream>>>(g, s.Fx, s.Fy, s.Fz, dev, dev + 3 * G);
    if ((st = fetch(6 * G)) == HV_OK) {
        std::fprintf(out, "VECTORS %s_%c float\n", "forces", 'p');
        std::fwrite(host, sizeof(unsigned), 3 * G, out);
        std::fprintf(out, "VECTORS %s_%c float\n", "forces", 'n');
        std::fwrite(host + 3 * G, sizeof(unsigned), 3 * G, out);
    }
    // density, potentials (init.hpp:186-213)
    const T *fields[2] = {s.rho, s.U};
    const char *names[2] = {"density", "potentials"};
    for (int f = 0; f < 2 && st == HV_OK; f++) {
        k_vtk_scalars<T><<<nb, 256, 0, c->stream>>>(g, fields[f], dev, dev + G, dev + 2 * G);
        if ((st = fetch(3 * G)) != HV_OK) break;
        const char tags[3] = {'p', 'n', 't'};
        for (int q = 0; q < 3; q++) {
            std::fprintf(out, "SCALARS %s_%c float 1\n", names[f], tags[q]);
            std::fprintf(out, "LOOKUP_TABLE default\n");
            std::fwrite(host + q * G, sizeof(unsigned), G, out);
        }
    }
    cudaFreeAsync(dev, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFreeHost(host);
    return st;
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" hv_status hv_write_vtk(hv_ctx *c, const char *path) {
    if (!c || !path) return HV_ERR_BAD_ARG;
    HV_CUDA(cudaSetDevice(c->device));
    FILE *out = std::fopen(path, "wb");
    if (!out) {
        set_last_error(std::string("cannot open ") + path);
        return HV_ERR_BAD_ARG;
    }
    hv_status st = c->prec == HV_F64 ? write_typed<double>(c, c->d64, out) : write_typed<float>(c, c->d32, out);
    if (std::fclose(out) != 0 && st == HV_OK) st = HV_ERR_BAD_ARG;
    return st;
}
