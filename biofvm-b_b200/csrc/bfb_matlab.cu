// bfb_matlab.cu -- the reference's MATLAB v4 snapshot of the field, packed on
// the device (Microenvironment::write_to_matlab, BioFVM_microenvironment.cpp:
// 1079-1107, with write_matlab4_header, BioFVM_matlab.cpp:535-584; the MPI
// variant BioFVM_parallel.cpp:528-678 writes the same bytes at one rank).
//
// File layout, little-endian:
//   5 x uint32: type 0 (full double matrix), rows = 4 + S, cols = V, imag 0,
//               name length (the name's characters, no terminator)
//   the name "multiscale_microenvironment"
//   V columns of 4 + S doubles: voxel centre x, y, z, voxel volume, then the
//   S densities of that voxel (voxel order n = (i*ny + j)*nz + k)
// Centres are lo + (i + 0.5)*dx per axis, fused as the reference build fuses
// `local_x_start + (i + 0.5)*dx` (BioFVM_parallel.cpp:129-143); the volume is
// (dx*dx)*dx (:156). FP32 fields are widened to double.
#include <cstdio>

#include "bfb_aux.cuh"

namespace bfb {

template <typename T>
__global__ void matlab_pack_kernel(const T *__restrict__ f, double *__restrict__ out, int nx, int ny, int nz, int S,
                                   int Lp, double x0, double y0, double z0, double dx, double vol) {
    const int rows = 4 + S;
    const long long V = (long long)nx * ny * nz;
    const long long total = V * rows;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long n = e / rows;
        const int r = (int)(e - n * rows);
        double v;
        if (r >= 4) {
            const long long row = n / nz;  // field rows (i, j) are Lp elements apart
            v = (double)f[row * Lp + (n - row * nz) * S + (r - 4)];
        } else if (r == 3) {
            v = vol;
        } else {
            const int k = (int)(n % nz), j = (int)((n / nz) % ny), i = (int)(n / ((long long)ny * nz));
            const int c = r == 0 ? i : (r == 1 ? j : k);
            const double lo = r == 0 ? x0 : (r == 1 ? y0 : z0);
            v = __fma_rn((double)c + 0.5, dx, lo);
        }
        out[e] = v;
    }
}

}  // namespace bfb

using namespace bfb;

extern "C" BFB_API int bfb_write_matlab(bfb_env env, const char *filename) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (!filename) return fail(BFB_ERR_INVALID_ARG, "filename is NULL");
    BFB_CUDA(cudaSetDevice(env->device));
    const int S = env->S;
    const long long V = env->V;
    const size_t count = (size_t)V * (4 + S);
    if (V > 0xffffffffLL || 4 + S > 0x7fffffff) return fail(BFB_ERR_SIZE, "bfb_write_matlab: matrix too large for MAT v4");
    double *dbuf = nullptr, *hbuf = nullptr;
    BFB_CUDA(cudaMalloc(&dbuf, count * sizeof(double)));
    cudaError_t e = cudaMallocHost(&hbuf, count * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(dbuf);
        return cuda_fail(e, "cudaMallocHost (bfb_write_matlab)");
    }
    const double dx = env->dx, vol = (dx * dx) * dx;
    const double y0 = env->bbox[1] + 0.0, z0 = env->bbox[2] + 0.0, x0 = env->bbox[0] + 0.0;
    const int blocks = 148 * 8;
    if (env->precision == BFB_FP64)
        matlab_pack_kernel<double><<<blocks, 256, 0, env->stream>>>(static_cast<const double *>(env->field), dbuf,
                                                                    env->nx, env->ny, env->nz, S, env->Lp, x0, y0, z0, dx, vol);
    else
        matlab_pack_kernel<float><<<blocks, 256, 0, env->stream>>>(static_cast<const float *>(env->field), dbuf,
                                                                   env->nx, env->ny, env->nz, S, env->Lp, x0, y0, z0, dx, vol);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hbuf, dbuf, count * sizeof(double), cudaMemcpyDeviceToHost, env->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(env->stream);
    cudaFree(dbuf);
    if (e != cudaSuccess) {
        cudaFreeHost(hbuf);
        return cuda_fail(e, "bfb_write_matlab");
    }
    if (int es = env_check_device_error(env)) {  // no file from an untrustworthy field
        cudaFreeHost(hbuf);
        return es;
    }
    static const char name[] = "multiscale_microenvironment";
    const unsigned header[5] = {0u, (unsigned)(4 + S), (unsigned)V, 0u, (unsigned)(sizeof(name) - 1)};
    std::FILE *fp = std::fopen(filename, "wb");
    int st = BFB_OK;
    if (!fp) {
        st = fail(BFB_ERR_INVALID_ARG, std::string("bfb_write_matlab: could not open ") + filename);
    } else {
        bool ok = std::fwrite(header, sizeof(unsigned), 5, fp) == 5 &&
                  std::fwrite(name, 1, sizeof(name) - 1, fp) == sizeof(name) - 1 &&
                  std::fwrite(hbuf, sizeof(double), count, fp) == count;
        ok = (std::fclose(fp) == 0) && ok;
        if (!ok) st = fail(BFB_ERR_STATE, std::string("bfb_write_matlab: write failed for ") + filename);
    }
    cudaFreeHost(hbuf);
    return st;
}
