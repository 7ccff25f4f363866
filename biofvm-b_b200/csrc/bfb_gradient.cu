// bfb_gradient.cu -- gradient vectors of the field, the consumer of the
// diffusion step that chemotaxis reads (Microenvironment::
// compute_all_gradient_vectors, BioFVM_microenvironment.cpp:1243-1402).
//
// Per voxel n and substrate q, component c of out[(n*S + q)*3 + c] is
//   (rho[+1] - rho[-1]) / (2*dx)   inside axis c,
//   (rho[+1] - rho[ 0]) / dx       at its low end,
//   (rho[ 0] - rho[-1]) / dx       at its high end,
// and 0 on an axis of one voxel (the reference leaves z untouched there,
// :1352-1354, and has no neighbour to read for x or y). The per-voxel path
// compute_gradient_vector (:1404-1535) divides its y and z end caps by dx
// instead of dy / dz; on the uniform mesh the LOD solver requires these are
// equal, so both reference paths give these values.
//
// FP64: each value is the reference's `g = rho[a]; g -= rho[b]; g /= h`, the
// division correctly rounded from r = RN(1/h) with one residual correction
// (div_rcp), bit for bit with the IEEE quotient. FP32: the difference is
// formed in FP64 from the two FP32 values and the quotient rounded once to
// FP32.
//
// One block per (i, j) row of nz*S contiguous elements; a thread takes
// elements t, t + blockDim, ... of the row. The x and y neighbours are the
// same element of the rows ny and 1 away, so the field is read from DRAM about
// once and its neighbour re-reads hit L2. The output is 3x the field; each
// warp writes 96 contiguous values per iteration (staging them in shared
// memory for 16-byte stores measured slower: 1.06 against 0.76 ms at 256^3 x 8).
#include "bfb_aux.cuh"
#include "bfb_line.cuh"

namespace bfb {

__device__ __forceinline__ double grad_diff(double a, double b, double h, double rh) {
    return div_rcp(__dsub_rn(a, b), h, rh);
}

template <typename T>
__global__ void __launch_bounds__(256) gradient_kernel(const T *__restrict__ f, T *__restrict__ out, int nx, int ny,
                                                       int nz, int S, double h1, double r1, double h2, double r2) {
    const long long row = blockIdx.x;  // i * ny + j
    const int i = (int)(row / ny), j = (int)(row - (long long)i * ny);
    const int L = nz * S;
    const size_t base = (size_t)row * L;
    const long long jx = (long long)ny * L, jy = L;
    const T *__restrict__ fr = f + base;
    T *__restrict__ o = out + base * 3;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const int k = t / S;
        const double v = (double)fr[t];
        double gx = 0.0, gy = 0.0, gz = 0.0;
        if (nx > 1) {
            if (i == 0) gx = grad_diff((double)fr[t + jx], v, h1, r1);
            else if (i == nx - 1) gx = grad_diff(v, (double)fr[t - jx], h1, r1);
            else gx = grad_diff((double)fr[t + jx], (double)fr[t - jx], h2, r2);
        }
        if (ny > 1) {
            if (j == 0) gy = grad_diff((double)fr[t + jy], v, h1, r1);
            else if (j == ny - 1) gy = grad_diff(v, (double)fr[t - jy], h1, r1);
            else gy = grad_diff((double)fr[t + jy], (double)fr[t - jy], h2, r2);
        }
        if (nz > 1) {
            if (k == 0) gz = grad_diff((double)fr[t + S], v, h1, r1);
            else if (k == nz - 1) gz = grad_diff(v, (double)fr[t - S], h1, r1);
            else gz = grad_diff((double)fr[t + S], (double)fr[t - S], h2, r2);
        }
        o[3 * (size_t)t] = (T)gx;
        o[3 * (size_t)t + 1] = (T)gy;
        o[3 * (size_t)t + 2] = (T)gz;
    }
}

}  // namespace bfb

using namespace bfb;

namespace {

int launch_gradients(bfb_env_s *env, void *out) {
    // h = dx; 2h = dx * 2.0 exactly as the reference forms two_dx (:1245-1255)
    const double h1 = env->dx, h2 = env->dx * 2.0;
    const double r1 = 1.0 / h1, r2 = 1.0 / h2;
    const unsigned rows = (unsigned)((long long)env->nx * env->ny);
    const int L = env->nz * env->S;
    const int threads = L >= 256 ? 256 : ((L + 31) / 32) * 32;
    if (env->precision == BFB_FP64)
        gradient_kernel<double><<<rows, threads, 0, env->stream>>>(static_cast<const double *>(env->field),
                                                                   static_cast<double *>(out), env->nx, env->ny,
                                                                   env->nz, env->S, h1, r1, h2, r2);
    else
        gradient_kernel<float><<<rows, threads, 0, env->stream>>>(static_cast<const float *>(env->field),
                                                                  static_cast<float *>(out), env->nx, env->ny, env->nz,
                                                                  env->S, h1, r1, h2, r2);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

}  // namespace

extern "C" {

BFB_API int bfb_compute_gradients(bfb_env env, void *out_dev) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (!out_dev) return fail(BFB_ERR_INVALID_ARG, "out_dev is NULL");
    BFB_CUDA(cudaSetDevice(env->device));
    return launch_gradients(env, out_dev);
}

BFB_API int bfb_get_gradients(bfb_env env, double *out_host) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (!out_host) return fail(BFB_ERR_INVALID_ARG, "out_host is NULL");
    BFB_CUDA(cudaSetDevice(env->device));
    const size_t n = 3 * (size_t)env->N;
    void *buf = nullptr;
    BFB_CUDA(cudaMalloc(&buf, n * env->elem));
    int st = launch_gradients(env, buf);
    cudaError_t e = cudaSuccess;
    if (!st) {
        if (env->precision == BFB_FP64) {
            e = cudaMemcpyAsync(out_host, buf, n * sizeof(double), cudaMemcpyDeviceToHost, env->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(env->stream);
        } else {
            std::vector<float> tmp(n);
            e = cudaMemcpyAsync(tmp.data(), buf, n * sizeof(float), cudaMemcpyDeviceToHost, env->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(env->stream);
            if (e == cudaSuccess)
                for (size_t q = 0; q < n; ++q) out_host[q] = tmp[q];
        }
    }
    cudaFree(buf);
    if (st) return st;
    if (e != cudaSuccess) return cuda_fail(e, "bfb_get_gradients");
    return BFB_OK;
}

}  // extern "C"
