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
// (div_rcp), bit for bit with the IEEE quotient. FP32: the same operations
// in FP32, h and 2h rounded once to FP32, the quotient by the binary32 form of
// the same correction (bit for bit with IEEE FP32 division).
//
// One block per (i, j) row of nz*S contiguous elements (field rows are Lp
// elements apart; the output is packed, 3*nz*S per row). The x and y
// neighbours are the same element of the rows ny and 1 away, so the field is
// read from DRAM about once and its neighbour re-reads hit L2. The output is
// 3x the field.
// - gradient_vec_kernel (rows of a multiple of 16 bytes, 16-byte aligned
//   field and output): a thread takes one 16-byte vector of the row (4 FP32
//   or 2 FP64 elements) per iteration, loads each neighbour as one vector,
//   and writes the vector's 3-interleaved gradients as three 16-byte stores,
//   so a warp writes 1.5 KB of contiguous output per iteration.
// - gradient_kernel (any other shape): one element per thread and
//   iteration, three 4- or 8-byte stores. (Staging its output in shared
//   memory for 16-byte stores measured slower: 1.06 against 0.76 ms at
//   256^3 x 8.)
#include "bfb_aux.cuh"
#include "bfb_line.cuh"

namespace bfb {

__device__ __forceinline__ double grad_diff(double a, double b, double h, double rh) {
    return div_rcp(__dsub_rn(a, b), h, rh);
}
// binary32 version of div_rcp: the correctly rounded t/h from r = RN(1/h)
// with one residual correction (Markstein), as IEEE division gives it
__device__ __forceinline__ float grad_diff(float a, float b, float h, float rh) {
    const float t = __fsub_rn(a, b);
    const float q0 = __fmul_rn(t, rh);
    const float e = __fmaf_rn(-q0, h, t);
    return __fmaf_rn(e, rh, q0);
}

template <typename T, int SC>  // SC: the substrate count when a compile-time constant (else 0)
__global__ void __launch_bounds__(256) gradient_kernel(const T *__restrict__ f, T *__restrict__ out, int nx, int ny,
                                                       int nz, int S_, int Lp, T h1, T r1, T h2, T r2) {
    const int S = SC > 0 ? SC : S_;
    const long long row = blockIdx.x;  // i * ny + j
    const int i = (int)(row / ny), j = (int)(row - (long long)i * ny);
    const int L = nz * S;
    const long long jx = (long long)ny * Lp, jy = Lp;  // field rows are Lp elements apart
    const T *__restrict__ fr = f + (size_t)row * Lp;
    T *__restrict__ o = out + (size_t)row * L * 3;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const int k = t / S;
        const T v = fr[t];
        T gx = T(0), gy = T(0), gz = T(0);
        if (nx > 1) {
            if (i == 0) gx = grad_diff(fr[t + jx], v, h1, r1);
            else if (i == nx - 1) gx = grad_diff(v, fr[t - jx], h1, r1);
            else gx = grad_diff(fr[t + jx], fr[t - jx], h2, r2);
        }
        if (ny > 1) {
            if (j == 0) gy = grad_diff(fr[t + jy], v, h1, r1);
            else if (j == ny - 1) gy = grad_diff(v, fr[t - jy], h1, r1);
            else gy = grad_diff(fr[t + jy], fr[t - jy], h2, r2);
        }
        if (nz > 1) {
            if (k == 0) gz = grad_diff(fr[t + S], v, h1, r1);
            else if (k == nz - 1) gz = grad_diff(v, fr[t - S], h1, r1);
            else gz = grad_diff(fr[t + S], fr[t - S], h2, r2);
        }
        o[3 * (size_t)t] = gx;
        o[3 * (size_t)t + 1] = gy;
        o[3 * (size_t)t + 2] = gz;
    }
}

// 16-byte vectors of the element type: 4 floats or 2 doubles
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using V = float4;
    static constexpr int n = 4;
};
template <>
struct Vec16<double> {
    using V = double2;
    static constexpr int n = 2;
};
template <typename T>
union Pack16 {
    typename Vec16<T>::V v;
    T s[Vec16<T>::n];
};
template <typename T>
__device__ __forceinline__ void ld16(const T *p, T (&x)[Vec16<T>::n]) {
    Pack16<T> u;
    u.v = __ldg(reinterpret_cast<const typename Vec16<T>::V *>(p));
#pragma unroll
    for (int e = 0; e < Vec16<T>::n; ++e) x[e] = u.s[e];
}
template <typename T>
__device__ __forceinline__ void st16(T *p, const T *x) {
    Pack16<T> u;
#pragma unroll
    for (int e = 0; e < Vec16<T>::n; ++e) u.s[e] = x[e];
    *reinterpret_cast<typename Vec16<T>::V *>(p) = u.v;
}

// One axis's values of a vector whose neighbours along that axis are `off`
// elements away; lo / hi: the vector lies on the axis's first / last plane.
template <typename T>
__device__ __forceinline__ void axis_grad(const T *p, long long off, bool lo, bool hi, const T (&v)[Vec16<T>::n],
                                          T (&g)[Vec16<T>::n], T h1, T r1, T h2, T r2) {
    constexpr int VW = Vec16<T>::n;
    T a[VW], b[VW];
    if (lo) {
        ld16(p + off, a);
#pragma unroll
        for (int e = 0; e < VW; ++e) g[e] = grad_diff(a[e], v[e], h1, r1);
    } else if (hi) {
        ld16(p - off, b);
#pragma unroll
        for (int e = 0; e < VW; ++e) g[e] = grad_diff(v[e], b[e], h1, r1);
    } else {
        ld16(p + off, a);
        ld16(p - off, b);
#pragma unroll
        for (int e = 0; e < VW; ++e) g[e] = grad_diff(a[e], b[e], h2, r2);
    }
}

// The vectorised form of gradient_kernel: same values, same operations per
// element. Requires nz*S a multiple of VW and 16-byte aligned f and out (the
// host checks both; a row of a multiple of VW elements is never padded, so
// the field's rows are then L elements apart too); every vector then lies in one row, its x / y neighbours
// are whole vectors, and so are its z neighbours when S is a multiple of VW
// (ZV; otherwise they are read per element).
template <typename T, int SC>
__global__ void __launch_bounds__(256) gradient_vec_kernel(const T *__restrict__ f, T *__restrict__ out, int nx,
                                                           int ny, int nz, int S_, int Lp, T h1, T r1, T h2, T r2) {
    constexpr int VW = Vec16<T>::n;
    constexpr bool ZV = SC > 0 && SC % VW == 0;
    const int S = SC > 0 ? SC : S_;
    const long long row = blockIdx.x;  // i * ny + j
    const int i = (int)(row / ny), j = (int)(row - (long long)i * ny);
    const int L = nz * S;
    const long long jx = (long long)ny * Lp, jy = Lp;
    const T *__restrict__ fr = f + (size_t)row * Lp;
    T *__restrict__ o = out + (size_t)row * L * 3;
    for (int t = threadIdx.x * VW; t < L; t += blockDim.x * VW) {
        T v[VW], g[3][VW];
        ld16(fr + t, v);
#pragma unroll
        for (int e = 0; e < VW; ++e) g[0][e] = g[1][e] = g[2][e] = T(0);
        if (nx > 1) axis_grad(fr + t, jx, i == 0, i == nx - 1, v, g[0], h1, r1, h2, r2);
        if (ny > 1) axis_grad(fr + t, jy, j == 0, j == ny - 1, v, g[1], h1, r1, h2, r2);
        if (nz <= 1) {
        } else if constexpr (ZV) {
            const int k = t / S;
            axis_grad(fr + t, (long long)S, k == 0, k == nz - 1, v, g[2], h1, r1, h2, r2);
        } else {
#pragma unroll
            for (int e = 0; e < VW; ++e) {
                const int k = (t + e) / S;
                const T *p = fr + t + e;
                if (k == 0) g[2][e] = grad_diff(p[S], v[e], h1, r1);
                else if (k == nz - 1) g[2][e] = grad_diff(v[e], p[-S], h1, r1);
                else g[2][e] = grad_diff(p[S], p[-S], h2, r2);
            }
        }
        T w[3 * VW];  // out[(t + e)*3 + c] for the vector's VW elements
#pragma unroll
        for (int e = 0; e < VW; ++e) {
#pragma unroll
            for (int c = 0; c < 3; ++c) w[3 * e + c] = g[c][e];
        }
        T *oq = o + 3 * (size_t)t;
#pragma unroll
        for (int q = 0; q < 3; ++q) st16(oq + q * VW, w + q * VW);
    }
}

}  // namespace bfb

using namespace bfb;

namespace {

template <typename T>
int launch_typed(bfb_env_s *env, void *out, T h1, T r1, T h2, T r2) {
    const unsigned rows = (unsigned)((long long)env->nx * env->ny);
    const int L = env->nz * env->S;
    const T *f = static_cast<const T *>(env->field);
    T *o = static_cast<T *>(out);
    cudaStream_t s = env->stream;
    const int nx = env->nx, ny = env->ny, nz = env->nz, S = env->S, Lp = env->Lp;
    constexpr int VW = Vec16<T>::n;
    const bool vec = L % VW == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(o) & 15) == 0;
    if (vec) {
        const int nv = L / VW;  // vectors per row
        const int threads = nv >= 256 ? 256 : ((nv + 31) / 32) * 32;
        switch (S) {
        case 1: gradient_vec_kernel<T, 1><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
        case 2: gradient_vec_kernel<T, 2><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
        case 4: gradient_vec_kernel<T, 4><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
        case 8: gradient_vec_kernel<T, 8><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
        default: gradient_vec_kernel<T, 0><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
        }
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }
    const int threads = L >= 256 ? 256 : ((L + 31) / 32) * 32;
    switch (S) {
    case 1: gradient_kernel<T, 1><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
    case 2: gradient_kernel<T, 2><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
    case 4: gradient_kernel<T, 4><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
    case 8: gradient_kernel<T, 8><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
    default: gradient_kernel<T, 0><<<rows, threads, 0, s>>>(f, o, nx, ny, nz, S, Lp, h1, r1, h2, r2); break;
    }
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

int launch_gradients(bfb_env_s *env, void *out) {
    // h = dx; 2h = dx * 2.0 exactly as the reference forms two_dx (:1245-1255)
    const double h1 = env->dx, h2 = env->dx * 2.0;
    if (env->precision == BFB_FP64) return launch_typed<double>(env, out, h1, 1.0 / h1, h2, 1.0 / h2);
    const float f1 = (float)h1, f2 = (float)h2;
    return launch_typed<float>(env, out, f1, 1.0f / f1, f2, 1.0f / f2);
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
    return env_check_device_error(env);
}

}  // extern "C"
