// bfb_aux.cu -- agents (secretion/uptake), checksum and precision conversion.
#include "bfb_aux.cuh"

#include <cub/cub.cuh>

#include <algorithm>

namespace bfb {

// ---------------------------------------------------------------------------
// Conversions
// ---------------------------------------------------------------------------
__global__ void d2f_kernel(const double *__restrict__ s, float *__restrict__ d, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] = __double2float_rn(s[e]);
}
__global__ void f2d_kernel(const float *__restrict__ s, double *__restrict__ d, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        d[e] = (double)s[e];
}
static unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 32); }

template <typename TS, typename TD>
__global__ void convert_rows_kernel(const TS *__restrict__ s, TD *__restrict__ d, long long rows, int L, int sp,
                                    int dp) {
    const long long n = rows * L;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / L, q = e - r * L;
        if constexpr (sizeof(TD) == 4)
            d[r * dp + q] = __double2float_rn(s[r * sp + q]);
        else
            d[r * dp + q] = (double)s[r * sp + q];
    }
}

int launch_convert_d2f_rows(const double *src, float *dst, long long rows, int L, int sp, int dp, cudaStream_t s) {
    if (sp == L && dp == L) return launch_convert_d2f(src, dst, rows * L, s);
    if (rows * L <= 0) return BFB_OK;
    convert_rows_kernel<double, float><<<grid_for(rows * L), 256, 0, s>>>(src, dst, rows, L, sp, dp);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}
int launch_convert_f2d_rows(const float *src, double *dst, long long rows, int L, int sp, int dp, cudaStream_t s) {
    if (sp == L && dp == L) return launch_convert_f2d(src, dst, rows * L, s);
    if (rows * L <= 0) return BFB_OK;
    convert_rows_kernel<float, double><<<grid_for(rows * L), 256, 0, s>>>(src, dst, rows, L, sp, dp);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

int launch_convert_d2f(const double *src, float *dst, long long n, cudaStream_t s) {
    if (n <= 0) return BFB_OK;
    d2f_kernel<<<grid_for(n), 256, 0, s>>>(src, dst, n);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}
int launch_convert_f2d(const float *src, double *dst, long long n, cudaStream_t s) {
    if (n <= 0) return BFB_OK;
    f2d_kernel<<<grid_for(n), 256, 0, s>>>(src, dst, n);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// ---------------------------------------------------------------------------
// Agent binning and constants.
//
// Binning restates Basic_Agent::assign_position -> update_voxel_index ->
// Cartesian_Mesh::nearest_voxel_local_index at one rank
// (BioFVM_basic_agent.cpp:112-153, BioFVM_parallel.cpp:418-522,
//  BioFVM_mesh.cpp:204-213):
//   invalid position (outside the closed box)  -> position rejected, the
//                                                agent keeps voxel 0
//   v = (int)floor((p - lo)/h) clamped to [0, (int)((hi - lo)/h) - 1]
//   index = x*lny*lnz + y*lnz + z with lny/lnz the truncated extents,
//   clamped to [0, V-1].
// Constants restate set_internal_uptake_constants (BioFVM_basic_agent.cpp:
// 155-176) with the reference build's fused axpy:
//   c = (dt*volume)/dV, t1 = (S*rho*)*c, t2 = fma(c, U, fma(c, S, 1)).
// ---------------------------------------------------------------------------
struct BinGeom {
    double lo[3], hi[3], h[3];
    int V;
    double dV;
};

__device__ __forceinline__ int bin_axis(double p, double lo, double hi, double h) {
    int v = (int)floor(__ddiv_rn(__dsub_rn(p, lo), h));
    const int g = (int)__ddiv_rn(__dsub_rn(hi, lo), h);
    if (v >= g) v = g - 1;
    if (v < 0) v = 0;
    return v;
}

__global__ void bin_agents_kernel(int n, int S, const double *__restrict__ pos, const double *__restrict__ vol,
                                  const double *__restrict__ sec, const double *__restrict__ upt,
                                  const double *__restrict__ sat, double dt, BinGeom g, int *__restrict__ voxel,
                                  double *__restrict__ t1, double *__restrict__ t2) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
    int idx = 0;  // a freshly created agent's current_voxel_index
    const bool valid = !(x < g.lo[0] || x > g.hi[0] || y < g.lo[1] || y > g.hi[1] || z < g.lo[2] || z > g.hi[2]);
    if (valid) {
        const int xi = bin_axis(x, g.lo[0], g.hi[0], g.h[0]);
        const int yi = bin_axis(y, g.lo[1], g.hi[1], g.h[1]);
        const int zi = bin_axis(z, g.lo[2], g.hi[2], g.h[2]);
        const int lny = (int)__ddiv_rn(__dsub_rn(g.hi[1], g.lo[1]), g.h[1]);
        const int lnz = (int)__ddiv_rn(__dsub_rn(g.hi[2], g.lo[2]), g.h[2]);
        idx = xi * lny * lnz + yi * lnz + zi;
        if (idx < 0) idx = 0;
        if (idx >= g.V) idx = g.V - 1;
    }
    voxel[a] = idx;
    const double c = __ddiv_rn(__dmul_rn(dt, vol[a]), g.dV);
    for (int d = 0; d < S; ++d) {
        const size_t e = (size_t)a * S + d;
        t1[e] = __dmul_rn(__dmul_rn(sec[e], sat[e]), c);
        t2[e] = __fma_rn(c, upt[e], __fma_rn(c, sec[e], 1.0));
    }
}

template <typename T>
__global__ void gather_constants_kernel(int n_active, int S, const int *__restrict__ order,
                                        const double *__restrict__ t1, const double *__restrict__ t2,
                                        T *__restrict__ o1, T *__restrict__ o2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_active * S) return;
    const int r = (int)(e / S), d = (int)(e % S);
    const int a = order[r];
    o1[e] = (T)t1[(size_t)a * S + d];
    o2[e] = (T)t2[(size_t)a * S + d];
}

// BioFVM_basic_agent.cpp:291-296 for all agents of one voxel, in list order.
template <typename T>
__global__ void cells_kernel(T *__restrict__ f, int S, int nz, int Lp, int n_occ, const int *__restrict__ seg_start,
                             const int *__restrict__ seg_voxel, const T *__restrict__ t1, const T *__restrict__ t2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    const int s = (int)(e / S), d = (int)(e % S);
    const size_t fe = voxel_elem(seg_voxel[s], d, nz, S, Lp);
    T x = f[fe];
    const int a1 = seg_start[s + 1];
    for (int a = seg_start[s]; a < a1; ++a) {
        const size_t q = (size_t)a * S + d;
        if constexpr (sizeof(T) == 8)
            x = __ddiv_rn(__dadd_rn(x, t1[q]), t2[q]);
        else
            x = __fdiv_rn(__fadd_rn(x, t1[q]), t2[q]);
    }
    f[fe] = x;
}

void agents_free(bfb_env_s *env) {
    cudaFree(env->agent_voxel);
    cudaFree(env->seg_start);
    cudaFree(env->seg_voxel);
    cudaFree(env->ag_t1);
    cudaFree(env->ag_t2);
    cudaFree(env->ag_order);
    env->ag_order = nullptr;
    env->agent_voxel = env->seg_start = env->seg_voxel = nullptr;
    env->ag_t1 = env->ag_t2 = nullptr;
    env->n_agents = env->n_occ = env->n_active = 0;
}

namespace {
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
    template <typename U>
    U *as() { return static_cast<U *>(p); }
};
}  // namespace

// Sort the active agents by voxel (stable: list order within a voxel) and
// build the per-voxel segments the cells kernel walks. d_vox/d_t1/d_t2 are
// device arrays in list order (d_t1/d_t2 FP64, [n][S]); active may be NULL.
static int index_agents(bfb_env_s *env, int n, const int *d_vox, const double *d_t1, const double *d_t2,
                        const uint8_t *active) {
    const int S = env->S;
    cudaStream_t s = env->stream;
    std::vector<int> h_vox(n);
    BFB_CUDA(cudaMemcpyAsync(h_vox.data(), d_vox, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    BFB_CUDA(cudaStreamSynchronize(s));
    std::vector<int> keys, idx;
    keys.reserve(n);
    idx.reserve(n);
    for (int a = 0; a < n; ++a) {
        if (!active || active[a]) {
            if (h_vox[a] < 0 || h_vox[a] >= env->V) return fail(BFB_ERR_INVALID_ARG, "agent voxel index out of range");
            keys.push_back(h_vox[a]);
            idx.push_back(a);
        }
    }
    const int na = (int)keys.size();
    env->n_active = na;
    if (na == 0) return BFB_OK;
    DevBuf d_keys, d_keys_sorted, d_idx, d_idx_sorted, d_unique, d_counts, d_nruns, d_tmp;
    BFB_CUDA(d_keys.alloc(sizeof(int) * na));
    BFB_CUDA(d_keys_sorted.alloc(sizeof(int) * na));
    BFB_CUDA(d_idx.alloc(sizeof(int) * na));
    BFB_CUDA(d_idx_sorted.alloc(sizeof(int) * na));
    BFB_CUDA(d_unique.alloc(sizeof(int) * na));
    BFB_CUDA(d_counts.alloc(sizeof(int) * na));
    BFB_CUDA(d_nruns.alloc(sizeof(int)));
    BFB_CUDA(cudaMemcpyAsync(d_keys.p, keys.data(), sizeof(int) * na, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_idx.p, idx.data(), sizeof(int) * na, cudaMemcpyHostToDevice, s));

    // Stable LSD radix sort by voxel: agents of one voxel stay in list order.
    int end_bit = 1;
    while (end_bit < 31 && (1LL << end_bit) < env->V) ++end_bit;
    size_t tmp_sort = 0, tmp_rle = 0;
    BFB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, d_keys.as<int>(), d_keys_sorted.as<int>(),
                                             d_idx.as<int>(), d_idx_sorted.as<int>(), na, 0, end_bit, s));
    BFB_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tmp_rle, d_keys_sorted.as<int>(), d_unique.as<int>(),
                                                d_counts.as<int>(), d_nruns.as<int>(), na, s));
    BFB_CUDA(d_tmp.alloc(std::max(tmp_sort, tmp_rle)));
    BFB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp_sort, d_keys.as<int>(), d_keys_sorted.as<int>(),
                                             d_idx.as<int>(), d_idx_sorted.as<int>(), na, 0, end_bit, s));
    BFB_CUDA(cub::DeviceRunLengthEncode::Encode(d_tmp.p, tmp_rle, d_keys_sorted.as<int>(), d_unique.as<int>(),
                                                d_counts.as<int>(), d_nruns.as<int>(), na, s));
    int n_occ = 0;
    BFB_CUDA(cudaMemcpyAsync(&n_occ, d_nruns.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BFB_CUDA(cudaStreamSynchronize(s));
    std::vector<int> counts(n_occ), starts(n_occ + 1, 0);
    BFB_CUDA(cudaMemcpy(counts.data(), d_counts.p, sizeof(int) * n_occ, cudaMemcpyDeviceToHost));
    for (int q = 0; q < n_occ; ++q) starts[q + 1] = starts[q] + counts[q];
    BFB_CUDA(cudaMalloc(&env->seg_start, sizeof(int) * (n_occ + 1)));
    BFB_CUDA(cudaMalloc(&env->seg_voxel, sizeof(int) * std::max(1, n_occ)));
    BFB_CUDA(cudaMemcpyAsync(env->seg_start, starts.data(), sizeof(int) * (n_occ + 1), cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(env->seg_voxel, d_unique.p, sizeof(int) * n_occ, cudaMemcpyDeviceToDevice, s));
    env->n_occ = n_occ;

    BFB_CUDA(cudaMalloc(&env->ag_order, sizeof(int) * na));
    BFB_CUDA(cudaMemcpyAsync(env->ag_order, d_idx_sorted.p, sizeof(int) * na, cudaMemcpyDeviceToDevice, s));
    BFB_CUDA(cudaMalloc(&env->ag_t1, env->elem * (size_t)na * S));
    BFB_CUDA(cudaMalloc(&env->ag_t2, env->elem * (size_t)na * S));
    const long long tot = (long long)na * S;
    const unsigned gb = (unsigned)((tot + 255) / 256);
    if (env->precision == BFB_FP64)
        gather_constants_kernel<double><<<gb, 256, 0, s>>>(na, S, d_idx_sorted.as<int>(), d_t1, d_t2,
                                                           (double *)env->ag_t1, (double *)env->ag_t2);
    else
        gather_constants_kernel<float><<<gb, 256, 0, s>>>(na, S, d_idx_sorted.as<int>(), d_t1, d_t2,
                                                          (float *)env->ag_t1, (float *)env->ag_t2);
    BFB_CUDA(cudaGetLastError());
    BFB_CUDA(cudaStreamSynchronize(s));  // temporaries are freed on return
    return BFB_OK;
}

int agents_build(bfb_env_s *env, int n, const double *pos, const double *volume, const double *sec,
                 const double *upt, const double *sat, const uint8_t *active, double dt) {
    agents_free(env);
    if (n == 0) return BFB_OK;
    const int S = env->S;
    cudaStream_t s = env->stream;
    DevBuf d_pos, d_vol, d_sec, d_upt, d_sat, d_t1, d_t2;
    BFB_CUDA(d_pos.alloc(sizeof(double) * 3 * n));
    BFB_CUDA(d_vol.alloc(sizeof(double) * n));
    BFB_CUDA(d_sec.alloc(sizeof(double) * n * S));
    BFB_CUDA(d_upt.alloc(sizeof(double) * n * S));
    BFB_CUDA(d_sat.alloc(sizeof(double) * n * S));
    BFB_CUDA(d_t1.alloc(sizeof(double) * n * S));
    BFB_CUDA(d_t2.alloc(sizeof(double) * n * S));
    BFB_CUDA(cudaMalloc(&env->agent_voxel, sizeof(int) * n));
    BFB_CUDA(cudaMemcpyAsync(d_pos.p, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_vol.p, volume, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_sec.p, sec, sizeof(double) * n * S, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_upt.p, upt, sizeof(double) * n * S, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_sat.p, sat, sizeof(double) * n * S, cudaMemcpyHostToDevice, s));

    BinGeom g;
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = env->bbox[a];
        g.hi[a] = env->bbox[3 + a];
        g.h[a] = env->dx;
    }
    g.V = (int)env->V;
    g.dV = (env->dx * env->dx) * env->dx;
    bin_agents_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, S, d_pos.as<double>(), d_vol.as<double>(),
                                                      d_sec.as<double>(), d_upt.as<double>(), d_sat.as<double>(), dt,
                                                      g, env->agent_voxel, d_t1.as<double>(), d_t2.as<double>());
    BFB_CUDA(cudaGetLastError());
    env->n_agents = n;
    return index_agents(env, n, env->agent_voxel, d_t1.as<double>(), d_t2.as<double>(), active);
}

int agents_build_constants(bfb_env_s *env, int n, const int *voxel, const double *t1, const double *t2,
                           const uint8_t *active) {
    agents_free(env);
    if (n == 0) return BFB_OK;
    const int S = env->S;
    cudaStream_t s = env->stream;
    DevBuf d_t1, d_t2;
    BFB_CUDA(d_t1.alloc(sizeof(double) * n * S));
    BFB_CUDA(d_t2.alloc(sizeof(double) * n * S));
    BFB_CUDA(cudaMalloc(&env->agent_voxel, sizeof(int) * n));
    BFB_CUDA(cudaMemcpyAsync(env->agent_voxel, voxel, sizeof(int) * n, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_t1.p, t1, sizeof(double) * n * S, cudaMemcpyHostToDevice, s));
    BFB_CUDA(cudaMemcpyAsync(d_t2.p, t2, sizeof(double) * n * S, cudaMemcpyHostToDevice, s));
    env->n_agents = n;
    return index_agents(env, n, env->agent_voxel, d_t1.as<double>(), d_t2.as<double>(), active);
}

int launch_cells(bfb_env_s *env, cudaStream_t s) {
    if (env->n_occ == 0) return BFB_OK;
    const long long tot = (long long)env->n_occ * env->S;
    const unsigned gb = (unsigned)((tot + 255) / 256);
    if (env->precision == BFB_FP64)
        cells_kernel<double><<<gb, 256, 0, s>>>((double *)env->field, env->S, env->nz, env->Lp, env->n_occ,
                                                env->seg_start,
                                                env->seg_voxel, (const double *)env->ag_t1, (const double *)env->ag_t2);
    else
        cells_kernel<float><<<gb, 256, 0, s>>>((float *)env->field, env->S, env->nz, env->Lp, env->n_occ,
                                               env->seg_start,
                                               env->seg_voxel, (const float *)env->ag_t1, (const float *)env->ag_t2);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// ---------------------------------------------------------------------------
// Checksum: fixed partition of voxels per block, one pass over the field,
// FP64 sums in a fixed order -> deterministic.
// A block sums voxels [v0, v1) (v0 a multiple of 4, so the block's first
// element is 16-byte aligned when the field is). The block's elements are cut
// into rows of W = R*S elements (W a multiple of the 16-byte vector width V);
// thread t reads vector t of every row, so one warp load covers 512
// consecutive bytes, every element is read once, and the element at position
// p = V*t + j of a row always belongs to substrate p mod S: the thread keeps
// one FP64 accumulator per vector lane j. The block then adds, per substrate
// d, the accumulators of positions d, d + S, ..., in order, and
// checksum_final_kernel adds the blocks' partial sums in block order.
// ---------------------------------------------------------------------------
constexpr int kSumBlocks = 296;  // 2 x 148 SMs
constexpr int kSumThreads = 256;
constexpr int kMaxSumS = 64;

template <typename T>
struct SumVec;
template <>
struct SumVec<float> {
    static constexpr int V = 4;
    using type = float4;
    __device__ static void add(const float4 &x, double (&a)[4]) {
        a[0] += (double)x.x, a[1] += (double)x.y, a[2] += (double)x.z, a[3] += (double)x.w;
    }
};
template <>
struct SumVec<double> {
    static constexpr int V = 2;
    using type = double2;
    __device__ static void add(const double2 &x, double (&a)[2]) { a[0] += x.x, a[1] += x.y; }
};

// W = R*S elements per row: the largest multiple of lcm(S, V) not above V*256
__host__ __device__ inline int sum_row_width(int S, int V) {
    int l = S;
    while (l % V) l += S;
    return (V * kSumThreads) / l * l;
}

template <typename T>
__global__ void __launch_bounds__(kSumThreads) checksum_partial_kernel(const T *__restrict__ f, long long V, int S,
                                                                       double *__restrict__ partials) {
    constexpr int VW = SumVec<T>::V;
    using VT = typename SumVec<T>::type;
    __shared__ double red[VW * kSumThreads];
    const int W = sum_row_width(S, VW);
    const int t = threadIdx.x;
    long long per = (V + gridDim.x - 1) / gridDim.x;
    per = (per + 3) / 4 * 4;
    const long long v0 = min(V, (long long)blockIdx.x * per), v1 = min(V, v0 + per);
    const long long e0 = v0 * S, ne = (v1 - v0) * S;  // the block's elements
    const T *__restrict__ base = f + e0;
    double acc[VW];
#pragma unroll
    for (int j = 0; j < VW; ++j) acc[j] = 0.0;
    const bool vec = (reinterpret_cast<uintptr_t>(base) & 15) == 0;
    const long long rows = ne / W;
    long long row = 0;
    if (vec && VW * t < W) {
        const VT *__restrict__ p = reinterpret_cast<const VT *>(base) + t;
        const long long stride = W / VW;  // vectors per row
        constexpr int kRowsInFlight = 8;  // 8 x 16 B per thread in flight
        for (; row + kRowsInFlight <= rows; row += kRowsInFlight) {
            VT x[kRowsInFlight];
#pragma unroll
            for (int u = 0; u < kRowsInFlight; ++u) x[u] = p[(row + u) * stride];
#pragma unroll
            for (int u = 0; u < kRowsInFlight; ++u) SumVec<T>::add(x[u], acc);
        }
        for (; row < rows; ++row) SumVec<T>::add(p[row * stride], acc);
    }
    if (!vec) row = 0;  // an unaligned field is read element by element
    // the rest (the last partial row, or all rows without 16-byte alignment)
    // element by element, each element to the accumulator of its row position
    if (VW * t < W)
        for (long long e = row * W + VW * t; e < ne; e += W)
#pragma unroll
            for (int j = 0; j < VW; ++j)
                if (e + j < ne) acc[j] += (double)base[e + j];
#pragma unroll
    for (int j = 0; j < VW; ++j) red[VW * t + j] = VW * t < W ? acc[j] : 0.0;
    __syncthreads();
    if (t < S) {
        double sum = 0.0;
        for (int q = t; q < W; q += S) sum += red[q];
        partials[(size_t)blockIdx.x * S + t] = sum;
    }
}

// The same sums over a field with padded rows (rows of L = nz*S elements, Lp
// apart): block b sums rows [r0, r1); thread t < W = R*S takes positions
// t, t + W, ... of every row, all of substrate t mod S; then, as above,
// thread d < S adds its substrate's W / S accumulators in order.
template <typename T>
__global__ void __launch_bounds__(kSumThreads) checksum_rows_kernel(const T *__restrict__ f, long long rows, int L,
                                                                    int Lp, int S, double *__restrict__ partials) {
    __shared__ double red[kSumThreads];
    const int W = kSumThreads / S * S;
    const int t = threadIdx.x;
    const long long per = (rows + gridDim.x - 1) / gridDim.x;
    const long long r0 = min(rows, (long long)blockIdx.x * per), r1 = min(rows, r0 + per);
    double acc = 0.0;
    if (t < W)
        for (long long r = r0; r < r1; ++r) {
            const T *__restrict__ row = f + (size_t)r * Lp;
            for (int q = t; q < L; q += W) acc += (double)row[q];
        }
    red[t] = t < W ? acc : 0.0;
    __syncthreads();
    if (t < S) {
        double sum = 0.0;
        for (int q = t; q < W; q += S) sum += red[q];
        partials[(size_t)blockIdx.x * S + t] = sum;
    }
}

__global__ void checksum_final_kernel(const double *__restrict__ partials, int nblocks, int S, double *__restrict__ out) {
    const int d = threadIdx.x;
    if (d >= S) return;
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += partials[(size_t)b * S + d];
    out[d] = acc;
}

int checksum_prepare(bfb_env_s *env) {
    if (env->partials) return BFB_OK;
    BFB_CUDA(cudaMalloc(&env->partials, sizeof(double) * (kSumBlocks * (size_t)env->S + env->S)));
    env->partial_blocks = kSumBlocks;
    return BFB_OK;
}

int launch_checksum(bfb_env_s *env, double *out_dev, cudaStream_t s) {
    if (env->S > kMaxSumS) return fail(BFB_ERR_UNSUPPORTED, "checksum supports at most 64 substrates");
    if (env->Lp != env->nz * env->S) {  // padded rows
        const long long rows = (long long)env->nx * env->ny;
        if (env->precision == BFB_FP64)
            checksum_rows_kernel<double><<<kSumBlocks, kSumThreads, 0, s>>>(
                (const double *)env->field, rows, env->nz * env->S, env->Lp, env->S, env->partials);
        else
            checksum_rows_kernel<float><<<kSumBlocks, kSumThreads, 0, s>>>(
                (const float *)env->field, rows, env->nz * env->S, env->Lp, env->S, env->partials);
        checksum_final_kernel<<<1, kMaxSumS, 0, s>>>(env->partials, kSumBlocks, env->S, out_dev);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }
    if (env->precision == BFB_FP64)
        checksum_partial_kernel<double><<<kSumBlocks, kSumThreads, 0, s>>>((const double *)env->field, env->V, env->S,
                                                                         env->partials);
    else
        checksum_partial_kernel<float><<<kSumBlocks, kSumThreads, 0, s>>>((const float *)env->field, env->V, env->S,
                                                                        env->partials);
    checksum_final_kernel<<<1, kMaxSumS, 0, s>>>(env->partials, kSumBlocks, env->S, out_dev);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// ---------------------------------------------------------------------------
// Field comparison: max|a-b|, max|b|, sum (a-b)^2, sum b^2 (FP64 partials per
// block, summed in block order on the host).
// ---------------------------------------------------------------------------
template <typename TA, typename TB>
__global__ void compare_kernel(const TA *__restrict__ a, int la, const TB *__restrict__ b, int lb, long long rows, int L,
                               double *__restrict__ part) {
    __shared__ double s0[256], s1[256], s2[256], s3[256];
    double mx = 0, mb = 0, sd = 0, sb = 0;
    const long long N = rows * L;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
        const long long r = (la == L && lb == L) ? 0 : e / L, q = e - r * L;
        const double x = (double)a[r * la + q], y = (double)b[r * lb + q], df = x - y;
        mx = fmax(mx, fabs(df));
        mb = fmax(mb, fabs(y));
        sd += df * df;
        sb += y * y;
    }
    s0[threadIdx.x] = mx;
    s1[threadIdx.x] = mb;
    s2[threadIdx.x] = sd;
    s3[threadIdx.x] = sb;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + w]);
            s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + w]);
            s2[threadIdx.x] += s2[threadIdx.x + w];
            s3[threadIdx.x] += s3[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x + 0] = s0[0];
        part[4 * blockIdx.x + 1] = s1[0];
        part[4 * blockIdx.x + 2] = s2[0];
        part[4 * blockIdx.x + 3] = s3[0];
    }
}

int compare_fields(const void *a, int pa, int la, const void *b, int pb, int lb, long long rows, int L, double *out4,
                   cudaStream_t s) {
    const int blocks = 592;
    double *part = nullptr;
    BFB_CUDA(cudaMalloc(&part, sizeof(double) * 4 * blocks));
    if (pa == BFB_FP64 && pb == BFB_FP64)
        compare_kernel<<<blocks, 256, 0, s>>>((const double *)a, la, (const double *)b, lb, rows, L, part);
    else if (pa == BFB_FP32 && pb == BFB_FP64)
        compare_kernel<<<blocks, 256, 0, s>>>((const float *)a, la, (const double *)b, lb, rows, L, part);
    else if (pa == BFB_FP64 && pb == BFB_FP32)
        compare_kernel<<<blocks, 256, 0, s>>>((const double *)a, la, (const float *)b, lb, rows, L, part);
    else
        compare_kernel<<<blocks, 256, 0, s>>>((const float *)a, la, (const float *)b, lb, rows, L, part);
    std::vector<double> h(4 * blocks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * 4 * blocks, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(part);
    if (e != cudaSuccess) return cuda_fail(e, "compare_fields");
    out4[0] = out4[1] = out4[2] = out4[3] = 0;
    for (int q = 0; q < blocks; ++q) {
        out4[0] = std::max(out4[0], h[4 * q]);
        out4[1] = std::max(out4[1], h[4 * q + 1]);
        out4[2] += h[4 * q + 2];
        out4[3] += h[4 * q + 3];
    }
    return BFB_OK;
}

// Checksum kernels on caller-provided scratch: `partials` holds at least
// nblocks*S doubles; out_dev receives S doubles. Launches only, no allocation.
int launch_checksum_raw(const void *field, int precision, long long V, int S, double *partials, int nblocks,
                        double *out_dev, cudaStream_t s) {
    if (precision == BFB_FP64)
        checksum_partial_kernel<double><<<nblocks, kSumThreads, 0, s>>>((const double *)field, V, S, partials);
    else
        checksum_partial_kernel<float><<<nblocks, kSumThreads, 0, s>>>((const float *)field, V, S, partials);
    checksum_final_kernel<<<1, kMaxSumS, 0, s>>>(partials, nblocks, S, out_dev);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

}  // namespace bfb
