// bfb_adjoint.cu -- reverse mode of the composite step (LOD diffusion-decay,
// then agent secretion/uptake), with checkpointing.
//
// Forward step (per substrate; A_a = tridiag(-c1, diag, -c1) of axis a,
// Dir the affine overwrite s = (1 - M) y + M g of the active faces):
//     s0 = Dir(u); y_x = A_x^-1 s0; s1 = Dir(y_x); y_y = A_y^-1 s1;
//     s2 = Dir(y_y); y_z = A_z^-1 s2; v = Dir(y_z); u' = Cells(v)
// Reverse, with lam = dL/du':
//     lam_v = Cells^T(lam; v)                    (per-agent dL/dtemp1, dL/dtemp2)
//     mu_z = A_z^-1 (1 - M) lam_v                (A symmetric: A^-T = A^-1, same factors)
//     mu_y = A_y^-1 (1 - M) mu_z,  mu_x = A_x^-1 (1 - M) mu_y,  dL/du = (1 - M) mu_x
//     dL/dc1 -= sum_a mu_a^T Lap y_a,  dL/dc2 -= sum_a mu_a^T y_a
// where Lap = dA/dc1 is tridiag(-1, 2, -1) with end diagonals 1 (0 when n = 1),
// c1 = dt D/dx^2 and c2 = dt lambda/3. The oracle holds the same derivation
// (oracle/lod_oracle.c: orc_lod_step_adjoint) for the tests.
//
// Each adjoint sweep is one kernel: a warp stages the stage input (s0, s1 or
// s2) and the incoming adjoint for 32 lines into shared memory, solves both
// systems with the forward factors (y_a and mu_a), adds mu.Lap y and mu.y per
// line into a slot of a partial-sum buffer, and writes mu_a. The per-substrate
// sums are reduced in a fixed order, so the gradients are deterministic.
//
// Checkpointing: the forward run keeps the field every K steps. The reverse
// pass walks the segments backwards; for each it recomputes the K steps from
// the checkpoint with out-of-place sweeps, keeping u, s1, s2 of every step and
// the pre-agent values at agent voxels, then reverses them.
#include <algorithm>
#include <vector>

#include "bfb_aux.cuh"
#include "bfb_tiles.cuh"

namespace bfb {

// One line solved in place with the forward factors (any right-hand side).
template <typename T>
__device__ __forceinline__ void thomas_inplace(LineSolver<T> &L, T *line, int ls, int n, int m0) {
    line[0] = L.first(line[0], line[min(1, n - 1) * ls]);
    const int hend = min(n - 1, m0);
    int k = 1;
    for (; k < hend; ++k) line[k * ls] = L.template fwd<false>(line[k * ls], k);
#pragma unroll 4
    for (; k < n - 1; ++k) line[k * ls] = L.template fwd<true>(line[k * ls], k);
    if (n > 1) L.template fwd<false>(line[(n - 1) * ls], n - 1);
    line[(n - 1) * ls] = L.out_last();
    const int tl = max(m0, 1);
    k = n - 2;
#pragma unroll 4
    for (; k >= tl; --k) line[k * ls] = L.template bwd<true>(line[k * ls], k);
    for (; k >= 0; --k) line[k * ls] = L.template bwd<false>(line[k * ls], k);
}

// mu.Lap y and mu.y along one line (FP64 accumulation)
template <typename T>
__device__ __forceinline__ void line_dots(const T *y, const T *mu, int ls, int n, double &dl, double &dy) {
    for (int m = 0; m < n; ++m) {
        const double ym = (double)y[m * ls], mm = (double)mu[m * ls];
        double lap = 0.0;
        if (n > 1) {
            if (m == 0) lap = ym - (double)y[ls];
            else if (m == n - 1) lap = ym - (double)y[(m - 1) * ls];
            else lap = 2.0 * ym - (double)y[(m - 1) * ls] - (double)y[(m + 1) * ls];
        }
        dl += mm * lap;
        dy += mm * ym;
    }
}

// Adjoint of one strided sweep (x: axis 0 with PRE_DIR, y: axis 1).
//   a.f  = stage input (u for x, with the step's leading Dirichlet applied here)
//   lam  = incoming adjoint; a.fo = mu out; part = [tiles*32][2] slot sums
template <typename T, bool PRE_DIR>
__global__ void __launch_bounds__(32) adjoint_strided_kernel(SweepArgs<T> a, const T *__restrict__ lam, StridedGeom g,
                                                             double *__restrict__ part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const long long tile = blockIdx.x;
    const int n = g.n;
    const long long P = g.P;
    T *smX = reinterpret_cast<T *>(smem_raw);
    T *smL = smX + (size_t)n * 32;
    const int slab = (int)(tile / g.ncb);
    const long long col0 = (tile % g.ncb) * 32;
    const int ncols = (int)min((long long)32, P - col0);
    const size_t off = (size_t)slab * g.slab_stride + col0;
    if (lane < ncols)
        for (int r = 0; r < n; ++r) {
            cp_async<sizeof(T)>(smX + r * 32 + lane, a.f + off + (size_t)r * P + lane);
            cp_async<sizeof(T)>(smL + r * 32 + lane, lam + off + (size_t)r * P + lane);
        }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    double dl = 0.0, dy = 0.0;
    if (lane < ncols) {
        const long long col = col0 + lane;
        const int S = a.S, d = (int)(col % S);
        int ci, cj, ck;
        if (g.axis == 0) {
            const long long t = col / S;
            ck = (int)(t % a.nz);
            cj = (int)(t / a.nz);
            ci = 0;
        } else {
            ck = (int)(col / S);
            ci = slab;
            cj = 0;
        }
        const unsigned m = a.dir.any ? a.dir.mask[d] : 0u;
        bool col_dir, lo_dir, hi_dir;
        if (g.axis == 0) {
            col_dir = ((m & 4u) && cj == 0) || ((m & 8u) && cj == a.ny - 1) || ((m & 16u) && ck == 0) ||
                      ((m & 32u) && ck == a.nz - 1);
            lo_dir = m & 1u;
            hi_dir = m & 2u;
        } else {
            col_dir = ((m & 1u) && ci == 0) || ((m & 2u) && ci == a.nx - 1) || ((m & 16u) && ck == 0) ||
                      ((m & 32u) && ck == a.nz - 1);
            lo_dir = m & 4u;
            hi_dir = m & 8u;
        }
        T *xl = smX + lane, *ll = smL + lane;
        if (PRE_DIR) {
            if (lo_dir) xl[0] = g.axis == 0 ? dir_value(a.dir, 0, cj, ck, d) : dir_value(a.dir, ci, 0, ck, d);
            if (hi_dir)
                xl[(n - 1) * 32] =
                    g.axis == 0 ? dir_value(a.dir, n - 1, cj, ck, d) : dir_value(a.dir, ci, n - 1, ck, d);
        }
        if (col_dir) {
            for (int r = 0; r < n; ++r) ll[r * 32] = T(0);
        } else {
            if (lo_dir) ll[0] = T(0);
            if (hi_dir) ll[(n - 1) * 32] = T(0);
        }
        LineSolver<T> L1(a, d), L2(a, d);
        thomas_inplace(L1, xl, 32, n, a.fac.m0);
        thomas_inplace(L2, ll, 32, n, a.fac.m0);
        line_dots(xl, ll, 32, n, dl, dy);
        T *out = a.fo + off + lane;
        for (int r = 0; r < n; ++r) out[(size_t)r * P] = ll[r * 32];
    }
    part[2 * ((size_t)tile * 32 + lane)] = dl;
    part[2 * ((size_t)tile * 32 + lane) + 1] = dy;
}

// Adjoint of the contiguous z sweep; line t = (r, d) of the tile is row
// row0 + r, substrate d, and lanes take lines t = lane, lane + 32, ...
// Slot t of the tile (LPT slots, a multiple of 32 >= R*S) gets that line's sums.
template <typename T>
__global__ void __launch_bounds__(32) adjoint_contig_kernel(SweepArgs<T> a, const T *__restrict__ lam, ContigGeom g,
                                                            int LPT, double *__restrict__ part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const long long tile = blockIdx.x;
    const long long row0 = tile * g.R;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = a.S, nz = g.nz, L = nz * S;
    T *smX = reinterpret_cast<T *>(smem_raw);
    T *smL = smX + (size_t)g.R * g.RS;
    const T *X = a.f + (size_t)row0 * L;
    const T *Lm = lam + (size_t)row0 * L;
    for (int e = lane; e < nr * L; e += 32) {
        const int r = e / L, q = e - r * L;
        cp_async<sizeof(T)>(smX + (size_t)r * g.RS + q, X + e);
        cp_async<sizeof(T)>(smL + (size_t)r * g.RS + q, Lm + e);
    }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    double *slot = part + 2 * (size_t)tile * LPT;
    for (int t = lane; t < LPT; t += 32) {
        double dl = 0.0, dy = 0.0;
        if (t < nr * S) {
            const int r = t / S, d = t - r * S;
            const long long row = row0 + r;
            const int i = (int)(row / a.ny), j = (int)(row % a.ny);
            const unsigned m = a.dir.any ? a.dir.mask[d] : 0u;
            const bool line_dir = ((m & 1u) && i == 0) || ((m & 2u) && i == a.nx - 1) || ((m & 4u) && j == 0) ||
                                  ((m & 8u) && j == a.ny - 1);
            const bool lo_dir = m & 16u, hi_dir = m & 32u;
            T *xl = smX + (size_t)r * g.RS + d, *ll = smL + (size_t)r * g.RS + d;
            if (line_dir) {
                for (int k = 0; k < nz; ++k) ll[k * S] = T(0);
            } else {
                if (lo_dir) ll[0] = T(0);
                if (hi_dir) ll[(nz - 1) * S] = T(0);
            }
            LineSolver<T> L1(a, d), L2(a, d);
            thomas_inplace(L1, xl, S, nz, a.fac.m0);
            thomas_inplace(L2, ll, S, nz, a.fac.m0);
            line_dots(xl, ll, S, nz, dl, dy);
        }
        slot[2 * t] = dl;
        slot[2 * t + 1] = dy;
    }
    __syncwarp();
    T *O = a.fo + (size_t)row0 * L;
    for (int e = lane; e < nr * L; e += 32) {
        const int r = e / L, q = e - r * L;
        O[e] = smL[(size_t)r * g.RS + q];
    }
}

// Per-substrate sums of the slot partials, in slot order: block d adds the
// slots of substrate d into gacc[d] (mu.Lap y) and gacc[S + d] (mu.y).
// Strided sweeps: 32 slots per tile, slot = column. Contiguous sweep: LPT
// slots per tile, slot = line (r, d) of the tile.
__global__ void adjoint_reduce_kernel(const double *__restrict__ part, long long ntiles, int strided, long long P,
                                      int ncb, int S, int LPT, int R, long long nrows, double *__restrict__ gacc) {
    __shared__ double s0[256], s1[256];
    const int d = blockIdx.x;
    const int per = strided ? 32 : LPT;
    const long long nslots = ntiles * per;
    double a0 = 0.0, a1 = 0.0;
    for (long long q = threadIdx.x; q < nslots; q += blockDim.x) {
        const long long tile = q / per;
        const int t = (int)(q % per);
        int dq;
        bool valid;
        if (strided) {
            const long long col = (tile % ncb) * 32 + t;
            valid = col < P;
            dq = (int)(col % S);
        } else {
            const int nr = (int)min((long long)R, nrows - tile * R);
            valid = t < nr * S;
            dq = t % S;
        }
        if (valid && dq == d) {
            a0 += part[2 * q];
            a1 += part[2 * q + 1];
        }
    }
    s0[threadIdx.x] = a0;
    s1[threadIdx.x] = a1;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s0[threadIdx.x] += s0[threadIdx.x + w];
            s1[threadIdx.x] += s1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        gacc[d] += s0[0];
        gacc[S + d] += s1[0];
    }
}

// dL/du = (1 - M) mu: zero the active-face entries.
template <typename T>
__global__ void adjoint_mask_kernel(T *f, DirFaces<T> dir) {
    const long long fx = (long long)dir.ny * dir.nz, fy = (long long)dir.nx * dir.nz, fz = (long long)dir.nx * dir.ny;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * (fx + fy + fz)) return;
    int i, j, k;
    if (t < 2 * fx) {
        const long long q = t % fx;
        i = (t / fx) ? dir.nx - 1 : 0;
        j = (int)(q / dir.nz);
        k = (int)(q % dir.nz);
    } else if ((t -= 2 * fx) < 2 * fy) {
        const long long q = t % fy;
        j = (t / fy) ? dir.ny - 1 : 0;
        i = (int)(q / dir.nz);
        k = (int)(q % dir.nz);
    } else {
        t -= 2 * fy;
        const long long q = t % fz;
        k = (t / fz) ? dir.nz - 1 : 0;
        i = (int)(q / dir.ny);
        j = (int)(q % dir.ny);
    }
    const size_t vb = (((size_t)i * dir.ny + j) * dir.nz + k) * dir.S;
    for (int d = 0; d < dir.S; ++d) {
        const unsigned m = dir.mask[d];
        if (((m & 1u) && i == 0) || ((m & 2u) && i == dir.nx - 1) || ((m & 4u) && j == 0) ||
            ((m & 8u) && j == dir.ny - 1) || ((m & 16u) && k == 0) || ((m & 32u) && k == dir.nz - 1))
            f[vb + d] = T(0);
    }
}

template <typename T>
__global__ void gather_occ_kernel(const T *__restrict__ f, const int *__restrict__ seg_voxel, int n_occ, int S,
                                  T *__restrict__ out) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    out[e] = f[(size_t)seg_voxel[e / S] * S + (e % S)];
}

template <typename T>
__global__ void cells_on_kernel(T *__restrict__ f, int S, int n_occ, const int *__restrict__ seg_start,
                                const int *__restrict__ seg_voxel, const T *__restrict__ t1,
                                const T *__restrict__ t2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    const int s = (int)(e / S), d = (int)(e % S);
    const size_t fe = (size_t)seg_voxel[s] * S + d;
    T x = f[fe];
    for (int q = seg_start[s]; q < seg_start[s + 1]; ++q) {
        const size_t z = (size_t)q * S + d;
        if constexpr (sizeof(T) == 8)
            x = __ddiv_rn(__dadd_rn(x, t1[z]), t2[z]);
        else
            x = __fdiv_rn(__fadd_rn(x, t1[z]), t2[z]);
    }
    f[fe] = x;
}

// Cells^T at one (voxel, substrate): the agents of the voxel applied
// x_k = (x_(k-1) + t1_k)/t2_k in list order; backwards,
// dL/dt1_k += g/t2_k, dL/dt2_k -= g x_k/t2_k, g <- g/t2_k. The x_k are
// replayed from the pre-agent value v (x_0).
template <typename T>
__global__ void cells_adjoint_kernel(T *__restrict__ lam, const T *__restrict__ vocc, int S, int n_occ,
                                     const int *__restrict__ seg_start, const int *__restrict__ seg_voxel,
                                     const T *__restrict__ t1, const T *__restrict__ t2, double *__restrict__ gt1,
                                     double *__restrict__ gt2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    const int s = (int)(e / S), d = (int)(e % S);
    const size_t fe = (size_t)seg_voxel[s] * S + d;
    const int q0 = seg_start[s], q1 = seg_start[s + 1];
    double g = (double)lam[fe];
    for (int k = q1 - 1; k >= q0; --k) {
        double x = (double)vocc[e];  // replay x_k
        for (int q = q0; q <= k; ++q) x = (x + (double)t1[(size_t)q * S + d]) / (double)t2[(size_t)q * S + d];
        const double tt = (double)t2[(size_t)k * S + d];
        gt1[(size_t)k * S + d] += g / tt;
        gt2[(size_t)k * S + d] -= g * x / tt;
        g /= tt;
    }
    lam[fe] = (T)g;
}

}  // namespace bfb

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace bfb {
int env_prepare_step(bfb_env_s *env, double dt, int flags);
template <typename T>
SweepArgs<T> env_sweep_args(bfb_env_s *env, int axis, double dt);
int env_tile_plan(bfb_env_s *env, int elem, StridedGeom *gx, StridedGeom *gy, ContigGeom *gz, int vb16[3]);
}  // namespace bfb

using namespace bfb;

namespace {

// Carves the call's buffers out of the env's workspace block (256-byte
// aligned). Pass 1 sizes the block (base == nullptr), pass 2 hands out pointers.
struct Carve {
    char *base = nullptr;
    size_t off = 0;
    template <typename U>
    void take(U **out, size_t bytes) {
        *out = base ? reinterpret_cast<U *>(base + off) : nullptr;
        off += (std::max<size_t>(bytes, 1) + 255) / 256 * 256;
    }
};

struct Buf {
    void *p = nullptr;
    CUtensorMap map[2];
    int ok[2] = {0, 0};
    int crow[2] = {0, 0};
};

template <typename T>
int adjoint_run(bfb_env_s *env, double dt, int n_steps, int flags, int K, const void *dL_dfinal, void *dL_dinitial,
                void *final_field, double *gD, double *gL, double *gsec, double *gupt, double *gsat) {
    const int S = env->S;
    const size_t N = (size_t)env->N;
    const size_t fb = N * sizeof(T);
    cudaStream_t st = env->stream;
    const bool cells = (flags & BFB_STEP_CELLS) && env->n_occ > 0;
    int rc = env_prepare_step(env, dt, BFB_STEP_DIFFUSION);
    if (rc) return rc;
    StridedGeom gx, gy;
    ContigGeom gz;
    int vb16[3];
    if ((rc = env_tile_plan(env, sizeof(T), &gx, &gy, &gz, vb16))) return rc;

    const int nseg = (n_steps + K - 1) / K;
    const int LPT = (gz.R * S + 31) / 32 * 32;  // partial slots per contiguous tile
    const long long slots_x = (long long)gx.n_slabs * gx.ncb * 32, slots_y = (long long)gy.n_slabs * gy.ncb * 32,
                    slots_z = (gz.nrows + gz.R - 1) / gz.R * LPT;
    const long long slots = std::max(slots_x, std::max(slots_y, slots_z));
    const size_t occ = (size_t)env->n_occ * S, nact = (size_t)env->n_active * S;
    std::vector<T *> ckpt(nseg);
    std::vector<Buf> U(K + 1), S1(K), S2(K);
    T *lam = nullptr, *mu = nullptr, *vocc = nullptr;
    double *part = nullptr, *gacc = nullptr, *gt1 = nullptr, *gt2 = nullptr;
    auto carve = [&](Carve &c) {
        for (auto &p : ckpt) c.take(&p, fb);
        for (auto *v : {&U, &S1, &S2})
            for (auto &b : *v) {
                T *p;
                c.take(&p, fb);
                b.p = p;
            }
        c.take(&lam, fb);
        c.take(&mu, fb);
        c.take(&part, sizeof(double) * 2 * slots);
        c.take(&gacc, sizeof(double) * 2 * S);
        c.take(&vocc, sizeof(T) * occ * K);
        c.take(&gt1, sizeof(double) * nact);
        c.take(&gt2, sizeof(double) * nact);
    };
    Carve sizing;
    carve(sizing);
    if (sizing.off > env->adj_ws_bytes) {
        BFB_CUDA(cudaStreamSynchronize(st));
        cudaFree(env->adj_ws);
        env->adj_ws = nullptr;
        env->adj_ws_bytes = 0;
        cudaError_t e = cudaMalloc(&env->adj_ws, sizing.off);
        if (e != cudaSuccess) {
            env->adj_ws = nullptr;
            return cuda_fail(e, "cudaMalloc (adjoint workspace)");
        }
        env->adj_ws_bytes = sizing.off;
    }
    Carve c;
    c.base = static_cast<char *>(env->adj_ws);
    carve(c);
    for (auto *v : {&U, &S1, &S2})
        for (auto &b : *v)
            for (int a = 0; a < 2; ++a)
                b.ok[a] = env->use_tma && make_sweep_tensor_map(&b.map[a], &b.crow[a], b.p, sizeof(T), a, env->nx,
                                                                env->ny, env->nz, S);
    BFB_CUDA(cudaMemsetAsync(gacc, 0, sizeof(double) * 2 * S, st));
    if (nact) {
        BFB_CUDA(cudaMemsetAsync(gt1, 0, sizeof(double) * nact, st));
        BFB_CUDA(cudaMemsetAsync(gt2, 0, sizeof(double) * nact, st));
    }

    // ---- forward with checkpoints (the env's own fast path)
    const int fwd_flags = BFB_STEP_DIFFUSION | (cells ? BFB_STEP_CELLS : 0);
    for (int c = 0; c < nseg; ++c) {
        BFB_CUDA(cudaMemcpyAsync(ckpt[c], env->field, fb, cudaMemcpyDeviceToDevice, st));
        const int len = std::min(K, n_steps - c * K);
        if ((rc = bfb_simulate(env, dt, len, fwd_flags))) return rc;
    }
    if (final_field) BFB_CUDA(cudaMemcpyAsync(final_field, env->field, fb, cudaMemcpyDeviceToDevice, st));
    BFB_CUDA(cudaMemcpyAsync(lam, dL_dfinal, fb, cudaMemcpyDeviceToDevice, st));

    // launch helpers
    const int warps = 1;
    auto fwd_sweep = [&](int axis, Buf &in, Buf &out) -> int {
        SweepArgs<T> a = env_sweep_args<T>(env, axis, dt);
        a.f = static_cast<T *>(in.p);
        a.fo = static_cast<T *>(out.p);
        if (axis < 2) {
            const bool tma = in.ok[axis] && out.ok[axis];
            return launch_strided<T>(a, axis, axis == 0, warps, tma ? &in.map[axis] : nullptr,
                                     tma ? &out.map[axis] : nullptr, in.crow[axis], st);
        }
        return launch_contig<T>(a, warps, env->use_tma != 0, st);
    };
    auto dirfaces = [&]() {
        SweepArgs<T> a = env_sweep_args<T>(env, 0, dt);
        return a.dir;
    };
    auto adj_sweep = [&](int axis, const T *X, const T *lin, T *mout) -> int {
        SweepArgs<T> a = env_sweep_args<T>(env, axis, dt);
        a.f = const_cast<T *>(X);
        a.fo = mout;
        if (axis < 2) {
            const StridedGeom &g = axis == 0 ? gx : gy;
            const size_t smem = 2 * (size_t)g.n * 32 * sizeof(T);
            if (smem > 227 * 1024) return fail(BFB_ERR_UNSUPPORTED, "adjoint: lines too long for shared memory");
            const unsigned blocks = (unsigned)((long long)g.n_slabs * g.ncb);
            if (axis == 0) {
                cudaFuncSetAttribute(adjoint_strided_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     227 * 1024);
                adjoint_strided_kernel<T, true><<<blocks, 32, smem, st>>>(a, lin, g, part);
            } else {
                cudaFuncSetAttribute(adjoint_strided_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     227 * 1024);
                adjoint_strided_kernel<T, false><<<blocks, 32, smem, st>>>(a, lin, g, part);
            }
            BFB_CUDA(cudaGetLastError());
            adjoint_reduce_kernel<<<S, 256, 0, st>>>(part, blocks, 1, g.P, g.ncb, S, 32, 0, 0, gacc);
        } else {
            const size_t smem = 2 * (size_t)gz.R * gz.RS * sizeof(T);
            if (smem > 227 * 1024) return fail(BFB_ERR_UNSUPPORTED, "adjoint: rows too long for shared memory");
            const unsigned blocks = (unsigned)((gz.nrows + gz.R - 1) / gz.R);
            cudaFuncSetAttribute(adjoint_contig_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            adjoint_contig_kernel<T><<<blocks, 32, smem, st>>>(a, lin, gz, LPT, part);
            BFB_CUDA(cudaGetLastError());
            adjoint_reduce_kernel<<<S, 256, 0, st>>>(part, blocks, 0, 0, 0, S, LPT, gz.R, gz.nrows, gacc);
        }
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    };
    const DirFaces<T> dir = dirfaces();
    const long long nface = 2 * ((long long)env->ny * env->nz + (long long)env->nx * env->nz +
                                 (long long)env->nx * env->ny);
    auto mask = [&](T *f) -> int {
        if (!dir.any) return BFB_OK;
        adjoint_mask_kernel<T><<<(unsigned)((nface + 255) / 256), 256, 0, st>>>(f, dir);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    };
    const unsigned occ_blocks = (unsigned)((occ + 255) / 256);
    const T *t1 = static_cast<const T *>(env->ag_t1), *t2 = static_cast<const T *>(env->ag_t2);

    // ---- reverse, segment by segment
    for (int c = nseg - 1; c >= 0; --c) {
        const int len = std::min(K, n_steps - c * K);
        BFB_CUDA(cudaMemcpyAsync(U[0].p, ckpt[c], fb, cudaMemcpyDeviceToDevice, st));
        for (int j = 0; j < len; ++j) {  // recompute, keeping every stage input
            if ((rc = fwd_sweep(0, U[j], S1[j])) || (rc = fwd_sweep(1, S1[j], S2[j])) ||
                (rc = fwd_sweep(2, S2[j], U[j + 1])))
                return rc;
            if (cells) {
                gather_occ_kernel<T><<<occ_blocks, 256, 0, st>>>(static_cast<T *>(U[j + 1].p), env->seg_voxel,
                                                                 env->n_occ, S, vocc + (size_t)j * occ);
                cells_on_kernel<T><<<occ_blocks, 256, 0, st>>>(static_cast<T *>(U[j + 1].p), S, env->n_occ,
                                                               env->seg_start, env->seg_voxel, t1, t2);
                BFB_CUDA(cudaGetLastError());
            }
        }
        for (int j = len - 1; j >= 0; --j) {  // reverse each step
            if (cells) {
                cells_adjoint_kernel<T><<<occ_blocks, 256, 0, st>>>(lam, vocc + (size_t)j * occ, S, env->n_occ,
                                                                    env->seg_start, env->seg_voxel, t1, t2, gt1, gt2);
                BFB_CUDA(cudaGetLastError());
            }
            if ((rc = adj_sweep(2, static_cast<T *>(S2[j].p), lam, mu))) return rc;
            if ((rc = adj_sweep(1, static_cast<T *>(S1[j].p), mu, lam))) return rc;
            if ((rc = adj_sweep(0, static_cast<T *>(U[j].p), lam, mu))) return rc;
            if ((rc = mask(mu))) return rc;
            std::swap(lam, mu);  // lam = dL/du of this step's input
        }
    }
    if (dL_dinitial) BFB_CUDA(cudaMemcpyAsync(dL_dinitial, lam, fb, cudaMemcpyDeviceToDevice, st));

    // ---- gradients to the caller
    std::vector<double> acc(2 * S);
    BFB_CUDA(cudaMemcpyAsync(acc.data(), gacc, sizeof(double) * 2 * S, cudaMemcpyDeviceToHost, st));
    std::vector<double> h1(nact), h2(nact);
    std::vector<int> order(env->n_active);
    if (nact) {
        BFB_CUDA(cudaMemcpyAsync(h1.data(), gt1, sizeof(double) * nact, cudaMemcpyDeviceToHost, st));
        BFB_CUDA(cudaMemcpyAsync(h2.data(), gt2, sizeof(double) * nact, cudaMemcpyDeviceToHost, st));
        BFB_CUDA(cudaMemcpyAsync(order.data(), env->ag_order, sizeof(int) * env->n_active, cudaMemcpyDeviceToHost,
                                 st));
    }
    BFB_CUDA(cudaStreamSynchronize(st));
    const double kD = -dt / (env->dx * env->dx), kL = -dt / 3.0;
    for (int d = 0; d < S; ++d) {
        if (gD) gD[d] = kD * acc[d];
        if (gL) gL[d] = kL * acc[S + d];
    }
    // temp1 = c S rho*, temp2 = 1 + c S + c U, c = dt*volume/dV (set_internal_uptake_constants)
    const size_t nlist = (size_t)env->n_agents * S;
    if (gsec) std::fill(gsec, gsec + nlist, 0.0);
    if (gupt) std::fill(gupt, gupt + nlist, 0.0);
    if (gsat) std::fill(gsat, gsat + nlist, 0.0);
    if ((gsec || gupt || gsat) && cells) {
        if (env->h_sec.empty())
            return fail(BFB_ERR_STATE, "adjoint: agents were set from cached constants; rates are unknown");
        const double dV = (env->dx * env->dx) * env->dx;
        for (int q = 0; q < env->n_active; ++q) {
            const int a = order[q];
            const double c = env->agent_dt * env->h_vol[a] / dV;
            for (int d = 0; d < S; ++d) {
                const size_t qa = (size_t)q * S + d, la = (size_t)a * S + d;
                if (gsec) gsec[la] = h1[qa] * c * env->h_sat[la] + h2[qa] * c;
                if (gupt) gupt[la] = h2[qa] * c;
                if (gsat) gsat[la] = h1[qa] * c * env->h_sec[la];
            }
        }
    }
    return BFB_OK;
}

}  // namespace

extern "C" BFB_API int bfb_adjoint_run(bfb_env env, double dt, int n_steps, int flags, int checkpoint_every,
                                       const void *dL_dfinal, void *dL_dinitial, void *final_field, double *dL_dD,
                                       double *dL_dlambda, double *dL_dsecretion, double *dL_duptake,
                                       double *dL_dsaturation) {
    if (!env) return fail(BFB_ERR_INVALID_ARG, "null bfb_env");
    if (n_steps < 1 || checkpoint_every < 1 || !(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "bad dt, n_steps or K");
    if (!dL_dfinal) return fail(BFB_ERR_INVALID_ARG, "dL_dfinal is NULL");
    if (!(flags & BFB_STEP_DIFFUSION) || (flags & ~(BFB_STEP_DIFFUSION | BFB_STEP_CELLS)))
        return fail(BFB_ERR_UNSUPPORTED, "adjoint: flags must be BFB_STEP_DIFFUSION [| BFB_STEP_CELLS]");
    BFB_CUDA(cudaSetDevice(env->device));
    const int K = std::min(checkpoint_every, n_steps);
    return env->precision == BFB_FP64
               ? adjoint_run<double>(env, dt, n_steps, flags, K, dL_dfinal, dL_dinitial, final_field, dL_dD,
                                     dL_dlambda, dL_dsecretion, dL_duptake, dL_dsaturation)
               : adjoint_run<float>(env, dt, n_steps, flags, K, dL_dfinal, dL_dinitial, final_field, dL_dD,
                                    dL_dlambda, dL_dsecretion, dL_duptake, dL_dsaturation);
}
