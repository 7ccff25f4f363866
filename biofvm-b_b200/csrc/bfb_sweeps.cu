// bfb_sweeps.cu -- Thomas sweep kernels (see bfb_sweeps.cuh for the design).
#include "bfb_sweeps.cuh"
#include "bfb_tiles.cuh"

#include <algorithm>
#include <mutex>

namespace bfb {


// ---------------------------------------------------------------------------
// One line, at line[m*ls] (m = 0..n-1), in shared or global memory.
//   pre(m, x)   input transform (bulk / pre-sweep Dirichlet), identity otherwise
//   out(m, y)   writes the result of row m (Dirichlet applied by the caller)
//   ready(r)    called before row r is first read; lets the strided kernel
//               wait for the cp.async group holding row r
// The per-lane factor pointers are already offset by the substrate d. The
// line pointer and stride are 64-bit so the global fallbacks can use it too.
// ---------------------------------------------------------------------------
struct LineFactors64 {
    const double *den, *cb, *rcp;
    double den_t, cb_t, rcp_t, c1;
    int S, m0;
};

template <class Pre, class Out, class Ready>
__device__ __forceinline__ void solve_line(double *line, long long ls, int n, const LineFactors64 &F, Pre pre,
                                           Out out, Ready ready) {
    ready(0);
    double prev = div_rcp(pre(0, line[0]), F.den[0], F.rcp[0]);
    line[0] = prev;
    const int hb = min(F.m0, n - 1);  // head rows [1, hb) read the tables
    for (int r = 1; r < hb; ++r) {
        ready(r);
        const size_t q = (size_t)r * F.S;
        prev = div_rcp(__fma_rn(F.c1, prev, pre(r, line[r * ls])), F.den[q], F.rcp[q]);
        line[r * ls] = prev;
    }
#pragma unroll 4
    for (int r = max(hb, 1); r < n - 1; ++r) {  // tail rows use register factors
        ready(r);
        prev = div_rcp(__fma_rn(F.c1, prev, pre(r, line[r * ls])), F.den_t, F.rcp_t);
        line[r * ls] = prev;
    }
    if (n > 1) {
        ready(n - 1);
        const size_t q = (size_t)(n - 1) * F.S;
        prev = div_rcp(__fma_rn(F.c1, prev, pre(n - 1, line[(n - 1) * ls])), F.den[q], F.rcp[q]);
    }
    double next = prev;
    out(n - 1, next);
    const int tl = max(F.m0, 0);
#pragma unroll 4
    for (int r = n - 2; r >= tl; --r) {
        next = __fma_rn(-F.cb_t, next, line[r * ls]);
        out(r, next);
    }
    for (int r = min(tl, n - 1) - 1; r >= 0; --r) {
        next = __fma_rn(-F.cb[(size_t)r * F.S], next, line[r * ls]);
        out(r, next);
    }
}

struct LineFactors32 {
    const float *rh, *rl, *a, *cb;
    float rh_t, rl_t, a_t, cb_t;
    float gh, gl;
    int S, m0;
};

template <class Pre, class Out, class Ready>
__device__ __forceinline__ void solve_line(float *line, long long ls, int n, const LineFactors32 &F, Pre pre, Out out,
                                           Ready ready) {
    ready(0);
    ready(min(1, n - 1));
    const float xb = pre(min(1, n - 1), line[min(1, n - 1) * ls]);  // deviation reference: row 1
    float p;
    {
        const float dlt = __fsub_rn(pre(0, line[0]), xb);
        p = __fmaf_rn(dlt, F.rh[0], __fmul_rn(dlt, F.rl[0]));
    }
    line[0] = p;
    const int hb = min(F.m0, n - 1);
    for (int r = 1; r < hb; ++r) {
        ready(r);
        const float dlt = __fsub_rn(pre(r, line[r * ls]), xb);
        const size_t q = (size_t)r * F.S;
        p = __fmaf_rn(F.a[q], p, __fmaf_rn(dlt, F.rh[q], __fmul_rn(dlt, F.rl[q])));
        line[r * ls] = p;
    }
#pragma unroll 4
    for (int r = max(hb, 1); r < n - 1; ++r) {
        ready(r);
        const float dlt = __fsub_rn(pre(r, line[r * ls]), xb);
        p = __fmaf_rn(F.a_t, p, __fmaf_rn(dlt, F.rh_t, __fmul_rn(dlt, F.rl_t)));
        line[r * ls] = p;
    }
    if (n > 1) {
        ready(n - 1);
        const float dlt = __fsub_rn(pre(n - 1, line[(n - 1) * ls]), xb);
        const size_t q = (size_t)(n - 1) * F.S;
        p = __fmaf_rn(F.a[q], p, __fmaf_rn(dlt, F.rh[q], __fmul_rn(dlt, F.rl[q])));
    }
    // y = g*xb + z, with g*xb added as (hi, lo) around the deviation
    float next = p;
    out(n - 1, __fmaf_rn(xb, F.gh, __fmaf_rn(xb, F.gl, next)));
    const int tl = max(F.m0, 0);
#pragma unroll 4
    for (int r = n - 2; r >= tl; --r) {
        next = __fmaf_rn(-F.cb_t, next, line[r * ls]);
        out(r, __fmaf_rn(xb, F.gh, __fmaf_rn(xb, F.gl, next)));
    }
    for (int r = min(tl, n - 1) - 1; r >= 0; --r) {
        next = __fmaf_rn(-F.cb[(size_t)r * F.S], next, line[r * ls]);
        out(r, __fmaf_rn(xb, F.gh, __fmaf_rn(xb, F.gl, next)));
    }
}

__device__ __forceinline__ LineFactors64 line_factors(const SweepArgs<double> &a, int d) {
    LineFactors64 F;
    F.den = a.fac.t0 + d;
    F.cb = a.fac.t1 + d;
    F.rcp = a.fac.t2 + d;
    F.S = a.S;
    F.m0 = a.fac.m0;
    F.c1 = a.c1[d];
    F.den_t = a.fac.tail[d];
    F.cb_t = a.fac.tail[a.S + d];
    F.rcp_t = a.fac.tail[2 * a.S + d];
    return F;
}

__device__ __forceinline__ LineFactors32 line_factors(const SweepArgs<float> &a, int d) {
    LineFactors32 F;
    F.rh = a.fac.t0 + d;
    F.rl = a.fac.t1 + d;
    F.a = a.fac.t2 + d;
    F.cb = a.fac.t3 + d;
    F.S = a.S;
    F.m0 = a.fac.m0;
    F.rh_t = a.fac.tail[d];
    F.rl_t = a.fac.tail[a.S + d];
    F.a_t = a.fac.tail[2 * a.S + d];
    F.cb_t = a.fac.tail[3 * a.S + d];
    F.gh = a.g[d];
    F.gl = a.g[a.S + d];
    return F;
}

// ---------------------------------------------------------------------------
// Strided sweep (x: axis 0, y: axis 1). One warp = one 32-column tile.
//   FUSE_PRE: x-sweep; applies the step's leading Dirichlet to rows 0 / n-1
//   BULK:     x-sweep; applies the bulk source/sink update on load
// The hot loops carry no Dirichlet test: rows 0 and n-1 are peeled, and a
// column lying wholly on an active face is overwritten after its solve.
// ---------------------------------------------------------------------------
template <typename T, int VB, bool FUSE_PRE, bool BULK>
__global__ void __launch_bounds__(128, 1) sweep_strided_kernel(SweepArgs<T> a, StridedGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile >= (long long)g.n_slabs * g.ncb) return;
    strided_tile<T, VB, FUSE_PRE, BULK>(a, g, tile, reinterpret_cast<T *>(smem_raw) + (size_t)warp * g.n * 32);
}

// ---------------------------------------------------------------------------
// Contiguous sweep (z). One warp = R consecutive (i,j) rows of nz*S elements.
// ---------------------------------------------------------------------------
template <typename T, int VB, int SC>
__global__ void __launch_bounds__(128, 1) sweep_contig_kernel(SweepArgs<T> a, ContigGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile * g.R >= g.nrows) return;
    contig_tile<T, VB, SC>(a, g, tile, reinterpret_cast<T *>(smem_raw) + (size_t)warp * g.R * g.RS);
}
// The same for S > 32 (a lane solves several lines of the tile).
template <typename T, int VB>
__global__ void __launch_bounds__(128, 1) sweep_contig_wide_kernel(SweepArgs<T> a, ContigGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile * g.R >= g.nrows) return;
    contig_tile_wide<T, VB>(a, g, tile, reinterpret_cast<T *>(smem_raw) + (size_t)warp * g.R * g.RS);
}

// ---------------------------------------------------------------------------
// Fallbacks for lines too long for shared memory: thread per line, the line
// read and written in place in global memory (the forward pass stores its
// intermediate values, so two reads and two writes per sweep).
// ---------------------------------------------------------------------------
template <typename T, bool FUSE_PRE>
__global__ void sweep_strided_global_kernel(SweepArgs<T> a, StridedGeom g) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.n_slabs * g.P) return;
    const int slab = (int)(t / g.P);
    const long long col = t % g.P;
    const int n = g.n;
    const StridedColumn col_at = strided_column(a, g, slab, col);
    if (!col_at.real) return;  // padding of a padded row: no line
    const int d = col_at.d, ci = col_at.ci, cj = col_at.cj, ck = col_at.ck;
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
    auto vox_dir = [&](int mm) -> T {
        return g.axis == 0 ? dir_value(a.dir, mm, cj, ck, d) : dir_value(a.dir, ci, mm, ck, d);
    };
    const long long P = g.P;
    T *line = a.fo + (size_t)slab * g.slab_stride + col;  // solved in place in the output
    if (a.fo != a.f) {
        const T *src = a.f + (size_t)slab * g.slab_stride + col;
        for (int r = 0; r < n; ++r) line[(size_t)r * P] = src[(size_t)r * P];
    }
    auto pre = [&](int r, T x) -> T {
        if constexpr (FUSE_PRE) {
            if (a.bulk.on) {
                const size_t e = (size_t)slab * g.slab_stride + (size_t)r * P + col;
                x = bulk_update(x, a.bulk.A[e], a.bulk.B[e], a.bulk.dt);
            }
            if ((r == 0 && lo_dir) || (r == n - 1 && hi_dir)) x = vox_dir(r);
        }
        return x;
    };
    auto out = [&](int r, T y) {
        if (col_dir || (r == 0 && lo_dir) || (r == n - 1 && hi_dir)) y = vox_dir(r);
        line[(size_t)r * P] = y;
    };
    auto ready = [](int) {};
    solve_line(line, P, n, line_factors(a, d), pre, out, ready);
}

template <typename T>
__global__ void sweep_contig_global_kernel(SweepArgs<T> a, long long nrows) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int S = a.S, nz = a.nz;
    if (t >= nrows * S) return;
    const long long row = t / S;
    const int d = (int)(t % S);
    const int i = (int)(row / a.ny), j = (int)(row % a.ny);
    const unsigned m = a.dir.any ? a.dir.mask[d] : 0u;
    const bool line_dir = ((m & 1u) && i == 0) || ((m & 2u) && i == a.nx - 1) || ((m & 4u) && j == 0) ||
                          ((m & 8u) && j == a.ny - 1);
    const bool lo_dir = m & 16u, hi_dir = m & 32u;
    T *line = a.fo + (size_t)row * a.Lp + d;  // solved in place in the output
    if (a.fo != a.f) {
        const T *src = a.f + (size_t)row * a.Lp + d;
        for (int k = 0; k < nz; ++k) line[(size_t)k * S] = src[(size_t)k * S];
    }
    auto pre = [](int, T x) -> T { return x; };
    auto out = [&](int k, T y) {
        if (line_dir || (k == 0 && lo_dir) || (k == nz - 1 && hi_dir)) y = dir_value(a.dir, i, j, k, d);
        line[(size_t)k * S] = y;
    };
    auto ready = [](int) {};
    solve_line(line, S, nz, line_factors(a, d), pre, out, ready);
}

// ---------------------------------------------------------------------------
// Standalone Dirichlet (apply_dirichlet_conditions) and bulk step.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void dirichlet_kernel(SweepArgs<T> a) {
    // one thread per face voxel slot of the union of the 6 faces, enumerated
    // face by face; edges are written more than once with the same value
    const long long fx = (long long)a.ny * a.nz, fy = (long long)a.nx * a.nz, fz = (long long)a.nx * a.ny;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = 2 * (fx + fy + fz);
    if (t >= total) return;
    int i, j, k;
    if (t < 2 * fx) {
        const int side = (int)(t / fx);
        const long long q = t % fx;
        i = side ? a.nx - 1 : 0;
        j = (int)(q / a.nz);
        k = (int)(q % a.nz);
    } else if ((t -= 2 * fx) < 2 * fy) {
        const int side = (int)(t / fy);
        const long long q = t % fy;
        j = side ? a.ny - 1 : 0;
        i = (int)(q / a.nz);
        k = (int)(q % a.nz);
    } else {
        t -= 2 * fy;
        const int side = (int)(t / fz);
        const long long q = t % fz;
        k = side ? a.nz - 1 : 0;
        i = (int)(q / a.ny);
        j = (int)(q % a.ny);
    }
    const size_t vb = ((size_t)i * a.ny + j) * a.Lp + (size_t)k * a.S;
    for (int d = 0; d < a.S; ++d) {
        if (on_active_face(a.dir.mask[d], i, j, k, a.nx, a.ny, a.nz)) a.f[vb + d] = dir_value(a.dir, i, j, k, d);
    }
}

template <typename T>
__global__ void bulk_kernel(T *f, const T *A, const T *B, T dt, long long N) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x)
        f[e] = bulk_update(f[e], A[e], B[e], dt);
}

// ---------------------------------------------------------------------------
// Host-side launchers
// ---------------------------------------------------------------------------
size_t strided_smem(int n, int elem, int warps) {
    const size_t b = (size_t)warps * n * 32 * elem;
    return b <= (size_t)kMaxSmem ? b : 0;
}

size_t contig_smem(int nz, int S, int Lp, int elem, int warps, int *R, int *RS) {
    (void)nz;
    const int L = Lp;  // a shared row holds a whole (padded) row
    int r = S <= 32 ? 32 / S : 1;
    int rs = L;
    if (r > 1) {
        rs = L + ((S - (L % 32)) % 32 + 32) % 32;  // smallest rs >= L with rs = S (mod 32)
    }
    *R = r;
    *RS = rs;
    const size_t b = (size_t)warps * r * rs * elem;
    return b <= (size_t)kMaxSmem ? b : 0;
}

template <typename T, int VB, bool FP>
static int go_strided(const SweepArgs<T> &a, const StridedGeom &g, int warps, size_t smem, cudaStream_t s) {
    const long long tiles = (long long)g.n_slabs * g.ncb;
    const long long blocks = (tiles + warps - 1) / warps;
    if (FP && a.bulk.on)
        sweep_strided_kernel<T, VB, FP, FP><<<(unsigned)blocks, warps * 32, smem, s>>>(a, g);
    else
        sweep_strided_kernel<T, VB, FP, false><<<(unsigned)blocks, warps * 32, smem, s>>>(a, g);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

template <typename T>
int launch_strided(const SweepArgs<T> &a, int axis, bool fuse_pre, int warps, const CUtensorMap *map,
                   const CUtensorMap *map_out, int crow, int lines, cudaStream_t s) {
    StridedGeom g = strided_geometry(a, axis);
    warps = std::max(1, std::min(warps, 4));
    // the x sweep's load-time Dirichlet and bulk update: without either, the
    // plain kernel computes the same
    fuse_pre = fuse_pre && (a.dir.any || a.bulk.on);
    if (map && map_out) {
        const int st = launch_strided_tma<T>(a, g, map, map_out, crow, lines, fuse_pre, warps, s);
        if (st != kNotApplicable) return st;
    }
    size_t smem = strided_smem(g.n, sizeof(T), warps);
    while (smem == 0 && warps > 1) smem = strided_smem(g.n, sizeof(T), --warps);
    if (smem == 0) {
        const long long threads = (long long)g.n_slabs * g.P;
        const unsigned blocks = (unsigned)((threads + 127) / 128);
        if (fuse_pre)
            sweep_strided_global_kernel<T, true><<<blocks, 128, 0, s>>>(a, g);
        else
            sweep_strided_global_kernel<T, false><<<blocks, 128, 0, s>>>(a, g);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }
    // 16-byte copies need every row start 16-byte aligned
    const bool al16 = ((g.P * (long long)sizeof(T)) % 16 == 0) && ((g.slab_stride * (long long)sizeof(T)) % 16 == 0) &&
                      ((reinterpret_cast<uintptr_t>(a.f) & 15) == 0);
    if (al16) {
        return fuse_pre ? go_strided<T, 16, true>(a, g, warps, smem, s) : go_strided<T, 16, false>(a, g, warps, smem, s);
    }
    return fuse_pre ? go_strided<T, (int)sizeof(T), true>(a, g, warps, smem, s)
                    : go_strided<T, (int)sizeof(T), false>(a, g, warps, smem, s);
}

bool contig_aligned_geom(int nz, int S, int Lp, int elem, int *R, int *RS) {
    if ((elem != 4 && elem != 8) || S > 32) return false;
    (void)nz;
    // A warp's access to element r*rs + k*S + d (lane (r, d)) is conflict-free
    // when no 4-byte bank holds more words of it than the element has words:
    // every element index mod `slots` at most `words` times (FP32: 32 slots,
    // once each; FP64: 16 slots of two banks, twice each -- the two
    // wavefronts that 256 bytes take anyway). Where that leaves fewer than 16
    // lanes busy (FP32 S = 1), two-way conflicts are allowed (measured at
    // 256^3 x 1 FP32: 0.053 ms against 0.073 for the cp.async tile; for other
    // S they cost more than the lanes they add).
    const int epv = 16 / elem, words = elem / 4, slots = 32 / words;
    const int base = (Lp + epv - 1) / epv * epv;  // a shared row holds a whole (padded) row
    for (int cap = 1; cap <= 2; ++cap) {
        int best_r = 0, best_rs = 0;
        for (int t = 0; t < slots / epv; ++t) {  // base + epv*t: every multiple of epv (mod slots) once
            const int rs = base + epv * t;
            int used[32] = {0};
            int r = 0;
            for (; r < 32 / S; ++r) {
                int add[32] = {0};
                bool ok = true;
                for (int d = 0; d < S; ++d) {
                    const int q = (int)(((long long)r * rs + d) % slots);
                    ok = ok && used[q] + ++add[q] <= words * cap;
                }
                if (!ok) break;
                for (int q = 0; q < slots; ++q) used[q] += add[q];
            }
            if (r > best_r) {
                best_r = r;
                best_rs = rs;
            }
        }
        if (best_r * S >= 16) {
            *R = best_r;
            *RS = best_rs;
            return true;
        }
    }
    return false;
}

template <typename T, int VB>
static int go_contig(const SweepArgs<T> &a, const ContigGeom &g, int warps, size_t smem, cudaStream_t s) {
    const long long tiles = (g.nrows + g.R - 1) / g.R;
    const long long blocks = (tiles + warps - 1) / warps;
#define BFB_CONTIG(SC) sweep_contig_kernel<T, VB, SC><<<(unsigned)blocks, warps * 32, smem, s>>>(a, g)
    switch (a.S) {  // the substrate count as a constant where it is a common one
    case 1: BFB_CONTIG(1); break;
    case 2: BFB_CONTIG(2); break;
    case 3: BFB_CONTIG(3); break;
    case 4: BFB_CONTIG(4); break;
    case 5: BFB_CONTIG(5); break;
    case 6: BFB_CONTIG(6); break;
    case 8: BFB_CONTIG(8); break;
    default:
        if (a.S > 32) sweep_contig_wide_kernel<T, VB><<<(unsigned)blocks, warps * 32, smem, s>>>(a, g);
        else BFB_CONTIG(0);
    }
#undef BFB_CONTIG
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// Rows per bulk-copy z tile for FP64: a tile holds whole rows, so few tiles
// fit an SM; where fewer rows per tile keep at least 1/16 more lines resident
// per SM (one-warp CTAs; 228 KB of shared memory per SM, 1 KB reserved per
// CTA), the tile takes that many. A stride free of bank conflicts for R rows
// is free of them for fewer.
static int z_rows_for_residency(int R, int RS, int S, int eb) {
    const long long smem_sm = 228 * 1024, reserve = 1024;
    auto lines = [&](int r) -> long long {
        const long long wb = (128 + (long long)r * RS * eb + 127) / 128 * 128;
        return smem_sm / (wb + reserve) * r * S;
    };
    const long long base = lines(R);
    int best = R;
    long long best_l = base;
    for (int r = R - 1; r >= 1 && r * S >= 16; --r)  // at least half the warp busy
        if (lines(r) > best_l) {
            best_l = lines(r);
            best = r;
        }
    return best_l >= base + base / 16 ? best : R;
}

template <typename T>
int launch_contig(const SweepArgs<T> &a, int warps, bool use_tma, cudaStream_t s, int chunks) {
    ContigGeom g;
    g.nz = a.nz;
    g.nrows = (long long)a.nx * a.ny;
    g.Lp = a.Lp;
    warps = std::max(1, std::min(warps, 4));
    size_t smem = contig_smem(a.nz, a.S, a.Lp, sizeof(T), warps, &g.R, &g.RS);
    while (smem == 0 && warps > 1) smem = contig_smem(a.nz, a.S, a.Lp, sizeof(T), --warps, &g.R, &g.RS);
    if (smem == 0) {
        const long long threads = g.nrows * a.S;
        sweep_contig_global_kernel<T><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(a, g.nrows);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }
    const long long L = a.Lp;  // row pitch: copies cover whole (padded) rows
    const bool base16 = (reinterpret_cast<uintptr_t>(a.f) & 15) == 0;
    const int eb = (int)sizeof(T);
    if (use_tma && base16 && (L * eb) % 16 == 0) {
        // the bulk-copy tile needs 16-byte shared rows: contig_smem's
        // conflict-free stride where it is one, else contig_aligned_geom's
        ContigGeom gt = g;
        const bool ok = ((long long)g.RS * eb) % 16 == 0 || contig_aligned_geom(a.nz, a.S, a.Lp, eb, &gt.R, &gt.RS);
        if (ok && eb == 8) gt.R = z_rows_for_residency(gt.R, gt.RS, a.S, eb);
        if (ok && (L * eb) * gt.R < (1 << 20)) {
            const int st = launch_contig_tma<T>(a, gt, warps, s, chunks);
            if (st != kNotApplicable) return st;
        }
    }
    if (base16 && (L * eb) % 16 == 0 && ((long long)g.RS * eb) % 16 == 0) return go_contig<T, 16>(a, g, warps, smem, s);
    if (eb < 8 && (L * eb) % 8 == 0 && ((long long)g.RS * eb) % 8 == 0) return go_contig<T, 8>(a, g, warps, smem, s);
    return go_contig<T, (int)sizeof(T)>(a, g, warps, smem, s);
}

template <typename T>
int launch_dirichlet(const SweepArgs<T> &a, cudaStream_t s) {
    if (!a.dir.any) return BFB_OK;
    const long long total = 2 * ((long long)a.ny * a.nz + (long long)a.nx * a.nz + (long long)a.nx * a.ny);
    dirichlet_kernel<T><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(a);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

template <typename T>
int launch_bulk(const SweepArgs<T> &a, long long N, cudaStream_t s) {
    if (!a.bulk.on) return BFB_OK;
    const long long blocks = std::min<long long>((N + 255) / 256, 148LL * 16);
    bulk_kernel<T><<<(unsigned)blocks, 256, 0, s>>>(a.f, a.bulk.A, a.bulk.B, a.bulk.dt, N);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// Opt every shared-memory kernel into the full 227 KB once per device, before
// any launch (so that nothing configures a kernel inside a stream capture).
template <typename K>
static void opt_in(K k) {
    cudaFuncSetAttribute((const void *)k, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
}

template <typename T, int VB>
static void opt_in_contig() {
    opt_in(sweep_contig_kernel<T, VB, 0>);
    opt_in(sweep_contig_kernel<T, VB, 1>);
    opt_in(sweep_contig_kernel<T, VB, 2>);
    opt_in(sweep_contig_kernel<T, VB, 3>);
    opt_in(sweep_contig_kernel<T, VB, 4>);
    opt_in(sweep_contig_kernel<T, VB, 5>);
    opt_in(sweep_contig_kernel<T, VB, 6>);
    opt_in(sweep_contig_kernel<T, VB, 8>);
}

void sweeps_prepare_device() {
    static std::mutex mu;
    static unsigned long long done = 0;  // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done & (1ull << (dev & 63))) return;
    opt_in(sweep_strided_kernel<double, 16, true, true>);
    opt_in(sweep_strided_kernel<double, 16, true, false>);
    opt_in(sweep_strided_kernel<double, 16, false, false>);
    opt_in(sweep_strided_kernel<double, 8, true, true>);
    opt_in(sweep_strided_kernel<double, 8, true, false>);
    opt_in(sweep_strided_kernel<double, 8, false, false>);
    opt_in(sweep_strided_kernel<float, 16, true, true>);
    opt_in(sweep_strided_kernel<float, 16, true, false>);
    opt_in(sweep_strided_kernel<float, 16, false, false>);
    opt_in(sweep_strided_kernel<float, 4, true, true>);
    opt_in(sweep_strided_kernel<float, 4, true, false>);
    opt_in(sweep_strided_kernel<float, 4, false, false>);
    opt_in_contig<double, 16>();
    opt_in_contig<double, 8>();
    opt_in_contig<float, 16>();
    opt_in_contig<float, 8>();
    opt_in_contig<float, 4>();
    opt_in(sweep_contig_wide_kernel<double, 16>);
    opt_in(sweep_contig_wide_kernel<double, 8>);
    opt_in(sweep_contig_wide_kernel<float, 16>);
    opt_in(sweep_contig_wide_kernel<float, 8>);
    opt_in(sweep_contig_wide_kernel<float, 4>);
    tma_prepare_device();
    tmem_prepare_device();
    done |= 1ull << (dev & 63);
}

template int launch_strided<double>(const SweepArgs<double> &, int, bool, int, const CUtensorMap *,
                                    const CUtensorMap *, int, int, cudaStream_t);
template int launch_strided<float>(const SweepArgs<float> &, int, bool, int, const CUtensorMap *, const CUtensorMap *,
                                   int, int, cudaStream_t);
template int launch_contig<double>(const SweepArgs<double> &, int, bool, cudaStream_t, int);
template int launch_contig<float>(const SweepArgs<float> &, int, bool, cudaStream_t, int);
template int launch_dirichlet<double>(const SweepArgs<double> &, cudaStream_t);
template int launch_dirichlet<float>(const SweepArgs<float> &, cudaStream_t);
template int launch_bulk<double>(const SweepArgs<double> &, long long, cudaStream_t);
template int launch_bulk<float>(const SweepArgs<float> &, long long, cudaStream_t);

}  // namespace bfb
