// bfb_tma.cu -- the sweeps with Blackwell's tensor memory accelerator (TMA).
//
// Same algorithm as the cp.async kernels in bfb_sweeps.cu (see bfb_sweeps.cuh),
// with the data movement handed to the TMA engine:
//   * strided x/y sweeps: one elected lane issues kChunks 2-D/3-D tensor
//     copies (cp.async.bulk.tensor, box = 32 lines x crow rows) per warp tile,
//     each completing on its own mbarrier; the forward elimination starts on
//     row group 0 while the later groups are still in flight. The back
//     substitution writes its results into the tile in shared memory, and each
//     finished row group is written back by a bulk tensor store while the
//     lower groups are still being computed.
//   * contiguous z sweep: the R rows of a warp tile are one contiguous block
//     of global memory; each row is one 1-D bulk copy (cp.async.bulk) into its
//     padded shared row, and one bulk store per row writes it back.
// Nothing here multicasts: every copy moves this GPU's memory into this CTA.
// Every mbarrier wait is bounded; a wait that runs out sets the env's error
// flag and the warp returns.
#include <cuda.h>

#include "bfb_tma.cuh"

namespace bfb {

// ---------------------------------------------------------------------------
// Strided sweep with TMA (rank 2: x, rank 3: y).
// ---------------------------------------------------------------------------
template <typename T, bool FUSE_PRE, bool BULK>
__global__ void __launch_bounds__(128)
    sweep_strided_tma_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap map_out,
                             SweepArgs<T> a, StridedGeom g, int crow) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile >= (long long)g.n_slabs * g.ncb) return;
    const int slab = (int)(tile / g.ncb);
    const int col0 = (int)((tile % g.ncb) * 32);
    const int n = g.n;
    const long long P = g.P;
    const int nch = (n + crow - 1) / crow;
    const int rank = g.axis == 0 ? 2 : 3;
    unsigned char *wbase = smem_raw + (size_t)warp * strided_tma_warp_bytes(n, crow, sizeof(T));
    const unsigned bar0 = smem_u32(wbase);
    T *__restrict__ sm = reinterpret_cast<T *>(wbase + 128);
    const unsigned sm_u32 = smem_u32(sm);
    const unsigned chunk_bytes = (unsigned)crow * 32u * (unsigned)sizeof(T);

    if (lane == 0) {
        for (int ch = 0; ch < nch; ++ch) mbar_init(bar0 + 8 * ch, 1);
        fence_mbar_init();
    }
    __syncwarp();
    if (lane == 0) {
        for (int ch = 0; ch < nch; ++ch) {
            mbar_expect_tx(bar0 + 8 * ch, chunk_bytes);
            tma_load(sm_u32 + ch * chunk_bytes, &map, col0, ch * crow, slab, rank, bar0 + 8 * ch);
        }
    }

    // ---- line coordinates of this lane (lanes past P run along on zeros)
    const long long col = (long long)col0 + lane;
    const bool valid = col < P;
    const int S = a.S;
    const int d = (int)(col % S);
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
    const unsigned m = (a.dir.any && valid) ? a.dir.mask[d] : 0u;
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
    const T *bA = nullptr, *bB = nullptr;
    if constexpr (BULK) {
        bA = a.bulk.A + (size_t)slab * g.slab_stride + col;
        bB = a.bulk.B + (size_t)slab * g.slab_stride + col;
    }
    auto load = [&](int r) -> T {
        T x = sm[r * 32 + lane];
        if constexpr (BULK) {
            if (valid) x = bulk_update(x, bA[(size_t)r * P], bB[(size_t)r * P], a.bulk.dt);
        }
        return x;
    };
    auto wait_group = [&](int ch) -> bool {
        if (mbar_wait(bar0 + 8 * ch, 0)) return true;
        if (lane == 0) atomicOr(a.err, 1);
        return false;
    };

    LineSolver<T> L(a, d);
    const int m0 = a.fac.m0;

    // a line's input row after the step's leading Dirichlet
    auto xin = [&](int q) -> T {
        T x = load(q);
        if (FUSE_PRE && ((q == 0 && lo_dir) || (q == n - 1 && hi_dir))) x = vox_dir(q);
        return x;
    };

    // ---- forward elimination, row group by row group as the copies land
    const int rref = min(1, n - 1);  // row of the deviation reference
    const int ref_ch = rref / crow;
    for (int ch = 0; ch <= ref_ch; ++ch)
        if (!wait_group(ch)) return;
    sm[lane] = L.first(xin(0), xin(rref));
    int r = 1;
    for (int ch = 0; ch < nch; ++ch) {
        if (ch > ref_ch && !wait_group(ch)) return;
        const int rend = min(n - 1, (ch + 1) * crow);
        const int hend = min(rend, m0);
        for (; r < hend; ++r) sm[r * 32 + lane] = L.template fwd<false>(load(r), r);
#pragma unroll 8
        for (; r < rend; ++r) sm[r * 32 + lane] = L.template fwd<true>(load(r), r);
    }
    if (n > 1) {
        T x = load(n - 1);
        if (FUSE_PRE && hi_dir) x = vox_dir(n - 1);
        L.template fwd<false>(x, n - 1);
    }

    // ---- back substitution into the tile; each finished row group is stored
    {
        T y = L.out_last();
        if (hi_dir || (lo_dir && n == 1)) y = vox_dir(n - 1);
        sm[(n - 1) * 32 + lane] = y;
    }
    const int tl = max(m0, 1);
    r = n - 2;
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int rlo = ch * crow;
        const int tstop = max(rlo, tl);
#pragma unroll 8
        for (; r >= tstop; --r) sm[r * 32 + lane] = L.template bwd<true>(sm[r * 32 + lane], r);
        const int hstop = max(rlo, 1);
        for (; r >= hstop; --r) sm[r * 32 + lane] = L.template bwd<false>(sm[r * 32 + lane], r);
        if (rlo == 0 && n > 1) {
            T y = L.template bwd<false>(sm[lane], 0);
            if (lo_dir) y = vox_dir(0);
            sm[lane] = y;
        }
        if (col_dir)  // the whole column lies on an active face of another axis
            for (int q = rlo; q < min(n, rlo + crow); ++q) sm[q * 32 + lane] = vox_dir(q);
        fence_async_smem();
        __syncwarp();
        if (lane == 0) {
            tma_store(&map_out, col0, rlo, slab, rank, sm_u32 + ch * chunk_bytes);
            bulk_commit();
        }
    }
    if (lane == 0) bulk_wait_read_all();  // the tile must outlive the stores' reads
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Contiguous z sweep with 1-D bulk copies.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) sweep_contig_tma_kernel(SweepArgs<T> a, ContigGeom g) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    const long long row0 = tile * g.R;
    if (row0 >= g.nrows) return;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = a.S, nz = g.nz;
    const int L = nz * S;
    const size_t wbytes = 128 + (size_t)g.R * g.RS * sizeof(T);
    unsigned char *wbase = smem_raw + (size_t)warp * ((wbytes + 127) / 128 * 128);
    const unsigned bar = smem_u32(wbase);
    T *__restrict__ sm = reinterpret_cast<T *>(wbase + 128);
    T *__restrict__ base = a.f + (size_t)row0 * L;
    T *__restrict__ obase = a.fo + (size_t)row0 * L;
    const unsigned row_bytes = (unsigned)L * (unsigned)sizeof(T);

    if (lane == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncwarp();
    if (lane == 0) {
        mbar_expect_tx(bar, row_bytes * (unsigned)nr);
        for (int r = 0; r < nr; ++r) bulk_load(smem_u32(sm + (size_t)r * g.RS), base + (size_t)r * L, row_bytes, bar);
    }
    if (!mbar_wait(bar, 0)) {
        if (lane == 0) atomicOr(a.err, 1);
        return;
    }

    const int m0 = a.fac.m0;
    for (int t = lane; t < nr * S; t += 32) {
        const int r = t / S, d = t - r * S;
        const long long row = row0 + r;
        const int i = (int)(row / a.ny), j = (int)(row % a.ny);
        const unsigned m = a.dir.any ? a.dir.mask[d] : 0u;
        const bool line_dir = ((m & 1u) && i == 0) || ((m & 2u) && i == a.nx - 1) || ((m & 4u) && j == 0) ||
                              ((m & 8u) && j == a.ny - 1);
        const bool lo_dir = m & 16u, hi_dir = m & 32u;
        T *line = sm + (size_t)r * g.RS + d;
        LineSolver<T> Ls(a, d);
        line[0] = Ls.first(line[0], line[min(1, nz - 1) * S]);
        const int hend = min(nz - 1, m0);
        int k = 1;
        for (; k < hend; ++k) line[k * S] = Ls.template fwd<false>(line[k * S], k);
#pragma unroll 8
        for (; k < nz - 1; ++k) line[k * S] = Ls.template fwd<true>(line[k * S], k);
        if (nz > 1) Ls.template fwd<false>(line[(nz - 1) * S], nz - 1);
        {
            const T y = Ls.out_last();
            line[(nz - 1) * S] = (hi_dir || (lo_dir && nz == 1)) ? dir_value(a.dir, i, j, nz - 1, d) : y;
        }
        const int tl = max(m0, 1);
        k = nz - 2;
#pragma unroll 8
        for (; k >= tl; --k) line[k * S] = Ls.template bwd<true>(line[k * S], k);
        for (; k >= 1; --k) line[k * S] = Ls.template bwd<false>(line[k * S], k);
        if (nz > 1) {
            const T y = Ls.template bwd<false>(line[0], 0);
            line[0] = lo_dir ? dir_value(a.dir, i, j, 0, d) : y;
        }
        if (line_dir)
            for (int q = 0; q < nz; ++q) line[q * S] = dir_value(a.dir, i, j, q, d);
    }
    fence_async_smem();
    __syncwarp();
    if (lane == 0) {
        for (int r = 0; r < nr; ++r) bulk_store(obase + (size_t)r * L, smem_u32(sm + (size_t)r * g.RS), row_bytes);
        bulk_commit();
        bulk_wait_read_all();
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Contiguous z sweep, pipelined: the tile's k range is cut into row groups of
// kc rows; group c of every row is one bulk copy on mbarrier c, so the
// forward elimination starts on group 0 while the later groups land, and the
// back substitution stores each finished group while the lower ones are
// still being computed. SC is the substrate count when it is a compile-time
// constant (1, 2, 4, 8), 0 otherwise; every lane owns at most one line
// (S <= 32 gives R = 32/S rows per warp).
// ---------------------------------------------------------------------------
template <typename T, int SC>
__global__ void __launch_bounds__(128) sweep_contig_pipe_kernel(SweepArgs<T> a, ContigGeom g, int kc) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    const long long row0 = tile * g.R;
    if (row0 >= g.nrows) return;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = SC > 0 ? SC : a.S;
    const int nz = g.nz;
    const int L = nz * S;
    const int nch = (nz + kc - 1) / kc;
    const size_t wbytes = (128 + (size_t)g.R * g.RS * sizeof(T) + 127) / 128 * 128;
    unsigned char *wbase = smem_raw + (size_t)warp * wbytes;
    const unsigned bar0 = smem_u32(wbase);
    T *__restrict__ sm = reinterpret_cast<T *>(wbase + 128);
    T *__restrict__ base = a.f + (size_t)row0 * L;
    T *__restrict__ obase = a.fo + (size_t)row0 * L;
    auto seg_bytes = [&](int c) -> unsigned { return (unsigned)((min(nz, (c + 1) * kc) - c * kc) * S * (int)sizeof(T)); };

    if (lane == 0) {
        for (int c = 0; c < nch; ++c) mbar_init(bar0 + 8 * c, 1);
        fence_mbar_init();
    }
    __syncwarp();
    if (lane == 0) {
        for (int c = 0; c < nch; ++c) {
            const unsigned b = seg_bytes(c);
            mbar_expect_tx(bar0 + 8 * c, b * (unsigned)nr);
            for (int r = 0; r < nr; ++r)
                bulk_load(smem_u32(sm + (size_t)r * g.RS + (size_t)c * kc * S), base + (size_t)r * L + (size_t)c * kc * S,
                          b, bar0 + 8 * c);
        }
    }
    auto wait_c = [&](int c) -> bool {
        if (mbar_wait(bar0 + 8 * c, 0)) return true;
        if (lane == 0) atomicOr(a.err, 1);
        return false;
    };

    const bool active = lane < nr * S;
    const int r = active ? lane / S : 0;
    const int d = active ? lane - r * S : 0;
    const long long row = row0 + r;
    const int i = (int)(row / a.ny), j = (int)(row % a.ny);
    const unsigned m = (a.dir.any && active) ? a.dir.mask[d] : 0u;
    const bool line_dir = ((m & 1u) && i == 0) || ((m & 2u) && i == a.nx - 1) || ((m & 4u) && j == 0) ||
                          ((m & 8u) && j == a.ny - 1);
    const bool lo_dir = m & 16u, hi_dir = m & 32u;
    T *line = sm + (size_t)r * g.RS + d;
    LineSolver<T> Ls(a, d);
    const int m0 = a.fac.m0;

    // ---- forward
    const int kref = min(1, nz - 1);  // row of the deviation reference
    const int ref_c = kref / kc;
    for (int c = 0; c <= ref_c; ++c)
        if (!wait_c(c)) return;
    if (active) line[0] = Ls.first(line[0], line[kref * S]);
    int k = 1;
    for (int c = 0; c < nch; ++c) {
        if (c > ref_c && !wait_c(c)) return;
        const int kend = min(nz - 1, (c + 1) * kc);
        if (active) {
            const int hend = min(kend, m0);
            for (; k < hend; ++k) line[k * S] = Ls.template fwd<false>(line[k * S], k);
#pragma unroll 8
            for (; k < kend; ++k) line[k * S] = Ls.template fwd<true>(line[k * S], k);
        }
        k = max(k, kend);
    }
    if (active && nz > 1) Ls.template fwd<false>(line[(nz - 1) * S], nz - 1);

    // ---- backward; each finished row group is stored for all rows of the tile
    if (active) {
        const T y = Ls.out_last();  // also seeds the back substitution
        line[(nz - 1) * S] = (hi_dir || (lo_dir && nz == 1)) ? dir_value(a.dir, i, j, nz - 1, d) : y;
    }
    const int tl = max(m0, 1);
    k = nz - 2;
    for (int c = nch - 1; c >= 0; --c) {
        const int klo = c * kc;
        if (active) {
            const int tstop = max(klo, tl);
#pragma unroll 8
            for (; k >= tstop; --k) line[k * S] = Ls.template bwd<true>(line[k * S], k);
            const int hstop = max(klo, 1);
            for (; k >= hstop; --k) line[k * S] = Ls.template bwd<false>(line[k * S], k);
            if (klo == 0 && nz > 1) {
                const T y = Ls.template bwd<false>(line[0], 0);
                line[0] = lo_dir ? dir_value(a.dir, i, j, 0, d) : y;
            }
            if (line_dir)
                for (int q = klo; q < min(nz, klo + kc); ++q) line[q * S] = dir_value(a.dir, i, j, q, d);
        }
        k = min(k, klo - 1);
        fence_async_smem();
        __syncwarp();
        if (lane == 0) {
            const unsigned b = seg_bytes(c);
            for (int q = 0; q < nr; ++q)
                bulk_store(obase + (size_t)q * L + (size_t)klo * S, smem_u32(sm + (size_t)q * g.RS + (size_t)klo * S), b);
            bulk_commit();
        }
    }
    if (lane == 0) bulk_wait_read_all();
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename T>
int launch_strided_tma(const SweepArgs<T> &a, const StridedGeom &g, const CUtensorMap *map,
                       const CUtensorMap *map_out, int crow, bool fuse_pre, int warps, cudaStream_t s) {
    const size_t wb = strided_tma_warp_bytes(g.n, crow, sizeof(T));
    while (warps > 1 && wb * warps > (size_t)kMaxSmem) --warps;
    if (wb * warps > (size_t)kMaxSmem) return kNotApplicable;  // the caller takes another kernel
    const long long tiles = (long long)g.n_slabs * g.ncb;
    const unsigned blocks = (unsigned)((tiles + warps - 1) / warps);
    const size_t smem = wb * warps;
    if (fuse_pre && a.bulk.on)
        sweep_strided_tma_kernel<T, true, true><<<blocks, warps * 32, smem, s>>>(*map, *map_out, a, g, crow);
    else if (fuse_pre)
        sweep_strided_tma_kernel<T, true, false><<<blocks, warps * 32, smem, s>>>(*map, *map_out, a, g, crow);
    else
        sweep_strided_tma_kernel<T, false, false><<<blocks, warps * 32, smem, s>>>(*map, *map_out, a, g, crow);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

template <typename T>
int launch_contig_tma(const SweepArgs<T> &a, const ContigGeom &g, int warps, cudaStream_t s, int chunks) {
    const size_t wb = (128 + (size_t)g.R * g.RS * sizeof(T) + 127) / 128 * 128;
    while (warps > 1 && wb * warps > (size_t)kMaxSmem) --warps;
    if (wb * warps > (size_t)kMaxSmem) return kNotApplicable;
    const long long tiles = (g.nrows + g.R - 1) / g.R;
    const unsigned blocks = (unsigned)((tiles + warps - 1) / warps);
    const size_t smem = wb * warps;
    if (a.S <= 32) {
        // row groups of kc k-rows whose byte length keeps every copy 16-byte aligned
        const int eb = (int)sizeof(T);
        int q = 16;
        for (int v = a.S * eb; v % 2 == 0 && q > 1; v /= 2) q /= 2;  // q = 16 / gcd(16, S*elem)
        int kc = (g.nz + chunks - 1) / chunks;
        kc = (kc + q - 1) / q * q;
        switch (a.S) {
        case 1: sweep_contig_pipe_kernel<T, 1><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 2: sweep_contig_pipe_kernel<T, 2><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 4: sweep_contig_pipe_kernel<T, 4><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 8: sweep_contig_pipe_kernel<T, 8><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        default: sweep_contig_pipe_kernel<T, 0><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        }
    } else {
        sweep_contig_tma_kernel<T><<<blocks, warps * 32, smem, s>>>(a, g);
    }
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

template int launch_strided_tma<double>(const SweepArgs<double> &, const StridedGeom &, const CUtensorMap *,
                                        const CUtensorMap *, int, bool, int, cudaStream_t);
template int launch_strided_tma<float>(const SweepArgs<float> &, const StridedGeom &, const CUtensorMap *,
                                       const CUtensorMap *, int, bool, int, cudaStream_t);
template int launch_contig_tma<double>(const SweepArgs<double> &, const ContigGeom &, int, cudaStream_t, int);
template int launch_contig_tma<float>(const SweepArgs<float> &, const ContigGeom &, int, cudaStream_t, int);

template <typename K>
static void opt_in_tma(K k) {
    cudaFuncSetAttribute((const void *)k, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
}

void tma_prepare_device() {
    opt_in_tma(sweep_strided_tma_kernel<double, true, true>);
    opt_in_tma(sweep_strided_tma_kernel<double, true, false>);
    opt_in_tma(sweep_strided_tma_kernel<double, false, false>);
    opt_in_tma(sweep_strided_tma_kernel<float, true, true>);
    opt_in_tma(sweep_strided_tma_kernel<float, true, false>);
    opt_in_tma(sweep_strided_tma_kernel<float, false, false>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 1>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 2>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 4>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 8>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 0>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 1>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 2>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 4>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 8>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 0>);
    opt_in_tma(sweep_contig_tma_kernel<double>);
    opt_in_tma(sweep_contig_tma_kernel<float>);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Tensor map of the field for the x (axis 0) or y (axis 1) sweep:
//   x: 2-D {P = ny*nz*S, nx},      box {32, crow}
//   y: 3-D {P = nz*S, ny, nx},     box {32, crow, 1}
// Returns false when the grid does not meet TMA's rules (row pitch a multiple
// of 16 bytes, box rows <= 256); the cp.async kernels handle those grids.
bool make_sweep_tensor_map(CUtensorMap *out, int *crow_out, void *field, int elem, int axis, int nx, int ny, int nz,
                           int S, int chunks) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int n = axis == 0 ? nx : ny;
    const long long P = axis == 0 ? (long long)ny * nz * S : (long long)nz * S;
    if (chunks < 1 || chunks > 16) return false;  // one mbarrier per row group in a 128-byte header
    const int crow = (n + chunks - 1) / chunks;
    if (crow > 256 || (P * elem) % 16 != 0 || (reinterpret_cast<uintptr_t>(field) & 15)) return false;
    if (P > 0xffffffffLL) return false;
    cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)n, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)(P * elem), (cuuint64_t)((long long)ny * P * elem)};
    cuuint32_t box[3] = {32, (cuuint32_t)crow, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t rank = axis == 0 ? 2 : 3;
    const CUresult r = fn(out, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank,
                          field, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    *crow_out = crow;
    return true;
}

}  // namespace bfb
