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

#include <algorithm>

#include "bfb_tma_tiles.cuh"

namespace bfb {

// ---------------------------------------------------------------------------
// Strided sweep with TMA (rank 2: x, rank 3: y).
// ---------------------------------------------------------------------------
// Register bound (here and for the z kernels below): the FP32 kernels compile
// spill-free in 96 registers per thread (107-117 without the bound), so that
// one-warp CTAs of small tiles, whose shared memory allows many per SM, fit 21
// per SM instead of 17. Large grids are bound by shared memory and do not
// change; many small envs stepped side by side do (256 grids of edges 32-160
// stepped one env at a time: 6.70 -> 6.35 ms per step).
template <typename T, bool FUSE_PRE, bool BULK>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 : 1)
    sweep_strided_tma_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap map_out,
                             SweepArgs<T> a, StridedGeom g, int crow) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile >= (long long)g.n_slabs * g.ncb) return;
    unsigned char *wbase = smem_raw + (size_t)warp * strided_tma_warp_bytes(g.n, crow, sizeof(T), g.tw);
    if (lane == 0) {
        const int nch = (g.n + crow - 1) / crow;
        for (int ch = 0; ch < nch; ++ch) mbar_init(smem_u32(wbase) + 8 * ch, 1);
        fence_mbar_init();
    }
    __syncwarp();
    strided_tma_tile<T, FUSE_PRE, BULK>(&map, &map_out, a, g, crow, tile, wbase, 0u);
}

// ---------------------------------------------------------------------------
// Contiguous z sweep with 1-D bulk copies.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 : 1) sweep_contig_tma_kernel(SweepArgs<T> a, ContigGeom g) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    const long long row0 = tile * g.R;
    if (row0 >= g.nrows) return;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = a.S, nz = g.nz;
    const int L = g.Lp;  // row pitch: whole padded rows are copied
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
// constant (1 to 6, 8), 0 otherwise; every lane owns at most one line
// (S <= 32 gives R = 32/S rows per warp).
// ---------------------------------------------------------------------------
template <typename T, int SC>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 5 : 1) sweep_contig_pipe_kernel(SweepArgs<T> a, ContigGeom g, int kc) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // tiles from the last rows to the first: the y sweep before this one ends
    // on the last (i, j) rows, whose lines are then still in L2
    const long long ntiles = (g.nrows + g.R - 1) / g.R;
    const long long slot = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (slot >= ntiles) return;
    const long long tile = ntiles - 1 - slot;
    const size_t wbytes = (128 + (size_t)g.R * g.RS * sizeof(T) + 127) / 128 * 128;
    unsigned char *wbase = smem_raw + (size_t)warp * wbytes;
    if (lane == 0) {
        const int nch = (g.nz + kc - 1) / kc;
        for (int c = 0; c < nch; ++c) mbar_init(smem_u32(wbase) + 8 * c, 1);
        fence_mbar_init();
    }
    __syncwarp();
    contig_pipe_tile<T, SC>(a, g, kc, tile, wbase, 0u);
}

// ---------------------------------------------------------------------------
// Watchdog self-test: one bounded wait on an mbarrier that nothing completes
// (no thread arrives on it and no copy targets it), so nothing is in flight
// when the wait gives up. It sets the error flag exactly as a stalled copy in
// a sweep would.
// ---------------------------------------------------------------------------
__global__ void watchdog_probe_kernel(int polls, int *err) {
    __shared__ __align__(8) unsigned long long bar;
    const unsigned b = smem_u32(&bar);
    if (threadIdx.x == 0) {
        mbar_init(b, 1);
        fence_mbar_init();
    }
    __syncwarp();
    bool done = false;
    for (int i = 0; i < polls && !done; ++i) done = mbar_try_wait(b, 0);
    if (!done && threadIdx.x == 0) atomicOr(err, 1);
}

int launch_watchdog_probe(int polls, int *err, cudaStream_t s) {
    watchdog_probe_kernel<<<1, 32, 0, s>>>(polls, err);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename T>
int launch_strided_tma(const SweepArgs<T> &a, const StridedGeom &g_in, const CUtensorMap *map,
                       const CUtensorMap *map_out, int crow, int lines, bool fuse_pre, int warps, cudaStream_t s) {
    StridedGeom g = g_in;  // warp tiles of the maps' width
    g.tw = lines;
    g.ncb = (int)((g.P + lines - 1) / lines);
    const size_t wb = strided_tma_warp_bytes(g.n, crow, sizeof(T), lines);
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
        case 3: sweep_contig_pipe_kernel<T, 3><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 4: sweep_contig_pipe_kernel<T, 4><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 5: sweep_contig_pipe_kernel<T, 5><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
        case 6: sweep_contig_pipe_kernel<T, 6><<<blocks, warps * 32, smem, s>>>(a, g, kc); break;
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
                                        const CUtensorMap *, int, int, bool, int, cudaStream_t);
template int launch_strided_tma<float>(const SweepArgs<float> &, const StridedGeom &, const CUtensorMap *,
                                       const CUtensorMap *, int, int, bool, int, cudaStream_t);
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
    opt_in_tma(sweep_contig_pipe_kernel<double, 3>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 4>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 5>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 6>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 8>);
    opt_in_tma(sweep_contig_pipe_kernel<double, 0>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 1>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 2>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 3>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 4>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 5>);
    opt_in_tma(sweep_contig_pipe_kernel<float, 6>);
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

// Tensor map of the field for the x (axis 0) or y (axis 1) sweep, with Lp the
// (i, j) rows' pitch in elements (nz*S, or more for a padded field):
//   x: 2-D {P = ny*Lp, nx},        box {lines, crow}
//   y: 3-D {P = Lp, ny, nx},       box {lines, crow, 1}
// Returns false when the grid does not meet TMA's rules (row pitch a multiple
// of 16 bytes, box rows <= 256); the cp.async kernels handle those grids.
bool make_sweep_tensor_map(CUtensorMap *out, int *crow_out, void *field, int elem, int axis, int nx, int ny, int nz,
                           int S, int chunks, int Lp, int lines) {
    (void)nz;
    (void)S;
    const int n = axis == 0 ? nx : ny;
    if (chunks < 1 || chunks > 16) return false;  // one mbarrier per row group in a 128-byte header
    const int crow = strided_box_rows(n, chunks, lines, elem);
    if (!make_sweep_tensor_map_rows(out, field, elem, axis, nx, ny, Lp, lines, crow)) return false;
    *crow_out = crow;
    return true;
}

bool make_sweep_tensor_map_rows(CUtensorMap *out, void *field, int elem, int axis, int nx, int ny, int Lp, int lines,
                                int crow) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    if (lines < 1 || lines > 32 || (lines * elem) % 16 != 0) return false;  // tile x offsets stay 16-byte aligned
    const int n = axis == 0 ? nx : ny;
    const long long P = axis == 0 ? (long long)ny * Lp : (long long)Lp;
    if (crow < 1 || crow > 256 || (P * elem) % 16 != 0 || (reinterpret_cast<uintptr_t>(field) & 15)) return false;
    if (P > 0xffffffffLL) return false;
    cuuint64_t dims[3] = {(cuuint64_t)P, (cuuint64_t)n, (cuuint64_t)nx};
    cuuint64_t strides[2] = {(cuuint64_t)(P * elem), (cuuint64_t)((long long)ny * P * elem)};
    cuuint32_t box[3] = {(cuuint32_t)lines, (cuuint32_t)crow, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t rank = axis == 0 ? 2 : 3;
    const CUresult r = fn(out, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank,
                          field, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Lines per strided TMA warp tile: 32, or for FP64 kNarrowLinesF64 where that
// keeps at least 1/8 more lines resident per SM (by the occupancy calculator:
// shared memory with its per-CTA reservation, registers and the CTA limit all
// count). At 256^3 x 8 FP64 the narrow tile keeps five warps per SM instead
// of three. FP32 tiles stay at 32 lines (narrower ones measured 3-10% slower
// at 128^3 to 256^3). The tile's row stride is a compile-time constant, so
// only these two widths are built.
int strided_tile_lines(int n, int elem, int chunks) {
    if (elem != 8) return 32;
    if (chunks < 1) chunks = 1;
    const void *kernel = (const void *)sweep_strided_tma_kernel<double, false, false>;
    auto resident = [&](int w) -> long long {  // lines per SM at width w (0: does not fit)
        const int crow = strided_box_rows(n, chunks, w, elem);
        const size_t wb = strided_tma_warp_bytes(n, crow, elem, w);
        if (crow > 256 || wb > (size_t)kMaxSmem) return 0;
        int ctas = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, kernel, 32, wb) != cudaSuccess) {
            (void)cudaGetLastError();
            return 0;
        }
        return (long long)ctas * w;
    };
    const long long base = resident(32), narrow = resident(kNarrowLinesF64);
    return narrow > 0 && narrow >= base + base / 8 ? kNarrowLinesF64 : 32;
}

}  // namespace bfb
