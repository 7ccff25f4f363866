// bfb_tma_tiles.cuh -- warp-tile bodies of the TMA sweeps, shared by the
// single-env kernels (bfb_tma.cu) and the batched persistent kernel
// (bfb_batch.cu). See bfb_tma.cu for the data movement and bfb_sweeps.cuh
// for the arithmetic.
#pragma once
#include "bfb_tma.cuh"

namespace bfb {

// The line solve of one strided warp tile (RS <= 32 lines of one slab, one
// lane per line; lanes past RS have no line), shared by the TMA tiles of
// the forward sweeps. Row q of this lane's line is col[q * RS] in shared
// memory. wait(ch) returns once row
// group ch (rows [ch*crow, (ch+1)*crow)) has landed, false when its bounded
// wait ran out; flush(ch) writes row group ch back once its rows are final
// (the back substitution finishes the groups from the last to the first).
// Returns false when a wait ran out.
template <typename T, bool FUSE_PRE, bool BULK, int RS, typename WAIT, typename FLUSH>
__device__ __forceinline__ bool strided_solve(const SweepArgs<T> &a, const StridedGeom &g, int crow, int slab,
                                              long long col0, T *__restrict__ col, WAIT wait, FLUSH flush) {
    constexpr int rs = RS;  // a compile-time row stride keeps the row loops free of address arithmetic
    const int lane = threadIdx.x & 31;
    const int n = g.n;
    const long long P = g.P;
    const int nch = (n + crow - 1) / crow;
    if (lane >= rs) {  // no line: follow the row groups' waits and flushes
        for (int ch = 0; ch < nch; ++ch)
            if (!wait(ch)) return false;
        for (int ch = nch - 1; ch >= 0; --ch) flush(ch);
        return true;
    }

    // ---- line coordinates of this lane (lanes past P and padding columns
    // run along; past P nothing is stored, padding holds no field value)
    const long long cl = col0 + lane;
    const StridedColumn col_at = strided_column(a, g, slab, cl);
    const bool valid = col_at.real;
    const int d = col_at.d, ci = col_at.ci, cj = col_at.cj, ck = col_at.ck;
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
        bA = a.bulk.A + (size_t)slab * g.slab_stride + cl;
        bB = a.bulk.B + (size_t)slab * g.slab_stride + cl;
    }
    auto load = [&](int r) -> T {
        T x = col[r * rs];
        if constexpr (BULK) {
            if (valid) x = bulk_update(x, bA[(size_t)r * P], bB[(size_t)r * P], a.bulk.dt);
        }
        return x;
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
        if (!wait(ch)) return false;
    col[0] = L.first(xin(0), xin(rref));
    int r = 1;
    auto st_col = [&](int q, T v) { col[q * rs] = v; };
    for (int ch = 0; ch < nch; ++ch) {
        if (ch > ref_ch && !wait(ch)) return false;
        const int rend = min(n - 1, (ch + 1) * crow);
        const int hend = min(rend, m0);
        r = head_forward(L, r, hend, load, st_col);
        r = tail_forward(L, r, rend, load, st_col);
    }
    if (n > 1) {
        T x = load(n - 1);
        if (FUSE_PRE && hi_dir) x = vox_dir(n - 1);
        L.template fwd<false>(x, n - 1);
    }

    // ---- back substitution into the tile; each finished row group is flushed
    {
        T y = L.out_last();
        if (hi_dir || (lo_dir && n == 1)) y = vox_dir(n - 1);
        col[(n - 1) * rs] = y;
    }
    const int tl = max(m0, 1);
    auto ld_col = [&](int q) { return col[q * rs]; };
    r = n - 2;
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int rlo = ch * crow;
        const int tstop = max(rlo, tl);
        r = tail_backward(L, r, tstop, ld_col, st_col);
        const int hstop = max(rlo, 1);
        r = head_backward(L, r, hstop, ld_col, st_col);
        if (rlo == 0 && n > 1) {
            T y = L.template bwd<false>(col[0], 0);
            if (lo_dir) y = vox_dir(0);
            col[0] = y;
        }
        if (col_dir)  // the whole column lies on an active face of another axis
            for (int q = rlo; q < min(n, rlo + crow); ++q) col[q * rs] = vox_dir(q);
        flush(ch);
    }
    return true;
}

// One warp tile of a strided sweep with TMA: TW lines of `tile`, in the
// warp's region `wbase` (128-byte header of row-group mbarriers, then the
// tile). The mbarriers are initialised by the caller; row group ch waits for
// parity bit ch of `phase`, and every call completes one phase of each of
// its row groups. Returns false (error flag set) when a bounded wait ran out.
template <typename T, bool FUSE_PRE, bool BULK, int TW>
__device__ __forceinline__ bool strided_tma_tile_w(const CUtensorMap *map, const CUtensorMap *map_out,
                                                   const SweepArgs<T> &a, const StridedGeom &g, int crow,
                                                   long long tile, unsigned char *wbase, unsigned phase) {
    const int lane = threadIdx.x & 31;
    const int slab = (int)(tile / g.ncb);
    const int col0 = (int)((tile % g.ncb) * TW);
    const int nch = (g.n + crow - 1) / crow;
    const int rank = g.axis == 0 ? 2 : 3;
    const unsigned bar0 = smem_u32(wbase);
    T *__restrict__ sm = reinterpret_cast<T *>(wbase + 128);
    const unsigned sm_u32 = smem_u32(sm);
    const unsigned chunk_bytes = (unsigned)crow * (unsigned)TW * (unsigned)sizeof(T);

    if (lane == 0) {
        for (int ch = 0; ch < nch; ++ch) {
            mbar_expect_tx(bar0 + 8 * ch, chunk_bytes);
            tma_load(sm_u32 + ch * chunk_bytes, map, col0, ch * crow, slab, rank, bar0 + 8 * ch);
        }
    }
    auto wait = [&](int ch) -> bool {
        if (mbar_wait(bar0 + 8 * ch, (phase >> ch) & 1u)) return true;
        if (lane == 0) atomicOr(a.err, 1);
        return false;
    };
    auto flush = [&](int ch) {
        fence_async_smem();
        __syncwarp();
        if (lane == 0) {
            tma_store(map_out, col0, ch * crow, slab, rank, sm_u32 + ch * chunk_bytes);
            bulk_commit();
        }
    };
    if (!strided_solve<T, FUSE_PRE, BULK, TW>(a, g, crow, slab, col0, sm + lane, wait, flush)) return false;
    if (lane == 0) bulk_wait_read_all();  // the tile must outlive the stores' reads
    __syncwarp();
    return true;
}

// The tile at the geometry's width: 32 lines, or kNarrowLinesF64 for FP64.
template <typename T, bool FUSE_PRE, bool BULK>
__device__ __forceinline__ bool strided_tma_tile(const CUtensorMap *map, const CUtensorMap *map_out,
                                                 const SweepArgs<T> &a, const StridedGeom &g, int crow, long long tile,
                                                 unsigned char *wbase, unsigned phase) {
    if constexpr (sizeof(T) == 8) {
        if (g.tw == kNarrowLinesF64)
            return strided_tma_tile_w<T, FUSE_PRE, BULK, kNarrowLinesF64>(map, map_out, a, g, crow, tile, wbase,
                                                                         phase);
    }
    return strided_tma_tile_w<T, FUSE_PRE, BULK, 32>(map, map_out, a, g, crow, tile, wbase, phase);
}

// One warp tile of the pipelined z sweep (rows row0 .. row0 + R - 1 of
// `tile`) in the warp's region `wbase`; mbarriers and `phase` as for
// strided_tma_tile. Returns false (error flag set) when a bounded wait ran out.
template <typename T, int SC>
__device__ __forceinline__ bool contig_pipe_tile(const SweepArgs<T> &a, const ContigGeom &g, int kc, long long tile,
                                                 unsigned char *wbase, unsigned phase) {
    const int lane = threadIdx.x & 31;
    const long long row0 = tile * g.R;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = SC > 0 ? SC : a.S;
    const int nz = g.nz;
    const int L = g.Lp;  // row pitch; the last row group copies a padded row's padding along
    const int nch = (nz + kc - 1) / kc;
    const unsigned bar0 = smem_u32(wbase);
    T *__restrict__ sm = reinterpret_cast<T *>(wbase + 128);
    T *__restrict__ base = a.f + (size_t)row0 * L;
    T *__restrict__ obase = a.fo + (size_t)row0 * L;
    auto seg_bytes = [&](int c) -> unsigned {
        const int end = c == nch - 1 ? L : (c + 1) * kc * S;
        return (unsigned)((end - c * kc * S) * (int)sizeof(T));
    };

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
        if (mbar_wait(bar0 + 8 * c, (phase >> c) & 1u)) return true;
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
        if (!wait_c(c)) return false;
    if (active) line[0] = Ls.first(line[0], line[kref * S]);
    int k = 1;
    for (int c = 0; c < nch; ++c) {
        if (c > ref_c && !wait_c(c)) return false;
        const int kend = min(nz - 1, (c + 1) * kc);
        if (active) {
            const int hend = min(kend, m0);
            k = head_forward(Ls, k, hend, [&](int q) { return line[q * S]; }, [&](int q, T v) { line[q * S] = v; });
            k = tail_forward(Ls, k, kend, [&](int q) { return line[q * S]; }, [&](int q, T v) { line[q * S] = v; });
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
            k = tail_backward(Ls, k, tstop, [&](int q) { return line[q * S]; }, [&](int q, T v) { line[q * S] = v; });
            const int hstop = max(klo, 1);
            k = head_backward(Ls, k, hstop, [&](int q) { return line[q * S]; }, [&](int q, T v) { line[q * S] = v; });
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
    return true;
}


}  // namespace bfb
