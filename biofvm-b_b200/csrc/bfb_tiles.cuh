// bfb_tiles.cuh -- one warp's tile of a strided (x, y) or contiguous (z)
// sweep, staged with cp.async. The single-env kernels (bfb_sweeps.cu) and the
// batched ensemble kernel (bfb_batch.cu) both run these.
#pragma once
#include "bfb_line.cuh"

namespace bfb {

// One strided tile (32 lines of one slab) by the calling warp; sm is the
// warp's shared-memory region of n*32 elements. Used by the single-env kernel
// below and by the batched ensemble kernel (bfb_batch.cu).
template <typename T, int VB, bool FUSE_PRE, bool BULK>
__device__ __forceinline__ void strided_tile(const SweepArgs<T> &a, const StridedGeom &g, long long tile, T *sm) {
    const int lane = threadIdx.x & 31;
    const int slab = (int)(tile / g.ncb);
    const long long col0 = (tile % g.ncb) * 32;
    const int ncols = (int)min((long long)32, g.P - col0);
    const int n = g.n;
    const long long P = g.P;
    T *__restrict__ base = a.f + (size_t)slab * g.slab_stride + col0;   // input
    T *__restrict__ obase = a.fo + (size_t)slab * g.slab_stride + col0; // output (== base in place)

    // ---- stage the tile: kChunks commit groups of rows
    const int crow = (n + kChunks - 1) / kChunks;
    const int nch = (n + crow - 1) / crow;  // non-empty groups
    constexpr int EPV = VB / (int)sizeof(T);  // elements per copy
    const bool vec = (VB > (int)sizeof(T)) && ncols == 32;
#pragma unroll 1
    for (int ch = 0; ch < kChunks; ++ch) {
        const int r0 = min(n, ch * crow), r1 = min(n, r0 + crow);
        if (vec) {
            constexpr int VPR = 32 / EPV;  // copies per row
            const int total = (r1 - r0) * VPR;
            for (int v = lane; v < total; v += 32) {
                const int r = r0 + v / VPR, q = (v % VPR) * EPV;
                cp_async<VB>(sm + r * 32 + q, base + (size_t)r * P + q);
            }
        } else if (lane < ncols) {
            // one element per lane and row: 32-bit shared addresses and a
            // global pointer stepped by the row pitch
            const T *gp = base + (size_t)r0 * P + lane;
            unsigned sp = (unsigned)__cvta_generic_to_shared(sm + r0 * 32 + lane);
#pragma unroll 4
            for (int r = r0; r < r1; ++r, gp += P, sp += 32 * (unsigned)sizeof(T)) cp_async_s<sizeof(T)>(sp, gp);
        }
        cp_commit();
    }
    // Group ch has landed for the whole warp after wait(ch). Every lane takes
    // the same nch waits: one lane's 16-byte copies fill rows other lanes read.
    auto wait = [&](int ch) {
        cp_wait_dyn(kChunks - 1 - ch);
        __syncwarp();
    };
    const bool valid = lane < ncols;
    if (!valid) {
        for (int ch = 0; ch < nch; ++ch) wait(ch);
        return;
    }

    // ---- line coordinates of this lane (padding columns of a padded row run
    // along with no Dirichlet value and no bulk term)
    const long long col = col0 + lane;
    const StridedColumn col_at = strided_column(a, g, slab, col);
    const int d = col_at.d, ci = col_at.ci, cj = col_at.cj, ck = col_at.ck;
    const unsigned m = (a.dir.any && col_at.real) ? a.dir.mask[d] : 0u;
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
            if (col_at.real) x = bulk_update(x, bA[(size_t)r * P], bB[(size_t)r * P], a.bulk.dt);
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

    // ---- forward elimination in shared memory, group by group as copies land
    const int rref = min(1, n - 1);  // row of the deviation reference
    const int ref_ch = rref / crow;
    for (int ch = 0; ch <= ref_ch; ++ch) wait(ch);
    sm[lane] = L.first(xin(0), xin(rref));
    int r = 1;
    auto st_sm = [&](int q, T v) { sm[q * 32 + lane] = v; };
    for (int ch = 0; ch < nch; ++ch) {
        if (ch > ref_ch) wait(ch);
        const int rend = min(n - 1, (ch + 1) * crow);
        const int hend = min(rend, m0);
        r = head_forward(L, r, hend, load, st_sm);
        r = tail_forward(L, r, rend, load, st_sm);
    }
    if (n > 1) {
        T x = load(n - 1);
        if (FUSE_PRE && hi_dir) x = vox_dir(n - 1);
        L.template fwd<false>(x, n - 1);
    }

    // ---- back substitution straight to global memory
    T *gp = obase + lane + (size_t)(n - 1) * P;
    {
        T y = L.out_last();
        if (hi_dir || (lo_dir && n == 1)) y = vox_dir(n - 1);
        *gp = y;
    }
    const int tl = max(m0, 1);
    T *__restrict__ go = obase + lane;
    auto ld_sm = [&](int q) { return sm[q * 32 + lane]; };
    // tail_backward and head_backward store rows n-2, n-3, ..., 1 in this
    // order: a pointer stepped down by the pitch replaces a 64-bit index
    // product per row
    T *gw = go + (size_t)max(n - 2, 0) * P;
    auto st_g = [&](int, T v) {
        *gw = v;
        gw -= P;
    };
    r = tail_backward(L, n - 2, tl, ld_sm, st_g);
    r = head_backward(L, r, 1, ld_sm, st_g);
    if (n > 1) {
        T y = L.template bwd<false>(sm[lane], 0);
        if (lo_dir) y = vox_dir(0);
        go[0] = y;
    }
    if (col_dir)  // the whole column is on an active face of another axis
        for (int q = 0; q < n; ++q) obase[lane + (size_t)q * P] = vox_dir(q);
}

// One contiguous tile (R rows) by the calling warp, any S (lanes loop over
// the tile's lines); sm is the warp's region of R*RS elements. The S > 32
// kernel runs it, and contig_tile_any for S > 32.
template <typename T, int VB>
__device__ __forceinline__ void contig_tile_wide(const SweepArgs<T> &a, const ContigGeom &g, long long tile, T *sm) {
    const int lane = threadIdx.x & 31;
    const long long row0 = tile * g.R;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = a.S, nz = g.nz;
    const int L = g.Lp;  // row pitch: a padded row's padding is copied along
    T *__restrict__ base = a.f + (size_t)row0 * L;
    T *__restrict__ obase = a.fo + (size_t)row0 * L;
    constexpr int EPV = VB / (int)sizeof(T);

    // ---- stage nr rows (one contiguous block of global memory) into padded rows
    {
        const int vpr = L / EPV;
        const int total = nr * vpr;
        for (int v = lane; v < total; v += 32) {
            const int r = v / vpr, q = (v - r * vpr) * EPV;
            cp_async<VB>(sm + (size_t)r * g.RS + q, base + (size_t)r * L + q);
        }
        cp_commit();
        cp_wait<0>();
        __syncwarp();
    }

    // ---- lane (r, d) solves line (row0 + r, d) in place
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
            const T y = Ls.out_last();  // also seeds the back substitution
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
    __syncwarp();

    // ---- copy the rows back out
    {
        const int vpr = L / EPV;
        const int total = nr * vpr;
        for (int v = lane; v < total; v += 32) {
            const int r = v / vpr, q = (v - r * vpr) * EPV;
            const T *src = sm + (size_t)r * g.RS + q;
            T *dst = obase + (size_t)r * L + q;
            if constexpr (VB == 16) {
                *reinterpret_cast<int4 *>(dst) = *reinterpret_cast<const int4 *>(src);
            } else if constexpr (VB == 8) {
                *reinterpret_cast<int2 *>(dst) = *reinterpret_cast<const int2 *>(src);
            } else {
                *dst = *src;
            }
        }
    }
}

// One contiguous tile (R = 32/S rows) by the calling warp for S <= 32; sm is
// the warp's region of R*RS elements. Used by the single-env cp.async kernel
// (bfb_sweeps.cu) and, through contig_tile_any, by bfb_batch.cu. Each row's k range is cut into two
// row groups, each one cp.async commit group of VB-byte copies (every row
// group starts VB-aligned), so the forward elimination starts on group 0
// while group 1 lands; the back substitution finishes group 1 first and the
// warp writes it out while it computes group 0. Lane (r, d) solves line
// (row0 + r, d) with the blocked row loops of bfb_line.cuh.
template <typename T, int VB, int SC = 0>
__device__ __forceinline__ void contig_tile(const SweepArgs<T> &a, const ContigGeom &g, long long tile, T *sm) {
    const int S = SC > 0 ? SC : a.S;  // SC: the substrate count when it is a compile-time constant
    const int lane = threadIdx.x & 31;
    const long long row0 = tile * g.R;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int nz = g.nz;
    const int L = g.Lp;  // row pitch: the last row group copies a padded row's padding along
    const int RS = g.RS;
    T *__restrict__ base = a.f + (size_t)row0 * L;
    T *__restrict__ obase = a.fo + (size_t)row0 * L;
    constexpr int EPV = VB / (int)sizeof(T);
    // k rows per group: a multiple of EPV / gcd(EPV, S), so that k0*S is a multiple of EPV
    int qa = EPV;
    for (int v = S; v % 2 == 0 && qa > 1; v /= 2) qa /= 2;
    int kc = (nz + 1) / 2;
    kc = (kc + qa - 1) / qa * qa;
    const int nch = (nz + kc - 1) / kc;  // 1 or 2
    auto span_of = [&](int c) { return (c == nch - 1 ? L : (c + 1) * kc * S) - c * kc * S; };

    for (int c = 0; c < nch; ++c) {
        const int k0 = c * kc, span = span_of(c), vspan = span / EPV;
        for (int r = 0; r < nr; ++r) {
            const T *src = base + (size_t)r * L + (size_t)k0 * S + lane * EPV;
            unsigned dst = (unsigned)__cvta_generic_to_shared(sm + (size_t)r * RS + (size_t)k0 * S + lane * EPV);
#pragma unroll 4
            for (int v = lane; v < vspan; v += 32, src += 32 * EPV, dst += 32 * VB) cp_async_s<VB>(dst, src);
        }
        cp_commit();
    }
    auto wait_c = [&](int c) {
        cp_wait_dyn(nch - 1 - c);
        __syncwarp();
    };
    auto store_c = [&](int c) {  // row group c of every row, shared -> global
        const int k0 = c * kc, span = span_of(c), vspan = span / EPV;
        for (int r = 0; r < nr; ++r) {
            const T *src = sm + (size_t)r * RS + (size_t)k0 * S;
            T *dst = obase + (size_t)r * L + (size_t)k0 * S;
            for (int v = lane; v < vspan; v += 32) {
                if constexpr (VB == 16) {
                    *reinterpret_cast<int4 *>(dst + v * EPV) = *reinterpret_cast<const int4 *>(src + v * EPV);
                } else if constexpr (VB == 8) {
                    *reinterpret_cast<int2 *>(dst + v * EPV) = *reinterpret_cast<const int2 *>(src + v * EPV);
                } else {
                    dst[v] = src[v];
                }
            }
        }
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
    T *line = sm + (size_t)r * RS + d;
    LineSolver<T> Ls(a, d);
    const int m0 = a.fac.m0;
    auto ld = [&](int q) { return line[q * S]; };
    auto st = [&](int q, T v) { line[q * S] = v; };

    // ---- forward
    const int kref = min(1, nz - 1);  // row of the deviation reference
    const int ref_c = kref / kc;
    for (int c = 0; c <= ref_c; ++c) wait_c(c);
    if (active) line[0] = Ls.first(line[0], line[kref * S]);
    int k = 1;
    for (int c = 0; c < nch; ++c) {
        if (c > ref_c) wait_c(c);
        const int kend = min(nz - 1, (c + 1) * kc);
        if (active) {
            k = head_forward(Ls, k, min(kend, m0), ld, st);
            k = tail_forward(Ls, k, kend, ld, st);
        }
        k = max(k, kend);
    }
    if (active && nz > 1) Ls.template fwd<false>(line[(nz - 1) * S], nz - 1);

    // ---- backward; each finished row group is written out for all rows
    if (active) {
        const T y = Ls.out_last();  // also seeds the back substitution
        line[(nz - 1) * S] = (hi_dir || (lo_dir && nz == 1)) ? dir_value(a.dir, i, j, nz - 1, d) : y;
    }
    const int tl = max(m0, 1);
    k = nz - 2;
    for (int c = nch - 1; c >= 0; --c) {
        const int klo = c * kc;
        if (active) {
            k = tail_backward(Ls, k, max(klo, tl), ld, st);
            k = head_backward(Ls, k, max(klo, 1), ld, st);
            if (klo == 0 && nz > 1) {
                const T y = Ls.template bwd<false>(line[0], 0);
                line[0] = lo_dir ? dir_value(a.dir, i, j, 0, d) : y;
            }
            if (line_dir)
                for (int q = klo; q < min(nz, klo + kc); ++q) line[q * S] = dir_value(a.dir, i, j, q, d);
        }
        k = min(k, klo - 1);
        __syncwarp();
        store_c(c);
    }
}

// contig_tile for S <= 32 (with the substrate count as a constant where it
// is a common one), contig_tile_wide otherwise.
template <typename T, int VB>
__device__ __forceinline__ void contig_tile_any(const SweepArgs<T> &a, const ContigGeom &g, long long tile, T *sm) {
    switch (a.S) {
    case 1: contig_tile<T, VB, 1>(a, g, tile, sm); break;
    case 2: contig_tile<T, VB, 2>(a, g, tile, sm); break;
    case 3: contig_tile<T, VB, 3>(a, g, tile, sm); break;
    case 4: contig_tile<T, VB, 4>(a, g, tile, sm); break;
    case 5: contig_tile<T, VB, 5>(a, g, tile, sm); break;
    case 6: contig_tile<T, VB, 6>(a, g, tile, sm); break;
    case 8: contig_tile<T, VB, 8>(a, g, tile, sm); break;
    default:
        if (a.S > 32) contig_tile_wide<T, VB>(a, g, tile, sm);
        else contig_tile<T, VB>(a, g, tile, sm);
    }
}

}  // namespace bfb
