// bfb_sweeps.cuh -- LOD Thomas sweeps for sm_100a.
//
// One LOD step of the reference (BioFVM_parallel.cpp:693-1395) is
//     Dir, X-sweep, Dir, Y-sweep, Dir, Z-sweep, Dir
// where every sweep solves, for each grid line and substrate, the symmetric
// tridiagonal system A y = u, A = tridiag(-c1, diag, -c1), with precomputed
// Thomas factors (forward: y0 = u0/den0, ym = (um + c1*y(m-1))/den_m; back:
// ym -= c_m * y(m+1)), and Dir overwrites the active outer faces.
//
// Field layout rho[((i*ny + j)*nz + k)*S + d]: z (with d) is contiguous, x is
// the slowest axis. So:
//   * x- and y-sweeps are STRIDED: a line's elements are P = ny*nz*S (x) or
//     nz*S (y) elements apart, and P consecutive lines form a contiguous row.
//     A warp owns 32 adjacent lines ("columns"); its n x 32 tile is staged
//     into shared memory with cp.async (16-byte copies when aligned), one lane
//     per line runs the recurrence in shared memory, and the back substitution
//     stores straight to global memory, 128 B (FP32) / 256 B (FP64) per warp
//     store. One read and one write of the field per sweep.
//   * the z-sweep is CONTIGUOUS: a line lives inside one (i,j) row of nz*S
//     contiguous elements. A warp stages R = 32/S whole rows (one contiguous
//     block of global memory) into padded shared rows, lane (r, d) solves line
//     (row r, substrate d) in place, and the warp copies the rows back out.
// Dirichlet is fused: the pre-X Dir (and, if enabled, the bulk source/sink
// update that precedes the step) on the X-sweep load, and each post-sweep Dir
// on that sweep's store. Because Dir is a pure overwrite of fixed positions
// and each sweep rewrites every element of its line, this is exactly the
// reference's sequence. The recurrence keeps the un-overwritten values.
//
// Factor tails: den_m and c_m converge to a floating-point fixed point after a
// few rows (den_m = c3 - c1^2/den_(m-1) contracts by (c1/den)^2 < 1/4), so
// every table is bitwise constant on rows [m0, n-2]. The host finds m0 per axis
// and the kernels keep those values in registers; only rows < m0 and row n-1
// read the tables. This is exact, not an approximation.
//
// Arithmetic:
//   FP64 -- the reference's operations in its order, bit for bit: the fused
//     u += c1*u_prev and u -= c*u_next of its -ffp-contract=fast build and a
//     correctly rounded division by den_m (reciprocal + one residual
//     correction, see div_rcp in bfb_sweeps.cu).
//   FP32 -- FP32 storage and FP32 arithmetic, in "deviation" form. With
//     xb = u_1 of the line (u_0 when n == 1; row 0 of a Dirichlet line holds
//     the boundary value) and g = 1/(1 + c2), A*1 = (1 + c2)*1 exactly (every
//     row of A sums to 1 + c2), so  A^{-1} u = g*xb + A^{-1}(u - xb).
//     The recurrence runs on u - xb with the reciprocal form
//     z_m = (u_m - xb)*r_m + a_m*z_(m-1)  (r = 1/den, a = c1/den), r and g
//     carried as hi+lo FP32 pairs. Rounding of the coefficients then acts only
//     on the deviation, which smooths out as the field diffuses, instead of on
//     the whole field, which makes plain FP32 Thomas drift ~1e-4 in 1000 steps.
#pragma once
#include "bfb_internal.cuh"

namespace bfb {

constexpr int kChunks = 4;  // default row groups per tile (async copy / TMA stages)

// Per-axis factor tables on the device (see bfb_capi.cu: upload_factors).
//   FP64: t0 = den, t1 = c (back-substitution coefficient), t2 = RN(1/den)
//   FP32: t0 = 1/den (hi), t1 = 1/den (lo), t2 = c1/den, t3 = c
// tail[q*S + d] = value of table q on rows [m0, n-2] (valid when m0 <= n-2).
// head[(q*S + d)*hpad + m] = table q, substrate d, row m < hpad: the rows
// below m0 again, one substrate's rows contiguous (hpad a multiple of 4), so
// that a lane reads four rows of a table with one 16-byte load.
template <typename T>
struct Factors {
    const T *t0, *t1, *t2, *t3;
    const T *tail;
    const T *head;
    int m0, hpad;
};

template <typename T>
struct SweepArgs {
    T *f;          // input field
    T *fo;         // output field (== f for the in-place sweeps of a step)
    int nx, ny, nz, S;
    int Lp;        // elements between consecutive (i, j) rows: nz*S, or nz*S rounded up to whole
                   // 16-byte vectors when the field is padded (bfb_env_s::Lp); rho(i,j,k,d) is at
                   // (i*ny + j)*Lp + k*S + d
    Factors<T> fac;
    const T *c1;   // FP64: [S] c1 = dt*D/dx^2
    const T *g;    // FP32: [2*S] g = 1/(1 + c2) as hi, lo
    DirFaces<T> dir;
    BulkTerms<T> bulk;
    int *err;      // device error flag: bounded waits that run out set bit 0
};

struct StridedGeom {
    int n;                 // line length
    long long P;           // lines per slab == element stride between line elements (x: ny*Lp,
                           // y: Lp; the columns q >= nz*S of a padded row are padding, not lines)
    long long slab_stride; // elements between slabs
    int n_slabs;
    int ncb;               // column blocks (warp tiles) per slab
    int axis;              // 0 = x, 1 = y
    int tw = 32;           // lines per warp tile: 32, or fewer for the TMA tiles (strided_tile_lines)
};

struct ContigGeom {
    int nz;
    long long nrows;       // nx * ny rows of nz*S elements
    int Lp;                // elements between consecutive rows (SweepArgs::Lp)
    int R;                 // rows per warp tile
    int RS;                // shared-memory row stride (elements), RS = S (mod 32)
};

// The voxel and substrate of strided column `cl` of slab `slab` (x: cl =
// j*Lp + q, y: cl = q, with q = k*S + d); `real` is false for columns past P
// and for the padding of a padded row (q >= nz*S), whose lanes run along but
// read no Dirichlet value or bulk term.
struct StridedColumn {
    int d, ci, cj, ck;
    bool real;
};
template <typename T>
__device__ __forceinline__ StridedColumn strided_column(const SweepArgs<T> &a, const StridedGeom &g, int slab,
                                                        long long cl) {
    StridedColumn c;
    long long q;
    if (g.axis == 0) {
        c.cj = (int)(cl / a.Lp);
        q = cl - (long long)c.cj * a.Lp;
        c.ci = 0;
    } else {
        q = cl;
        c.ci = slab;
        c.cj = 0;
    }
    c.real = cl < g.P && q < (long long)a.nz * a.S;
    c.ck = (int)(q / a.S);
    c.d = (int)(q - (long long)c.ck * a.S);
    return c;
}

// launchers (bfb_sweeps.cu). `map` (may be NULL) is the field's tensor map
// for this axis; with it the TMA kernels run, otherwise cp.async ones.
template <typename T>
int launch_strided(const SweepArgs<T> &a, int axis, bool fuse_pre, int warps, const CUtensorMap *map,
                   const CUtensorMap *map_out, int crow, int lines, cudaStream_t s);
template <typename T>
int launch_contig(const SweepArgs<T> &a, int warps, bool use_tma, cudaStream_t s, int chunks = kChunks);

// TMA kernels (bfb_tma.cu); they return kNotApplicable when the tile does
// not fit in shared memory, and the caller then takes another kernel.
constexpr int kNotApplicable = 1;
template <typename T>
int launch_strided_tma(const SweepArgs<T> &a, const StridedGeom &g, const CUtensorMap *map,
                       const CUtensorMap *map_out, int crow, int lines, bool fuse_pre, int warps, cudaStream_t s);
template <typename T>
int launch_contig_tma(const SweepArgs<T> &a, const ContigGeom &g, int warps, cudaStream_t s, int chunks);
// `chunks` row groups per tile: box rows = ceil(n / chunks) (<= 256); Lp the
// (i, j) rows' pitch in elements; `lines` the box's columns (the lines of one
// warp tile, <= 32, a whole number of 16-byte vectors).
bool make_sweep_tensor_map(CUtensorMap *out, int *crow_out, void *field, int elem, int axis, int nx, int ny, int nz,
                           int S, int chunks, int Lp, int lines);
// The same with the box's rows given (crow <= 256).
bool make_sweep_tensor_map_rows(CUtensorMap *out, void *field, int elem, int axis, int nx, int ny, int Lp, int lines,
                                int crow);
// Lines per strided TMA warp tile for lines of n rows in `chunks` row groups:
// the width that keeps the most lines resident per SM (a line's rows all sit
// in shared memory, so FP64 tiles of 32 long lines leave few warps per SM and
// a narrower tile fits more of them); 32 on ties.
int strided_tile_lines(int n, int elem, int chunks);
// FP64 x/y sweeps with each line's forward results in tensor memory
// (bfb_tmem.cu): lines of 16 to 256 rows, 32-line tiles, tensor maps of
// 16-row boxes. launch_strided_tmem returns kNotApplicable for other lines.
bool tmem_sweep_fits(int n);
bool make_tmem_sweep_map(CUtensorMap *out, void *field, int axis, int nx, int ny, int Lp);
int launch_strided_tmem(const SweepArgs<double> &a, const StridedGeom &g, const CUtensorMap *map,
                        const CUtensorMap *map_out, bool fuse_pre, cudaStream_t s);
void tmem_prepare_device();
// The x sweep of an x-slab of a larger grid in two halves (bfb_slab.cu, FP64):
// the forward half over lines [line0, line1) of the slab's ny*Lp columns,
// starting from prev_in[line] (the previous slab's last forward value; NULL
// for the grid's first slab) and giving its own last one in prev_out (may be
// NULL); the backward half starting from next_in[line] (the next slab's first
// back-substituted value; NULL for the grid's last slab) and giving its own
// in next_out (may be NULL). a.nx is the slab's plane count and the factor
// tables are the whole line's; x0 is the slab's first plane of nglob.
int launch_slab_x_forward(const SweepArgs<double> &a, int x0, int nglob, long long line0, long long line1,
                          const double *prev_in, double *prev_out, cudaStream_t s);
int launch_slab_x_backward(const SweepArgs<double> &a, int x0, int nglob, long long line0, long long line1,
                           const double *next_in, double *next_out, cudaStream_t s);
// The strided geometry of a sweep over args a (axis 0: x, 1: y), 32-line tiles.
template <typename T>
inline StridedGeom strided_geometry(const SweepArgs<T> &a, int axis) {
    StridedGeom g;
    g.axis = axis;
    if (axis == 0) {
        g.n = a.nx;
        g.P = (long long)a.ny * a.Lp;
        g.slab_stride = 0;
        g.n_slabs = 1;
    } else {
        g.n = a.ny;
        g.P = a.Lp;
        g.slab_stride = (long long)a.ny * a.Lp;
        g.n_slabs = a.nx;
    }
    g.ncb = (int)((g.P + 31) / 32);
    return g;
}
void tma_prepare_device();
// One bounded mbarrier wait that nothing completes, `polls` polls long; sets
// *err like a stalled copy would (bfb_watchdog_selftest).
int launch_watchdog_probe(int polls, int *err, cudaStream_t s);
template <typename T>
int launch_dirichlet(const SweepArgs<T> &a, cudaStream_t s);
template <typename T>
int launch_bulk(const SweepArgs<T> &a, long long N, cudaStream_t s);

// shared-memory bytes a strided / contiguous CTA needs (0 if it does not fit);
// Lp is the z rows' pitch in elements (a shared row holds a whole padded row)
size_t strided_smem(int n, int elem, int warps);
size_t contig_smem(int nz, int S, int Lp, int elem, int warps, int *R, int *RS);
// Rows per warp tile R and shared row stride RS for the bulk-copy z tile where
// contig_smem's conflict-free stride (RS = S mod 32) is not a multiple of 16
// bytes (S not a multiple of 4 in FP32, odd S in FP64): RS >= nz*S a multiple
// of 16 bytes, chosen among its residues so that the most rows keep the warp's
// accesses free of bank conflicts (lane (r, d) reads element r*RS + k*S + d),
// or with two-way conflicts where conflict-free strides keep fewer than 16
// lanes busy (FP32 S = 1); false when even that leaves fewer than 16.
bool contig_aligned_geom(int nz, int S, int Lp, int elem, int *R, int *RS);

// Opt the shared-memory kernels into 227 KB, once per device.
void sweeps_prepare_device();

}  // namespace bfb
