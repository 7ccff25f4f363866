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
// c1 = dt D/dx^2 and c2 = dt lambda/3 (A = (1 + c2) I + c1 Lap). The oracle
// holds the same derivation (oracle/lod_oracle.c: orc_lod_step_adjoint).
//
// Kernels. One adjoint sweep is two launches:
//   * the solve mu_a = A_a^-1 (1 - M) lam: the forward sweep's kernels with
//     the mask on the load (x / y: TMA tiles of 32 lines in row groups on
//     per-group mbarriers, z: 1-D bulk copies of whole rows), one read and
//     one write of the field;
//   * the sums mu.Lap y and mu.y over the new mu and the forward sweep's
//     stored output s_(a+1) = Dir(y_a): one thread per line, two reads.
// Staging y beside the adjoint in the solve's shared memory instead halves
// the lines in flight per SM and left that kernel latency-bound at ~12% of
// HBM bandwidth (one warp per SM sub-partition); the split costs one extra
// read of mu and keeps both launches bandwidth-bound. Grids the TMA path
// cannot describe use cp.async kernels that do both steps in one launch.
// y_a differs from the stored s_(a+1) only on active faces. On lines that lie
// inside a face of another axis the masked adjoint is zero, so mu is zero and
// y does not matter; at the two ends of a line on the sweep's own faces, y is
// rebuilt from the end row of A y = s, whose right side is the face value:
//   y_0 = (g_0 + c1 y_1) / (1 + c1 + c2)  (and the mirror at n-1; a 2x2 solve
//   when n = 2 and both ends are faces; g/(1 + c2) when n = 1).
// dL/du = (1 - M) mu_x is not formed: its two readers mask on their own
// loads (the agents' adjoint of the step before, and the z solve), and
// adjoint_mask_kernel masks the returned dL/d(initial field).
// Per-substrate sums: each warp reduces its lanes per substrate and adds the
// result to its own slot of a partial buffer, across all steps; one kernel at
// the end adds the slots in a fixed order. Gradients are run-to-run identical.
//
// Checkpointing: the forward pass keeps the field at the start of every
// K-step segment except the last, whose stage fields it writes directly. The
// reverse pass walks the segments backwards; each earlier segment is
// recomputed from its checkpoint with out-of-place sweeps that keep, per step,
// s1, s2 and the step's output (and the pre-agent values at occupied voxels).
#include <algorithm>
#include <vector>

#include "bfb_aux.cuh"
#include "bfb_tiles.cuh"
#include "bfb_tma.cuh"

namespace bfb {

// Terms of the adjoint sweeps besides the forward's SweepArgs.
struct AdjTerms {
    const double *c1;  // [S] dt*D/dx^2
    const double *c2;  // [S] dt*lambda/3
    double *part;      // [tiles of this sweep][S][2] running sums (mu.Lap y, mu.y)
};

__device__ __forceinline__ double shfl_xor_d(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }

// Adds this warp's per-substrate sums of (dl, dy) to slot[d][2]. Lanes
// without a line pass dl = dy = 0. `d` is the lane's substrate.
__device__ __forceinline__ void tile_partials(double dl, double dy, int d, int S, double *__restrict__ slot) {
    const int lane = threadIdx.x & 31;
    if (32 % S == 0) {  // lanes of one substrate are lane = d (mod S)
        for (int o = 16; o >= S; o >>= 1) {
            dl += shfl_xor_d(dl, o);
            dy += shfl_xor_d(dy, o);
        }
        if (lane < S) {
            slot[2 * lane] += dl;
            slot[2 * lane + 1] += dy;
        }
    } else {
        for (int q = 0; q < S; ++q) {
            double u = d == q ? dl : 0.0, w = d == q ? dy : 0.0;
            for (int o = 16; o > 0; o >>= 1) {
                u += shfl_xor_d(u, o);
                w += shfl_xor_d(w, o);
            }
            if (lane == 0) {
                slot[2 * q] += u;
                slot[2 * q + 1] += w;
            }
        }
    }
}

// The forward sweep's y at a line's two ends when they lie on the sweep's own
// active faces (see the file comment); FP64.
struct EndFix {
    bool lo = false, hi = false;
    double y0 = 0.0, yn = 0.0;
    __device__ __forceinline__ void make(bool lo_dir, bool hi_dir, int n, double c1, double c2, double g0, double gn,
                                         double y1_stored, double yn2_stored) {
        lo = lo_dir;
        hi = hi_dir;
        if (!lo && !hi) return;
        const double a1 = 1.0 + c1 + c2;
        if (n == 1) {
            y0 = yn = g0 / (1.0 + c2);
        } else if (n == 2 && lo && hi) {
            const double det = a1 * a1 - c1 * c1;
            y0 = (a1 * g0 + c1 * gn) / det;
            yn = (c1 * g0 + a1 * gn) / det;
        } else {
            // with n == 2 and one face end, the other end's stored value is y itself
            if (lo) y0 = (g0 + c1 * y1_stored) / a1;
            if (hi) yn = (gn + c1 * yn2_stored) / a1;
        }
    }
};

// mu.Lap y and mu.y at row m of a line; yv(q) returns y at row q (FP64).
template <typename YV>
__device__ __forceinline__ void dots_at(int m, int n, double mu, YV yv, double &dl, double &dy) {
    const double yc = yv(m);
    double lap = 0.0;
    if (n > 1) {
        if (m == 0)
            lap = yc - yv(1);
        else if (m == n - 1)
            lap = yc - yv(n - 2);
        else
            lap = 2.0 * yc - yv(m - 1) - yv(m + 1);
    }
    dl += mu * lap;
    dy += mu * yc;
}

// ---------------------------------------------------------------------------
// Strided adjoint solve with TMA (rank 2: x, rank 3: y): mu = A^-1 (1 - M) lam
// for the 32 lines of a warp, with the forward sweep's pipeline (one tile,
// row groups on their own mbarriers, finished groups stored while the lower
// ones are computed). The sums over mu and y are left to adjoint_dots_kernel.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128, 1)
    adjoint_solve_strided_tma_kernel(const __grid_constant__ CUtensorMap map_l,
                                     const __grid_constant__ CUtensorMap map_mu, SweepArgs<T> a, StridedGeom g,
                                     int crow) {
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
    unsigned char *wbase = smem_raw + (size_t)warp * strided_tma_warp_bytes(n, crow, sizeof(T), 32);
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
            tma_load(sm_u32 + ch * chunk_bytes, &map_l, col0, ch * crow, slab, rank, bar0 + 8 * ch);
        }
    }

    const long long col = (long long)col0 + lane;
    const bool valid = col < P;
    const int S = a.S;
    const int d = (int)(col % S);
    int ci, cj, ck;
    if (g.axis == 0) {
        const long long q = col / S;
        ck = (int)(q % a.nz);
        cj = (int)(q / a.nz);
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
    auto wait_group = [&](int ch) -> bool {
        if (mbar_wait(bar0 + 8 * ch, 0)) return true;
        if (lane == 0) atomicOr(a.err, 1);
        return false;
    };
    // masked adjoint: interior rows lose only whole lines on other faces,
    // the end rows also their own faces
    auto xin = [&](int q) -> T { return col_dir ? T(0) : sm[q * 32 + lane]; };
    auto xend = [&](int q) -> T {
        return (col_dir || (q == 0 && lo_dir) || (q == n - 1 && hi_dir)) ? T(0) : sm[q * 32 + lane];
    };
    LineSolver<T> L(a, d);
    const int m0 = a.fac.m0;

    // ---- forward elimination, row group by row group as the copies land
    const int rref = min(1, n - 1);
    const int ref_ch = rref / crow;
    for (int ch = 0; ch <= ref_ch; ++ch)
        if (!wait_group(ch)) return;
    sm[lane] = L.first(xend(0), xend(rref));
    int r = 1;
    for (int ch = 0; ch < nch; ++ch) {
        if (ch > ref_ch && !wait_group(ch)) return;
        const int rend = min(n - 1, (ch + 1) * crow);
        const int hend = min(rend, m0);
        auto st = [&](int q, T v) { sm[q * 32 + lane] = v; };
        r = head_forward(L, r, hend, xin, st);
        r = tail_forward(L, r, rend, xin, st);
    }
    if (n > 1) L.template fwd<false>(xend(n - 1), n - 1);

    // ---- back substitution into the tile; each finished row group is stored
    sm[(n - 1) * 32 + lane] = L.out_last();
    const int tl = max(m0, 1);
    r = n - 2;
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int rlo = ch * crow;
        const int tstop = max(rlo, tl);
        auto ld = [&](int q) { return sm[q * 32 + lane]; };
        auto st = [&](int q, T v) { sm[q * 32 + lane] = v; };
        r = tail_backward(L, r, tstop, ld, st);
        r = head_backward(L, r, max(rlo, 1), ld, st);
        if (rlo == 0 && n > 1) sm[lane] = L.template bwd<false>(sm[lane], 0);
        fence_async_smem();
        __syncwarp();
        if (lane == 0) {
            tma_store(&map_mu, col0, rlo, slab, rank, sm_u32 + ch * chunk_bytes);
            bulk_commit();
        }
    }
    if (lane == 0) bulk_wait_read_all();
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Strided adjoint sweep with cp.async (grids TMA cannot describe).
//   a.f: incoming adjoint, yin: stored s_(a+1), a.fo: output mu
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(32) adjoint_strided_kernel(SweepArgs<T> a, const T *__restrict__ yin, StridedGeom g,
                                                             AdjTerms t) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const long long tile = blockIdx.x;
    const int n = g.n;
    const long long P = g.P;
    T *sl = reinterpret_cast<T *>(smem_raw);
    T *sy = sl + (size_t)n * 32;
    const int slab = (int)(tile / g.ncb);
    const long long col0 = (tile % g.ncb) * 32;
    const int ncols = (int)min((long long)32, P - col0);
    const size_t off = (size_t)slab * g.slab_stride + col0;
    if (lane < ncols)
        for (int r = 0; r < n; ++r) {
            cp_async<sizeof(T)>(sl + r * 32 + lane, a.f + off + (size_t)r * P + lane);
            cp_async<sizeof(T)>(sy + r * 32 + lane, yin + off + (size_t)r * P + lane);
        }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    const bool valid = lane < ncols;
    const long long col = col0 + lane;
    const int S = a.S, d = (int)(col % S);
    double dl = 0.0, dy = 0.0;
    if (valid) {
        int ci, cj, ck;
        if (g.axis == 0) {
            const long long q = col / S;
            ck = (int)(q % a.nz);
            cj = (int)(q / a.nz);
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
        T *ll = sl + lane;
        const T *yl = sy + lane;
        if (col_dir) {
            for (int q = 0; q < n; ++q) ll[q * 32] = T(0);
        } else {
            if (lo_dir) ll[0] = T(0);
            if (hi_dir) ll[(n - 1) * 32] = T(0);
        }
        EndFix fx;
        if (!col_dir && (lo_dir || hi_dir)) {
            auto gv = [&](int q) -> double {
                return (double)(g.axis == 0 ? dir_value(a.dir, q, cj, ck, d) : dir_value(a.dir, ci, q, ck, d));
            };
            fx.make(lo_dir, hi_dir, n, t.c1[d], t.c2[d], gv(0), gv(n - 1), n > 1 ? (double)yl[32] : 0.0,
                    n > 1 ? (double)yl[(n - 2) * 32] : 0.0);
        }
        auto yv = [&](int q) -> double {
            if (q == 0 && fx.lo) return fx.y0;
            if (q == n - 1 && fx.hi) return fx.yn;
            return (double)yl[q * 32];
        };
        LineSolver<T> Ls(a, d);
        const int m0 = a.fac.m0;
        ll[0] = Ls.first(ll[0], ll[min(1, n - 1) * 32]);
        const int hend = min(n - 1, m0);
        int k = 1;
        for (; k < hend; ++k) ll[k * 32] = Ls.template fwd<false>(ll[k * 32], k);
        for (; k < n - 1; ++k) ll[k * 32] = Ls.template fwd<true>(ll[k * 32], k);
        if (n > 1) Ls.template fwd<false>(ll[(n - 1) * 32], n - 1);
        T *out = a.fo + off + lane;
        T mu = Ls.out_last();
        dots_at(n - 1, n, (double)mu, yv, dl, dy);
        out[(size_t)(n - 1) * P] = mu;
        const int tl = max(m0, 1);
        for (k = n - 2; k >= tl; --k) {
            mu = Ls.template bwd<true>(ll[k * 32], k);
            dots_at(k, n, (double)mu, yv, dl, dy);
            out[(size_t)k * P] = mu;
        }
        for (; k >= 0; --k) {
            mu = Ls.template bwd<false>(ll[k * 32], k);
            dots_at(k, n, (double)mu, yv, dl, dy);
            out[(size_t)k * P] = mu;
        }
    }
    tile_partials(dl, dy, d, S, t.part + (size_t)tile * S * 2);
}

// ---------------------------------------------------------------------------
// Contiguous (z) adjoint solve, the forward pipe kernel's pipeline; S <= 32,
// lane (r, d) owns line (row0 + r, d). SC: substrate count when a
// compile-time constant.
// ---------------------------------------------------------------------------
template <typename T, int SC>
__global__ void __launch_bounds__(128, 1) adjoint_solve_contig_pipe_kernel(SweepArgs<T> a, ContigGeom g, int kc) {
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
    const T *__restrict__ base = a.f + (size_t)row0 * L;
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
    auto xin = [&](int q) -> T { return line_dir ? T(0) : line[q * S]; };
    auto xend = [&](int q) -> T {
        return (line_dir || (q == 0 && lo_dir) || (q == nz - 1 && hi_dir)) ? T(0) : line[q * S];
    };
    LineSolver<T> Ls(a, d);
    const int m0 = a.fac.m0;

    const int kref = min(1, nz - 1);
    const int ref_c = kref / kc;
    for (int c = 0; c <= ref_c; ++c)
        if (!wait_c(c)) return;
    if (active) line[0] = Ls.first(xend(0), xend(kref));
    int k = 1;
    for (int c = 0; c < nch; ++c) {
        if (c > ref_c && !wait_c(c)) return;
        const int kend = min(nz - 1, (c + 1) * kc);
        if (active) {
            const int hend = min(kend, m0);
            auto st = [&](int q, T v) { line[q * S] = v; };
            k = head_forward(Ls, k, hend, xin, st);
            k = tail_forward(Ls, k, kend, xin, st);
        }
        k = max(k, kend);
    }
    if (active && nz > 1) Ls.template fwd<false>(xend(nz - 1), nz - 1);

    if (active) line[(nz - 1) * S] = Ls.out_last();
    const int tl = max(m0, 1);
    k = nz - 2;
    for (int c = nch - 1; c >= 0; --c) {
        const int klo = c * kc;
        if (active) {
            const int tstop = max(klo, tl);
            auto ld = [&](int q) { return line[q * S]; };
            auto st = [&](int q, T v) { line[q * S] = v; };
            k = tail_backward(Ls, k, tstop, ld, st);
            k = head_backward(Ls, k, max(klo, 1), ld, st);
            if (klo == 0 && nz > 1) line[0] = Ls.template bwd<false>(line[0], 0);
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
// The sums of one adjoint sweep: sum_m mu_m y_m and the edge form of
// mu.Lap y, sum_(m < n-1) (mu_m - mu_(m+1)) (y_m - y_(m+1)), with y's face
// ends rebuilt (EndFix). Each line is cut into segments of `seg` rows; one
// thread walks one segment of VEC adjacent lines (rows [s*seg, s*seg + seg)
// and the edge out of its last row) with 16-byte loads when VEC > 1.
// Element m of line l is at (l / inner) * n * inner + (l % inner) + m * inner;
// thread g takes lines VEC * (g % (nlines / VEC)) + [0, VEC) and segment
// g / (nlines / VEC), so consecutive threads read consecutive addresses on
// the x and y axes and consecutive substrates on z. blockDim = S * 2^p, so
// slot VEC * threadIdx.x + u of the block belongs to substrate
// (VEC * threadIdx.x + u) % S and the per-substrate sums are a fixed-order
// tree.
// ---------------------------------------------------------------------------
template <typename T, int VEC>
__device__ __forceinline__ void load_vec(const T *p, double (&o)[VEC]) {
    if constexpr (VEC == 1) {
        o[0] = (double)p[0];
    } else {
        if constexpr (sizeof(T) == 8) {
            static_assert(VEC == 2, "FP64 rows are read 2 at a time");
            const double2 v = *reinterpret_cast<const double2 *>(p);
            o[0] = v.x;
            o[1] = v.y;
        } else {
            static_assert(VEC == 4, "FP32 rows are read 4 at a time");
            const float4 v = *reinterpret_cast<const float4 *>(p);
            o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w;
        }
    }
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) adjoint_dots_kernel(const T *__restrict__ mu, const T *__restrict__ y,
                                                           DirFaces<T> dir, int axis, int n, long long inner,
                                                           long long nlines, int seg, AdjTerms t) {
    __shared__ double s0[256 * VEC], s1[256 * VEC];
    const int S = dir.S;
    const int tid = threadIdx.x;
    const long long ngroups = nlines / VEC;
    const long long gidx = (long long)blockIdx.x * blockDim.x + tid;
    const long long nsegs = (long long)((n + seg - 1) / seg);
    double dl[VEC], dyy[VEC];
#pragma unroll
    for (int u = 0; u < VEC; ++u) dl[u] = dyy[u] = 0.0;
    if (gidx < ngroups * nsegs) {
        const long long l0 = (gidx % ngroups) * VEC;
        const int q0 = (int)(gidx / ngroups) * seg;
        const int q1 = min(n, q0 + seg);  // rows [q0, q1); edges (m, m+1) for m in [q0, q1), m + 1 < n
        const long long outer = l0 / inner;
        const size_t base = (size_t)outer * n * inner + (size_t)(l0 - outer * inner);
        const T *__restrict__ mp = mu + base;
        const T *__restrict__ yp = y + base;
        // rebuilt ends, read by the segments holding rows 0, n-2 and n-1
        EndFix fx[VEC];
        bool any_fix = false;
        if (dir.any && (q0 == 0 || q1 >= n - 1)) {
#pragma unroll
            for (int u = 0; u < VEC; ++u) {
                const int d = (int)((l0 + u) % S);
                const unsigned msk = dir.mask[d];
                const bool lo = msk & (1u << (2 * axis)), hi = msk & (2u << (2 * axis));
                if (!(lo || hi)) continue;
                any_fix = true;
                const long long v0 = (long long)((base + u) / S);  // voxel of element 0
                const long long yz = (long long)dir.ny * dir.nz;
                const int vi = (int)(v0 / yz), vj = (int)((v0 / dir.nz) % dir.ny), vk = (int)(v0 % dir.nz);
                auto gv = [&](int q) -> double {
                    int ii = vi, jj = vj, kk = vk;
                    if (axis == 0) ii = q; else if (axis == 1) jj = q; else kk = q;
                    return (double)dir_value(dir, ii, jj, kk, d);
                };
                fx[u].make(lo, hi, n, t.c1[d], t.c2[d], gv(0), gv(n - 1), n > 1 ? (double)yp[inner + u] : 0.0,
                           n > 1 ? (double)yp[(size_t)(n - 2) * inner + u] : 0.0);
            }
        }
        auto yrow = [&](int q, double (&o)[VEC]) {
            load_vec<T, VEC>(yp + (size_t)q * inner, o);
            if (any_fix) {
#pragma unroll
                for (int u = 0; u < VEC; ++u) {
                    if (q == 0 && fx[u].lo) o[u] = fx[u].y0;
                    if (q == n - 1 && fx[u].hi) o[u] = fx[u].yn;
                }
            }
        };
        double mprev[VEC], yprev[VEC], dl2[VEC], dy2[VEC];
        load_vec<T, VEC>(mp + (size_t)q0 * inner, mprev);
        yrow(q0, yprev);
#pragma unroll
        for (int u = 0; u < VEC; ++u) {
            dyy[u] = mprev[u] * yprev[u];
            dl2[u] = dy2[u] = 0.0;
        }
        // own interior rows (q0, qa): plain loads, two independent accumulator chains
        const int qa = min(q1, n - 1);
        int q = q0 + 1;
#pragma unroll 2
        for (; q + 1 < qa; q += 2) {
            double ma[VEC], ya[VEC], mb[VEC], yb[VEC];
            load_vec<T, VEC>(mp + (size_t)q * inner, ma);
            load_vec<T, VEC>(yp + (size_t)q * inner, ya);
            load_vec<T, VEC>(mp + (size_t)(q + 1) * inner, mb);
            load_vec<T, VEC>(yp + (size_t)(q + 1) * inner, yb);
#pragma unroll
            for (int u = 0; u < VEC; ++u) {
                dl[u] += (mprev[u] - ma[u]) * (yprev[u] - ya[u]);
                dyy[u] += ma[u] * ya[u];
                dl2[u] += (ma[u] - mb[u]) * (ya[u] - yb[u]);
                dy2[u] += mb[u] * yb[u];
                mprev[u] = mb[u];
                yprev[u] = yb[u];
            }
        }
        for (; q < qa; ++q) {
            double ma[VEC], ya[VEC];
            load_vec<T, VEC>(mp + (size_t)q * inner, ma);
            load_vec<T, VEC>(yp + (size_t)q * inner, ya);
#pragma unroll
            for (int u = 0; u < VEC; ++u) {
                dl[u] += (mprev[u] - ma[u]) * (yprev[u] - ya[u]);
                dyy[u] += ma[u] * ya[u];
                mprev[u] = ma[u];
                yprev[u] = ya[u];
            }
        }
        // row qa closes the segment: its own last row n-1, or the next segment's first row
        if (qa > q0) {
            double ma[VEC], ya[VEC];
            load_vec<T, VEC>(mp + (size_t)qa * inner, ma);
            yrow(qa, ya);
            const bool own = qa < q1;
#pragma unroll
            for (int u = 0; u < VEC; ++u) {
                dl[u] += (mprev[u] - ma[u]) * (yprev[u] - ya[u]);
                if (own) dyy[u] += ma[u] * ya[u];
            }
        }
#pragma unroll
        for (int u = 0; u < VEC; ++u) {
            dl[u] += dl2[u];
            dyy[u] += dy2[u];
        }
    }
#pragma unroll
    for (int u = 0; u < VEC; ++u) {
        s0[VEC * tid + u] = dl[u];
        s1[VEC * tid + u] = dyy[u];
    }
    __syncthreads();
    const int slots = VEC * blockDim.x;
    for (int h = slots / S / 2; h >= 1; h >>= 1) {
        for (int i = tid; i < h * S; i += blockDim.x) {
            s0[i] += s0[i + h * S];
            s1[i] += s1[i + h * S];
        }
        __syncthreads();
    }
    if (tid < S) {
        double *slot = t.part + ((size_t)blockIdx.x * S + tid) * 2;
        slot[0] += s0[tid];
        slot[1] += s1[tid];
    }
}

// Contiguous adjoint sweep with cp.async (any S; lines t = lane, lane + 32, ...).
template <typename T>
__global__ void __launch_bounds__(32) adjoint_contig_kernel(SweepArgs<T> a, const T *__restrict__ yin, ContigGeom g,
                                                            AdjTerms t) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const long long tile = blockIdx.x;
    const long long row0 = tile * g.R;
    const int nr = (int)min((long long)g.R, g.nrows - row0);
    const int S = a.S, nz = g.nz, L = nz * S;
    T *sl = reinterpret_cast<T *>(smem_raw);
    T *sy = sl + (size_t)g.R * g.RS;
    const T *Lm = a.f + (size_t)row0 * L;
    const T *Y = yin + (size_t)row0 * L;
    for (int e = lane; e < nr * L; e += 32) {
        const int r = e / L, q = e - r * L;
        cp_async<sizeof(T)>(sl + (size_t)r * g.RS + q, Lm + e);
        cp_async<sizeof(T)>(sy + (size_t)r * g.RS + q, Y + e);
    }
    cp_commit();
    cp_wait<0>();
    __syncwarp();
    double *slot = t.part + (size_t)tile * S * 2;
    const int rounds = (g.R * S + 31) / 32;
    for (int rd = 0; rd < rounds; ++rd) {
        const int tt = rd * 32 + lane;
        double dl = 0.0, dy = 0.0;
        int d = -1;
        if (tt < nr * S) {
            const int r = tt / S;
            d = tt - r * S;
            const long long row = row0 + r;
            const int i = (int)(row / a.ny), j = (int)(row % a.ny);
            const unsigned m = a.dir.any ? a.dir.mask[d] : 0u;
            const bool line_dir = ((m & 1u) && i == 0) || ((m & 2u) && i == a.nx - 1) || ((m & 4u) && j == 0) ||
                                  ((m & 8u) && j == a.ny - 1);
            const bool lo_dir = m & 16u, hi_dir = m & 32u;
            T *ll = sl + (size_t)r * g.RS + d;
            const T *yl = sy + (size_t)r * g.RS + d;
            if (line_dir) {
                for (int q = 0; q < nz; ++q) ll[q * S] = T(0);
            } else {
                if (lo_dir) ll[0] = T(0);
                if (hi_dir) ll[(nz - 1) * S] = T(0);
            }
            EndFix fx;
            if (!line_dir && (lo_dir || hi_dir))
                fx.make(lo_dir, hi_dir, nz, t.c1[d], t.c2[d], (double)dir_value(a.dir, i, j, 0, d),
                        (double)dir_value(a.dir, i, j, nz - 1, d), nz > 1 ? (double)yl[S] : 0.0,
                        nz > 1 ? (double)yl[(nz - 2) * S] : 0.0);
            auto yv = [&](int q) -> double {
                if (q == 0 && fx.lo) return fx.y0;
                if (q == nz - 1 && fx.hi) return fx.yn;
                return (double)yl[q * S];
            };
            LineSolver<T> Ls(a, d);
            const int m0 = a.fac.m0;
            ll[0] = Ls.first(ll[0], ll[min(1, nz - 1) * S]);
            const int hend = min(nz - 1, m0);
            int k = 1;
            for (; k < hend; ++k) ll[k * S] = Ls.template fwd<false>(ll[k * S], k);
            for (; k < nz - 1; ++k) ll[k * S] = Ls.template fwd<true>(ll[k * S], k);
            if (nz > 1) Ls.template fwd<false>(ll[(nz - 1) * S], nz - 1);
            T mu = Ls.out_last();
            dots_at(nz - 1, nz, (double)mu, yv, dl, dy);
            ll[(nz - 1) * S] = mu;
            const int tl = max(m0, 1);
            for (k = nz - 2; k >= tl; --k) {
                mu = Ls.template bwd<true>(ll[k * S], k);
                dots_at(k, nz, (double)mu, yv, dl, dy);
                ll[k * S] = mu;
            }
            for (; k >= 0; --k) {
                mu = Ls.template bwd<false>(ll[k * S], k);
                dots_at(k, nz, (double)mu, yv, dl, dy);
                ll[k * S] = mu;
            }
        }
        tile_partials(dl, dy, d, S, slot);
    }
    __syncwarp();
    T *O = a.fo + (size_t)row0 * L;
    for (int e = lane; e < nr * L; e += 32) {
        const int r = e / L, q = e - r * L;
        O[e] = sl[(size_t)r * g.RS + q];
    }
}

// gacc[d] = sum over slots of part[slot][d][0], gacc[S + d] likewise for [1];
// block d adds its slots in a fixed order.
__global__ void adjoint_reduce_kernel(const double *__restrict__ part, long long nslots, int S, double *__restrict__ gacc) {
    __shared__ double s0[256], s1[256];
    const int d = blockIdx.x;
    double a0 = 0.0, a1 = 0.0;
    for (long long q = threadIdx.x; q < nslots; q += blockDim.x) {
        a0 += part[(q * S + d) * 2];
        a1 += part[(q * S + d) * 2 + 1];
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
        gacc[d] = s0[0];
        gacc[S + d] = s1[0];
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
    for (int d = 0; d < dir.S; ++d)
        if (on_active_face(dir.mask[d], i, j, k, dir.nx, dir.ny, dir.nz)) f[vb + d] = T(0);
}

// Agents' update of a recomputed step, keeping the pre-agent values v.
template <typename T>
__global__ void cells_keep_kernel(T *__restrict__ f, int S, int n_occ, const int *__restrict__ seg_start,
                                  const int *__restrict__ seg_voxel, const T *__restrict__ t1, const T *__restrict__ t2,
                                  T *__restrict__ vkeep) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    const int s = (int)(e / S), d = (int)(e % S);
    const size_t fe = (size_t)seg_voxel[s] * S + d;
    T x = f[fe];
    vkeep[e] = x;
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
// replayed from the pre-agent value v = x_0, which is also written back into
// the step's output w (turning it into Dir(y_z) for the z adjoint).
// With `dir` active (every step but the run's last), lam is the next step's
// mu_x, and its active-face entries are masked here: the next step's leading
// Dirichlet overwrote those voxels.
template <typename T>
__global__ void cells_adjoint_kernel(T *__restrict__ lam, T *__restrict__ w, const T *__restrict__ vkeep, int S,
                                     int n_occ, const int *__restrict__ seg_start, const int *__restrict__ seg_voxel,
                                     const T *__restrict__ t1, const T *__restrict__ t2, double *__restrict__ gt1,
                                     double *__restrict__ gt2, DirFaces<T> dir) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)n_occ * S) return;
    const int s = (int)(e / S), d = (int)(e % S);
    const int vox = seg_voxel[s];
    const size_t fe = (size_t)vox * S + d;
    const int q0 = seg_start[s], q1 = seg_start[s + 1];
    const T v = vkeep[e];
    double g = (double)lam[fe];
    if (dir.any) {
        const int k = vox % dir.nz, j = (vox / dir.nz) % dir.ny, i = vox / (dir.nz * dir.ny);
        if (on_active_face(dir.mask[d], i, j, k, dir.nx, dir.ny, dir.nz)) g = 0.0;
    }
    for (int k = q1 - 1; k >= q0; --k) {
        double x = (double)v;  // replay x_k
        for (int q = q0; q <= k; ++q) x = (x + (double)t1[(size_t)q * S + d]) / (double)t2[(size_t)q * S + d];
        const double tt = (double)t2[(size_t)k * S + d];
        gt1[(size_t)k * S + d] += g / tt;
        gt2[(size_t)k * S + d] -= g * x / tt;
        g /= tt;
    }
    lam[fe] = (T)g;
    w[fe] = v;
}

}  // namespace bfb

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace bfb {
int env_prepare_step(bfb_env_s *env, double dt, int flags);
template <typename T>
SweepArgs<T> env_sweep_args(bfb_env_s *env, int axis, double dt);
int env_tile_plan(bfb_env_s *env, int elem, int Lp, StridedGeom *gx, StridedGeom *gy, ContigGeom *gz, int vb16[3]);
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

// A field-sized buffer with its x (0) and y (1) tensor maps.
struct Buf {
    void *p = nullptr;
    CUtensorMap map[2];
    int ok[2] = {0, 0};
    int crow[2] = {0, 0};
};

template <typename K>
void opt_in(K k) {
    cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
}

template <typename T>
void opt_in_all() {
    static int done_dev = -1;  // per instantiation (precision)
    int dev = 0;
    cudaGetDevice(&dev);
    if (done_dev == dev) return;
    opt_in(adjoint_solve_strided_tma_kernel<T>);
    opt_in(adjoint_strided_kernel<T>);
    opt_in(adjoint_solve_contig_pipe_kernel<T, 1>);
    opt_in(adjoint_solve_contig_pipe_kernel<T, 2>);
    opt_in(adjoint_solve_contig_pipe_kernel<T, 4>);
    opt_in(adjoint_solve_contig_pipe_kernel<T, 8>);
    opt_in(adjoint_solve_contig_pipe_kernel<T, 0>);
    opt_in(adjoint_contig_kernel<T>);
    done_dev = dev;
}

template <typename T>
struct Adjoint {
    bfb_env_s *env = nullptr;
    double dt = 0;
    cudaStream_t st = nullptr;
    int S = 0;
    StridedGeom gx, gy;
    ContigGeom gz;
    int kc = 0;  // z row-group length of the pipelined kernel (0: the cp.async kernel)
    const double *coef = nullptr;  // [2S]: c1, c2
    double *part_x = nullptr, *part_y = nullptr, *part_z = nullptr;
    long long tiles_z = 0;
    bool sums = true;  // the per-line sums for dL/dD and dL/dlambda (skipped when neither is asked for)

    // tensor maps with the env's row-group counts (so the recompute runs the
    // env's tuned launch shape) and warp tiles of 32 lines (the adjoint
    // kernels' tiles); workspace buffers are packed (rows nz*S apart)
    void map(Buf &b) {
        for (int a = 0; a < 2; ++a)
            b.ok[a] = env->use_tma && make_sweep_tensor_map(&b.map[a], &b.crow[a], b.p, sizeof(T), a, env->nx,
                                                            env->ny, env->nz, S, env->tuning.chunks[a], env->nz * S,
                                                            32);
    }
    // the env's sweep arguments over packed workspace buffers
    SweepArgs<T> args(int axis) const {
        SweepArgs<T> a = env_sweep_args<T>(env, axis, dt);
        a.Lp = env->nz * S;
        return a;
    }

    // one forward sweep, out of place, in the env's launch shape
    int fwd(int axis, Buf &in, Buf &out) {
        SweepArgs<T> a = args(axis);
        a.f = static_cast<T *>(in.p);
        a.fo = static_cast<T *>(out.p);
        const int warps = env->tuning.warps[axis];
        if (axis < 2) {
            const bool tma = env->tuning.tma[axis] && in.ok[axis] && out.ok[axis];
            return launch_strided<T>(a, axis, axis == 0, warps, tma ? &in.map[axis] : nullptr,
                                     tma ? &out.map[axis] : nullptr, in.crow[axis], 32, st);
        }
        return launch_contig<T>(a, warps, env->use_tma && env->tuning.tma[2], st, env->tuning.chunks[2]);
    }

    // the sums of one sweep over the stored y and the new mu
    // lines per thread (16-byte loads) and rows per thread in the sums kernel
    // (measured at 256^3 x 8 FP32: 4 lines x 64 rows beats 1 x 64, 4 x 16 and
    // 4 x 32, and ties with 4 x 128)
    static constexpr int kVec = sizeof(T) == 8 ? 2 : 4;
    static constexpr int kDotSeg = sizeof(T) == 8 ? 32 : 64;
    int dots_threads() const {
        int threads = S;
        while (threads * 2 <= 256) threads *= 2;
        return threads;
    }
    static int axis_len(const bfb_env_s *e, int axis) { return axis == 0 ? e->nx : (axis == 1 ? e->ny : e->nz); }
    long long axis_inner(int axis) const {
        return axis == 0 ? (long long)env->ny * env->nz * S : (axis == 1 ? (long long)env->nz * S : S);
    }
    int dots_vec(int axis) const { return axis_inner(axis) % kVec == 0 ? kVec : 1; }
    long long dots_blocks(int axis) const {
        const int n = axis_len(env, axis);
        const int sg = dots_vec(axis) == kVec ? kDotSeg : 64;
        const long long work = (long long)env->N / n / dots_vec(axis) * ((n + sg - 1) / sg);
        return (work + dots_threads() - 1) / dots_threads();
    }
    int dots(int axis, const SweepArgs<T> &a, const T *mu, const T *y, const AdjTerms &t) {
        const int n = axis_len(env, axis);
        const long long nlines = (long long)env->N / n;
        const unsigned blocks = (unsigned)dots_blocks(axis);
        if (dots_vec(axis) == kVec)
            adjoint_dots_kernel<T, kVec><<<blocks, dots_threads(), 0, st>>>(mu, y, a.dir, axis, n, axis_inner(axis),
                                                                             nlines, kDotSeg, t);
        else
            adjoint_dots_kernel<T, 1><<<blocks, dots_threads(), 0, st>>>(mu, y, a.dir, axis, n, axis_inner(axis),
                                                                          nlines, 64, t);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }

    // one adjoint sweep: lam (in) and y (stored forward output) -> mu (out)
    int adj(int axis, Buf &lam, Buf &y, Buf &mu) {
        SweepArgs<T> a = args(axis);
        a.f = static_cast<T *>(lam.p);
        a.fo = static_cast<T *>(mu.p);
        const AdjTerms t{coef, coef + S, axis == 0 ? part_x : (axis == 1 ? part_y : part_z)};
        const T *yp = static_cast<const T *>(y.p);
        if (axis < 2) {
            const StridedGeom &g = axis == 0 ? gx : gy;
            const unsigned tiles = (unsigned)((long long)g.n_slabs * g.ncb);
            if (lam.ok[axis] && mu.ok[axis]) {
                const int crow = lam.crow[axis];
                const size_t wb = strided_tma_warp_bytes(g.n, crow, sizeof(T), 32);
                if (wb <= (size_t)kMaxSmem) {
                    adjoint_solve_strided_tma_kernel<T><<<tiles, 32, wb, st>>>(lam.map[axis], mu.map[axis], a, g, crow);
                    BFB_CUDA(cudaGetLastError());
                    return sums ? dots(axis, a, static_cast<const T *>(mu.p), yp, t) : BFB_OK;
                }
            }
            const size_t smem = 2 * (size_t)g.n * 32 * sizeof(T);
            if (smem > (size_t)kMaxSmem) return fail(BFB_ERR_UNSUPPORTED, "adjoint: lines too long for shared memory");
            adjoint_strided_kernel<T><<<tiles, 32, smem, st>>>(a, yp, g, t);
            BFB_CUDA(cudaGetLastError());
            return BFB_OK;
        }
        const unsigned tiles = (unsigned)tiles_z;
        if (kc > 0) {
            const size_t wb = (128 + (size_t)gz.R * gz.RS * sizeof(T) + 127) / 128 * 128;
            switch (S) {
            case 1: adjoint_solve_contig_pipe_kernel<T, 1><<<tiles, 32, wb, st>>>(a, gz, kc); break;
            case 2: adjoint_solve_contig_pipe_kernel<T, 2><<<tiles, 32, wb, st>>>(a, gz, kc); break;
            case 4: adjoint_solve_contig_pipe_kernel<T, 4><<<tiles, 32, wb, st>>>(a, gz, kc); break;
            case 8: adjoint_solve_contig_pipe_kernel<T, 8><<<tiles, 32, wb, st>>>(a, gz, kc); break;
            default: adjoint_solve_contig_pipe_kernel<T, 0><<<tiles, 32, wb, st>>>(a, gz, kc); break;
            }
            BFB_CUDA(cudaGetLastError());
            return sums ? dots(2, a, static_cast<const T *>(mu.p), yp, t) : BFB_OK;
        }
        const size_t smem = 2 * (size_t)gz.R * gz.RS * sizeof(T);
        if (smem > (size_t)kMaxSmem) return fail(BFB_ERR_UNSUPPORTED, "adjoint: rows too long for shared memory");
        adjoint_contig_kernel<T><<<tiles, 32, smem, st>>>(a, yp, gz, t);
        BFB_CUDA(cudaGetLastError());
        return BFB_OK;
    }
};

template <typename T>
int adjoint_run(bfb_env_s *env, double dt, int n_steps, int flags, int K, const void *dL_dfinal, void *dL_dinitial,
                void *final_field, double *gD, double *gL, double *gsec, double *gupt, double *gsat) {
    const int S = env->S;
    const size_t fb = (size_t)env->N * sizeof(T);
    cudaStream_t st = env->stream;
    const bool cells = (flags & BFB_STEP_CELLS) && env->n_occ > 0;
    int rc = env_prepare_step(env, dt, BFB_STEP_DIFFUSION);
    if (rc) return rc;
    Adjoint<T> A;
    A.env = env;
    A.dt = dt;
    A.st = st;
    A.sums = gD || gL;
    A.S = S;
    int vb16[3];
    if ((rc = env_tile_plan(env, sizeof(T), env->nz * S, &A.gx, &A.gy, &A.gz, vb16))) return rc;
    opt_in_all<T>();
    const long long tiles_x = (long long)A.gx.n_slabs * A.gx.ncb, tiles_y = (long long)A.gy.n_slabs * A.gy.ncb;
    A.tiles_z = (A.gz.nrows + A.gz.R - 1) / A.gz.R;
    {   // pipelined z solve: the forward pipe kernel's alignment rules
        const long long L = (long long)env->nz * S;
        const int eb = (int)sizeof(T);
        const size_t wb = (128 + (size_t)A.gz.R * A.gz.RS * eb + 127) / 128 * 128;
        if (env->use_tma && S <= 32 && (L * eb) % 16 == 0 && ((long long)A.gz.RS * eb) % 16 == 0 &&
            wb <= (size_t)kMaxSmem) {
            int q = 16;
            for (int v = S * eb; v % 2 == 0 && q > 1; v /= 2) q /= 2;  // q = 16 / gcd(16, S*elem)
            const int kc = (env->nz + kChunks - 1) / kChunks;
            A.kc = (kc + q - 1) / q * q;
        }
    }

    // ---- workspace
    const int nseg = (n_steps + K - 1) / K;
    const size_t occ = (size_t)env->n_occ * S;
    const size_t nact = (size_t)env->n_active * S;
    // partial-sum slots per axis: tiles of the fused fallback kernels or blocks of the sums kernel
    const long long reg_x = std::max(tiles_x, A.dots_blocks(0)), reg_y = std::max(tiles_y, A.dots_blocks(1)),
                    reg_z = std::max(A.tiles_z, A.dots_blocks(2));
    const long long slots = reg_x + reg_y + reg_z;
    std::vector<T *> ckpt(nseg - 1);
    std::vector<Buf> S1(K), S2(K), W(K);
    Buf lam, mu, ck;
    // the env's field rows are padded where nz*S elements are not whole 16-byte
    // vectors; the workspace is packed, and the last segment then starts from
    // a packed copy of the field (head)
    const bool padded = env->Lp != env->nz * S;
    T *head = nullptr;
    T *vkeep = nullptr;
    double *part = nullptr, *gacc = nullptr, *gt1 = nullptr, *gt2 = nullptr, *coef = nullptr;
    auto carve = [&](Carve &c) {
        for (auto &p : ckpt) c.take(&p, fb);
        for (auto *v : {&S1, &S2, &W})
            for (auto &b : *v) {
                T *p;
                c.take(&p, fb);
                b.p = p;
            }
        for (Buf *b : {&lam, &mu}) {
            T *p;
            c.take(&p, fb);
            b->p = p;
        }
        c.take(&head, padded ? fb : 0);
        c.take(&part, sizeof(double) * 2 * S * slots);
        c.take(&gacc, sizeof(double) * 2 * S);
        c.take(&coef, sizeof(double) * 2 * S);
        c.take(&vkeep, sizeof(T) * occ * K);
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
        const cudaError_t e = cudaMalloc(&env->adj_ws, sizing.off);
        if (e != cudaSuccess) {
            env->adj_ws = nullptr;
            return cuda_fail(e, "cudaMalloc (adjoint workspace)");
        }
        env->adj_ws_bytes = sizing.off;
    }
    Carve c;
    c.base = static_cast<char *>(env->adj_ws);
    carve(c);
    for (auto *v : {&S1, &S2, &W})
        for (auto &b : *v) A.map(b);
    A.map(lam);
    A.map(mu);
    A.part_x = part;
    A.part_y = part + 2 * S * reg_x;
    A.part_z = part + 2 * S * (reg_x + reg_y);
    // c1 and c2 as the factor precompute forms them, at the dt the factors hold
    const double fdt = env->factor_dt;
    std::vector<double> hcoef(2 * S);
    for (int d = 0; d < S; ++d) {
        double c1 = env->D[d] * fdt;
        c1 /= env->dx;
        c1 /= env->dx;
        double c2 = env->lambda[d] * fdt;
        c2 /= 3.0;
        hcoef[d] = c1;
        hcoef[S + d] = c2;
    }
    A.coef = coef;
    BFB_CUDA(cudaMemcpyAsync(coef, hcoef.data(), sizeof(double) * 2 * S, cudaMemcpyHostToDevice, st));
    BFB_CUDA(cudaMemsetAsync(part, 0, sizeof(double) * 2 * S * slots, st));
    if (nact) {
        BFB_CUDA(cudaMemsetAsync(gt1, 0, sizeof(double) * nact, st));
        BFB_CUDA(cudaMemsetAsync(gt2, 0, sizeof(double) * nact, st));
    }
    const unsigned occ_blocks = (unsigned)((occ + 255) / 256);
    const T *t1 = static_cast<const T *>(env->ag_t1), *t2 = static_cast<const T *>(env->ag_t2);

    // len forward steps from `in`, keeping s1, s2 and every step's output
    auto segment = [&](Buf &in, int len) -> int {
        for (int j = 0; j < len; ++j) {
            int r;
            if ((r = A.fwd(0, j == 0 ? in : W[j - 1], S1[j])) || (r = A.fwd(1, S1[j], S2[j])) ||
                (r = A.fwd(2, S2[j], W[j])))
                return r;
            if (cells) {
                cells_keep_kernel<T><<<occ_blocks, 256, 0, st>>>(static_cast<T *>(W[j].p), S, env->n_occ,
                                                                 env->seg_start, env->seg_voxel, t1, t2,
                                                                 vkeep + (size_t)j * occ);
                BFB_CUDA(cudaGetLastError());
            }
        }
        return BFB_OK;
    };

    // field (rows Lp apart) <-> packed workspace
    const size_t row_b = (size_t)env->nz * S * sizeof(T), field_b = (size_t)env->Lp * sizeof(T);
    const size_t nrows = (size_t)env->nx * env->ny;
    auto from_field = [&](T *dst) {
        return padded ? cudaMemcpy2DAsync(dst, row_b, env->field, field_b, row_b, nrows, cudaMemcpyDeviceToDevice, st)
                      : cudaMemcpyAsync(dst, env->field, fb, cudaMemcpyDeviceToDevice, st);
    };

    // ---- forward: checkpoints of the earlier segments, stage fields of the last
    const int fwd_flags = BFB_STEP_DIFFUSION | (cells ? BFB_STEP_CELLS : 0);
    for (int s = 0; s < nseg - 1; ++s) {
        BFB_CUDA(from_field(ckpt[s]));
        if ((rc = bfb_simulate(env, dt, K, fwd_flags))) return rc;
    }
    const int last_len = n_steps - (nseg - 1) * K;
    {
        Buf f;  // the field itself where its rows are packed, else a packed copy
        if (padded) BFB_CUDA(from_field(head));
        f.p = padded ? static_cast<void *>(head) : env->field;
        A.map(f);
        if ((rc = segment(f, last_len))) return rc;
    }
    if (padded)
        BFB_CUDA(cudaMemcpy2DAsync(env->field, field_b, W[last_len - 1].p, row_b, row_b, nrows,
                                   cudaMemcpyDeviceToDevice, st));
    else
        BFB_CUDA(cudaMemcpyAsync(env->field, W[last_len - 1].p, fb, cudaMemcpyDeviceToDevice, st));
    if (final_field) BFB_CUDA(cudaMemcpyAsync(final_field, W[last_len - 1].p, fb, cudaMemcpyDeviceToDevice, st));
    BFB_CUDA(cudaMemcpyAsync(lam.p, dL_dfinal, fb, cudaMemcpyDeviceToDevice, st));

    // ---- reverse, segment by segment
    const DirFaces<T> dirf = env_sweep_args<T>(env, 0, dt).dir;
    Buf *pl = &lam, *pm = &mu;
    for (int s = nseg - 1; s >= 0; --s) {
        const int len = s == nseg - 1 ? last_len : K;
        if (s < nseg - 1) {
            ck.p = ckpt[s];
            A.map(ck);
            if ((rc = segment(ck, len))) return rc;
        }
        for (int j = len - 1; j >= 0; --j) {
            if (cells) {
                DirFaces<T> dj = dirf;
                if (s == nseg - 1 && j == len - 1) dj.any = 0;  // dL/d(final field) is not masked
                cells_adjoint_kernel<T><<<occ_blocks, 256, 0, st>>>(
                    static_cast<T *>(pl->p), static_cast<T *>(W[j].p), vkeep + (size_t)j * occ, S, env->n_occ,
                    env->seg_start, env->seg_voxel, t1, t2, gt1, gt2, dj);
                BFB_CUDA(cudaGetLastError());
            }
            if ((rc = A.adj(2, *pl, W[j], *pm))) return rc;
            if ((rc = A.adj(1, *pm, S2[j], *pl))) return rc;
            if ((rc = A.adj(0, *pl, S1[j], *pm))) return rc;
            std::swap(pl, pm);  // *pl = dL/du of this step's input
        }
    }
    if (dL_dinitial) {
        if (dirf.any) {
            const long long nface = 2 * ((long long)env->ny * env->nz + (long long)env->nx * env->nz +
                                         (long long)env->nx * env->ny);
            adjoint_mask_kernel<T><<<(unsigned)((nface + 255) / 256), 256, 0, st>>>(static_cast<T *>(pl->p), dirf);
            BFB_CUDA(cudaGetLastError());
        }
        BFB_CUDA(cudaMemcpyAsync(dL_dinitial, pl->p, fb, cudaMemcpyDeviceToDevice, st));
    }
    adjoint_reduce_kernel<<<S, 256, 0, st>>>(part, slots, S, gacc);
    BFB_CUDA(cudaGetLastError());

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
    int herr = 0;
    BFB_CUDA(cudaMemcpy(&herr, env->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(BFB_ERR_WATCHDOG, "adjoint: a device-side wait ran out of its iteration limit");
    const double kD = -fdt / (env->dx * env->dx), kL = -fdt / 3.0;
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
            const double cc = env->agent_dt * env->h_vol[a] / dV;
            for (int d = 0; d < S; ++d) {
                const size_t qa = (size_t)q * S + d, la = (size_t)a * S + d;
                if (gsec) gsec[la] = h1[qa] * cc * env->h_sat[la] + h2[qa] * cc;
                if (gupt) gupt[la] = h2[qa] * cc;
                if (gsat) gsat[la] = h1[qa] * cc * env->h_sec[la];
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
    if (env->nx_global) return fail(BFB_ERR_UNSUPPORTED, "reverse mode runs on whole grids, not x-slab envs");
    if (n_steps < 1 || checkpoint_every < 1 || !(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "bad dt, n_steps or K");
    NvtxRange range("bfb_adjoint_run");
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
