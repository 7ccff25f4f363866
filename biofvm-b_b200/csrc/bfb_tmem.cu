// bfb_tmem.cu -- the FP64 strided (x/y) sweep with each line's forward
// results held in tensor memory (TMEM), Blackwell's per-SM 256 KB memory of
// the tensor cores, here used as plain storage.
//
// Why: an FP64 line solve is a chain of dependent FP64 operations per row, so
// a sweep runs as fast as the number of lines in flight per SM allows. In the
// shared-memory tiles (bfb_tma_tiles.cuh) every row of every line in flight
// sits in shared memory, which holds at most ~110 lines of 256 doubles per
// SM. Here the forward elimination's results go to TMEM instead: a CTA of
// four warps allocates all 512 TMEM columns, and lane l of warp w owns TMEM
// lane 32w + l -- 512 32-bit columns, one 256-row FP64 line. Shared memory
// only stages row groups of 16 rows through two small rings per warp:
//   * input: 6 slots, each one TMA tensor copy of 16 rows x 32 lines on its
//     own mbarrier, refilled as soon as the forward pass has read it, with
//     the next row group of the tile or, past the tile's last, of the warp's
//     next tile (so the next tile's first rows arrive during this tile's back
//     substitution);
//   * output: 3 slots that the back substitution fills (rows descending) and
//     that one TMA tensor store each writes back; a slot is reused once the
//     store issued from it has read it.
// The operations per row are those of the shared-memory tiles (the same
// LineSolver<double> calls in the same order), so the results are bit for
// bit the same. Rows are moved to and from TMEM eight at a time
// (tcgen05.st / tcgen05.ld, shape 32x32b, 16 columns).
//
// Measured at 256^3 x 8 FP64 (CUDA events): x/y 0.78 / 0.80 ms against 0.44 /
// 0.44 ms for the shared-memory tiles, and about 2x slower at 200^3 and
// 128^3 too: TMEM holds 128 lines per SM, not many more than the 110 that the
// 22-line shared-memory tiles keep resident, and each line advances about
// half as fast (one warp per scheduler, and the row-group and TMEM traffic
// around every 8 or 16 rows). So the tiles are an explicit choice (tuning
// value 2) that bfb_autotune does not try.
//
// Every wait is bounded: an mbarrier wait that runs out sets the env's error
// flag, and the warp stops taking tiles; all warps still meet at the end,
// where warp 0 frees the TMEM. One CTA per SM (its shared memory is more than
// half an SM's), so an allocation never waits for another CTA's columns.
#include <cuda.h>

#include <algorithm>

#include "bfb_tma_tiles.cuh"

namespace bfb {

namespace {

constexpr int kTmemGroup = 16;  // rows per row group (TMA box rows)
constexpr int kTmemIn = 6;      // input ring slots per warp
constexpr int kTmemOut = 3;     // output ring slots per warp
constexpr int kTmemWarps = 4;   // one per TMEM lane quadrant
constexpr int kTmemCols = 512;  // all of an SM's TMEM columns
constexpr int kTmemMaxRows = kTmemCols / 2;  // FP64: two 32-bit columns per row
constexpr unsigned kTmemSlotBytes = kTmemGroup * 32 * 8;
constexpr size_t kTmemWarpBytes = 128 + (size_t)(kTmemIn + kTmemOut) * kTmemSlotBytes;
constexpr size_t kTmemCtaBytes = 128 + kTmemWarps * kTmemWarpBytes;

// ---- tcgen05 (tensor memory) -------------------------------------------------
// All of these are .sync.aligned: every lane of the warp executes them together.
__device__ __forceinline__ void tmem_alloc(unsigned dst_smem, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// eight doubles of this lane's TMEM row, columns [taddr, taddr + 16)
__device__ __forceinline__ void tmem_st8(unsigned taddr, const double (&v)[8]) {
    unsigned r[16];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v[u]);
        r[2 * u] = (unsigned)b;
        r[2 * u + 1] = (unsigned)(b >> 32);
    }
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
// issues the load of eight doubles; they are valid after tmem_wait_ld(r)
__device__ __forceinline__ void tmem_ld8(unsigned taddr, unsigned (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
// waits for the issued loads; the registers are operands so that no use of
// them is scheduled before the wait
__device__ __forceinline__ void tmem_wait_ld(unsigned (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}
__device__ __forceinline__ double tmem_dbl(const unsigned (&r)[16], int u) {
    return __longlong_as_double((long long)(((unsigned long long)r[2 * u + 1] << 32) | r[2 * u]));
}
template <int N>
__device__ __forceinline__ void bulk_wait_read_n() {
    asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}

// One warp's tiles (32 lines each): tile w, w + W, ... of the sweep. Returns
// false when a bounded wait ran out (the error flag is set).
template <bool FUSE_PRE, bool BULK>
__device__ bool tmem_warp_tiles(const CUtensorMap *map, const CUtensorMap *map_out, const SweepArgs<double> &a,
                                const StridedGeom &g, unsigned char *wbase, unsigned tbase) {
    const int lane = threadIdx.x & 31;
    const int n = g.n;
    const long long P = g.P;
    const int ng = (n + kTmemGroup - 1) / kTmemGroup;
    const long long ntiles = (long long)g.n_slabs * g.ncb;
    const long long stride = (long long)gridDim.x * kTmemWarps;
    const long long first = (long long)blockIdx.x * kTmemWarps + (threadIdx.x >> 5);
    if (first >= ntiles) return true;
    const int rank = g.axis == 0 ? 2 : 3;
    const unsigned bar0 = smem_u32(wbase);
    double *in_ring = reinterpret_cast<double *>(wbase + 128);
    double *out_ring = in_ring + (size_t)kTmemIn * kTmemGroup * 32;
    const unsigned in_u32 = smem_u32(in_ring), out_u32 = smem_u32(out_ring);
    if (lane == 0) {
        for (int s = 0; s < kTmemIn; ++s) mbar_init(bar0 + 8 * s, 1);
        fence_mbar_init();
    }
    __syncwarp();

    // producer (lane 0): the next row group to load, group pg of tile pt
    long long pt = first;
    int pg = 0;
    unsigned issued = 0, used = 0, out_seq = 0;
    auto issue_next = [&]() {
        if (pt >= ntiles) return;
        const int s = (int)(issued % kTmemIn);
        mbar_expect_tx(bar0 + 8 * s, kTmemSlotBytes);
        tma_load(in_u32 + s * kTmemSlotBytes, map, (int)((pt % g.ncb) * 32), pg * kTmemGroup, (int)(pt / g.ncb), rank,
                 bar0 + 8 * s);
        ++issued;
        if (++pg == ng) {
            pg = 0;
            pt += stride;
        }
    };
    if (lane == 0)
        for (int s = 0; s < kTmemIn; ++s) issue_next();

    bool ok = true;
    const int m0 = a.fac.m0;
    const int tl = max(m0, 1);
    for (long long tile = first; tile < ntiles && ok; tile += stride) {
        const int slab = (int)(tile / g.ncb);
        const int col0 = (int)((tile % g.ncb) * 32);
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
        auto vox_dir = [&](int mm) -> double {
            return g.axis == 0 ? dir_value(a.dir, mm, cj, ck, d) : dir_value(a.dir, ci, mm, ck, d);
        };
        const double *bA = nullptr, *bB = nullptr;
        if constexpr (BULK) {
            bA = a.bulk.A + (size_t)slab * g.slab_stride + cl;
            bB = a.bulk.B + (size_t)slab * g.slab_stride + cl;
        }
        auto upd = [&](double x, int q) -> double {
            if constexpr (BULK) {
                if (valid) x = bulk_update(x, bA[(size_t)q * P], bB[(size_t)q * P], a.bulk.dt);
            }
            return x;
        };
        LineSolver<double> L(a, d);

        // ---- forward elimination, group by group from the input ring, eight
        // rows at a time into TMEM
        for (int gi = 0; gi < ng; ++gi) {
            const int s = (int)(used % kTmemIn);
            const bool landed = mbar_wait(bar0 + 8 * s, (used / kTmemIn) & 1u);
            if (!__all_sync(0xffffffffu, landed)) {
                if (lane == 0) atomicOr(a.err, 1);
                ok = false;
                break;
            }
            const double *slot = in_ring + (size_t)s * kTmemGroup * 32 + lane;
#pragma unroll 1
            for (int half = 0; half < 2; ++half) {
                const int b = gi * kTmemGroup + half * 8;
                if (b >= n) break;
                const double *rows = slot + half * 8 * 32;
                double y[8];
                if (b >= tl && b + 8 <= n - 1) {  // tail rows only: factors in registers
#pragma unroll
                    for (int u = 0; u < 8; ++u) y[u] = upd(rows[u * 32], b + u);
#pragma unroll
                    for (int u = 0; u < 8; ++u) y[u] = L.tstep(y[u]);
                } else {
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int q = b + u;
                        double v = 0.0;
                        if (q < n) {
                            double x = upd(rows[u * 32], q);
                            if (FUSE_PRE && ((q == 0 && lo_dir) || (q == n - 1 && hi_dir))) x = vox_dir(q);
                            if (q == 0)
                                v = L.first(x, x);
                            else if (q == n - 1 || q < m0)
                                v = L.template fwd<false>(x, q);
                            else
                                v = L.tstep(x);
                        }
                        y[u] = v;
                    }
                }
                __syncwarp();
                tmem_st8(tbase + 2 * b, y);
            }
            ++used;
            __syncwarp();  // every lane has read the slot: refill it
            if (lane == 0) issue_next();
        }
        if (!ok) break;
        __syncwarp();
        tmem_wait_st();

        // ---- back substitution, eight rows at a time from TMEM (the next
        // block's load in flight while this one is computed), into the output
        // ring; each finished group is stored
        const int btop = ((n - 1) / 8) * 8;
        unsigned ra[16], rb[16];
        __syncwarp();
        tmem_ld8(tbase + 2 * btop, ra);
        tmem_wait_ld(ra);
        double *oslot = nullptr;            // this lane's column of the current group's output slot
        int cur_h = -1, cur_s = 0, ob = 0;  // ob: the group's first row
#pragma unroll 1
        for (int b = btop; b >= 0; b -= 8) {
            if (b >= 8) {
                __syncwarp();
                tmem_ld8(tbase + 2 * (b - 8), rb);
            }
            const int h = b / kTmemGroup;
            if (h != cur_h) {  // a new group: its slot's last store must have read it
                cur_s = (int)(out_seq % kTmemOut);
                if (lane == 0 && out_seq >= (unsigned)kTmemOut) bulk_wait_read_n<kTmemOut - 1>();
                __syncwarp();
                oslot = out_ring + (size_t)cur_s * kTmemGroup * 32 + lane;
                ob = h * kTmemGroup;
                cur_h = h;
            }
            if (b >= tl && b + 8 <= n - 1) {  // tail rows only
                double v[8];
#pragma unroll
                for (int u = 7; u >= 0; --u) v[u] = L.bstep(tmem_dbl(ra, u));
#pragma unroll
                for (int u = 7; u >= 0; --u) oslot[(b + u - ob) * 32] = col_dir ? vox_dir(b + u) : v[u];
            } else {
#pragma unroll
                for (int u = 7; u >= 0; --u) {
                    const int q = b + u;
                    if (q > n - 1) continue;
                    double xq;
                    if (q == n - 1)
                        xq = L.out_last();
                    else if (q >= tl)
                        xq = L.bstep(tmem_dbl(ra, u));
                    else
                        xq = L.template bwd<false>(tmem_dbl(ra, u), q);
                    if (col_dir || (q == 0 && lo_dir) || (q == n - 1 && (hi_dir || (lo_dir && n == 1))))
                        xq = vox_dir(q);
                    oslot[(q - ob) * 32] = xq;
                }
            }
            if ((b % kTmemGroup) == 0) {  // the group's lowest rows are done: store it
                fence_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tma_store(map_out, col0, h * kTmemGroup, slab, rank, out_u32 + cur_s * kTmemSlotBytes);
                    bulk_commit();
                }
                ++out_seq;
            }
            if (b >= 8) {
                __syncwarp();
                tmem_wait_ld(rb);
#pragma unroll
                for (int u = 0; u < 16; ++u) ra[u] = rb[u];
            }
        }
    }
    // loads still in flight (a wait ran out): let them land before the CTA ends
    for (; used < issued; ++used) {
        const int s = (int)(used % kTmemIn);
        (void)mbar_wait(bar0 + 8 * s, (used / kTmemIn) & 1u);
    }
    if (lane == 0) bulk_wait_read_all();  // the output ring must outlive the stores' reads
    __syncwarp();
    return ok;
}

template <bool FUSE_PRE, bool BULK>
__global__ void __launch_bounds__(kTmemWarps * 32, 1)
    sweep_strided_tmem_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap map_out,
                              SweepArgs<double> a, StridedGeom g) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    unsigned *taddr_slot = reinterpret_cast<unsigned *>(smem_raw);
    if (warp == 0) {
        tmem_alloc(smem_u32(taddr_slot), kTmemCols);
        tmem_relinquish();
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const unsigned tmem = *taddr_slot;
    unsigned char *wbase = smem_raw + 128 + (size_t)warp * kTmemWarpBytes;
    tmem_warp_tiles<FUSE_PRE, BULK>(&map, &map_out, a, g, wbase, tmem + ((unsigned)(warp * 32) << 16));
    tmem_fence_before_sync();
    __syncthreads();  // every warp is done with its TMEM lanes
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 148;
        cached[dev] = n;
    }
    return cached[dev];
}

}  // namespace

bool tmem_sweep_fits(int n) { return n >= kTmemGroup && n <= kTmemMaxRows; }

bool make_tmem_sweep_map(CUtensorMap *out, void *field, int axis, int nx, int ny, int Lp) {
    return make_sweep_tensor_map_rows(out, field, 8, axis, nx, ny, Lp, 32, kTmemGroup);
}

void tmem_prepare_device() {
    for (const void *k : {(const void *)sweep_strided_tmem_kernel<true, true>,
                          (const void *)sweep_strided_tmem_kernel<true, false>,
                          (const void *)sweep_strided_tmem_kernel<false, false>})
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmemCtaBytes);
}

int launch_strided_tmem(const SweepArgs<double> &a, const StridedGeom &g_in, const CUtensorMap *map,
                        const CUtensorMap *map_out, bool fuse_pre, cudaStream_t s) {
    if (!tmem_sweep_fits(g_in.n) || !map || !map_out) return kNotApplicable;
    StridedGeom g = g_in;
    g.tw = 32;
    g.ncb = (int)((g.P + 31) / 32);
    const long long tiles = (long long)g.n_slabs * g.ncb;
    const long long blocks = std::min<long long>(sm_count(), (tiles + kTmemWarps - 1) / kTmemWarps);
    const unsigned grid = (unsigned)std::max<long long>(1, blocks);
    if (fuse_pre && a.bulk.on)
        sweep_strided_tmem_kernel<true, true><<<grid, kTmemWarps * 32, kTmemCtaBytes, s>>>(*map, *map_out, a, g);
    else if (fuse_pre)
        sweep_strided_tmem_kernel<true, false><<<grid, kTmemWarps * 32, kTmemCtaBytes, s>>>(*map, *map_out, a, g);
    else
        sweep_strided_tmem_kernel<false, false><<<grid, kTmemWarps * 32, kTmemCtaBytes, s>>>(*map, *map_out, a, g);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

}  // namespace bfb
