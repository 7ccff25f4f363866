// bfb_batch.cu -- many independent microenvironments stepped together.
//
// A batch references N envs of uneven shapes and substrate counts (same
// device and precision). Every tile runs the single-env kernels' warp-tile
// code: the TMA tiles (bfb_tma_tiles.cuh; the env's own tensor maps, read from
// global memory) where the env's grid and launch shape allow them, else the
// cp.async tiles (bfb_tiles.cuh). One step is captured once in a CUDA graph and
// replayed, in one of two modes:
//
// Staged (default): one launch per stage over a flat grid of tiles, one warp
// per tile (batch_stage_kernel). Per stage, the envs are listed by group, tile
// path and tile size (d_perm) with the prefix of their tile counts (d_tpre);
// a launch covers one class -- one group, one path, tiles within a factor 2 of
// each other -- so that its kernel compiles one path and its shared memory per
// warp fits the class. Each group of envs (about equal work) runs its chain of
// stage launches on its own stream, forked from and joined to the batch stream
// inside the graph; stream order alone orders the stages, so no warp waits.
//
// Persistent: one launch of batch_step_kernel per step, a grid of resident
// CTAs whose warps pull work items from a device queue (one atomic counter).
// An item is `tiles_per_item` adjacent warp tiles of one env and one stage;
// the items of one step are ordered
//     [x items of env 0..N-1][y items ...][z items ...][cell chunks ...]
// and an item of env k waits (bounded) until env k has finished every item of
// the previous stage. It only ever waits for items that running warps took
// earlier, so the launch cannot deadlock, whether or not the whole grid is
// resident. A finished item is published with its bulk stores complete
// (cp.async.bulk.wait_group), a proxy fence and a release; a consumer
// acquires, then fences before its own tensor loads.
//
// bfb_batch_simulate_loop runs the same envs one bfb_simulate call at a time
// (the per-instance launch loop); bfb_batch_autotune picks the mode, warps per
// CTA and tiles per item.
#include <algorithm>
#include <vector>

#include "bfb_aux.cuh"
#include "bfb_tiles.cuh"
#include "bfb_tma_tiles.cuh"

namespace bfb {

constexpr int kCellChunk = 1024;       // (voxel, substrate) pairs per cells item
constexpr int kDepWaitLimit = 1 << 24;  // polls (with ~100 ns back-off) before a dependency wait is declared lost

template <typename T>
struct BatchInst {
    SweepArgs<T> ax[3];  // per-axis arguments (factor tables differ per axis)
    StridedGeom gx, gy;
    ContigGeom gz;
    int vb16[3];         // 16-byte copies allowed (row pitch alignment) for x, y, z
    int tiles[3];        // warp tiles per sweep stage
    int items[4];        // work items per stage: x, y, z (tiles_per_item tiles each), cell chunks
    int tma[3];          // TMA tiles for x, y (tensor maps) and z (bulk copies)
    int crow[2];         // rows per TMA box (x, y)
    int kc;              // z row-group length of the pipelined tile
    const CUtensorMap *map[2];  // the env field's x / y tensor maps, in global memory
    T *f;                // the env's field, (i, j) rows Lp elements apart
    int S, nz, Lp, n_occ;
    const int *seg_start, *seg_voxel;
    const T *t1, *t2;
};

template <typename T>
struct BatchParams {
    const BatchInst<T> *inst;
    const int *prefix;        // [4][n+1]: items before env k in stage s
    int stage_base[5];        // first item of each stage; stage_base[4] = total
    int *done;                // [n][4] finished items per env and stage
    unsigned int *queue;
    int *err;
    int n;
    int warp_bytes;           // per-warp shared memory: 128-byte mbarrier header + the largest tile
    int stages;               // 3 (diffusion) or 4 (diffusion + cells)
    int tiles_per_item;
};

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// Waits until at most `newer` of this thread's most recent bulk groups are
// still pending (the older ones have completed); counts above 16 wait for 16.
template <int N>
__device__ __forceinline__ void bulk_wait_group() {
    asm volatile("cp.async.bulk.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_older(int newer) {
    switch (newer) {
    case 0: bulk_wait_group<0>(); break;
    case 1: bulk_wait_group<1>(); break;
    case 2: bulk_wait_group<2>(); break;
    case 3: bulk_wait_group<3>(); break;
    case 4: bulk_wait_group<4>(); break;
    case 5: bulk_wait_group<5>(); break;
    case 6: bulk_wait_group<6>(); break;
    case 7: bulk_wait_group<7>(); break;
    case 8: bulk_wait_group<8>(); break;
    case 9: bulk_wait_group<9>(); break;
    case 10: bulk_wait_group<10>(); break;
    case 11: bulk_wait_group<11>(); break;
    case 12: bulk_wait_group<12>(); break;
    case 13: bulk_wait_group<13>(); break;
    case 14: bulk_wait_group<14>(); break;
    case 15: bulk_wait_group<15>(); break;
    default: bulk_wait_group<16>(); break;
    }
}
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
}
__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *m) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<unsigned long long>(m)) : "memory");
}

template <typename T>
__device__ void cells_chunk(const BatchInst<T> &I, int chunk) {
    const int lane = threadIdx.x & 31;
    const long long total = (long long)I.n_occ * I.S;
    const long long e0 = (long long)chunk * kCellChunk;
    const long long e1 = min(total, e0 + kCellChunk);
    for (long long e = e0 + lane; e < e1; e += 32) {
        const int sidx = (int)(e / I.S), d = (int)(e % I.S);
        const size_t fe = voxel_elem(I.seg_voxel[sidx], d, I.nz, I.S, I.Lp);
        T x = I.f[fe];
        const int a1 = I.seg_start[sidx + 1];
        for (int q = I.seg_start[sidx]; q < a1; ++q) {
            const size_t z = (size_t)q * I.S + d;
            if constexpr (sizeof(T) == 8)
                x = __ddiv_rn(__dadd_rn(x, I.t1[z]), I.t2[z]);
            else
                x = __fdiv_rn(__fadd_rn(x, I.t1[z]), I.t2[z]);
        }
        I.f[fe] = x;
    }
}

// __launch_bounds__(128, 1): without the minimum-blocks hint the compiler
// holds this kernel (every tile variant inlined) to 80 registers and spills;
// with it, it takes 222 (FP32), so one-warp CTAs fit 9 per SM. TMA_ONLY
// leaves out the cp.async tiles, for batches whose every env takes the TMA
// tiles: FP32 then compiles spill-free in 128 registers (16 per SM).
template <typename T, bool TMA_ONLY>
__global__ void __launch_bounds__(128, (TMA_ONLY && sizeof(T) == 4) ? 4 : 1) batch_step_kernel(BatchParams<T> p) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned char *wbase = smem_raw + (size_t)warp * p.warp_bytes;
    T *sm = reinterpret_cast<T *>(wbase + 128);
    // the warp's row-group mbarriers, reused by every TMA tile it runs: bit c
    // of `phase` is the parity row group c waits for next
    if (lane == 0) {
        for (int c = 0; c < 16; ++c) mbar_init(smem_u32(wbase) + 8 * c, 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned phase = 0;
    const unsigned total = (unsigned)p.stage_base[p.stages];
    // The item finished last is published lazily: its bulk stores complete
    // while the warp already loads the next item. It is published before the
    // warp waits on any dependency (it may be the one waited for) and on exit.
    int pend_k = -1, pend_stage = 0;
    int groups = 0;  // bulk store groups the current item has committed so far
    auto publish = [&]() {
        if (pend_k < 0) return;
        if (lane == 0) {
            bulk_wait_older(groups);     // its bulk stores (older than the current item's) have completed ...
            fence_proxy_async_global();  // ... are ordered with the generic release below ...
            __threadfence();
            atomicAdd(p.done + 4 * pend_k + pend_stage, 1);  // ... and published
        }
        __syncwarp();
        pend_k = -1;
    };
    while (true) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(p.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        int stage = 0;
        while (item >= (unsigned)p.stage_base[stage + 1]) ++stage;
        const int r = (int)(item - (unsigned)p.stage_base[stage]);
        const int *pre = p.prefix + (size_t)stage * (p.n + 1);
        int lo = 0, hi = p.n;  // env k with pre[k] <= r < pre[k+1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (pre[mid] <= r) lo = mid; else hi = mid;
        }
        const int k = lo;
        const int it = r - pre[k];
        const BatchInst<T> &I = p.inst[k];
        groups = 0;
        if (stage < 2 && I.tma[stage] && lane == 0) prefetch_tensormap(I.map[stage]);
        if (stage > 0) {  // env k's previous stage must be complete
            const int need = I.items[stage - 1];
            const int *cnt = p.done + 4 * k + (stage - 1);
            if (ld_acquire(cnt) < need) {
                publish();
                int polls = 0;
                while (ld_acquire(cnt) < need) {
                    if (++polls > kDepWaitLimit) {
                        if (lane == 0) atomicOr(p.err, 2);
                        return;
                    }
                    __nanosleep(100);
                }
            }
            fence_proxy_async_global();  // this warp's tensor loads read what the acquire made visible
        }
        bool ok = true;
        if (stage < 3) {
            const int t0 = it * p.tiles_per_item, t1 = min(I.tiles[stage], t0 + p.tiles_per_item);
            for (int tile = t0; tile < t1 && ok; ++tile) {
                if (stage < 2 && I.tma[stage]) {
                    const StridedGeom &g = stage == 0 ? I.gx : I.gy;
                    const int crow = I.crow[stage];
                    ok = stage == 0 ? strided_tma_tile<T, true, false>(I.map[0], I.map[0], I.ax[0], g, crow, tile,
                                                                       wbase, phase)
                                    : strided_tma_tile<T, false, false>(I.map[1], I.map[1], I.ax[1], g, crow, tile,
                                                                        wbase, phase);
                    phase ^= (1u << ((g.n + crow - 1) / crow)) - 1u;
                    groups += (g.n + crow - 1) / crow;  // one store group per row group
                } else if (stage == 2 && I.tma[2]) {
                    switch (I.S) {  // the substrate count as a constant where it is a common one
                    case 1: ok = contig_pipe_tile<T, 1>(I.ax[2], I.gz, I.kc, tile, wbase, phase); break;
                    case 2: ok = contig_pipe_tile<T, 2>(I.ax[2], I.gz, I.kc, tile, wbase, phase); break;
                    case 4: ok = contig_pipe_tile<T, 4>(I.ax[2], I.gz, I.kc, tile, wbase, phase); break;
                    case 8: ok = contig_pipe_tile<T, 8>(I.ax[2], I.gz, I.kc, tile, wbase, phase); break;
                    default: ok = contig_pipe_tile<T, 0>(I.ax[2], I.gz, I.kc, tile, wbase, phase); break;
                    }
                    phase ^= (1u << ((I.gz.nz + I.kc - 1) / I.kc)) - 1u;
                    groups += (I.gz.nz + I.kc - 1) / I.kc;
                } else if constexpr (!TMA_ONLY) {
                    if (stage == 0) {
                        if (I.vb16[0]) strided_tile<T, 16, true, false>(I.ax[0], I.gx, tile, sm);
                        else strided_tile<T, (int)sizeof(T), true, false>(I.ax[0], I.gx, tile, sm);
                    } else if (stage == 1) {
                        if (I.vb16[1]) strided_tile<T, 16, false, false>(I.ax[1], I.gy, tile, sm);
                        else strided_tile<T, (int)sizeof(T), false, false>(I.ax[1], I.gy, tile, sm);
                    } else {
                        if (I.vb16[2]) contig_tile_any<T, 16>(I.ax[2], I.gz, tile, sm);
                        else contig_tile_any<T, (int)sizeof(T)>(I.ax[2], I.gz, tile, sm);
                    }
                }
                __syncwarp();  // the tile's shared memory is reused by the next tile
            }
        } else {
            cells_chunk(I, it);
        }
        if (!ok) return;  // a bounded wait ran out; the error flag is set
        publish();        // the item before this one; this item's stores stay in flight
        pend_k = k;
        pend_stage = stage;
        groups = 0;
    }
    publish();
}

// One stage of a class of envs of a batch as one launch (the staged mode).
// The stage's envs are listed in `perm` by tile path and by the shared memory
// their tiles need, and tpre[j] counts the stage's tiles (agent chunks for
// STAGE 3) of the listed envs before j. A launch covers the envs
// perm[lo .. hi): one tile path (PATH: kPathTma, kPathCp16 or kPathCpElem,
// compiled alone so that the kernel needs no more registers than that path)
// and similar tile sizes (so that its shared memory per warp fits them
// without waste). Warp g of its grid runs tile tpre[lo] + g - tpre[j] of env
// perm[j], where tpre[j] <= tpre[lo] + g < tpre[j + 1], with that env's own
// tile code, as bfb_simulate's kernels do; the stages follow one another in
// stream order, so no warp waits for another.
constexpr int kPathTma = 0, kPathCp16 = 1, kPathCpElem = 2;
// Register bound: the FP32 TMA sweep stages compile spill-free in 128
// registers per thread (160 without the bound), so that one-warp CTAs of
// small tiles fit 16 per SM instead of 12 (256 uneven grids of edges 32-160,
// staged: 6.76 -> 6.32 ms per step); the other paths would spill under it and
// keep the default.
template <typename T, int STAGE, int PATH>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && PATH == kPathTma && STAGE < 3) ? 4 : 1)
    batch_stage_kernel(const BatchInst<T> *__restrict__ inst, const int *__restrict__ perm,
                       const int *__restrict__ tpre, int lo, int hi, int warp_bytes) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gt = __ldg(tpre + lo) + blockIdx.x * (blockDim.x >> 5) + warp;
    if (gt >= __ldg(tpre + hi)) return;
    while (hi - lo > 1) {  // j with tpre[j] <= gt < tpre[j + 1]
        const int mid = (lo + hi) >> 1;
        if (__ldg(tpre + mid) <= gt) lo = mid; else hi = mid;
    }
    const BatchInst<T> &I = inst[__ldg(perm + lo)];
    const int tile = gt - __ldg(tpre + lo);
    if constexpr (STAGE == 3) {
        cells_chunk(I, tile);
    } else {
        unsigned char *wbase = smem_raw + (size_t)warp * warp_bytes;
        T *sm = reinterpret_cast<T *>(wbase + 128);
        const SweepArgs<T> ax = I.ax[STAGE];
        if constexpr (PATH == kPathTma) {
            const int nch = STAGE < 2 ? ((STAGE == 0 ? I.gx.n : I.gy.n) + I.crow[STAGE] - 1) / I.crow[STAGE]
                                      : (I.gz.nz + I.kc - 1) / I.kc;
            if (lane == 0) {
                for (int c = 0; c < nch; ++c) mbar_init(smem_u32(wbase) + 8 * c, 1);
                fence_mbar_init();
            }
            __syncwarp();
            if constexpr (STAGE < 2) {
                const StridedGeom g = STAGE == 0 ? I.gx : I.gy;
                const CUtensorMap *mp = I.map[STAGE];
                strided_tma_tile<T, STAGE == 0, false>(mp, mp, ax, g, I.crow[STAGE], tile, wbase, 0u);
            } else {
                const ContigGeom gz = I.gz;
                switch (I.S) {  // the substrate count as a constant where it is a common one
                case 1: contig_pipe_tile<T, 1>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 2: contig_pipe_tile<T, 2>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 3: contig_pipe_tile<T, 3>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 4: contig_pipe_tile<T, 4>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 5: contig_pipe_tile<T, 5>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 6: contig_pipe_tile<T, 6>(ax, gz, I.kc, tile, wbase, 0u); break;
                case 8: contig_pipe_tile<T, 8>(ax, gz, I.kc, tile, wbase, 0u); break;
                default: contig_pipe_tile<T, 0>(ax, gz, I.kc, tile, wbase, 0u); break;
                }
            }
        } else {
            constexpr int VB = PATH == kPathCp16 ? 16 : (int)sizeof(T);
            if constexpr (STAGE < 2) {
                const StridedGeom g = STAGE == 0 ? I.gx : I.gy;
                strided_tile<T, VB, STAGE == 0, false>(ax, g, tile, sm);
            } else {
                contig_tile_any<T, VB>(ax, I.gz, tile, sm);
            }
        }
    }
}

}  // namespace bfb

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct bfb_batch_s {
    std::vector<bfb_env> envs;
    int device = 0, precision = BFB_FP64, n = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    void *d_inst = nullptr;
    int *d_prefix = nullptr, *d_done = nullptr, *d_err = nullptr;
    unsigned int *d_queue = nullptr;
    int stage_base[5][2] = {};  // [stage][flags: 0 = diffusion, 1 = diffusion + cells]
    void *d_maps = nullptr;     // [n][2] CUtensorMap (64-byte aligned)
    int warp_bytes = 0;
    int warps = 1;
    int tiles_per_item = 2;
    int mode = BFB_BATCH_MODE_STAGED;
    int grid[5] = {0, 0, 0, 0, 0};  // resident CTAs for warps = 1..4
    bool tma_only = false;          // every env's x, y and z stages take TMA tiles
    // staged mode, per stage s: envs listed by tile size (d_perm[s]), tiles before
    // list entry j (d_tpre[s][j]), and classes of list entries [lo, hi) launched
    // together with `bytes` of shared memory per warp
    int *d_tpre = nullptr;  // [4][n+1]
    int *d_perm = nullptr;  // [4][n]
    struct StageClass {
        int lo, hi, bytes, total, path, group;
    };
    std::vector<StageClass> classes[4];
    // the env groups run side by side on these streams, each its own chain of
    // stage launches (forked from and joined to the batch stream inside the
    // captured graph)
    static constexpr int kSide = 8;
    int n_groups = 1;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kSide] = {};
    cudaGraphExec_t graph = nullptr;        // one step
    cudaGraphExec_t graph_multi = nullptr;  // kMultiSteps steps (both built together)
    static constexpr int kMultiSteps = 8;
    int graph_flags = -1;
    double graph_dt = 0;
    std::vector<uint64_t> graph_epochs;
};

namespace bfb {
// from bfb_capi.cu
int env_prepare_step(bfb_env_s *env, double dt, int flags);
template <typename T>
SweepArgs<T> env_sweep_args(bfb_env_s *env, int axis, double dt);
int env_tile_plan(bfb_env_s *env, int elem, int Lp, StridedGeom *gx, StridedGeom *gy, ContigGeom *gz, int vb16[3]);
int env_run_steps(bfb_env_s *env, double dt, int n, int flags, cudaStream_t s);
}  // namespace bfb

using namespace bfb;

template <typename T>
static int batch_upload(bfb_batch_s *b, double dt) {
    std::vector<BatchInst<T>> inst(b->n);
    std::vector<CUtensorMap> maps(2 * (size_t)b->n);
    std::vector<int> prefix(4 * (size_t)(b->n + 1), 0), tpre(4 * (size_t)(b->n + 1), 0), perm(4 * (size_t)b->n);
    std::vector<size_t> ebytes(3 * (size_t)b->n, 0);  // shared memory of env k's tile in stage s
    std::vector<int> epath(3 * (size_t)b->n, 0);      // tile path of env k in stage s
    const int eb = (int)sizeof(T);
    size_t tile_bytes = 0;
    const CUtensorMap *dmaps = static_cast<const CUtensorMap *>(b->d_maps);
    for (int k = 0; k < b->n; ++k) {
        bfb_env_s *e = b->envs[k];
        BatchInst<T> &I = inst[k];
        for (int a = 0; a < 3; ++a) I.ax[a] = env_sweep_args<T>(e, a, dt);
        int st = env_tile_plan(e, sizeof(T), e->Lp, &I.gx, &I.gy, &I.gz, I.vb16);
        if (st) return st;
        I.tiles[0] = I.gx.n_slabs * I.gx.ncb;
        I.tiles[1] = I.gy.n_slabs * I.gy.ncb;
        I.tiles[2] = (int)((I.gz.nrows + I.gz.R - 1) / I.gz.R);
        for (int a = 0; a < 3; ++a) I.items[a] = (I.tiles[a] + b->tiles_per_item - 1) / b->tiles_per_item;
        I.items[3] = (int)(((long long)e->n_occ * e->S + kCellChunk - 1) / kCellChunk);
        // TMA tiles where the env's own launch shape would use them, as wide
        // as the env's maps' boxes
        for (int a = 0; a < 2; ++a) {
            StridedGeom &g = a == 0 ? I.gx : I.gy;
            const int lines = e->tma_lines[a];
            I.tma[a] = e->use_tma && e->tuning.tma[a] && e->tma_ok[a] &&
                       strided_tma_warp_bytes(g.n, e->tma_crow[a], eb, lines) <= (size_t)kMaxSmem;
            if (I.tma[a]) {
                g.tw = lines;
                g.ncb = (int)((g.P + lines - 1) / lines);
                I.tiles[a] = g.n_slabs * g.ncb;
                I.items[a] = (I.tiles[a] + b->tiles_per_item - 1) / b->tiles_per_item;
            }
            I.crow[a] = e->tma_crow[a];
            maps[2 * (size_t)k + a] = e->tmap[a];
            I.map[a] = dmaps + 2 * (size_t)k + a;
            const size_t tb = I.tma[a] ? strided_tma_warp_bytes(g.n, I.crow[a], eb, lines) - 128 : (size_t)g.n * 32 * eb;
            tile_bytes = std::max(tile_bytes, tb);
            ebytes[(size_t)a * b->n + k] = tb;
        }
        {
            const long long L = e->Lp;  // row pitch
            const bool base16 = (reinterpret_cast<uintptr_t>(e->field) & 15) == 0;
            const bool tma_ok = e->use_tma && e->tuning.tma[2] && e->S <= 32 && base16 && (L * eb) % 16 == 0;
            if (tma_ok && ((long long)I.gz.RS * eb) % 16 != 0 &&
                contig_aligned_geom(e->nz, e->S, e->Lp, eb, &I.gz.R, &I.gz.RS)) {  // 16-byte shared rows, fewer rows
                I.tiles[2] = (int)((I.gz.nrows + I.gz.R - 1) / I.gz.R);
                I.items[2] = (I.tiles[2] + b->tiles_per_item - 1) / b->tiles_per_item;
            }
            I.tma[2] = tma_ok && ((long long)I.gz.RS * eb) % 16 == 0 && (L * eb) * I.gz.R < (1 << 20);
            int q = 16;
            for (int v = e->S * eb; v % 2 == 0 && q > 1; v /= 2) q /= 2;  // q = 16 / gcd(16, S*elem)
            const int chunks = e->tuning.chunks[2];
            const int kc = (e->nz + chunks - 1) / chunks;
            I.kc = (kc + q - 1) / q * q;
            if ((e->nz + I.kc - 1) / I.kc > 16) I.tma[2] = 0;  // one mbarrier per row group
            tile_bytes = std::max(tile_bytes, (size_t)I.gz.R * I.gz.RS * eb);
            ebytes[2 * (size_t)b->n + k] = (size_t)I.gz.R * I.gz.RS * eb;
        }
        I.f = static_cast<T *>(e->field);
        I.S = e->S;
        I.nz = e->nz;
        I.Lp = e->Lp;
        I.n_occ = e->n_occ;
        I.seg_start = e->seg_start;
        I.seg_voxel = e->seg_voxel;
        I.t1 = static_cast<const T *>(e->ag_t1);
        I.t2 = static_cast<const T *>(e->ag_t2);
        for (int s = 0; s < 4; ++s) prefix[(size_t)s * (b->n + 1) + k + 1] = prefix[(size_t)s * (b->n + 1) + k] + I.items[s];
    }
    // staged mode: envs in up to kSide groups of about equal work (largest
    // first, each to the least loaded group); per stage, each group's envs by
    // tile path, then by decreasing tile size, cut into classes of one path
    // whose smallest tile needs more than half the class's largest (at most 4
    // classes per group and path)
    auto warp_of = [](size_t bytes) { return (int)((128 + bytes + 127) / 128 * 128); };
    std::vector<int> group(b->n, 0);
    {
        b->n_groups = std::min(b->n, (int)bfb_batch_s::kSide);
        std::vector<int> order(b->n);
        for (int k = 0; k < b->n; ++k) order[k] = k;
        auto work = [&](int k) { return (double)b->envs[k]->N; };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) > work(y); });
        std::vector<double> load(b->n_groups, 0.0);
        for (int k : order) {
            const int gsel = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            group[k] = gsel;
            load[gsel] += work(k);
        }
    }
    for (int k = 0; k < b->n; ++k)
        for (int s = 0; s < 3; ++s) {
            const BatchInst<T> &I = inst[k];
            epath[(size_t)s * b->n + k] = I.tma[s] ? kPathTma : (I.vb16[s] ? kPathCp16 : kPathCpElem);
        }
    for (int s = 0; s < 4; ++s) {
        int *ps = perm.data() + (size_t)s * b->n;
        for (int k = 0; k < b->n; ++k) ps[k] = k;
        const size_t *bs = s < 3 ? ebytes.data() + (size_t)s * b->n : nullptr;
        const int *pa = s < 3 ? epath.data() + (size_t)s * b->n : nullptr;
        std::stable_sort(ps, ps + b->n, [&](int x, int y) {
            if (group[x] != group[y]) return group[x] < group[y];
            if (!bs) return false;
            return pa[x] != pa[y] ? pa[x] < pa[y] : bs[x] > bs[y];
        });
        int *ts = tpre.data() + (size_t)s * (b->n + 1);
        for (int j = 0; j < b->n; ++j) {
            const BatchInst<T> &I = inst[ps[j]];
            ts[j + 1] = ts[j] + (s < 3 ? I.tiles[s] : I.items[3]);
        }
        b->classes[s].clear();
        for (int j = 0; j < b->n;) {
            const int path = pa ? pa[ps[j]] : kPathTma, grp = group[ps[j]];
            int end = j + 1;  // the group's envs of this path are [j, end)
            while (end < b->n && group[ps[end]] == grp && (!pa || pa[ps[end]] == path)) ++end;
            for (int cls = 0; j < end; ++cls) {
                int hi = j + 1;
                if (bs) {
                    while (hi < end && 2 * bs[ps[hi]] > bs[ps[j]]) ++hi;
                    if (cls == 3) hi = end;  // at most 4 classes per path
                } else {
                    hi = end;
                }
                const int total = ts[hi] - ts[j];
                if (total > 0) b->classes[s].push_back({j, hi, bs ? warp_of(bs[ps[j]]) : 0, total, path, grp});
                j = hi;
            }
        }
    }
    const size_t warp_bytes = (128 + tile_bytes + 127) / 128 * 128;
    if (warp_bytes > (size_t)kMaxSmem) return fail(BFB_ERR_UNSUPPORTED, "batch: an env's tile does not fit in shared memory");
    b->warp_bytes = (int)warp_bytes;
    for (int f = 0; f < 2; ++f) {
        b->stage_base[0][f] = 0;
        for (int s = 0; s < 4; ++s) {
            const int cnt = (s == 3 && f == 0) ? 0 : prefix[(size_t)s * (b->n + 1) + b->n];
            b->stage_base[s + 1][f] = b->stage_base[s][f] + cnt;
        }
    }
    BFB_CUDA(cudaMemcpy(b->d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice));
    BFB_CUDA(cudaMemcpy(b->d_inst, inst.data(), sizeof(BatchInst<T>) * b->n, cudaMemcpyHostToDevice));
    BFB_CUDA(cudaMemcpy(b->d_prefix, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice));
    BFB_CUDA(cudaMemcpy(b->d_tpre, tpre.data(), sizeof(int) * tpre.size(), cudaMemcpyHostToDevice));
    BFB_CUDA(cudaMemcpy(b->d_perm, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice));
    b->tma_only = true;
    for (int k = 0; k < b->n; ++k) b->tma_only = b->tma_only && inst[k].tma[0] && inst[k].tma[1] && inst[k].tma[2];
    const void *step_kernel = b->tma_only ? (const void *)batch_step_kernel<T, true>
                                          : (const void *)batch_step_kernel<T, false>;
    BFB_CUDA(cudaFuncSetAttribute(step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem));
    for (const void *k :
         {(const void *)batch_stage_kernel<T, 0, kPathTma>, (const void *)batch_stage_kernel<T, 0, kPathCp16>,
          (const void *)batch_stage_kernel<T, 0, kPathCpElem>, (const void *)batch_stage_kernel<T, 1, kPathTma>,
          (const void *)batch_stage_kernel<T, 1, kPathCp16>, (const void *)batch_stage_kernel<T, 1, kPathCpElem>,
          (const void *)batch_stage_kernel<T, 2, kPathTma>, (const void *)batch_stage_kernel<T, 2, kPathCp16>,
          (const void *)batch_stage_kernel<T, 2, kPathCpElem>})
        BFB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem));
    int sms = 0;
    BFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    for (int w = 1; w <= 4; ++w) {
        int per_sm = 0;
        const size_t bytes = (size_t)w * warp_bytes;
        if (bytes > (size_t)kMaxSmem) {
            b->grid[w] = 0;
            continue;
        }
        BFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel, 32 * w, bytes));
        b->grid[w] = per_sm * sms;
    }
    return BFB_OK;
}

// The staged mode: one launch per stage, each over every env's tiles.
template <typename T>
static int batch_launch_staged(bfb_batch_s *b, int flags, cudaStream_t s) {
    const BatchInst<T> *inst = static_cast<const BatchInst<T> *>(b->d_inst);
    const int stages = (flags & BFB_STEP_CELLS) ? 4 : 3;
    cudaStream_t main = s;
    // one group: the batch stream; several: a side stream per group, forked
    // here and joined after the step's last stage
    const int nside = b->n_groups > 1 ? b->n_groups : 0;
    if (nside) {
        BFB_CUDA(cudaEventRecord(b->fork_ev, main));
        for (int i = 0; i < nside; ++i) BFB_CUDA(cudaStreamWaitEvent(b->side[i], b->fork_ev, 0));
    }
    for (int q = 0; q < stages; ++q) {
        const int *tp = b->d_tpre + (size_t)q * (b->n + 1);
        const int *pm = b->d_perm + (size_t)q * b->n;
        const int ncls = (int)b->classes[q].size();
        for (int ci = 0; ci < ncls; ++ci) {
            const auto &c = b->classes[q][ci];
            s = nside ? b->side[c.group] : main;
            int w = b->warps;
            while (w > 1 && (size_t)w * c.bytes > (size_t)kMaxSmem) --w;
            const unsigned blocks = (unsigned)((c.total + w - 1) / w);
            const size_t bytes = (size_t)w * c.bytes;
#define BFB_STAGE_LAUNCH(Q, PATH) \
    batch_stage_kernel<T, Q, PATH><<<blocks, 32 * w, Q < 3 ? bytes : 0, s>>>(inst, pm, tp, c.lo, c.hi, c.bytes)
            const int key = 3 * q + (q < 3 ? c.path : 0);
            switch (key) {
            case 0: BFB_STAGE_LAUNCH(0, kPathTma); break;
            case 1: BFB_STAGE_LAUNCH(0, kPathCp16); break;
            case 2: BFB_STAGE_LAUNCH(0, kPathCpElem); break;
            case 3: BFB_STAGE_LAUNCH(1, kPathTma); break;
            case 4: BFB_STAGE_LAUNCH(1, kPathCp16); break;
            case 5: BFB_STAGE_LAUNCH(1, kPathCpElem); break;
            case 6: BFB_STAGE_LAUNCH(2, kPathTma); break;
            case 7: BFB_STAGE_LAUNCH(2, kPathCp16); break;
            case 8: BFB_STAGE_LAUNCH(2, kPathCpElem); break;
            default: BFB_STAGE_LAUNCH(3, kPathTma); break;
            }
#undef BFB_STAGE_LAUNCH
            BFB_CUDA(cudaGetLastError());
        }
    }
    for (int i = 0; i < nside; ++i) {
        BFB_CUDA(cudaEventRecord(b->join_ev[i], b->side[i]));
        BFB_CUDA(cudaStreamWaitEvent(main, b->join_ev[i], 0));
    }
    return BFB_OK;
}

// The graph mode: `steps` steps of each env as bfb_simulate launches them, on
// the env's own stream, forked from and joined back into `s` (captured, the
// envs are independent branches of one graph, each running its steps back to
// back without waiting for the other envs between steps).
static int batch_launch_graph(bfb_batch_s *b, double dt, int flags, int steps, cudaStream_t s) {
    BFB_CUDA(cudaEventRecord(b->fork_ev, s));
    for (bfb_env e : b->envs) BFB_CUDA(cudaStreamWaitEvent(e->stream, b->fork_ev, 0));
    for (bfb_env e : b->envs) {
        const int st = env_run_steps(e, dt, steps, flags, e->stream);
        if (st) return st;
        BFB_CUDA(cudaEventRecord(b->join_ev[0], e->stream));
        BFB_CUDA(cudaStreamWaitEvent(s, b->join_ev[0], 0));
    }
    return BFB_OK;
}

template <typename T>
static int batch_launch(bfb_batch_s *b, int flags, cudaStream_t s) {
    if (b->mode == BFB_BATCH_MODE_STAGED) return batch_launch_staged<T>(b, flags, s);
    const int f = (flags & BFB_STEP_CELLS) ? 1 : 0;
    BatchParams<T> p;
    p.inst = static_cast<const BatchInst<T> *>(b->d_inst);
    p.prefix = b->d_prefix;
    for (int q = 0; q < 5; ++q) p.stage_base[q] = b->stage_base[q][f];
    p.done = b->d_done;
    p.queue = b->d_queue;
    p.err = b->d_err;
    p.n = b->n;
    p.warp_bytes = b->warp_bytes;
    p.stages = f ? 4 : 3;
    p.tiles_per_item = b->tiles_per_item;
    BFB_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), s));
    BFB_CUDA(cudaMemsetAsync(b->d_done, 0, sizeof(int) * 4 * b->n, s));
    int w = b->warps;
    while (w > 1 && b->grid[w] == 0) --w;  // the widest CTA that fits
    const size_t bytes = (size_t)w * b->warp_bytes;
    const int grid = std::max(1, b->grid[w]);
    if (b->tma_only)
        batch_step_kernel<T, true><<<grid, 32 * w, bytes, s>>>(p);
    else
        batch_step_kernel<T, false><<<grid, 32 * w, bytes, s>>>(p);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

static void batch_drop_graph(bfb_batch_s *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->graph_multi) cudaGraphExecDestroy(b->graph_multi);
    b->graph = nullptr;
    b->graph_multi = nullptr;
    b->graph_flags = -1;
}

extern "C" {

BFB_API int bfb_batch_create(bfb_batch *out, int n_envs, const bfb_env *envs) {
    if (!out || !envs || n_envs < 1) return fail(BFB_ERR_INVALID_ARG, "bfb_batch_create: need n_envs >= 1 envs");
    *out = nullptr;
    for (int k = 0; k < n_envs; ++k)
        if (!envs[k]) return fail(BFB_ERR_INVALID_ARG, "bfb_batch_create: null env");
    const int dev = envs[0]->device, prec = envs[0]->precision;
    for (int k = 1; k < n_envs; ++k)
        if (envs[k]->device != dev || envs[k]->precision != prec)
            return fail(BFB_ERR_INVALID_ARG, "bfb_batch_create: all envs must share device and precision");
    BFB_CUDA(cudaSetDevice(dev));
    bfb_batch_s *b = new bfb_batch_s();
    b->envs.assign(envs, envs + n_envs);
    b->device = dev;
    b->precision = prec;
    b->n = n_envs;
    const size_t inst_bytes = prec == BFB_FP64 ? sizeof(BatchInst<double>) : sizeof(BatchInst<float>);
    cudaError_t e = cudaMalloc(&b->d_inst, inst_bytes * n_envs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_prefix, sizeof(int) * 4 * (n_envs + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tpre, sizeof(int) * 4 * (n_envs + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_perm, sizeof(int) * 4 * n_envs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_done, sizeof(int) * 4 * n_envs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_maps, sizeof(CUtensorMap) * 2 * n_envs);  // 256-byte aligned
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    for (int i = 0; i < bfb_batch_s::kSide && e == cudaSuccess; ++i) {
        e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join_ev[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        const int st = cuda_fail(e, "bfb_batch_create");
        bfb_batch_destroy(b);
        return st;
    }
    b->stream = b->own_stream;
    *out = b;
    return BFB_OK;
}

BFB_API int bfb_batch_destroy(bfb_batch b) {
    if (!b) return BFB_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    cudaFree(b->d_inst);
    cudaFree(b->d_prefix);
    cudaFree(b->d_tpre);
    cudaFree(b->d_perm);
    cudaFree(b->d_done);
    cudaFree(b->d_err);
    cudaFree(b->d_queue);
    cudaFree(b->d_maps);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    for (int i = 0; i < bfb_batch_s::kSide; ++i) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->join_ev[i]) cudaEventDestroy(b->join_ev[i]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    delete b;
    return BFB_OK;
}

BFB_API int bfb_batch_set_option(bfb_batch b, int option, int value) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    if (option == BFB_BATCH_OPT_WARPS_PER_CTA && value >= 1 && value <= 4)
        b->warps = value;
    else if (option == BFB_BATCH_OPT_TILES_PER_ITEM && value >= 1 && value <= 64)
        b->tiles_per_item = value;
    else if (option == BFB_BATCH_OPT_MODE && (value == BFB_BATCH_MODE_PERSISTENT || value == BFB_BATCH_MODE_STAGED ||
                                             value == BFB_BATCH_MODE_GRAPH))
        b->mode = value;
    else
        return fail(BFB_ERR_INVALID_ARG, "bfb_batch_set_option: unknown option or value");
    batch_drop_graph(b);
    return BFB_OK;
}

BFB_API int bfb_batch_get_option(bfb_batch b, int option, int *value) {
    if (!b || !value) return fail(BFB_ERR_INVALID_ARG, "bfb_batch_get_option: null argument");
    if (option == BFB_BATCH_OPT_WARPS_PER_CTA)
        *value = b->warps;
    else if (option == BFB_BATCH_OPT_TILES_PER_ITEM)
        *value = b->tiles_per_item;
    else if (option == BFB_BATCH_OPT_MODE)
        *value = b->mode;
    else
        return fail(BFB_ERR_INVALID_ARG, "bfb_batch_get_option: unknown option");
    return BFB_OK;
}

BFB_API int bfb_batch_synchronize(bfb_batch b) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    BFB_CUDA(cudaSetDevice(b->device));
    BFB_CUDA(cudaStreamSynchronize(b->stream));
    int flag = 0;
    BFB_CUDA(cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    for (bfb_env e : b->envs) {
        int f2 = 0;
        BFB_CUDA(cudaMemcpy(&f2, e->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        flag |= f2;
    }
    if (flag) return fail(BFB_ERR_WATCHDOG, "batch: a device-side wait ran out of its iteration limit");
    return BFB_OK;
}

// `steps` steps of the batch in its mode, captured from its stream into one
// graph (the envs' streams are idle: the caller synchronised them).
static int batch_capture(bfb_batch_s *b, double dt, int flags, int steps, cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    BFB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = BFB_OK;
    if (b->mode == BFB_BATCH_MODE_GRAPH)
        st = batch_launch_graph(b, dt, flags, steps, b->stream);
    else
        for (int q = 0; q < steps && !st; ++q)
            st = b->precision == BFB_FP64 ? batch_launch<double>(b, flags, b->stream)
                                          : batch_launch<float>(b, flags, b->stream);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    return BFB_OK;
}

BFB_API int bfb_batch_simulate(bfb_batch b, double dt, int n_steps, int flags) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    if (n_steps < 0 || !(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "bad dt or n_steps");
    if (!(flags & BFB_STEP_DIFFUSION) || (flags & ~(BFB_STEP_DIFFUSION | BFB_STEP_CELLS)))
        return fail(BFB_ERR_UNSUPPORTED, "batch: flags must be BFB_STEP_DIFFUSION [| BFB_STEP_CELLS]");
    BFB_CUDA(cudaSetDevice(b->device));
    NvtxRange range("bfb_batch_simulate");
    // every env's factors, Dirichlet faces and agents as bfb_simulate would use them
    bool changed = b->graph_flags != flags || b->graph_dt != dt || b->graph_epochs.size() != b->envs.size();
    for (int k = 0; k < b->n; ++k) {
        int st = env_prepare_step(b->envs[k], dt, flags);
        if (st) return st;
        if (!changed && b->graph_epochs[k] != b->envs[k]->epoch) changed = true;
    }
    if (changed || !b->graph) {
        batch_drop_graph(b);
        int st = b->mode == BFB_BATCH_MODE_GRAPH ? BFB_OK  // the envs' own launches need no tables
                 : b->precision == BFB_FP64     ? batch_upload<double>(b, dt)
                                                : batch_upload<float>(b, dt);
        if (st) return st;
        for (bfb_env e : b->envs) BFB_CUDA(cudaStreamSynchronize(e->stream));
        if ((st = batch_capture(b, dt, flags, 1, &b->graph))) return st;
        if ((st = batch_capture(b, dt, flags, bfb_batch_s::kMultiSteps, &b->graph_multi))) return st;
        b->graph_flags = flags;
        b->graph_dt = dt;
        b->graph_epochs.resize(b->n);
        for (int k = 0; k < b->n; ++k) b->graph_epochs[k] = b->envs[k]->epoch;
    } else {
        for (bfb_env e : b->envs) BFB_CUDA(cudaStreamSynchronize(e->stream));
    }
    int left = n_steps;
    for (; b->graph_multi && left >= bfb_batch_s::kMultiSteps; left -= bfb_batch_s::kMultiSteps)
        BFB_CUDA(cudaGraphLaunch(b->graph_multi, b->stream));
    for (; left > 0; --left) BFB_CUDA(cudaGraphLaunch(b->graph, b->stream));
    return BFB_OK;
}

BFB_API int bfb_batch_autotune(bfb_batch b, double dt, int flags, int trials, int *chosen, double *best_ms) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    if (!(dt > 0) || trials < 1) return fail(BFB_ERR_INVALID_ARG, "dt must be > 0 and trials >= 1");
    BFB_CUDA(cudaSetDevice(b->device));
    // the trial steps advance the fields: keep copies and put them back
    std::vector<void *> saved(b->n, nullptr);
    int st = BFB_OK;
    for (int k = 0; k < b->n && !st; ++k) {
        bfb_env_s *e = b->envs[k];
        cudaError_t ce = cudaStreamSynchronize(e->stream);
        if (ce == cudaSuccess) ce = cudaMalloc(&saved[k], e->elem * e->Np);
        if (ce == cudaSuccess) ce = cudaMemcpy(saved[k], e->field, e->elem * e->Np, cudaMemcpyDeviceToDevice);
        if (ce != cudaSuccess) st = cuda_fail(ce, "bfb_batch_autotune: field copy");
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!st) {
        cudaError_t ce = cudaEventCreate(&e0);
        if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
        if (ce != cudaSuccess) st = cuda_fail(ce, "cudaEventCreate");
    }
    const int old_w = b->warps, old_t = b->tiles_per_item, old_m = b->mode;
    int best_w = old_w, best_t = old_t, best_m = old_m;
    double best = -1.0;
    // staged: warps per CTA only (tiles per item is a persistent-mode knob)
    struct Shape {
        int mode, w, tpi;
    };
    std::vector<Shape> shapes;
    for (int w : {1, 2, 4}) shapes.push_back({BFB_BATCH_MODE_STAGED, w, old_t});
    for (int w : {1, 2, 4})
        for (int tpi : {1, 2, 4, 8}) shapes.push_back({BFB_BATCH_MODE_PERSISTENT, w, tpi});
    shapes.push_back({BFB_BATCH_MODE_GRAPH, old_w, old_t});
    for (const Shape &sh : shapes) {
        {
            const int w = sh.w, tpi = sh.tpi;
            if (st) break;
            b->mode = sh.mode;
            b->warps = w;
            b->tiles_per_item = tpi;
            batch_drop_graph(b);
            // builds both graphs and warms; then `trials` launches of the multi-step graph
            const int steps = trials * bfb_batch_s::kMultiSteps;
            if ((st = bfb_batch_simulate(b, dt, bfb_batch_s::kMultiSteps, flags))) break;
            cudaError_t ce = cudaEventRecord(e0, b->stream);
            if (ce == cudaSuccess && (st = bfb_batch_simulate(b, dt, steps, flags))) break;
            if (ce == cudaSuccess) ce = cudaEventRecord(e1, b->stream);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
            float ms = 0;
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
            if (ce != cudaSuccess) {
                st = cuda_fail(ce, "bfb_batch_autotune: timing");
                break;
            }
            if (best < 0 || ms / steps < best) {
                best = ms / steps;
                best_w = w;
                best_t = tpi;
                best_m = sh.mode;
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (!st) st = bfb_batch_synchronize(b);
    for (int k = 0; k < b->n; ++k) {
        if (!saved[k]) continue;
        bfb_env_s *e = b->envs[k];
        const cudaError_t ce = cudaMemcpy(e->field, saved[k], e->elem * e->Np, cudaMemcpyDeviceToDevice);
        if (ce != cudaSuccess && !st) st = cuda_fail(ce, "bfb_batch_autotune: field restore");
        cudaFree(saved[k]);
    }
    b->warps = st ? old_w : best_w;
    b->tiles_per_item = st ? old_t : best_t;
    b->mode = st ? old_m : best_m;
    batch_drop_graph(b);
    if (st) return st;
    if (chosen) {
        chosen[0] = best_w;
        chosen[1] = best_t;
    }
    if (best_ms) *best_ms = best;
    return BFB_OK;
}

BFB_API int bfb_batch_simulate_loop(bfb_batch b, double dt, int n_steps, int flags) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    BFB_CUDA(cudaSetDevice(b->device));
    // every env's stream starts after the work queued on the batch stream, and
    // the batch stream waits for every env's last step, so events on the batch
    // stream bracket the whole loop
    BFB_CUDA(cudaEventRecord(b->fork_ev, b->stream));
    for (bfb_env e : b->envs) BFB_CUDA(cudaStreamWaitEvent(e->stream, b->fork_ev, 0));
    for (int q = 0; q < n_steps; ++q)
        for (bfb_env e : b->envs) {
            const int st = bfb_simulate(e, dt, 1, flags);
            if (st) return st;
        }
    for (bfb_env e : b->envs) {
        BFB_CUDA(cudaEventRecord(b->join_ev[0], e->stream));
        BFB_CUDA(cudaStreamWaitEvent(b->stream, b->join_ev[0], 0));
    }
    BFB_CUDA(cudaStreamSynchronize(b->stream));
    return BFB_OK;
}

BFB_API int bfb_batch_set_stream(bfb_batch b, void *stream) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    BFB_CUDA(cudaSetDevice(b->device));
    cudaStream_t want = stream ? (cudaStream_t)stream : b->own_stream;
    if (want != b->stream) BFB_CUDA(cudaStreamSynchronize(b->stream));
    b->stream = want;  // the captured step graph is launched into whichever stream is current
    return BFB_OK;
}

}  // extern "C"
