// bfb_batch.cu -- many independent microenvironments in one persistent launch.
//
// A batch references N envs of uneven shapes and substrate counts (same
// device and precision). One LOD step of all of them is one launch of
// batch_step_kernel: a grid of resident one-warp CTAs pulls work items from a
// device queue (one atomic counter). The items of one step are ordered
//     [x tiles of env 0..N-1][y tiles ...][z tiles ...][cell chunks ...]
// and an item of env k waits (bounded) until env k has finished every item of
// the previous stage. It only ever waits for items that running warps took
// earlier, so the launch cannot deadlock, whether or not the whole grid is
// resident. Each item runs the same warp-level tile code as the single-env
// kernels (bfb_tiles.cuh). The step (counter resets + launch) is captured
// once in a CUDA graph and replayed. bfb_batch_simulate_loop runs the same
// envs one bfb_simulate call at a time, the per-instance launch loop the
// persistent launch is compared with.
#include <algorithm>
#include <vector>

#include "bfb_aux.cuh"
#include "bfb_tiles.cuh"

namespace bfb {

constexpr int kCellChunk = 1024;       // (voxel, substrate) pairs per cells item
constexpr int kDepWaitLimit = 1 << 24;  // polls (with ~100 ns back-off) before a dependency wait is declared lost

template <typename T>
struct BatchInst {
    SweepArgs<T> ax[3];  // per-axis arguments (factor tables differ per axis)
    StridedGeom gx, gy;
    ContigGeom gz;
    int vb16[3];         // 16-byte copies allowed (row pitch alignment) for x, y, z
    int items[4];        // work items per stage: x tiles, y tiles, z tiles, cell chunks
    T *f;
    int S, n_occ;
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
    int smem_elems;           // per-warp shared-memory elements
    int stages;               // 3 (diffusion) or 4 (diffusion + cells)
};

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T>
__device__ void cells_chunk(const BatchInst<T> &I, int chunk) {
    const int lane = threadIdx.x & 31;
    const long long total = (long long)I.n_occ * I.S;
    const long long e0 = (long long)chunk * kCellChunk;
    const long long e1 = min(total, e0 + kCellChunk);
    for (long long e = e0 + lane; e < e1; e += 32) {
        const int sidx = (int)(e / I.S), d = (int)(e % I.S);
        const size_t fe = (size_t)I.seg_voxel[sidx] * I.S + d;
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

template <typename T>
__global__ void __launch_bounds__(128) batch_step_kernel(BatchParams<T> p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    T *sm = reinterpret_cast<T *>(smem_raw) + (size_t)warp * p.smem_elems;
    const unsigned total = (unsigned)p.stage_base[p.stages];
    while (true) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(p.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) return;
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
        const int tile = r - pre[k];
        const BatchInst<T> &I = p.inst[k];
        if (stage > 0) {  // env k's previous stage must be complete
            const int need = I.items[stage - 1];
            const int *cnt = p.done + 4 * k + (stage - 1);
            int it = 0;
            while (ld_acquire(cnt) < need) {
                if (++it > kDepWaitLimit) {
                    if (lane == 0) atomicOr(p.err, 2);
                    return;
                }
                __nanosleep(100);
            }
        }
        switch (stage) {
        case 0:
            if (I.vb16[0]) strided_tile<T, 16, true, false>(I.ax[0], I.gx, tile, sm);
            else strided_tile<T, (int)sizeof(T), true, false>(I.ax[0], I.gx, tile, sm);
            break;
        case 1:
            if (I.vb16[1]) strided_tile<T, 16, false, false>(I.ax[1], I.gy, tile, sm);
            else strided_tile<T, (int)sizeof(T), false, false>(I.ax[1], I.gy, tile, sm);
            break;
        case 2:
            if (I.vb16[2]) contig_tile<T, 16>(I.ax[2], I.gz, tile, sm);
            else contig_tile<T, (int)sizeof(T)>(I.ax[2], I.gz, tile, sm);
            break;
        default: cells_chunk(I, tile); break;
        }
        __syncwarp();  // the tile's shared memory is reused by the next item
        if (lane == 0) {
            __threadfence();
            atomicAdd(p.done + 4 * k + stage, 1);
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
    int smem_elems = 0;
    int warps = 1;
    int grid[5] = {0, 0, 0, 0, 0};  // resident CTAs for warps = 1..4
    cudaGraphExec_t graph = nullptr;
    int graph_flags = -1;
    double graph_dt = 0;
    std::vector<uint64_t> graph_epochs;
};

namespace bfb {
// from bfb_capi.cu
int env_prepare_step(bfb_env_s *env, double dt, int flags);
template <typename T>
SweepArgs<T> env_sweep_args(bfb_env_s *env, int axis, double dt);
int env_tile_plan(bfb_env_s *env, int elem, StridedGeom *gx, StridedGeom *gy, ContigGeom *gz, int vb16[3]);
}  // namespace bfb

using namespace bfb;

template <typename T>
static int batch_upload(bfb_batch_s *b, double dt) {
    std::vector<BatchInst<T>> inst(b->n);
    std::vector<int> prefix(4 * (size_t)(b->n + 1), 0);
    size_t smem = 0;
    for (int k = 0; k < b->n; ++k) {
        bfb_env_s *e = b->envs[k];
        BatchInst<T> &I = inst[k];
        for (int a = 0; a < 3; ++a) I.ax[a] = env_sweep_args<T>(e, a, dt);
        int st = env_tile_plan(e, sizeof(T), &I.gx, &I.gy, &I.gz, I.vb16);
        if (st) return st;
        I.items[0] = I.gx.n_slabs * I.gx.ncb;
        I.items[1] = I.gy.n_slabs * I.gy.ncb;
        I.items[2] = (int)((I.gz.nrows + I.gz.R - 1) / I.gz.R);
        I.items[3] = (int)(((long long)e->n_occ * e->S + kCellChunk - 1) / kCellChunk);
        I.f = static_cast<T *>(e->field);
        I.S = e->S;
        I.n_occ = e->n_occ;
        I.seg_start = e->seg_start;
        I.seg_voxel = e->seg_voxel;
        I.t1 = static_cast<const T *>(e->ag_t1);
        I.t2 = static_cast<const T *>(e->ag_t2);
        for (int s = 0; s < 4; ++s) prefix[(size_t)s * (b->n + 1) + k + 1] = prefix[(size_t)s * (b->n + 1) + k] + I.items[s];
        smem = std::max(smem, (size_t)I.gx.n * 32);
        smem = std::max(smem, (size_t)I.gy.n * 32);
        smem = std::max(smem, (size_t)I.gz.R * I.gz.RS);
    }
    if (smem * sizeof(T) > 227 * 1024) return fail(BFB_ERR_UNSUPPORTED, "batch: an env's tile does not fit in shared memory");
    b->smem_elems = (int)smem;
    for (int f = 0; f < 2; ++f) {
        b->stage_base[0][f] = 0;
        for (int s = 0; s < 4; ++s) {
            const int cnt = (s == 3 && f == 0) ? 0 : prefix[(size_t)s * (b->n + 1) + b->n];
            b->stage_base[s + 1][f] = b->stage_base[s][f] + cnt;
        }
    }
    BFB_CUDA(cudaMemcpy(b->d_inst, inst.data(), sizeof(BatchInst<T>) * b->n, cudaMemcpyHostToDevice));
    BFB_CUDA(cudaMemcpy(b->d_prefix, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice));
    BFB_CUDA(cudaFuncSetAttribute(batch_step_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    for (int w = 1; w <= 4; ++w) {
        int per_sm = 0;
        const size_t bytes = (size_t)w * smem * sizeof(T);
        if (bytes > 227 * 1024) {
            b->grid[w] = 0;
            continue;
        }
        BFB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_step_kernel<T>, 32 * w, bytes));
        int sms = 0;
        BFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
        b->grid[w] = per_sm * sms;
    }
    return BFB_OK;
}

template <typename T>
static int batch_launch(bfb_batch_s *b, int flags, cudaStream_t s) {
    const int f = (flags & BFB_STEP_CELLS) ? 1 : 0;
    BatchParams<T> p;
    p.inst = static_cast<const BatchInst<T> *>(b->d_inst);
    p.prefix = b->d_prefix;
    for (int q = 0; q < 5; ++q) p.stage_base[q] = b->stage_base[q][f];
    p.done = b->d_done;
    p.queue = b->d_queue;
    p.err = b->d_err;
    p.n = b->n;
    p.smem_elems = b->smem_elems;
    p.stages = f ? 4 : 3;
    BFB_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), s));
    BFB_CUDA(cudaMemsetAsync(b->d_done, 0, sizeof(int) * 4 * b->n, s));
    const int w = b->warps;
    const size_t bytes = (size_t)w * b->smem_elems * sizeof(T);
    const int grid = std::max(1, b->grid[w]);
    batch_step_kernel<T><<<grid, 32 * w, bytes, s>>>(p);
    BFB_CUDA(cudaGetLastError());
    return BFB_OK;
}

static void batch_drop_graph(bfb_batch_s *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
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
    if (e == cudaSuccess) e = cudaMalloc(&b->d_done, sizeof(int) * 4 * n_envs);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
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
    cudaFree(b->d_done);
    cudaFree(b->d_err);
    cudaFree(b->d_queue);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
    return BFB_OK;
}

BFB_API int bfb_batch_set_option(bfb_batch b, int option, int value) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    if (option != BFB_BATCH_OPT_WARPS_PER_CTA || value < 1 || value > 4)
        return fail(BFB_ERR_INVALID_ARG, "bfb_batch_set_option: unknown option or value");
    b->warps = value;
    batch_drop_graph(b);
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

BFB_API int bfb_batch_simulate(bfb_batch b, double dt, int n_steps, int flags) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    if (n_steps < 0 || !(dt > 0)) return fail(BFB_ERR_INVALID_ARG, "bad dt or n_steps");
    if (!(flags & BFB_STEP_DIFFUSION) || (flags & ~(BFB_STEP_DIFFUSION | BFB_STEP_CELLS)))
        return fail(BFB_ERR_UNSUPPORTED, "batch: flags must be BFB_STEP_DIFFUSION [| BFB_STEP_CELLS]");
    BFB_CUDA(cudaSetDevice(b->device));
    // every env's factors, Dirichlet faces and agents as bfb_simulate would use them
    bool changed = b->graph_flags != flags || b->graph_dt != dt || b->graph_epochs.size() != b->envs.size();
    for (int k = 0; k < b->n; ++k) {
        int st = env_prepare_step(b->envs[k], dt, flags);
        if (st) return st;
        if (!changed && b->graph_epochs[k] != b->envs[k]->epoch) changed = true;
    }
    if (changed || !b->graph) {
        batch_drop_graph(b);
        int st = b->precision == BFB_FP64 ? batch_upload<double>(b, dt) : batch_upload<float>(b, dt);
        if (st) return st;
        for (bfb_env e : b->envs) BFB_CUDA(cudaStreamSynchronize(e->stream));
        cudaGraph_t g = nullptr;
        BFB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        st = b->precision == BFB_FP64 ? batch_launch<double>(b, flags, b->stream) : batch_launch<float>(b, flags, b->stream);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->graph = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        b->graph_flags = flags;
        b->graph_dt = dt;
        b->graph_epochs.resize(b->n);
        for (int k = 0; k < b->n; ++k) b->graph_epochs[k] = b->envs[k]->epoch;
    } else {
        for (bfb_env e : b->envs) BFB_CUDA(cudaStreamSynchronize(e->stream));
    }
    for (int q = 0; q < n_steps; ++q) BFB_CUDA(cudaGraphLaunch(b->graph, b->stream));
    return BFB_OK;
}

BFB_API int bfb_batch_simulate_loop(bfb_batch b, double dt, int n_steps, int flags) {
    if (!b) return fail(BFB_ERR_INVALID_ARG, "null bfb_batch");
    for (int q = 0; q < n_steps; ++q)
        for (bfb_env e : b->envs) {
            const int st = bfb_simulate(e, dt, 1, flags);
            if (st) return st;
        }
    for (bfb_env e : b->envs) BFB_CUDA(cudaStreamSynchronize(e->stream));
    return BFB_OK;
}

}  // extern "C"
